/*
 * ORACLE -- test infrastructure only.  A sequential CPU restatement of the
 * reference spike_pstrsv preprocessing and solve (src/spike_pstrsv.c,
 * src/spike_pstrsv_ops.c, src/matrix_partitioning.c), used by the tests,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg as the CHECKER of
 * the CUDA path.  Nothing in the product links or calls this library.
 *
 * Pinned against the reference's own sources compiled as oracle/_ref (see the
 * Makefile): partition bounds, every flag/interval/offset array, the D/R_new,
 * D0/D1/D2 and reduced-system CSR pools, mapR, mapReducedX and the dense spike
 * matrix S compare bit-exact; x compares by tolerance because the reference
 * solve has a benign race on x (src/spike_pstrsv.c:213-229).
 *
 * 'L' is defined through the reversal mirror J L J (upper triangular), on
 * which the reference's 'U' algorithm runs; the reference's own 'L' branches
 * are unimplemented (src/spike_pstrsv.c:234-237).
 */
#ifndef SPIKE_ORACLE_H
#define SPIKE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct spko spko;

spko *spko_create(void);
void spko_destroy(spko *s);

/* Preprocess A (n rows, CSR a/ia/ja, 0-based) into P partitions.
 * uplo 'U'/'u' or 'L'/'l'.  flb = FORCE_LOAD_BALANCE.  starts/ends: optional
 * caller partition bounds (the IS_MATRIX_PARTITIONED path), else NULL.
 * Returns 0 on success, <0 on rejected input, 1 when the reference would
 * exit(1) because the dense S estimate exceeds its 16 GiB cap. */
int spko_preproc(spko *s, const double *a, const int *ia, const int *ja, int n, int P,
                 char uplo, int flb, const int *starts, const int *ends);

/* Solve A x = b with the preprocessed structure.  b is not modified. */
int spko_solve(const spko *s, const double *b, double *x);

/* Read back a named state array (reference global names, e.g. "ID", "T2",
 * "mapR", "S", "start_intervals").  Returns a pointer owned by s and stores
 * the element count and element type ('d' double, 'i' int32, 'q' int64,
 * 'c' char). */
const void *spko_array(const spko *s, const char *name, long long *count, char *type);

/* Scalars: "numRowsReducedSystem", "numNnzsReducedSystem",
 * "reducedSystemSolverStart", "isReducedSystemNecessary", "totalArea". */
long long spko_scalar(const spko *s, const char *name);

/* Plain sequential substitutions (runtime_analysis.c:37-65 / ops.c:1179-1194,
 * 1264-1279): U with the diagonal first in each row, L with it last. */
void spko_udsol(int n, const double *a, const int *ia, const int *ja, const double *b, double *x);
void spko_ldsol(int n, const double *a, const int *ia, const int *ja, const double *b, double *x);

#ifdef __cplusplus
}
#endif
#endif
