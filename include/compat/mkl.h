/*
 * The subset of Intel MKL's C interface that the reference's drivers call
 * (test/runtime_analysis.c, example_usage.c, src/matrix_reordering.c), so they
 * build against this library without MKL: put include/compat first on the
 * include path and link libspike_pstrsv_mklcompat.so.
 *
 * The triangular-solve comparators the reference profiler times against its own
 * solver (mkl_cspblas_dcsrtrsv, runtime_analysis.c:67-77, and the
 * inspector-executor mkl_sparse_d_trsv, :79-87, :345-381) run on the GPU with
 * cuSPARSE SpSV: the matrix and the SpSV analysis are made resident on the first
 * call for a matrix (or at mkl_sparse_optimize), and each call then copies x to
 * the GPU, solves and copies y back, so a timed call is an end-to-end solve from
 * host arrays.  mkl_cspblas_dcsrtrsv keeps one resident matrix per distinct
 * (a, ia, ja, m, uplo, transa, diag): a caller that changes those arrays in
 * place must call spk_mkl_release_cache() first.
 * The remaining entry points are host code with MKL's documented meaning:
 * mkl_malloc / mkl_free (aligned malloc / free: arrays from this mkl_malloc,
 * from matrixMarketToCSR and from the reordering may be released with either),
 * cblas_dcopy, mkl_dcsrmv (y := alpha op(A) x + beta y for a general CSR,
 * zero- or one-based per matdescra[3], transa 'N' or 'T'), mkl_set_num_threads
 * and mkl_get_max_threads (thread count for the host loops, OpenMP).
 * Enumeration values are this header's own; only the names follow MKL.
 */
#ifndef SPK_COMPAT_MKL_H
#define SPK_COMPAT_MKL_H

#include <stddef.h>

#ifndef MKL_INT
#define MKL_INT int
#endif

#ifdef __cplusplus
extern "C" {
#endif

void *mkl_malloc(size_t size, int alignment);
void mkl_free(void *p);
void mkl_set_num_threads(int n);
int mkl_get_max_threads(void);

void cblas_dcopy(const MKL_INT n, const double *x, const MKL_INT incx, double *y, const MKL_INT incy);

void mkl_dcsrmv(const char *transa, const MKL_INT *m, const MKL_INT *k, const double *alpha, const char *matdescra,
                const double *val, const MKL_INT *indx, const MKL_INT *pntrb, const MKL_INT *pntre, const double *x,
                const double *beta, double *y);

/* y = op(A)^-1 x for a zero-based triangular CSR (uplo 'U'/'L', transa 'N'/'T',
 * diag 'N' non-unit or 'U' unit) on the GPU (cuSPARSE SpSV). */
void mkl_cspblas_dcsrtrsv(const char *uplo, const char *transa, const char *diag, const MKL_INT *m, const double *a,
                          const MKL_INT *ia, const MKL_INT *ja, const double *x, double *y);

typedef enum {
    SPARSE_STATUS_SUCCESS = 0,
    SPARSE_STATUS_NOT_INITIALIZED = 1,
    SPARSE_STATUS_ALLOC_FAILED = 2,
    SPARSE_STATUS_INVALID_VALUE = 3,
    SPARSE_STATUS_EXECUTION_FAILED = 4,
    SPARSE_STATUS_INTERNAL_ERROR = 5,
    SPARSE_STATUS_NOT_SUPPORTED = 6
} sparse_status_t;
typedef enum { SPARSE_OPERATION_NON_TRANSPOSE = 0, SPARSE_OPERATION_TRANSPOSE = 1 } sparse_operation_t;
typedef enum { SPARSE_INDEX_BASE_ZERO = 0, SPARSE_INDEX_BASE_ONE = 1 } sparse_index_base_t;
typedef enum {
    SPARSE_MATRIX_TYPE_GENERAL = 0,
    SPARSE_MATRIX_TYPE_TRIANGULAR = 1
} sparse_matrix_type_t;
typedef enum { SPARSE_FILL_MODE_LOWER = 0, SPARSE_FILL_MODE_UPPER = 1 } sparse_fill_mode_t;
typedef enum { SPARSE_DIAG_NON_UNIT = 0, SPARSE_DIAG_UNIT = 1 } sparse_diag_type_t;
struct matrix_descr {
    sparse_matrix_type_t type;
    sparse_fill_mode_t mode;
    sparse_diag_type_t diag;
};
typedef struct spk_mkl_sparse_matrix *sparse_matrix_t;

/* A handle over the caller's CSR arrays (not copied until mkl_sparse_optimize or
 * the first mkl_sparse_d_trsv, which upload them with the descriptor of the
 * last mkl_sparse_set_sv_hint, or of that trsv call). */
sparse_status_t mkl_sparse_d_create_csr(sparse_matrix_t *A, const sparse_index_base_t indexing, const MKL_INT rows,
                                        const MKL_INT cols, MKL_INT *rows_start, MKL_INT *rows_end,
                                        MKL_INT *col_indx, double *values);
sparse_status_t mkl_sparse_set_sv_hint(const sparse_matrix_t A, const sparse_operation_t operation,
                                       const struct matrix_descr descr, const MKL_INT expected_calls);
sparse_status_t mkl_sparse_optimize(sparse_matrix_t A);
/* y = alpha op(A)^-1 x on the GPU (cuSPARSE SpSV). */
sparse_status_t mkl_sparse_d_trsv(const sparse_operation_t operation, const double alpha, const sparse_matrix_t A,
                                  const struct matrix_descr descr, const double *x, double *y);
sparse_status_t mkl_sparse_destroy(sparse_matrix_t A);

/* Drop every matrix mkl_cspblas_dcsrtrsv keeps resident (no MKL counterpart). */
void spk_mkl_release_cache(void);

#ifdef __cplusplus
}
#endif

#endif /* SPK_COMPAT_MKL_H */
