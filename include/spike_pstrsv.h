/*
 * spike_pstrsv on NVIDIA B200 (sm_100a): C ABI.
 *
 * Part 1 is a drop-in for the reference library's public API
 * (cuguilke/spike_pstrsv src/spike_pstrsv.h:7-38): the same five entry points,
 * with the same argument meaning, plus the globals its profiler links against
 * (src/spike_pstrsv_globals.h:53-79, src/spike_pstrsv_ops.h:15 and :238).
 * `nthreads` is the partition count P of the Spike decomposition; the same P
 * must be passed to preprocessing and to the solve, as in the reference.
 * Pointers may be host or device memory (classified with
 * cudaPointerGetAttributes).  The preprocessed matrix stays resident on the
 * GPU until the next spike_pstrsv_preproc or free_PSTRSV3 (the reference keeps
 * it in static arrays the same way).
 *
 * Part 2 is a handle-based extension (spk_*) with explicit status codes, device
 * pointers and caller streams; it has no counterpart in the reference.
 *
 * No MKL, CUDA or C++ types appear in any signature.
 */
#ifndef SPIKE_PSTRSV_B200_H
#define SPIKE_PSTRSV_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#ifndef MKL_INT
typedef int MKL_INT; /* 32-bit, as under the LP64 interface the reference links (Makefile.sample:15) */
#define SPK_DEFINED_MKL_INT 1
#endif

/* ========================================================================== */
/* Part 1: the reference API                                                   */
/* ========================================================================== */

/* Replaces spike_pstrsv_preproc (src/spike_pstrsv.h:7, src/spike_pstrsv.c:40-81).
 * Builds the partition, dependency and spike structure of the n x n triangular
 * CSR matrix (a, ia, ja; 0-based, columns sorted per row, diagonal first in
 * each row for 'U' and last for 'L') on the GPU.  uplo 'L' runs the reference
 * 'U' algorithm on the reversal mirror J L J (the reference leaves 'L' as a
 * TODO, src/spike_pstrsv.c:234-237). */
void spike_pstrsv_preproc(double *a, MKL_INT *ia, MKL_INT *ja, int n, int nthreads, const char uplo);

/* Replaces _spike_pstrsv_preproc (src/spike_pstrsv.h:14, src/spike_pstrsv.c:83-140):
 * as above, accumulating per-phase seconds into the *_timer_pstrsv3 globals. */
void _spike_pstrsv_preproc(double *a, MKL_INT *ia, MKL_INT *ja, int n, int nthreads, const char uplo);

/* Replaces spike_pstrsv (src/spike_pstrsv.h:21, src/spike_pstrsv.c:142-147):
 * preprocessing followed by one solve. */
void spike_pstrsv(const char uplo, int m, double *a, MKL_INT *ia, MKL_INT *ja, double *b, double *x,
                  int nthreads);

/* Replaces spike_pstrsv_solve (src/spike_pstrsv.h:31, src/spike_pstrsv.c:149-239):
 * solves A x = b with the structure of the last preprocessing call.  x is
 * written; b is left unchanged unless SPK_CLOBBER_B is set, in which case it
 * receives the corrected right-hand side b - R_new x as the reference leaves
 * it (src/spike_pstrsv.c:213-215). */
void spike_pstrsv_solve(const char uplo, int m, double *b, double *x, int nthreads);

/* Replaces _spike_pstrsv_solve (src/spike_pstrsv.h:38, src/spike_pstrsv.c:241-355):
 * as above, accumulating per-phase seconds into the timer globals. */
void _spike_pstrsv_solve(const char uplo, int m, double *b, double *x, int nthreads);

/* Replaces free_PSTRSV3 (src/spike_pstrsv_ops.h:15, src/spike_pstrsv_ops.c:122-127):
 * releases the resident preprocessed state. */
void free_PSTRSV3(void);

/* Replaces logPSTRSV3 (src/spike_pstrsv_ops.h:238, src/spike_pstrsv_ops.c:1311-1332):
 * prints the structure summary in the reference's text format. */
void logPSTRSV3(int nthreads);

/* Flags with the reference's names and defaults (src/spike_pstrsv_ops.c:63-65). */
extern char PSTRSV_VERBOSE;        /* 1: logPSTRSV3 after preprocessing */
extern char FORCE_LOAD_BALANCE;    /* 1 (default): optimizeLoadBalance step */
extern char IS_MATRIX_PARTITIONED; /* 1: use partition_starts/ends as set by the caller (rows of the
                                      caller's matrix, also for 'L'), then reset */
extern char SPK_CLOBBER_B;         /* 1: write the corrected right-hand side back into b */
extern char SPK_EXACT;             /* 1: no spike truncation (see spk_set_truncation) */

/* Partition bounds (src/spike_pstrsv_globals.h:14-16), sized for SPK_MAX_EXPORTED_PARTS. */
#define SPK_MAX_EXPORTED_PARTS 65536
extern MKL_INT partition_numRows[SPK_MAX_EXPORTED_PARTS];
extern MKL_INT partition_starts[SPK_MAX_EXPORTED_PARTS];
extern MKL_INT partition_ends[SPK_MAX_EXPORTED_PARTS];
extern MKL_INT numRowsReducedSystem;

/* Phase timers in seconds (src/spike_pstrsv_globals.h:58-79).  The per-thread
 * arrays keep the reference's names; the GPU phases are device-wide, so the
 * time of a phase is stored at index 0. */
extern double memoryAlloc_timer_pstrsv3;
extern double preprocessD_timer_pstrsv3;
extern double preprocessR_timer_pstrsv3;
extern double setDependents_timer_pstrsv3;
extern double preprocessS_timer_pstrsv3;
extern double preprocessMappings_timer_pstrsv3;
extern double produceCompressedR_timer_pstrsv3;
extern double produceS_timer_pstrsv3;
extern double produceReducedSystem_timer_pstrsv3;
extern double init_vars_pstrsv3;
extern double reduced_solver_timer_pstrsv3;
extern double temp_timer[SPK_MAX_EXPORTED_PARTS];
extern double waitBefore_timer_pstrsv3[SPK_MAX_EXPORTED_PARTS];
extern double computeY_timer[SPK_MAX_EXPORTED_PARTS];
extern double solveIndependent_timer[SPK_MAX_EXPORTED_PARTS];
extern double subtract_Rx_timer[SPK_MAX_EXPORTED_PARTS];
extern double waitAfter_timer_pstrsv3[SPK_MAX_EXPORTED_PARTS];
extern double solveD2_timer[SPK_MAX_EXPORTED_PARTS];
extern double solveD_timer[SPK_MAX_EXPORTED_PARTS];

/* ========================================================================== */
/* Part 2: handle API (no counterpart in the reference)                        */
/* ========================================================================== */

enum {
    SPK_OK = 0,
    SPK_ERR_ARG = -1,        /* invalid argument (sizes, uplo, P) */
    SPK_ERR_INPUT = -2,      /* malformed CSR: empty row, unsorted/out-of-range column, diagonal not in place */
    SPK_ERR_NOMEM = -3,      /* device allocation failed */
    SPK_ERR_CUDA = -4,       /* CUDA runtime error */
    SPK_ERR_STATE = -5,      /* no preprocessed system / mismatched m, P or uplo */
    SPK_ERR_TOO_LARGE = -6,  /* dense spike estimate over the 16 GiB cap (reference exits, ops.c:352-360) */
    SPK_ERR_TIMEOUT = -7     /* a bounded device wait gave up */
};

typedef struct spk_system spk_system;

/* Message and code of the last failure on the calling thread. */
const char *spk_last_error(void);
int spk_last_error_code(void);

int spk_create(spk_system **out);
int spk_destroy(spk_system *s);

/* Preprocess (a, ia, ja) into nparts partitions.  Host or device pointers.
 * flb: FORCE_LOAD_BALANCE.  starts/ends: optional host arrays of nparts
 * contiguous partition bounds (the IS_MATRIX_PARTITIONED path), else NULL, in
 * the caller's row order: for uplo 'L', partition t (rows [starts[t], ends[t])
 * of L) is partition nparts-1-t of the mirror J L J, which the structure
 * arrays describe. */
int spk_preproc(spk_system *s, const double *a, const int *ia, const int *ja, int n, int nparts,
                char uplo, int flb, const int *starts, const int *ends);

/* Solve with device pointers b (n doubles, not modified) and x (n doubles) on
 * `stream` (a cudaStream_t passed as void*; NULL = the legacy default stream).
 * Asynchronous with respect to the host. */
int spk_solve_device(spk_system *s, const double *b, double *x, void *stream);

/* Solve with host or device pointers; synchronous. */
int spk_solve(spk_system *s, const double *b, double *x);

/* Batched solve of nrhs right-hand sides, device arrays, column-major (column k
 * of B at B + k*ldb, of X at X + k*ldx), asynchronous on `stream` unless a
 * residual is requested or tol >= 0.  The matrix is read once per group of up
 * to 16 right-hand sides.
 *   mode SPK_MODE_FP64:    FP64 tile solves.
 *   mode SPK_MODE_FP32_IR: FP32 tile solves (FP32 values, FP32 accumulation), FP64
 *     residual R = B - A X and FP64 update X += solve_fp32(R), repeated until the
 *     scaled residual ||R||inf / (||A||inf ||X||inf + ||B||inf) of every column is
 *     <= tol (tol < 0: exactly maxit corrections, no host synchronisation).
 * iters (optional) receives the corrections applied, resid (optional, forces a
 * final residual) the largest scaled residual. */
enum { SPK_MODE_FP64 = 0, SPK_MODE_FP32_IR = 1 };
int spk_solve_batch(spk_system *s, int nrhs, const double *B, long long ldb, double *X, long long ldx, int mode,
                    double tol, int maxit, void *stream, int *iters, double *resid);

/* MatrixMarket coordinate file (real, integer or double values) into a 0-based
 * CSR (src/misc.h:35, src/misc.c:109-245): uplo 'U' keeps row <= column, 'L'
 * row >= column, 'N' all entries; symm 'Y' mirrors the off-diagonal entries of a
 * symmetric file ('S' and 'N' read the entries as they are); entries sorted by
 * (row, column); *numRows is the column count.  Host code, no GPU.  The arrays
 * come from posix_memalign: release them with free() (or spk_mtx_free), not
 * mkl_free.  On failure the pointers are NULL and the reason is printed. */
void matrixMarketToCSR(const char *filename, double **a, MKL_INT **ia, MKL_INT **ja, int *numRows, const char uplo,
                       const char symm);
/* The same with a status code (SPK_ERR_INPUT for unreadable, malformed or pattern
 * files) and the entry count. */
int spk_mtx_read(const char *path, char uplo, char symm, double **a, int **ia, int **ja, int *n, int *nnz);
void spk_mtx_free(double *a, int *ia, int *ja);

/* Replace pathToMatrixName and strconcat (src/misc.h, src/misc.c:254-297), which
 * the reference's profiler calls: base name of a path without its extension,
 * and the concatenation of two strings, both malloc'd (free()). */
char *pathToMatrixName(const char *filepath);
char *strconcat(const char *str1, const char *str2);

/* Partition-aware reordering (src/matrix_reordering.h:16-41,
 * src/matrix_reordering.c:18-356), host CSR arrays from malloc/posix_memalign
 * (matrixMarketToCSR's), freed and replaced where a function returns a new
 * matrix.
 * matrixReordering: (*a, *ia, *ja) is the full n x n matrix.  Unless the
 * nthreads equal partitions already decouple (matrixAnalysis), the rows are
 * renumbered for nthreads partitions and the matrix becomes the upper (uplo
 * 'U') or lower (otherwise) triangle of the renumbered matrix, with
 * partition_starts/ends/numRows set and IS_MATRIX_PARTITIONED = 1 for the next
 * spike_pstrsv_preproc.  The partitioner replaces the reference's METIS k-way
 * call: a reverse Cuthill-McKee order of the pattern of A + A^T cut into
 * nthreads contiguous ranges of nearly equal nonzero count; the rows are
 * renumbered in that order (so each partition keeps the narrow band; the
 * reference keeps a METIS part's rows in their original order).  The graph,
 * the renumbering and the triangle are built on the GPU.
 * matrixAnalysis: 1 (and the matrix replaced by its triangle, re-read from
 * matrixFileName, or taken in memory when it is NULL) when no entry of the
 * triangle couples two equal partitions, else 0.
 * matrixSymmetrization: A <- A + A^T, values summed, sorted columns.
 * matrixDuplication: copies of the three arrays. */
void matrixReordering(double **a, MKL_INT **ia, MKL_INT **ja, int numRows, int nthreads, const char uplo,
                      const char symm, const char *matrixFileName);
int matrixAnalysis(int numRows, int nthreads, double **a, MKL_INT **ia, MKL_INT **ja, const char uplo,
                   const char symm, const char *matrixFileName);
void matrixSymmetrization(double **a, MKL_INT **ia, MKL_INT **ja, int numRows);
void matrixDuplication(int numRows, double *a, MKL_INT *ia, MKL_INT *ja, double **a_dup, MKL_INT **ia_dup,
                       MKL_INT **ja_dup);
/* Status-returning reordering (no reference counterpart): matrixReordering's
 * renumbering and triangle without the matrixAnalysis shortcut; perm (optional,
 * n ints) receives the original row of every new row (the RCM order). */
int spk_reorder(double **a, int **ia, int **ja, int n, int nparts, char uplo, int *perm);
/* The reordering's partitioner alone, host code (no GPU): order[q] = the row at
 * position q of the reverse Cuthill-McKee order, part[r] = the partition of row
 * r (both optional, n ints). */
int spk_reorder_plan(int n, const int *ia, const int *ja, int nparts, int *order, int *part);

/* Lend the system device memory for the batched solves' work columns (no
 * reference counterpart): with a workspace set, spk_solve_batch carves its
 * work, residual and correction columns (32 x n FP64 each, as needed; FP32 +
 * refinement adds 32 FP64 columns of the reduced system's unknowns) from it
 * instead of buffers it allocates and keeps with the system, and the system's
 * own batch buffers are released.  spk_workspace_bytes gives the size a mode
 * needs (mode SPK_MODE_FP64 or SPK_MODE_FP32_IR; with_residual: FP64 batches
 * that report their residual).  One workspace can serve many systems whose
 * batches do not overlap on the GPU; NULL, 0 detaches it.  256-byte aligned
 * device memory; a batch that needs more returns SPK_ERR_TOO_LARGE. */
int spk_set_workspace(spk_system *s, void *dev_ptr, long long bytes);
long long spk_workspace_bytes(const spk_system *s, int mode, int with_residual);

/* Batched FP64 solve that allocates no device memory; no counterpart in the
 * reference.  For callers that must not allocate once they are serving: a
 * process whose HBM is already committed under a fixed budget (where a new
 * cudaMalloc can fail), or a latency-critical loop where cudaMalloc/cudaFree
 * would synchronize the device and stall work on other streams.
 * spk_solve_batch grows a per-system work buffer on first use and whenever a
 * larger batch arrives; this call instead uses one fixed 4 MiB scratch array
 * (524,288 FP64 values) compiled into the library, one per device.  The
 * right-hand sides are solved in groups of at most 524,288 / n columns;
 * systems of more than 524,288 rows are rejected with SPK_ERR_TOO_LARGE.
 * The first call on each device looks the scratch up (cudaGetSymbolAddress,
 * which may load the library's device code there): make that first call, on
 * every device you use, before any stream capture begins.  All calls on a
 * device share the scratch, so calls whose work overlaps on the GPU (other
 * streams, threads or systems) race and give wrong results: serialize them.
 * Nothing in the scratch has to start at zero.  FP64 only (SPK_MODE_FP64, no
 * residual), device arrays only, systems on the sliced-ELL layout only
 * (spk_debug_scalar(s, "ell") == 1; others get SPK_ERR_ARG). */
int spk_solve_batch_noalloc(spk_system *s, int nrhs, const double *B, long long ldb, double *X, long long ldx,
                            void *stream);

/* Wait for the system's work and report a device-side failure (a bounded wait
 * in a kernel that gave up) as SPK_ERR_TIMEOUT. */
int spk_check(spk_system *s);

/* Spike truncation threshold tau on absolute spike-row sums.  For rows of a
 * block whose spike row sums to <= tau the coupling correction is at most
 * tau * ||x||_inf, so the solve keeps the block-local value there, and reduced
 * rows with sum <= tau are left out of the reduced solve.  Default 2^-60 (below
 * FP64 resolution); tau < 0 = exact mode (nothing dropped).  Legacy entry
 * points use 2^-60, or exact mode when SPK_EXACT is set. */
int spk_set_truncation(spk_system *s, double tau);

/* Per-phase device timing with CUDA events recorded on the solve's stream:
 * spk_set_profiling(s, 1) enables it; spk_phase_times returns (and resets) the
 * accumulated milliseconds of phase 1 (block-local D1 solves), phase 2 (reduced
 * system) and phase 3+4 (coupled D2/D solves) and the number of solves timed. */
int spk_set_profiling(spk_system *s, int on);
int spk_phase_times(spk_system *s, double *ms3, long long *solves);

/* Structure introspection (reference global names: "ID", "T2", "mapR", "S",
 * "start_intervals", ...): copies up to `capacity` elements to host memory
 * `dst` and stores the full element count and type code ('d' double, 'i'
 * int32, 'q' int64, 'c' char).  dst may be NULL to query the size. */
int spk_debug_array(const spk_system *s, const char *name, void *dst, long long capacity,
                    long long *count, char *type);
long long spk_debug_scalar(const spk_system *s, const char *name);

/* One phase of the chain solve over U rows [row_lo, row_hi) (U order: for
 * uplo 'L', U row r is caller row n-1-r), on device arrays b and x in the
 * caller's order, on `stream`.  No reference counterpart: it is the building
 * block of a solve whose rows are sharded over several GPUs.  Phase 1 solves
 * every chain that starts in the range with zero coupling and stores its final
 * rows; phase 4 re-solves the coupled rows of every chain that ends in the range,
 * reading x at the `chain_reach` rows below each chain.  A shard therefore runs
 * phase 1, receives x of the first chain_reach rows of the next shard (final
 * after that shard's phase 1), then runs phase 4.  Chain bounds:
 * spk_debug_array "chain_tasks1" / "chain_tasks4" (lo, hi, st_lo, st_hi per
 * task).  SPK_ERR_STATE unless spk_debug_scalar(s, "chain") == 1. */
int spk_chain_phase(spk_system *s, int phase, int row_lo, int row_hi, const double *b, double *x, void *stream);

/* Serving residency (no reference counterpart): release every device pool of a
 * system solved by chains that its solves never read (the CSR copy, the
 * reference's D / T2 / spike / reduced-system pools, the partition task lists),
 * keeping the chain layout, 1/diag, the sliced-ELL copy and the chain tasks.
 * spk_solve, spk_solve_device and spk_solve_batch then always take the chain
 * kernels; spk_set_truncation, spk_solve_batch_noalloc and group membership
 * return SPK_ERR_STATE until the system is preprocessed again, and the
 * released pools read back empty through spk_debug_array.  *freed (may be
 * NULL) receives the bytes released.  SPK_ERR_STATE unless
 * spk_debug_scalar(s, "chain") == 1. */
int spk_compact(spk_system *s, long long *freed);

/* Tuning knobs of a system solved by chains (no reference counterpart; the
 * reference's only knob is nthreads).  spk_debug_scalar(s, name) reads them back.
 *   "rows":       rows per chain task of the one-right-hand-side solve (rounded
 *                 up to whole 32-row tiles, doubled at most three times until
 *                 every chain keeps its first rows final; SPK_ERR_ARG if none)
 *   "batch_rows": the same for the batched solve's own chains
 *   "stages":     2 or 3 tiles staged ahead by the one-right-hand-side kernel
 *   "batch_path": 1 batched solves on the chain kernels, 0 on the partition
 *                 kernels (not after spk_compact), -1 automatic (default)
 * Preprocessing sets the defaults again.  Not concurrent with the system's
 * solves: the device is synchronized before task lists are replaced.
 * SPK_ERR_STATE unless spk_debug_scalar(s, "chain") == 1. */
int spk_tune(spk_system *s, const char *name, long long value);

/* Test hook (no reference counterpart): spk_debug_set(s, "fail_waits", 1) makes
 * every solve kernel of s report a failed bounded wait at entry, before it
 * issues any copy, until the failure has been reported once (SPK_ERR_TIMEOUT
 * from the synchronous solve or spk_check); the next solve then runs normally.
 * It exercises the error path of the bounded waits without a real hang. */
int spk_debug_set(spk_system *s, const char *name, long long value);

/* Many systems solved by one captured launch sequence (no reference
 * counterpart).  count preprocessed systems (sliced-ELL layout), system i with
 * nrhs[i] right-hand sides in device array B[i] (column-major, leading dimension
 * ldb[i]) and solutions X[i] (ldx[i]).  The columns are split into width classes
 * 16/8/4/2/1; per class one launch runs the phase-1 tasks of every system from a
 * flat work list (longest tasks first), one the reduced solves, one phase 3+4
 * (FP32 + refinement adds residual and update launches per step).  The sequence
 * is captured on `stream` (not the legacy default stream) into a CUDA graph that
 * spk_group_solve replays; the arrays must stay in place.  mode SPK_MODE_FP64 or
 * SPK_MODE_FP32_IR with `iters` fixed refinement steps.  spk_group_residual
 * returns the largest scaled residual over all systems and columns;
 * spk_group_info: "kernels" (launches in the graph), "virtual_systems",
 * "columns", "task_items", "pool_bytes". */
typedef struct spk_group spk_group;
int spk_group_create(spk_group **out, int count, spk_system *const *systems, const int *nrhs,
                     const double *const *B, const long long *ldb, double *const *X, const long long *ldx, int mode,
                     int iters, void *stream);
int spk_group_solve(spk_group *g, void *stream);
int spk_group_residual(spk_group *g, void *stream, double *worst);
long long spk_group_info(const spk_group *g, const char *name);
int spk_group_destroy(spk_group *g);

/* Serving loop (no reference counterpart; the reference has one global system
 * and no request handling).  The server keeps preprocessed systems resident in
 * HBM under hbm_budget_bytes (footprint admission; idle systems are destroyed in
 * least-recently-used order when a matrix must be admitted) and serves solve
 * requests with nslots worker threads, each with its own CUDA stream: a free
 * worker packs up to 32 queued right-hand sides of the matrix whose oldest
 * request waited longest into one spk_solve_batch, so requests that arrive
 * while other batches run join the next batch and batches of different
 * matrices overlap on the device.  Requests take host arrays (column-major,
 * leading dimension n) that must stay valid until spk_server_wait returns.
 * SPK_MODE_FP32_IR batches take one FP64-residual correction step; every batch's
 * scaled residual is checked against 1e-12 (a batch above it is solved again in
 * FP64). */
typedef struct spk_server spk_server;
int spk_server_create(spk_server **out, long long hbm_budget_bytes, int nslots);
int spk_server_destroy(spk_server *srv);
/* Register (or replace, when idle) matrix `id`; the server keeps a host copy of
 * the CSR arrays and preprocesses it when a batch first needs it. */
int spk_server_put_matrix(spk_server *srv, int id, const double *a, const int *ia, const int *ja, int n,
                          int nparts, char uplo);
int spk_server_submit(spk_server *srv, int id, int nrhs, const double *b, double *x, int mode, long long *ticket);
/* Block until the request is done: latency (submit to result in x, seconds), the
 * batch's scaled residual (FP32_IR; -1 otherwise), refinement steps and the
 * batch's right-hand-side count. */
int spk_server_wait(spk_server *srv, long long ticket, double *latency_s, double *resid, int *iters,
                    int *batch_rhs);
/* out[0..15]: resident bytes, staging bytes, resident systems, evictions,
 * preprocessings, batches, right-hand sides batched, requests completed, budget,
 * batches retried after releasing idle systems when device memory ran out,
 * batches solved again in FP64 because their scaled residual was above 1e-12
 * (requests still above it fail with SPK_ERR_INPUT), and microseconds spent
 * (summed over the workers) in host staging in, the solves with their device
 * copies, host staging out and preprocessing, and systems compacted
 * (spk_compact) to make room before any eviction. */
int spk_server_stats(spk_server *srv, long long *out, int count);

/* The system used by the Part-1 entry points (NULL before the first preproc). */
spk_system *spk_legacy_system(void);

#ifdef __cplusplus
}
#endif

#endif /* SPIKE_PSTRSV_B200_H */
