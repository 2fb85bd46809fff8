/*
 * Minimal stand-in for Intel MKL's <mkl.h>, used ONLY to compile the
 * reference spike_pstrsv sources into a CPU checker library (test
 * infrastructure, never shipped, never on the GPU product path).
 *
 * Intel MKL is not installed in this environment.  The reference solver
 * files need only a handful of MKL entry points; each one below is written
 * from MKL's public documented semantics:
 *   - MKL_INT is 32-bit under the LP64 interface the reference links
 *     (Makefile.sample:15, -lmkl_intel_lp64).
 *   - mkl_malloc/mkl_free: aligned allocation (posix_memalign/free).
 *   - mkl_set_num_threads: no-op (the reference only sets 1 thread for the
 *     dead mkl_dcsrsm calls, spike_pstrsv_ops.c:1034).
 *   - cblas_dcopy: y := x with strides.
 *   - mkl_dcsrmv: y := alpha*A*x + beta*y for a general, zero-based CSR
 *     given by (val, indx, pntrb, pntre); row i of A occupies
 *     val[pntrb[i]-pntrb[0] .. pntre[i]-pntrb[0]).  The sum is accumulated
 *     left to right in CSR order.  MKL's own summation order is not
 *     published, so parity at this call site is ulp-level, not bitwise.
 *   - mkl_dcsrsm: reachable only from dead code (produceS_PSTRSV3,
 *     produceS_PSTRSV3_Parallel_OLD); it aborts if ever called.
 *   - mkl_dcsrcoo (matrix_reordering.c:186-187, job = {2, 0, 0, 0, nnz, 0}):
 *     zero-based coordinate format to zero-based CSR with the column indices
 *     sorted increasingly within each row.
 *   - mkl_dcsradd: only reached by matrixSymmetrization for unsymmetric input;
 *     it aborts if called (the checker runs the reordering on symmetric input).
 */
#ifndef SPK_MKL_SHIM_H
#define SPK_MKL_SHIM_H

#include <stddef.h>

typedef int MKL_INT;

#ifdef __cplusplus
extern "C" {
#endif

void *mkl_malloc(size_t size, int alignment);
void mkl_free(void *p);
void mkl_set_num_threads(int n);
void cblas_dcopy(const MKL_INT n, const double *x, const MKL_INT incx, double *y, const MKL_INT incy);
void mkl_dcsrmv(const char *transa, const MKL_INT *m, const MKL_INT *k, const double *alpha,
                const char *matdescra, const double *val, const MKL_INT *indx,
                const MKL_INT *pntrb, const MKL_INT *pntre, const double *x,
                const double *beta, double *y);
void mkl_dcsrsm(const char *transa, const MKL_INT *m, const MKL_INT *n, const double *alpha,
                const char *matdescra, const double *val, const MKL_INT *indx,
                const MKL_INT *pntrb, const MKL_INT *pntre, const double *b,
                const MKL_INT *ldb, double *c, const MKL_INT *ldc);
void mkl_dcsrcoo(const MKL_INT *job, const MKL_INT *n, double *acsr, MKL_INT *ja, MKL_INT *ia,
                 MKL_INT *nnz, double *acoo, MKL_INT *rowind, MKL_INT *colind, MKL_INT *info);
void mkl_dcsradd(const char *trans, const MKL_INT *request, const MKL_INT *sort, const MKL_INT *m,
                 const MKL_INT *n, double *a, MKL_INT *ja, MKL_INT *ia, const double *beta, double *b,
                 MKL_INT *jb, MKL_INT *ib, double *c, MKL_INT *jc, MKL_INT *ic, const MKL_INT *nzmax,
                 MKL_INT *info);

#ifdef __cplusplus
}
#endif

#endif
