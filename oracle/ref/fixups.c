/*
 * Support code linked into the CPU checker build of the reference sources
 * (oracle/_ref/libspike_ref.so).  Test infrastructure only.
 *
 * 1. The MKL entry points declared in shim/mkl.h, written from MKL's
 *    documented semantics (MKL is absent here; parity at the mkl_dcsrmv call
 *    site, src/spike_pstrsv.c:215, is therefore unpinned at the ulp level).
 * 2. mkl_malloc over-allocates by 64 KiB and zero-fills: pmemset_d zeroes
 *    step + step%P elements in its last thread instead of the remainder
 *    (src/spike_pstrsv_ops.c:1290-1292), so zeroing R_dense
 *    (src/spike_pstrsv_ops.c:368) can run up to P-1 elements past the end, or
 *    stop short of it and leave recycled heap contents in the spike block.
 * 3. spk_ref_initGlobals: the reference's initGlobals_PSTRSV3
 *    (src/spike_pstrsv_ops.c:69-106) passes BYTE counts to pmemset_d /
 *    pmemset_i, which take ELEMENT counts (src/spike_pstrsv_ops.c:1281-1309),
 *    so it zeroes 4-8x past the intended extent and overruns the pools once
 *    nnz > MAXNNZS/8.  src/spike_pstrsv.c is compiled with
 *    -DinitGlobals_PSTRSV3=spk_ref_initGlobals so its call lands here: the
 *    same arrays are zeroed over the element counts the reference intended.
 *    The buggy definition still exists in the library but is never called.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "mkl.h"
#include "prelude.h"

/* Defined (non-static) in src/spike_pstrsv_ops.c:51-62 but not in the header. */
extern MKL_INT mapReducedX[MAXSIZE];
extern char hasToCalculateSs[MAXTHREADCOUNT];

void *mkl_malloc(size_t size, int alignment)
{
    void *p = NULL;
    if (alignment < (int)sizeof(void *)) alignment = (int)sizeof(void *);
    if (posix_memalign(&p, (size_t)alignment, size + (64u << 10)) != 0) return NULL;
    memset(p, 0, size + (64u << 10));
    return p;
}

void mkl_free(void *p) { free(p); }

void mkl_set_num_threads(int n) { (void)n; }

void cblas_dcopy(const MKL_INT n, const double *x, const MKL_INT incx, double *y, const MKL_INT incy)
{
    for (MKL_INT i = 0; i < n; i++) y[(long)i * incy] = x[(long)i * incx];
}

void mkl_dcsrmv(const char *transa, const MKL_INT *m, const MKL_INT *k, const double *alpha,
                const char *matdescra, const double *val, const MKL_INT *indx,
                const MKL_INT *pntrb, const MKL_INT *pntre, const double *x,
                const double *beta, double *y)
{
    (void)k;
    if (!(transa[0] == 'N' || transa[0] == 'n') || !(matdescra[0] == 'G' || matdescra[0] == 'g') ||
        !(matdescra[3] == 'C' || matdescra[3] == 'c')) {
        fprintf(stderr, "mkl shim: only transa='N', general, zero-based CSR is supported\n");
        abort();
    }
    const MKL_INT base = pntrb[0];
    for (MKL_INT i = 0; i < *m; i++) {
        double sum = 0.0;
        for (MKL_INT j = pntrb[i] - base; j < pntre[i] - base; j++) sum += val[j] * x[indx[j]];
        y[i] = (*alpha) * sum + (*beta) * y[i];
    }
}

void mkl_dcsrsm(const char *transa, const MKL_INT *m, const MKL_INT *n, const double *alpha,
                const char *matdescra, const double *val, const MKL_INT *indx,
                const MKL_INT *pntrb, const MKL_INT *pntre, const double *b,
                const MKL_INT *ldb, double *c, const MKL_INT *ldc)
{
    (void)transa; (void)m; (void)n; (void)alpha; (void)matdescra; (void)val; (void)indx;
    (void)pntrb; (void)pntre; (void)b; (void)ldb; (void)c; (void)ldc;
    fprintf(stderr, "mkl shim: mkl_dcsrsm is only reachable from dead reference code\n");
    abort();
}

void spk_ref_initGlobals(int n, int nnz, int nthreads)
{
    size_t nn = (size_t)nnz, rows = (size_t)n;
    memset(D, 0, sizeof(double) * 2 * nn);
    memset(ID, 0, sizeof(MKL_INT) * 2 * (rows + 1));
    memset(JD, 0, sizeof(MKL_INT) * 2 * nn);
    memset(dependents, 0, sizeof(MKL_INT) * rows);
    memset(T, 0, sizeof(double) * nn);
    memset(JT, 0, sizeof(MKL_INT) * nn);
    memset(IT, 0, sizeof(MKL_INT) * (rows + 1));
    memset(T2, 0, sizeof(double) * 3 * nn);
    memset(JT2, 0, sizeof(MKL_INT) * 3 * nn);
    memset(IT2, 0, sizeof(MKL_INT) * 3 * (rows + 1));
    memset(mapReducedX, 0, sizeof(MKL_INT) * rows);
    memset(reducedX, 0, sizeof(double) * rows);
    size_t p = (size_t)nthreads;
    memset(starts_mapR, 0, sizeof(MKL_INT) * p);
    memset(ends_mapR, 0, sizeof(MKL_INT) * p);
    memset(starts_R, 0, sizeof(MKL_INT) * p);
    memset(ends_R, 0, sizeof(MKL_INT) * p);
    memset(starts_D, 0, sizeof(MKL_INT) * p);
    memset(ends_D, 0, sizeof(MKL_INT) * p);
    memset(starts_D0, 0, sizeof(MKL_INT) * p);
    memset(ends_D0, 0, sizeof(MKL_INT) * p);
    memset(starts_D1, 0, sizeof(MKL_INT) * p);
    memset(ends_D1, 0, sizeof(MKL_INT) * p);
    memset(starts_D2, 0, sizeof(MKL_INT) * p);
    memset(ends_D2, 0, sizeof(MKL_INT) * p);
    memset(starts_S, 0, sizeof(long long) * p);
    memset(ends_S, 0, sizeof(long long) * p);
    memset(numRows_S, 0, sizeof(MKL_INT) * p);
    memset(numCols_S, 0, sizeof(MKL_INT) * p);
    memset(start_intervals, 0, sizeof(MKL_INT) * p);
    memset(end_intervals, 0, sizeof(MKL_INT) * p);
    memset(hasDependences, 0, p);
    memset(hasReflections, 0, p);
    memset(hasToCalculateSs, 0, p);
    memset(isOptimizeds, 0, p);
    isReducedSystemNecessary = 0;
}
