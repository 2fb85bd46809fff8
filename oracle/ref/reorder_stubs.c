/*
 * Support code for compiling the reference's matrix_reordering.c into the CPU
 * checker library (oracle/_ref/libspike_ref.so).  Test infrastructure only.
 *
 * - mkl_dcsrcoo, job[0] = 2 (MKL's documented conversion from the coordinate
 *   format to CSR with column indices sorted increasingly in each row; job[1] =
 *   job[2] = 0: zero-based both ways).  Entries with equal (row, column) keep
 *   their coordinate order.
 * - mkl_dcsradd aborts: matrixSymmetrization (src/matrix_reordering.c:29-80) is
 *   only reached for unsymmetric input, which the checker does not use.
 * - METIS_SetDefaultOptions / METIS_PartGraphKway: the partitioner returns the
 *   vector injected by spk_ref_set_partition, so that the reference's steps
 *   after METIS (src/matrix_reordering.c:143-298) run on a known partition.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "mkl.h"
#include "metis.h"

void mkl_dcsrcoo(const MKL_INT *job, const MKL_INT *n, double *acsr, MKL_INT *ja, MKL_INT *ia,
                 MKL_INT *nnz, double *acoo, MKL_INT *rowind, MKL_INT *colind, MKL_INT *info)
{
    if (job[0] != 2 || job[1] != 0 || job[2] != 0) {
        fprintf(stderr, "mkl shim: mkl_dcsrcoo supports job = {2, 0, 0, ...} only\n");
        abort();
    }
    const MKL_INT m = *n, nz = *nnz;
    MKL_INT *next = (MKL_INT *)calloc((size_t)m + 1, sizeof(MKL_INT));
    if (!next) { *info = 1; return; }
    for (MKL_INT k = 0; k < nz; k++) next[rowind[k] + 1]++;
    for (MKL_INT r = 0; r < m; r++) next[r + 1] += next[r];
    memcpy(ia, next, sizeof(MKL_INT) * ((size_t)m + 1));
    for (MKL_INT k = 0; k < nz; k++) {
        MKL_INT q = next[rowind[k]]++;
        acsr[q] = acoo[k];
        ja[q] = colind[k];
    }
    for (MKL_INT r = 0; r < m; r++)  /* insertion sort by column, stable */
        for (MKL_INT q = ia[r] + 1; q < ia[r + 1]; q++) {
            MKL_INT c = ja[q], p = q;
            double v = acsr[q];
            while (p > ia[r] && ja[p - 1] > c) { ja[p] = ja[p - 1]; acsr[p] = acsr[p - 1]; p--; }
            ja[p] = c;
            acsr[p] = v;
        }
    free(next);
    *info = 0;
}

void mkl_dcsradd(const char *trans, const MKL_INT *request, const MKL_INT *sort, const MKL_INT *m,
                 const MKL_INT *n, double *a, MKL_INT *ja, MKL_INT *ia, const double *beta, double *b,
                 MKL_INT *jb, MKL_INT *ib, double *c, MKL_INT *jc, MKL_INT *ic, const MKL_INT *nzmax,
                 MKL_INT *info)
{
    (void)trans; (void)request; (void)sort; (void)m; (void)n; (void)a; (void)ja; (void)ia; (void)beta;
    (void)b; (void)jb; (void)ib; (void)c; (void)jc; (void)ic; (void)nzmax; (void)info;
    fprintf(stderr, "mkl shim: mkl_dcsradd is not available in the checker build\n");
    abort();
}

static int *g_part = NULL;
static int g_part_n = 0;

void spk_ref_set_partition(const int *part, int n)
{
    free(g_part);
    g_part = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (!g_part) { g_part_n = 0; return; }
    memcpy(g_part, part, sizeof(int) * (size_t)n);
    g_part_n = n;
}

int METIS_SetDefaultOptions(idx_t *options)
{
    for (int i = 0; i < METIS_NOPTIONS; i++) options[i] = -1;
    return METIS_OK;
}

int METIS_PartGraphKway(idx_t *nvtxs, idx_t *ncon, idx_t *xadj, idx_t *adjncy, idx_t *vwgt, idx_t *vsize,
                        idx_t *adjwgt, idx_t *nparts, real_t *tpwgts, real_t *ubvec, idx_t *options,
                        idx_t *objval, idx_t *part)
{
    (void)ncon; (void)xadj; (void)adjncy; (void)vwgt; (void)vsize; (void)adjwgt; (void)nparts;
    (void)tpwgts; (void)ubvec; (void)options;
    if (!g_part || g_part_n != *nvtxs) {
        fprintf(stderr, "metis shim: no injected partition for %d vertices\n", (int)*nvtxs);
        abort();
    }
    memcpy(part, g_part, sizeof(int) * (size_t)g_part_n);
    *objval = 0;
    return METIS_OK;
}
