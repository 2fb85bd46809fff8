/*
 * ORACLE -- test infrastructure only (see spike_oracle.h).
 *
 * A sequential, deterministic CPU restatement of the reference Spike
 * preprocessing and solve for the upper-triangular case.  Each step names the
 * reference function and lines it follows.  State lives in one struct instead
 * of the reference's static pools, and sizes are exact instead of the
 * compile-time limits (src/spike_pstrsv_globals.h:4-8).
 *
 * Deliberate, documented differences from the reference binary:
 *  - initGlobals_PSTRSV3 overruns (byte counts passed as element counts,
 *    src/spike_pstrsv_ops.c:71-82); here every array is sized and zeroed exactly.
 *  - optimizeLoadBalance reads uninitialised locals (totalLoss, bestCut;
 *    src/spike_pstrsv_ops.c:383, 537-541, 563) and adds INF per block in signed
 *    int.  Restated as the reference behaves when those locals read as 0 and the
 *    sum wraps (the checker build uses -ftrivial-auto-var-init=zero -fwrapv):
 *    totalLoss = 0 when the cut search does not run, an unassigned bestCut is
 *    -1 (what that build produces in every probe), and the INF sum wraps
 *    modulo 2^32.  One divergence: if the decision would keep a split whose D1
 *    range starts before row 0 (block 0 with bestCut -1, where the reference
 *    reads ID[-1]), the decision is reverted instead.
 *  - a zero-row triangular solve is skipped; the reference writes x[-1]
 *    relative to the segment (src/spike_pstrsv_ops.c:1186 with n = 0).
 *  - the solve runs its steps in one fixed order (all SpMV corrections before
 *    all D2 solves), i.e. one of the interleavings the reference's racy OpenMP
 *    region allows (src/spike_pstrsv.c:213-229).
 *  - nthreads > n (empty partitions) is rejected; the reference reads ia[] out
 *    of bounds there (src/matrix_partitioning.c:56-59).
 */
#include "spike_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define SPKO_INF 2147483640
#define SPKO_MEMSIZE 17179869184LL

struct spko {
    int n, nnz, P, flb;
    char uplo;
    /* upper-triangular matrix the algorithm runs on (J L J for 'L') */
    double *ua;
    int *uia, *uja;
    /* matrixPartitioning */
    int *pnum, *ps, *pe;
    /* D and R_new pool: D/JD entries, ID row pointers (2n+1) */
    double *D;
    int *ID, *JD;
    int *startsD, *endsD, *startsR, *endsR;
    int *dep;
    int redNec;
    char *hasDep, *hasRefl, *hasS, *isOpt;
    int *nRowsS, *nColsS;
    long long *startsS, *endsS;
    int *si, *ei;
    /* D0, D1, D2 pool */
    double *T2;
    int *IT2, *JT2;
    int nIT2rows;
    int *sD0, *eD0, *sD1, *eD1, *sD2, *eD2;
    /* compressed R column maps and dense spikes */
    int *mapR, *sMapR, *eMapR;
    int nMapR;
    double *S;
    long long totalArea;
    /* reduced system */
    int *mapRedX;
    int nRed, rss, nnzRed;
    double *T;
    int *IT, *JT;
    long long nT;
};

static int imax(int a, int b) { return a > b ? a : b; }

static void spko_free_state(spko *s)
{
    void **ptrs[] = {(void **)&s->ua, (void **)&s->uia, (void **)&s->uja, (void **)&s->pnum,
                     (void **)&s->ps, (void **)&s->pe, (void **)&s->D, (void **)&s->ID,
                     (void **)&s->JD, (void **)&s->startsD, (void **)&s->endsD,
                     (void **)&s->startsR, (void **)&s->endsR, (void **)&s->dep,
                     (void **)&s->hasDep, (void **)&s->hasRefl, (void **)&s->hasS,
                     (void **)&s->isOpt, (void **)&s->nRowsS, (void **)&s->nColsS,
                     (void **)&s->startsS, (void **)&s->endsS, (void **)&s->si, (void **)&s->ei,
                     (void **)&s->T2, (void **)&s->IT2, (void **)&s->JT2, (void **)&s->sD0,
                     (void **)&s->eD0, (void **)&s->sD1, (void **)&s->eD1, (void **)&s->sD2,
                     (void **)&s->eD2, (void **)&s->mapR, (void **)&s->sMapR, (void **)&s->eMapR,
                     (void **)&s->S, (void **)&s->mapRedX, (void **)&s->T, (void **)&s->IT,
                     (void **)&s->JT};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) {
        free(*ptrs[i]);
        *ptrs[i] = NULL;
    }
}

spko *spko_create(void) { return (spko *)calloc(1, sizeof(spko)); }

void spko_destroy(spko *s)
{
    if (!s) return;
    spko_free_state(s);
    free(s);
}

/* matrix_partitioning.c:18-36 -- k = n/P rows each, leftovers to the last block.
 * Caller bounds (the IS_MATRIX_PARTITIONED path) are in the caller's row order:
 * for 'L' caller partition t, rows [starts[t], ends[t]) of L, is partition
 * P-1-t of the mirror J L J, rows [n-ends[t], n-starts[t]). */
static void partition_rows(spko *s, const int *starts, const int *ends)
{
    int P = s->P, n = s->n;
    if (starts && ends) {
        for (int t = 0; t < P; t++) {
            int c = s->uplo == 'L' ? P - 1 - t : t;
            s->ps[t] = s->uplo == 'L' ? n - ends[c] : starts[c];
            s->pe[t] = s->uplo == 'L' ? n - starts[c] : ends[c];
            s->pnum[t] = s->pe[t] - s->ps[t];
        }
        return;
    }
    int k = n / P, left = n % P;
    for (int t = 0; t < P; t++) {
        s->pnum[t] = k;
        s->ps[t] = k * t;
        s->pe[t] = s->ps[t] + k;
    }
    s->pnum[P - 1] += left;
    s->pe[P - 1] += left;
}

/* matrix_partitioning.c:38-76 -- D = in-block entries, columns left-aligned. */
static void build_D(spko *s)
{
    const int *ia = s->uia, *ja = s->uja;
    const double *a = s->ua;
    long long w = 0;
    for (int t = 0; t < s->P; t++) {
        int ps = s->ps[t], pe = s->pe[t];
        s->startsD[t] = ps;
        for (int r = ps; r < pe; r++) {
            s->ID[r] = (int)w;
            for (int j = ia[r]; j < ia[r + 1]; j++) {
                int c = ja[j];
                if (ps <= c && c < pe) {
                    s->D[w] = a[j];
                    s->JD[w] = c - ps;
                    w++;
                }
            }
        }
        s->endsD[t] = pe;
    }
    s->ID[s->n] = (int)w;
}

/* spike_pstrsv_ops.c:129-182 ('U' branch) -- mark every column >= pe of blocks
 * 0..P-2 as a dependent (a row of the reduced system). */
static void set_dependents(spko *s)
{
    const int *ia = s->uia, *ja = s->uja;
    s->nRed = 0;
    s->redNec = 0;
    memset(s->dep, 0, sizeof(int) * (size_t)s->n);
    for (int t = 0; t < s->P - 1; t++) {
        int ps = s->ps[t], pe = s->pe[t];
        for (int j = ia[ps]; j < ia[pe]; j++) {
            int c = ja[j];
            if (pe <= c) {
                s->redNec = 1;
                s->hasDep[t] = 1;
                if (!s->dep[c]) s->nRed++;
                s->dep[c] = 1;
            }
        }
    }
}

/* spike_pstrsv_ops.c:184-212 ('U' branch) -- backward scan for the row of the
 * last coupling nonzero (column >= end); start-1 when the block has none. */
static int interval_end(const spko *s, int start, int end)
{
    const int *ia = s->uia, *ja = s->uja;
    int result = end - 1;
    for (int i = ia[end] - 1; i >= ia[start]; i--) {
        if (end <= ja[i]) break;
        if (i == ia[result]) result--;
    }
    return result;
}

/* spike_pstrsv_ops.c:375-565 ('U' branch), with the uninitialised reads
 * resolved as described at the top of this file. */
static void optimize_load_balance(spko *s)
{
    const int *ia = s->uia, *ja = s->uja;
    const int P = s->P;
    int gain, loss, minLoss = SPKO_INF;
    unsigned int totalLoss = 0; /* wraps like the reference's signed sum */
    int nnz_R, nnz_D, nnz_D1 = 0, nnz_D2 = 0, nnz_P = 0;
    int cost1 = 0, cost2 = 0, curCost1 = 0, curCost2 = 0, newCost1 = 0, newCost2 = 0;

    /* current costs (ops.c:389-455) */
    for (int i = 0; i < P; i++) {
        int start = s->ps[i], end = s->pe[i];
        nnz_R = 0;
        if (s->hasRefl[i]) {
            int sI = start + s->si[i], eI = start + s->ei[i];
            nnz_D1 = nnz_D2 = nnz_P = 0;
            int row = start;
            for (int j = ia[start]; j < ia[end]; j++) {
                int col = ja[j];
                if (j == ia[row + 1]) row++;
                if (end <= col)
                    nnz_R++;
                else if (sI > row) {
                    if (eI > col) nnz_D2++; else nnz_P++;
                } else if (eI > row) {
                    if (eI > col) nnz_D2++; else nnz_P++;
                    nnz_D1++;
                } else
                    nnz_D1++;
            }
            cost1 = imax(cost1, nnz_D1);
            cost2 = imax(cost2, nnz_R + nnz_P + nnz_D2);
        } else {
            nnz_D = ia[end] - ia[start];
            for (int j = ia[start]; j < ia[end]; j++)
                if (end < ja[j]) nnz_R++;
            curCost2 = imax(curCost2, nnz_R + nnz_D);
            s->isOpt[i] = nnz_R == 0 ? 2 : 0;
        }
    }
    curCost1 = cost1;
    curCost2 = imax(curCost2, cost2);

    /* probable costs (ops.c:457-506); nnz_P carries over from the last block above */
    for (int i = 0; i < P; i++) {
        int start = s->ps[i], end = s->pe[i];
        nnz_R = 0;
        if (!s->hasRefl[i] && s->isOpt[i] != 2) {
            int eI = start + s->ei[i], sI = eI - 1;
            nnz_D1 = nnz_D2 = nnz_R = 0;
            int row = start;
            for (int j = ia[start]; j < ia[end]; j++) {
                int col = ja[j];
                if (j == ia[row + 1]) row++;
                if (end <= col)
                    nnz_R++;
                else if (sI > row) {
                    if (eI > col) nnz_D2++; else nnz_P++;
                } else if (eI > row) {
                    if (eI > col) nnz_D2++; else nnz_P++;
                    nnz_D1++;
                } else
                    nnz_D1++;
            }
            newCost1 = imax(newCost1, nnz_D1);
            newCost2 = imax(newCost2, nnz_R + nnz_P + nnz_D2);
            s->isOpt[i] = 1;
        }
    }
    newCost2 = imax(newCost2, cost2);

    loss = imax(0, newCost1 - curCost1);
    gain = imax(0, curCost2 - newCost2);
    if (gain > loss) {
        /* cut search for blocks without any coupling (ops.c:515-555) */
        for (int i = 0; i < P; i++) {
            if (s->isOpt[i] != 2) continue;
            int start = s->ps[i], end = s->pe[i];
            int bestCut = -1, row = 0;
            nnz_D2 = nnz_P = 0;
            nnz_D = ia[end] - ia[start];
            for (int j = ia[start]; j < ia[end]; j++) {
                int col = ja[j];
                if (j == ia[row + 1]) {
                    nnz_D1 = nnz_D - (nnz_D2 + nnz_P);
                    cost1 = imax(0, nnz_D1 - newCost1);
                    cost2 = imax(0, nnz_D2 + nnz_P - newCost2);
                    loss = cost1 + cost2;
                    if (loss <= minLoss)
                        minLoss = loss;
                    else
                        bestCut = row - 1;
                    break; /* unconditional in the reference (ops.c:541) */
                }
                if (col <= row) nnz_D2++; else nnz_P++;
            }
            s->si[i] = bestCut;
            s->ei[i] = bestCut + 1;
            totalLoss += (unsigned int)minLoss;
        }
    }
    int revert = (int)totalLoss > 0;
    for (int i = 0; i < P && !revert; i++)
        if (s->isOpt[i] && s->ps[i] + s->si[i] < 0) revert = 1;
    if (revert) memset(s->isOpt, 0, (size_t)P);
}

/* spike_pstrsv_ops.c:567-644 and 682-723 ('U' branches) -- D1 = rows [si, k)
 * with columns shifted by si; D2 = rows [0, ei) restricted to columns < ei.
 * An empty row range still records one empty row, as the reference does. */
static void separate_D_sections(spko *s, int row)
{
    long long w = s->IT2[row];
    for (int t = 0; t < s->P; t++) {
        if (s->hasRefl[t] || s->isOpt[t]) {
            int stop = s->si[t];
            int lo = s->ps[t] + stop, hi = s->pe[t];
            s->sD1[t] = row;
            for (int r = lo; r < hi; r++) {
                for (int q = s->ID[r]; q < s->ID[r + 1]; q++) {
                    s->T2[w] = s->D[q];
                    s->JT2[w] = s->JD[q] - stop;
                    w++;
                }
                s->IT2[++row] = (int)w;
            }
            if (lo >= hi) s->IT2[++row] = (int)w;
            s->eD1[t] = row;
        } else {
            s->sD1[t] = s->eD1[t] = 0;
        }
    }
    for (int t = 0; t < s->P; t++) {
        if (s->hasRefl[t] || s->isOpt[t]) {
            int stop = s->ei[t];
            int lo = s->ps[t], hi = s->ps[t] + stop;
            s->sD2[t] = row;
            for (int r = lo; r < hi; r++) {
                for (int q = s->ID[r]; q < s->ID[r + 1]; q++) {
                    int c = s->JD[q];
                    if (c < stop) {
                        s->T2[w] = s->D[q];
                        s->JT2[w] = c;
                        w++;
                    }
                }
                s->IT2[++row] = (int)w;
            }
            if (lo >= hi) s->IT2[++row] = (int)w;
            s->eD2[t] = row;
        } else {
            s->sD2[t] = s->eD2[t] = 0;
        }
    }
    s->nIT2rows = row;
}

/* spike_pstrsv_ops.c:214-373 ('U' branch) -- intervals, S sizes, D0 extraction,
 * load balance, D1/D2 extraction and the dense S allocation. */
static int build_S_layout(spko *s)
{
    const int *ia = s->uia, *ja = s->uja;
    int row = 0;
    long long w = 0;
    s->totalArea = 0;
    s->IT2[0] = 0;
    s->nIT2rows = 0;
    if (!s->redNec) return 0;
    for (int t = 0; t < s->P; t++) {
        long long colCount = 0, rowCount = 0;
        int ps = s->ps[t], pe = s->pe[t];
        int minDR = pe, maxIR;
        if (t == 0) {
            maxIR = interval_end(s, ps, pe);
            s->ei[0] = maxIR - ps + 1;
            s->si[0] = s->ei[0];
            s->startsS[0] = s->endsS[0] = 0;
            continue;
        }
        for (int r = ps; r < pe; r++) {
            if (s->dep[r]) {
                minDR = r;
                s->hasRefl[t] = 1;
                break;
            }
        }
        if (s->hasRefl[t]) {
            int gap = minDR - ps;
            for (int j = ia[minDR]; j < ia[pe]; j++) {
                int c = ja[j];
                if (pe <= c && s->dep[c] != 2 + t) {
                    colCount++;
                    s->dep[c] = 2 + t;
                }
            }
            if (colCount > 0) s->hasS[t] = 1;
            s->nColsS[t] = (int)colCount;
            maxIR = interval_end(s, ps, pe);
            s->nRowsS[t] = imax(1 + maxIR - minDR, 0);
            rowCount = s->nRowsS[t];
            s->si[t] = minDR - ps;
            s->ei[t] = (maxIR < minDR) ? s->si[t] + 1 : maxIR - ps + 1;
            /* D0: rows [si, ei), columns in [si, ei), shifted by si (ops.c:300-323) */
            s->sD0[t] = row;
            for (int r = ps + s->si[t]; r < ps + s->ei[t]; r++) {
                for (int q = s->ID[r]; q < s->ID[r + 1]; q++) {
                    int c = s->JD[q];
                    if (s->si[t] <= c && c < s->ei[t]) {
                        s->T2[w] = s->D[q];
                        s->JT2[w] = c - gap;
                        w++;
                    }
                }
                s->IT2[++row] = (int)w;
            }
            s->eD0[t] = row;
        } else {
            maxIR = interval_end(s, ps, pe);
            s->ei[t] = maxIR - ps + 1;
            s->si[t] = s->ei[t];
        }
        s->startsS[t] = s->endsS[t - 1];
        s->endsS[t] = s->startsS[t] + (long long)(int)(colCount * rowCount);
        s->totalArea += colCount * rowCount;
    }
    s->totalArea += 40 - (s->totalArea % 40);
    if (s->flb) optimize_load_balance(s);
    if (s->totalArea * (long long)sizeof(double) * 3 > SPKO_MEMSIZE) return 1;
    separate_D_sections(s, row);
    s->S = (double *)calloc((size_t)s->totalArea, sizeof(double));
    return s->S ? 0 : -3;
}

/* spike_pstrsv_ops.c:772-827 ('U' branch) -- R_new = R_old (columns >= pe) plus
 * D3 (rows above border = ps+ei, columns >= border) for split blocks; stored
 * after D in the same pool, row pointers ID[n .. 2n]. */
static void build_R(spko *s)
{
    const int *ia = s->uia, *ja = s->uja;
    const double *a = s->ua;
    int n = s->n;
    long long w = s->ID[n];
    for (int t = 0; t < s->P; t++) {
        int ps = s->ps[t], pe = s->pe[t];
        int border = s->ei[t] + ps;
        int split = s->hasRefl[t] || s->isOpt[t];
        s->startsR[t] = n + ps;
        for (int r = ps; r < pe; r++) {
            s->ID[n + r] = (int)w;
            for (int j = ia[r]; j < ia[r + 1]; j++) {
                int c = ja[j];
                int inD3 = split && border <= c && border > r;
                if (inD3 || pe <= c) {
                    s->hasDep[t] = 1;
                    s->D[w] = a[j];
                    s->JD[w] = c;
                    w++;
                }
            }
        }
        s->endsR[t] = n + pe;
    }
    s->ID[2 * n] = (int)w;
}

/* spike_pstrsv_ops.c:860-886 -- mapR offsets per block (numCols_S each). */
static int build_mappings(spko *s)
{
    int size = 0;
    for (int t = 0; t < s->P; t++) {
        s->sMapR[t] = size;
        size += s->nColsS[t];
        s->eMapR[t] = size;
    }
    s->nMapR = size;
    s->mapR = (int *)calloc((size_t)size + 1, sizeof(int));
    return s->mapR ? 0 : -3;
}

/* spike_pstrsv_ops.c:888-959 -- per block with spikes: sorted distinct
 * out-of-block columns of R_new rows [si, ei) -> mapR, and the dense
 * row-major R (numRows_S x numCols_S) scattered into S. */
static int build_compressed_R(spko *s)
{
    int n = s->n;
    int *mark = (int *)calloc((size_t)n, sizeof(int));
    if (!mark) return -3;
    for (int t = 0; t < s->P; t++) {
        if (!s->hasS[t]) continue;
        int ps = s->ps[t], pe = s->pe[t];
        int rlo = n + ps + s->si[t], rhi = n + ps + s->ei[t];
        memset(mark, 0, sizeof(int) * (size_t)n);
        for (int q = s->ID[rlo]; q < s->ID[rhi]; q++) {
            int c = s->JD[q];
            if (!(ps <= c && c < pe)) mark[c] = 1;
        }
        int counter = 0;
        for (int i = 0; i < n; i++) {
            if (mark[i]) {
                s->mapR[s->sMapR[t] + counter] = i;
                mark[i] += counter;
                counter++;
            }
        }
        if (counter != s->nColsS[t]) {
            free(mark);
            return -4; /* the reference would scatter out of its dense block */
        }
        long long cc = s->nColsS[t];
        double *X = s->S + s->startsS[t];
        for (int r = rlo; r < rhi; r++) {
            for (int q = s->ID[r]; q < s->ID[r + 1]; q++) {
                int c = s->JD[q];
                if (!(ps <= c && c < pe)) X[(long long)(r - rlo) * cc + (mark[c] - 1)] = s->D[q];
            }
        }
    }
    free(mark);
    return 0;
}

/* spike_pstrsv_ops.c:1021-1069 with __udsol2 (ops.c:1196-1228) -- in-place
 * dense multi-RHS back substitution S = D0^{-1} R over the spike columns.
 * Per element: products subtracted in CSR order, then one division by the
 * diagonal (the first entry of the row); no fused multiply-add. */
static void spike_sweep(spko *s)
{
    for (int t = 0; t < s->P; t++) {
        int rc = s->nRowsS[t], cc = s->nColsS[t];
        if (!(s->hasS[t] && rc > 0)) continue;
        double *X = s->S + s->startsS[t];
        const int *IA = s->IT2 + s->sD0[t];
        double *last = X + (long long)(rc - 1) * cc;
        for (int l = 0; l < cc; l++) last[l] /= s->T2[IA[rc - 1]];
        for (int k = rc - 2; k >= 0; k--) {
            double *xk = X + (long long)k * cc;
            for (int j = IA[k] + 1; j < IA[k + 1]; j++) {
                double tv = s->T2[j];
                const double *xc = X + (long long)s->JT2[j] * cc;
                for (int l = 0; l < cc; l++) {
                    double p = tv * xc[l];
                    xk[l] = xk[l] - p;
                }
            }
            double dv = s->T2[IA[k]];
            for (int l = 0; l < cc; l++) xk[l] /= dv;
        }
    }
}

/* spike_pstrsv_ops.c:1071-1150 ('U' branch) -- reduced ids, then rows for the
 * dependents of blocks 1..P-2 holding the nonzero spike entries (val != 0),
 * columns mapped to reduced ids; unit diagonal implicit. */
static int build_reduced(spko *s)
{
    int n = s->n, idx = 0;
    s->mapRedX = (int *)calloc((size_t)s->nRed + 1, sizeof(int));
    if (!s->mapRedX) return -3;
    for (int i = 0; i < n; i++) {
        if (s->dep[i]) {
            s->mapRedX[idx] = i;
            idx++;
            s->dep[i] = idx;
        }
    }
    s->nRed = idx;
    s->IT = (int *)calloc((size_t)idx + 2, sizeof(int));
    if (!s->IT) return -3;
    /* pass 1 counts, pass 2 fills */
    for (int pass = 0; pass < 2; pass++) {
        long long w = 0;
        int row = 1;
        for (int t = 1; t < s->P - 1; t++) {
            int ps = s->ps[t], pe = s->pe[t];
            int first = -1;
            long long cc = s->nColsS[t];
            for (int i = ps; i < pe; i++) {
                if (!s->dep[i]) continue;
                if (first < 0) first = i;
                int rowS = i - first;
                if (s->hasRefl[t] && s->hasS[t] && rowS < s->nRowsS[t]) {
                    const double *Srow = s->S + s->startsS[t] + (long long)rowS * cc;
                    for (int j = 0; j < cc; j++) {
                        double v = Srow[j];
                        if (v != 0) {
                            if (pass) {
                                s->T[w] = v;
                                s->JT[w] = s->dep[s->mapR[s->sMapR[t] + j]] - 1;
                            }
                            w++;
                        }
                    }
                }
                if (pass) s->IT[row] = (int)w;
                row++;
            }
        }
        if (!pass) {
            s->nT = w;
            s->T = (double *)calloc((size_t)w + 1, sizeof(double));
            s->JT = (int *)calloc((size_t)w + 1, sizeof(int));
            if (!s->T || !s->JT) return -3;
        } else {
            s->rss = row - 1;
            s->nnzRed = (int)(w + s->nRed);
        }
    }
    return 0;
}

#define ALLOC(p, cnt, type)                                               \
    do {                                                                  \
        (p) = (type *)calloc((size_t)(cnt) + 1, sizeof(type));            \
        if (!(p)) return -3;                                              \
    } while (0)

int spko_preproc(spko *s, const double *a, const int *ia, const int *ja, int n, int P,
                 char uplo, int flb, const int *starts, const int *ends)
{
    spko_free_state(s);
    if (n <= 0 || P <= 0 || P > n) return -1;
    int nnz = ia[n];
    s->n = n;
    s->nnz = nnz;
    s->P = P;
    s->flb = flb;
    s->uplo = (uplo == 'l' || uplo == 'L') ? 'L' : 'U';
    ALLOC(s->ua, nnz, double);
    ALLOC(s->uia, n + 1, int);
    ALLOC(s->uja, nnz, int);
    if (s->uplo == 'U') {
        memcpy(s->ua, a, sizeof(double) * (size_t)nnz);
        memcpy(s->uia, ia, sizeof(int) * (size_t)(n + 1));
        memcpy(s->uja, ja, sizeof(int) * (size_t)nnz);
    } else {
        for (int r = 0; r <= n; r++) s->uia[r] = nnz - ia[n - r];
        for (int q = 0; q < nnz; q++) {
            s->uja[q] = n - 1 - ja[nnz - 1 - q];
            s->ua[q] = a[nnz - 1 - q];
        }
    }
    for (int r = 0; r < n; r++)
        if (s->uia[r + 1] <= s->uia[r]) return -2; /* empty row */
    ALLOC(s->pnum, P, int);
    ALLOC(s->ps, P, int);
    ALLOC(s->pe, P, int);
    ALLOC(s->D, 2LL * nnz, double);
    ALLOC(s->ID, 2LL * n + 1, int);
    ALLOC(s->JD, 2LL * nnz, int);
    ALLOC(s->startsD, P, int);
    ALLOC(s->endsD, P, int);
    ALLOC(s->startsR, P, int);
    ALLOC(s->endsR, P, int);
    ALLOC(s->dep, n, int);
    ALLOC(s->hasDep, P, char);
    ALLOC(s->hasRefl, P, char);
    ALLOC(s->hasS, P, char);
    ALLOC(s->isOpt, P, char);
    ALLOC(s->nRowsS, P, int);
    ALLOC(s->nColsS, P, int);
    ALLOC(s->startsS, P, long long);
    ALLOC(s->endsS, P, long long);
    ALLOC(s->si, P, int);
    ALLOC(s->ei, P, int);
    ALLOC(s->T2, 3LL * nnz, double);
    ALLOC(s->IT2, 3LL * (n + P) + 1, int);
    ALLOC(s->JT2, 3LL * nnz, int);
    ALLOC(s->sD0, P, int);
    ALLOC(s->eD0, P, int);
    ALLOC(s->sD1, P, int);
    ALLOC(s->eD1, P, int);
    ALLOC(s->sD2, P, int);
    ALLOC(s->eD2, P, int);
    ALLOC(s->sMapR, P, int);
    ALLOC(s->eMapR, P, int);

    partition_rows(s, starts, ends);
    for (int t = 0; t < P; t++)
        if (s->pnum[t] <= 0 || (t > 0 && s->ps[t] != s->pe[t - 1])) return -1;
    if (s->ps[0] != 0 || s->pe[P - 1] != n) return -1;
    build_D(s);
    set_dependents(s);
    int rc = build_S_layout(s);
    if (rc) return rc;
    build_R(s);
    if ((rc = build_mappings(s))) return rc;
    if (!s->S) {
        s->S = (double *)calloc(1, sizeof(double));
        if (!s->S) return -3;
    }
    if ((rc = build_compressed_R(s))) return rc;
    spike_sweep(s);
    return build_reduced(s);
}

/* Back substitution with the diagonal first in each row (ops.c:1179-1194). */
static void udsol(int n, double *x, const double *b, const double *A, const int *IA, const int *JA)
{
    if (n <= 0) return;
    x[n - 1] = b[n - 1] / A[IA[n - 1]];
    for (int k = n - 2; k >= 0; k--) {
        double t = b[k];
        for (int j = IA[k] + 1; j < IA[k + 1]; j++) t -= A[j] * x[JA[j]];
        x[k] = t / A[IA[k]];
    }
}

/* spike_pstrsv.c:149-239 ('U' branch) in one fixed order:
 * D1 solves -> gather -> unit-upper reduced solve (ops.c:1247-1262) -> scatter
 * -> R_new SpMV corrections (mkl_dcsrmv with alpha=-1, beta=1) -> D2/D solves. */
int spko_solve(const spko *s, const double *bin, double *xout)
{
    int n = s->n;
    double *b = (double *)malloc(sizeof(double) * (size_t)n);
    double *x = (double *)calloc((size_t)n, sizeof(double));
    double *red = (double *)calloc((size_t)s->nRed + 1, sizeof(double));
    if (!b || !x || !red) {
        free(b); free(x); free(red);
        return -3;
    }
    if (s->uplo == 'U')
        memcpy(b, bin, sizeof(double) * (size_t)n);
    else
        for (int i = 0; i < n; i++) b[i] = bin[n - 1 - i];

    if (s->redNec) {
        for (int t = 0; t < s->P; t++) {
            if (s->hasRefl[t] || s->isOpt[t]) {
                int ps = s->ps[t], st = s->si[t];
                udsol(s->pnum[t] - st, x + ps + st, b + ps + st, s->T2, s->IT2 + s->sD1[t], s->JT2);
            }
        }
        for (int i = 0; i < s->nRed; i++) red[i] = x[s->mapRedX[i]];
        for (int k = s->rss - 1; k >= 0; k--) {
            double t = 0;
            for (int j = s->IT[k]; j < s->IT[k + 1]; j++) t += s->T[j] * red[s->JT[j]];
            red[k] -= t;
        }
        for (int i = 0; i < s->rss; i++) x[s->mapRedX[i]] = red[i];
        for (int t = 0; t < s->P; t++) {
            if (!s->hasDep[t]) continue;
            for (int r = s->ps[t]; r < s->pe[t]; r++) {
                double sum = 0.0;
                for (int q = s->ID[n + r]; q < s->ID[n + r + 1]; q++) sum += s->D[q] * x[s->JD[q]];
                b[r] = (-1.0) * sum + (1.0) * b[r];
            }
        }
        for (int t = 0; t < s->P; t++) {
            int ps = s->ps[t];
            if (s->hasRefl[t] || s->isOpt[t])
                udsol(s->ei[t], x + ps, b + ps, s->T2, s->IT2 + s->sD2[t], s->JT2);
            else
                udsol(s->pnum[t], x + ps, b + ps, s->D, s->ID + ps, s->JD);
        }
    } else {
        for (int t = 0; t < s->P; t++) {
            int ps = s->ps[t];
            udsol(s->pnum[t], x + ps, b + ps, s->D, s->ID + ps, s->JD);
        }
    }
    if (s->uplo == 'U')
        memcpy(xout, x, sizeof(double) * (size_t)n);
    else
        for (int i = 0; i < n; i++) xout[i] = x[n - 1 - i];
    free(b);
    free(x);
    free(red);
    return 0;
}

void spko_udsol(int n, const double *a, const int *ia, const int *ja, const double *b, double *x)
{
    udsol(n, x, b, a, ia, ja);
}

/* runtime_analysis.c:52-65 / ops.c:1264-1279: forward substitution, diagonal last. */
void spko_ldsol(int n, const double *a, const int *ia, const int *ja, const double *b, double *x)
{
    if (n <= 0) return;
    x[0] = b[0] / a[ia[1] - 1];
    for (int k = 1; k < n; k++) {
        double t = b[k];
        for (int j = ia[k]; j < ia[k + 1] - 1; j++) t -= a[j] * x[ja[j]];
        x[k] = t / a[ia[k + 1] - 1];
    }
}

const void *spko_array(const spko *s, const char *name, long long *count, char *type)
{
    int n = s->n, P = s->P;
#define RET(ptr, cnt, ty)        \
    do {                         \
        *count = (long long)(cnt); \
        *type = (ty);            \
        return (const void *)(ptr); \
    } while (0)
    if (!strcmp(name, "partition_starts")) RET(s->ps, P, 'i');
    if (!strcmp(name, "partition_ends")) RET(s->pe, P, 'i');
    if (!strcmp(name, "partition_numRows")) RET(s->pnum, P, 'i');
    if (!strcmp(name, "D")) RET(s->D, s->ID[2 * n], 'd');
    if (!strcmp(name, "JD")) RET(s->JD, s->ID[2 * n], 'i');
    if (!strcmp(name, "ID")) RET(s->ID, 2LL * n + 1, 'i');
    if (!strcmp(name, "starts_D")) RET(s->startsD, P, 'i');
    if (!strcmp(name, "ends_D")) RET(s->endsD, P, 'i');
    if (!strcmp(name, "starts_R")) RET(s->startsR, P, 'i');
    if (!strcmp(name, "ends_R")) RET(s->endsR, P, 'i');
    if (!strcmp(name, "dependents")) RET(s->dep, n, 'i');
    if (!strcmp(name, "hasDependences")) RET(s->hasDep, P, 'c');
    if (!strcmp(name, "hasReflections")) RET(s->hasRefl, P, 'c');
    if (!strcmp(name, "hasToCalculateSs")) RET(s->hasS, P, 'c');
    if (!strcmp(name, "isOptimizeds")) RET(s->isOpt, P, 'c');
    if (!strcmp(name, "numRows_S")) RET(s->nRowsS, P, 'i');
    if (!strcmp(name, "numCols_S")) RET(s->nColsS, P, 'i');
    if (!strcmp(name, "starts_S")) RET(s->startsS, P, 'q');
    if (!strcmp(name, "ends_S")) RET(s->endsS, P, 'q');
    if (!strcmp(name, "start_intervals")) RET(s->si, P, 'i');
    if (!strcmp(name, "end_intervals")) RET(s->ei, P, 'i');
    if (!strcmp(name, "T2")) RET(s->T2, s->IT2[s->nIT2rows], 'd');
    if (!strcmp(name, "JT2")) RET(s->JT2, s->IT2[s->nIT2rows], 'i');
    if (!strcmp(name, "IT2")) RET(s->IT2, s->nIT2rows + 1, 'i');
    if (!strcmp(name, "starts_D0")) RET(s->sD0, P, 'i');
    if (!strcmp(name, "ends_D0")) RET(s->eD0, P, 'i');
    if (!strcmp(name, "starts_D1")) RET(s->sD1, P, 'i');
    if (!strcmp(name, "ends_D1")) RET(s->eD1, P, 'i');
    if (!strcmp(name, "starts_D2")) RET(s->sD2, P, 'i');
    if (!strcmp(name, "ends_D2")) RET(s->eD2, P, 'i');
    if (!strcmp(name, "mapR")) RET(s->mapR, s->nMapR, 'i');
    if (!strcmp(name, "starts_mapR")) RET(s->sMapR, P, 'i');
    if (!strcmp(name, "ends_mapR")) RET(s->eMapR, P, 'i');
    if (!strcmp(name, "S")) RET(s->S, s->totalArea, 'd');
    if (!strcmp(name, "mapReducedX")) RET(s->mapRedX, s->nRed, 'i');
    if (!strcmp(name, "T")) RET(s->T, s->nT, 'd');
    if (!strcmp(name, "JT")) RET(s->JT, s->nT, 'i');
    if (!strcmp(name, "IT")) RET(s->IT, s->rss + 1, 'i');
    if (!strcmp(name, "U_ia")) RET(s->uia, n + 1, 'i');
    if (!strcmp(name, "U_ja")) RET(s->uja, s->nnz, 'i');
    if (!strcmp(name, "U_a")) RET(s->ua, s->nnz, 'd');
#undef RET
    *count = 0;
    *type = 0;
    return NULL;
}

long long spko_scalar(const spko *s, const char *name)
{
    if (!strcmp(name, "numRowsReducedSystem")) return s->nRed;
    if (!strcmp(name, "numNnzsReducedSystem")) return s->nnzRed;
    if (!strcmp(name, "reducedSystemSolverStart")) return s->rss;
    if (!strcmp(name, "isReducedSystemNecessary")) return s->redNec;
    if (!strcmp(name, "totalArea")) return s->totalArea;
    return -1;
}
