// Device-side Spike preprocessing for sm_100a.
//
// Every O(nnz) step of the reference's preprocessing pipeline
// (src/spike_pstrsv.c:40-81) runs as a data-parallel kernel over rows or
// nonzeros: classify -> count -> exclusive scan -> scatter.  Only O(P)
// per-partition bookkeeping (interval arithmetic, the load-balance decision)
// runs on the host, on per-partition reductions copied back from the device.
// The produced pools are bit-identical to the reference's global arrays.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <ctime>

#include "spk_internal.cuh"

namespace spk {

namespace {

constexpr int kInf = 2147483640;                        // INF (spike_pstrsv_globals.h:7)
constexpr long long kMemSize = 17179869184LL;           // MEMSIZE (spike_pstrsv_globals.h:8)

struct PartDev {        // per-partition metadata read by the kernels
    int ps, pe, si, ei;
    int minDR, nRowsS, nColsS, sMapR;
    long long startsS;
    int flags;          // bit0: split (hasReflection || isOptimized), bit1: hasReflection, bit2: hasToCalculateS
    int pad;
};

struct Seg {            // one partition's slice of the D0 | D1 | D2 pool
    int out0;           // first pool row
    int nrows;          // pool rows (1 for an empty range: the reference records one empty row)
    int glo;            // first global row (meaningless for an artifact row)
    int clo, chi;       // kept local columns: clo <= JD < chi
    int shift;          // subtracted from JD
    int artifact;       // 1: the single empty row of an empty range
};

inline double now_s() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

__device__ __forceinline__ int lower_bound_i(const int *a, int lo, int hi, int key) {
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ int part_of(const int *__restrict__ ps, int P, int r) {
    int lo = 0, hi = P - 1;  // largest t with ps[t] <= r
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (ps[mid] <= r) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ---- input -----------------------------------------------------------------

// J L J: row r of U is row n-1-r of L reversed, column c -> n-1-c.
__global__ void k_mirror(int n, int nnz, const int *__restrict__ lia, const int *__restrict__ lja,
                         const double *__restrict__ la, int *__restrict__ uia,
                         int *__restrict__ uja, double *__restrict__ ua) {
    long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i <= n; i += stride)
        uia[i] = nnz - lia[n - i];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nnz; q += stride) {
        uja[q] = n - 1 - lja[nnz - 1 - q];
        ua[q] = la[nnz - 1 - q];
    }
}

// Row-wise input contract of the reference solver: nonempty rows, strictly
// increasing in-range columns, diagonal first (spike_pstrsv_ops.c:1179-1194).
// The smallest offending row wins; key = row * 8 + code.
__global__ void k_validate(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                           unsigned long long *__restrict__ err) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    int b = ia[r], e = ia[r + 1];
    int code = 0;
    if (e <= b) code = 1;
    else if (ja[b] != r) code = 2;
    else {
        for (int q = b + 1; q < e; q++) {
            int c = ja[q];
            if (c <= ja[q - 1] || c >= n) { code = 3; break; }
        }
    }
    if (code) atomicMin(err, (unsigned long long)r * 8ull + (unsigned long long)code);
}

// ---- dependents and intervals ------------------------------------------------

// setDependents_PSTRSV3 (ops.c:129-182) and the coupling half of getIntervalEnd
// (ops.c:184-212): dependents[col] = 1 for columns >= pe of blocks 0..P-2,
// hasDependences, and the last row holding a coupling nonzero per block.
__global__ void k_dependents(int n, int P, const int *__restrict__ ps, const int *__restrict__ pe,
                             const int *__restrict__ ia, const int *__restrict__ ja,
                             int *__restrict__ dep, int *__restrict__ maxIR,
                             int *__restrict__ hasDep) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    int t = part_of(ps, P, r);
    if (t >= P - 1) return;
    int end = pe[t];
    int b = ia[r], e = ia[r + 1];
    int q0 = lower_bound_i(ja, b, e, end);
    if (q0 >= e) return;
    atomicMax(&maxIR[t], r);
    hasDep[t] = 1;
    for (int q = q0; q < e; q++) dep[ja[q]] = 1;
}

// First dependent row per block (the minDependentRow scan, ops.c:256-264).
__global__ void k_min_dependent(int n, int P, const int *__restrict__ ps,
                                const int *__restrict__ dep, int *__restrict__ minDR) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n || !dep[r]) return;
    atomicMin(&minDR[part_of(ps, P, r)], r);
}

// Coupling nonzeros of rows [minDependentRow, pe) of reflected blocks; their
// distinct columns per block are numCols_S (ops.c:272-285) and, sorted, mapR
// (ops.c:923-943).  Pass 1 counts per row, pass 2 writes (block, column) keys.
__global__ void k_coupling_keys(int n, int P, const int *__restrict__ ps, const int *__restrict__ pe,
                                const int *__restrict__ minDR, const char *__restrict__ refl,
                                const int *__restrict__ ia, const int *__restrict__ ja,
                                int *__restrict__ cnt, const int *__restrict__ off,
                                unsigned long long *__restrict__ keys) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    int t = part_of(ps, P, r);
    int c = 0, q0 = 0, e = 0;
    if (t >= 1 && t < P - 1 && refl[t] && r >= minDR[t]) {
        int b = ia[r];
        e = ia[r + 1];
        q0 = lower_bound_i(ja, b, e, pe[t]);
        c = e - q0;
    }
    if (!keys) {
        cnt[r] = c;
        return;
    }
    unsigned long long hi = (unsigned long long)t << 32;
    int w = off[r];
    for (int q = q0; q < q0 + c; q++) keys[w++] = hi | (unsigned int)ja[q];
}

__global__ void k_count_cols(int nk, const unsigned long long *__restrict__ keys,
                             int *__restrict__ colCount, int *__restrict__ mapR) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nk) return;
    unsigned long long k = keys[i];
    atomicAdd(&colCount[(int)(k >> 32)], 1);
    mapR[i] = (int)(k & 0xffffffffull);
}

// optimizeLoadBalance counters (ops.c:389-505) per block:
//  [0..3] current-cost classification with the block's intervals: R, D1, D2, P
//  [4]    columns strictly beyond the block end (ops.c:441-446)
//  [5..8] probable-cost classification with eI = start+ei, sI = eI-1: R, D1, D2, P
//  [9]    all entries of the block's rows (ia[end] - ia[start])
constexpr int kLB = 10;
__global__ void k_lb_counts(int n, int P, const int *__restrict__ ps, const int *__restrict__ pe,
                            const int *__restrict__ si, const int *__restrict__ ei,
                            const int *__restrict__ ia, const int *__restrict__ ja,
                            int *__restrict__ out) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    int t = part_of(ps, P, r);
    int start = ps[t], end = pe[t];
    int sI = start + si[t], eI = start + ei[t];
    int eI2 = start + ei[t], sI2 = eI2 - 1;
    int c[kLB] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    c[9] = ia[r + 1] - ia[r];
    for (int q = ia[r]; q < ia[r + 1]; q++) {
        int col = ja[q];
        if (end <= col) c[0]++;
        else if (sI > r) { if (eI > col) c[2]++; else c[3]++; }
        else if (eI > r) { if (eI > col) c[2]++; else c[3]++; c[1]++; }
        else c[1]++;
        if (end < col) c[4]++;
        if (end <= col) c[5]++;
        else if (sI2 > r) { if (eI2 > col) c[7]++; else c[8]++; }
        else if (eI2 > r) { if (eI2 > col) c[7]++; else c[8]++; c[6]++; }
        else c[6]++;
    }
    for (int k = 0; k < kLB; k++)
        if (c[k]) atomicAdd(&out[t * kLB + k], c[k]);
}

// ---- D and R_new pools (matrix_partitioning.c:38-76, ops.c:772-827) --------------

__global__ void k_dr_counts(int n, int P, const PartDev *__restrict__ pd, const int *__restrict__ ps,
                            const int *__restrict__ ia, const int *__restrict__ ja,
                            int *__restrict__ nD, int *__restrict__ nR, int *__restrict__ hasDep) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) {
        if (r == n) { nD[n] = 0; nR[n] = 0; }
        return;
    }
    int t = part_of(ps, P, r);
    PartDev p = pd[t];
    int b = ia[r], e = ia[r + 1];
    int dlo = lower_bound_i(ja, b, e, p.ps);
    int dhi = lower_bound_i(ja, dlo, e, p.pe);
    int border = p.ps + p.ei;
    int thr = ((p.flags & 1) && r < border) ? border : p.pe;
    int rlo = lower_bound_i(ja, b, e, thr);
    nD[r] = dhi - dlo;
    nR[r] = e - rlo;
    if (e > rlo) hasDep[t] = 1;
}

__global__ void k_dr_scatter(int n, int P, const PartDev *__restrict__ pd, const int *__restrict__ ps,
                             const int *__restrict__ ia, const int *__restrict__ ja,
                             const double *__restrict__ a, const int *__restrict__ ID,
                             double *__restrict__ D, int *__restrict__ JD) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    int t = part_of(ps, P, r);
    PartDev p = pd[t];
    int b = ia[r], e = ia[r + 1];
    int dlo = lower_bound_i(ja, b, e, p.ps);
    int dhi = lower_bound_i(ja, dlo, e, p.pe);
    int w = ID[r];
    for (int q = dlo; q < dhi; q++, w++) {
        D[w] = a[q];
        JD[w] = ja[q] - p.ps;
    }
    int border = p.ps + p.ei;
    int thr = ((p.flags & 1) && r < border) ? border : p.pe;
    w = ID[n + r];
    for (int q = lower_bound_i(ja, b, e, thr); q < e; q++, w++) {
        D[w] = a[q];
        JD[w] = ja[q];
    }
}

__global__ void k_add_offset(int count, const int *__restrict__ in, int v, int *__restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = in[i] + v;
}

// ---- D0 | D1 | D2 pool (ops.c:300-323, 567-770) -------------------------------

__device__ __forceinline__ int seg_of(const Seg *__restrict__ segs, int nseg, int w) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (segs[mid].out0 <= w) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void k_t2_counts(int R, const Seg *__restrict__ segs, int nseg, const int *__restrict__ ID,
                            const int *__restrict__ JD, int *__restrict__ cnt) {
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= R) {
        if (w == R) cnt[R] = 0;
        return;
    }
    Seg s = segs[seg_of(segs, nseg, w)];
    if (s.artifact) { cnt[w] = 0; return; }
    int r = s.glo + (w - s.out0);
    int b = ID[r], e = ID[r + 1];
    int lo = lower_bound_i(JD, b, e, s.clo);
    int hi = lower_bound_i(JD, lo, e, s.chi);
    cnt[w] = hi - lo;
}

__global__ void k_t2_scatter(int R, const Seg *__restrict__ segs, int nseg, const int *__restrict__ ID,
                             const int *__restrict__ JD, const double *__restrict__ D,
                             const int *__restrict__ IT2, double *__restrict__ T2,
                             int *__restrict__ JT2) {
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= R) return;
    Seg s = segs[seg_of(segs, nseg, w)];
    if (s.artifact) return;
    int r = s.glo + (w - s.out0);
    int b = ID[r], e = ID[r + 1];
    int lo = lower_bound_i(JD, b, e, s.clo);
    int hi = lower_bound_i(JD, lo, e, s.chi);
    int o = IT2[w];
    for (int q = lo; q < hi; q++, o++) {
        T2[o] = D[q];
        JT2[o] = JD[q] - s.shift;
    }
}

// ---- compressed R and spikes (ops.c:888-959, 1021-1069) ------------------------

__global__ void k_scatter_rdense(int n, int P, const PartDev *__restrict__ pd, const int *__restrict__ ps,
                                 const int *__restrict__ ID, const int *__restrict__ JD,
                                 const double *__restrict__ D, const int *__restrict__ mapR,
                                 double *__restrict__ S) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    int t = part_of(ps, P, r);
    PartDev p = pd[t];
    if (!(p.flags & 4) || r < p.ps + p.si || r >= p.ps + p.ei) return;
    long long row = r - (p.ps + p.si);
    double *Srow = S + p.startsS + row * p.nColsS;
    const int *map = mapR + p.sMapR;
    for (int q = ID[n + r]; q < ID[n + r + 1]; q++) {
        int c = JD[q];
        if (p.ps <= c && c < p.pe) continue;
        Srow[lower_bound_i(map, 0, p.nColsS, c)] = D[q];
    }
}

// __udsol2 (ops.c:1196-1228): S = D0^{-1} R in place, one thread per spike
// column, rows bottom-up.  Each element takes the products in CSR order and one
// division, with explicit round-to-nearest operations so that no multiply-add
// is contracted: the result is bitwise identical to the reference.
__global__ void k_spike_sweep(const int *__restrict__ plist, const PartDev *__restrict__ pd,
                              const int *__restrict__ sD0, const int *__restrict__ IT2,
                              const int *__restrict__ JT2, const double *__restrict__ T2,
                              double *__restrict__ S) {
    int t = plist[blockIdx.x];
    PartDev p = pd[t];
    const int rc = p.nRowsS, cc = p.nColsS;
    const int *IA = IT2 + sD0[t];
    double *X = S + p.startsS;
    for (int l = threadIdx.x; l < cc; l += blockDim.x) {
        long long o = (long long)(rc - 1) * cc + l;
        X[o] = __ddiv_rn(X[o], T2[IA[rc - 1]]);
        for (int k = rc - 2; k >= 0; k--) {
            long long ok = (long long)k * cc + l;
            double x = X[ok];
            int j0 = IA[k], j1 = IA[k + 1];
            for (int j = j0 + 1; j < j1; j++) {
                double pr = __dmul_rn(T2[j], X[(long long)JT2[j] * cc + l]);
                x = __dsub_rn(x, pr);
            }
            X[ok] = __ddiv_rn(x, T2[j0]);
        }
    }
}

// ---- reduced system (ops.c:1071-1150) -----------------------------------------

__global__ void k_flags(int n, const int *__restrict__ dep, int *__restrict__ f) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) f[i] = dep[i] ? 1 : 0;
    else if (i == n) f[n] = 0;
}

__global__ void k_reduced_ids(int n, const int *__restrict__ redIdx, int *__restrict__ dep,
                              int *__restrict__ mapRedX) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !dep[i]) return;
    int k = redIdx[i];
    mapRedX[k] = i;
    dep[i] = k + 1;
}

__global__ void k_reduced_rows(int rss, int P, const int *__restrict__ ps, const PartDev *__restrict__ pd,
                               const int *__restrict__ mapRedX, const double *__restrict__ S,
                               const int *__restrict__ mapR, const int *__restrict__ dep,
                               int *__restrict__ cnt, const int *__restrict__ IT,
                               double *__restrict__ T, int *__restrict__ JT) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= rss) {
        if (!T && k == rss) cnt[rss] = 0;
        return;
    }
    int i = mapRedX[k];
    int t = part_of(ps, P, i);
    PartDev p = pd[t];
    int rowS = i - p.minDR;
    int c = 0;
    if ((p.flags & 2) && (p.flags & 4) && rowS < p.nRowsS) {
        const double *Srow = S + p.startsS + (long long)rowS * p.nColsS;
        int w = T ? IT[k] : 0;
        for (int j = 0; j < p.nColsS; j++) {
            double v = Srow[j];
            if (v != 0) {
                if (T) {
                    T[w] = v;
                    JT[w] = dep[mapR[p.sMapR + j]] - 1;
                    w++;
                }
                c++;
            }
        }
    }
    if (!T) cnt[k] = c;
}

__global__ void k_level_offsets(int P, const int *__restrict__ ps, const int *__restrict__ redIdx,
                                int n, int *__restrict__ lvl) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < P) lvl[t] = redIdx[ps[t]];
    else if (t == P) lvl[P] = redIdx[n];
}

// ---- host helpers -------------------------------------------------------------

inline int blocks_for(long long n, int bs = 256) { return (int)((n + bs - 1) / bs); }

int exclusive_scan(const int *in, int *out, int count, cudaStream_t st) {
    size_t tmp = 0;
    SPK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, count, st));
    DBuf<unsigned char> t(st);
    SPK_TRY(t.alloc(tmp));
    SPK_CUDA(cub::DeviceScan::ExclusiveSum(t.p, tmp, in, out, count, st));
    return SPK_OK;
}

template <typename T>
int to_host(std::vector<T> &h, const T *d, size_t count, cudaStream_t st) {
    h.resize(count);
    if (count) SPK_CUDA(cudaMemcpyAsync(h.data(), d, count * sizeof(T), cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaStreamSynchronize(st));
    return SPK_OK;
}

template <typename T>
int to_device(DBuf<T> &d, const std::vector<T> &h, cudaStream_t st) {
    SPK_TRY(d.alloc(h.size()));
    if (!h.empty())
        SPK_CUDA(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    return SPK_OK;
}

struct PhaseClock {
    double *acc;
    cudaStream_t st;
    double t0;
    PhaseClock(double *a, cudaStream_t s) : acc(a), st(s), t0(0) {
        if (acc) { cudaStreamSynchronize(st); t0 = now_s(); }
    }
    void lap(int slot) {
        if (!acc) return;
        cudaStreamSynchronize(st);
        double t1 = now_s();
        acc[slot] += t1 - t0;
        t0 = t1;
    }
};

// optimizeLoadBalance decision (ops.c:375-565) on per-block counters, with the
// reference's uninitialised reads fixed to the values its binary produces:
// totalLoss 0 when the cut search does not run, an unassigned bestCut -1, the
// INF sum wrapping modulo 2^32.  A split that would start D1 before row 0 (block
// 0 with bestCut -1, where the reference reads ID[-1]) reverts the decision.
void load_balance(std::vector<Part> &parts, const std::vector<int> &cnt,
                  const std::vector<int> &row0_cols) {
    const int P = (int)parts.size();
    auto imax = [](int a, int b) { return a > b ? a : b; };
    int cost1 = 0, cost2 = 0, curCost1 = 0, curCost2 = 0, newCost1 = 0, newCost2 = 0;
    int nnz_P = 0, minLoss = kInf;
    unsigned int totalLoss = 0;
    for (int i = 0; i < P; i++) {
        const int *c = &cnt[i * kLB];
        if (parts[i].hasRefl) {
            nnz_P = c[3];
            cost1 = imax(cost1, c[1]);
            cost2 = imax(cost2, c[0] + c[3] + c[2]);
        } else {
            curCost2 = imax(curCost2, c[4] + c[9]);
            parts[i].isOpt = c[4] == 0 ? 2 : 0;
        }
    }
    curCost1 = cost1;
    curCost2 = imax(curCost2, cost2);
    for (int i = 0; i < P; i++) {
        if (!parts[i].hasRefl && parts[i].isOpt != 2) {
            const int *c = &cnt[i * kLB];
            nnz_P += c[8];
            newCost1 = imax(newCost1, c[6]);
            newCost2 = imax(newCost2, c[5] + nnz_P + c[7]);
            parts[i].isOpt = 1;
        }
    }
    newCost2 = imax(newCost2, cost2);
    int loss = imax(0, newCost1 - curCost1);
    int gain = imax(0, curCost2 - newCost2);
    if (gain > loss) {
        for (int i = 0; i < P; i++) {
            if (parts[i].isOpt != 2) continue;
            int start = parts[i].ps, end = parts[i].pe;
            int bestCut = -1;
            // The reference's cut loop starts its row counter at 0, so it can only
            // meet a row boundary (ia[1]) when the block starts at row 0 or 1, and
            // it breaks at that first boundary (ops.c:528-549).
            if (start <= 1 && end >= 2) {
                int nnz_D = cnt[i * kLB + 9];
                int d2 = 0, pp = 0;
                if (start == 0)
                    for (int c : row0_cols) { if (c <= 0) d2++; else pp++; }
                int nnz_D1 = nnz_D - (d2 + pp);
                int c1 = imax(0, nnz_D1 - newCost1);
                int c2 = imax(0, d2 + pp - newCost2);
                int l = c1 + c2;
                if (l <= minLoss) minLoss = l; else bestCut = -1;  // row - 1 with row = 0
            }
            parts[i].si = bestCut;
            parts[i].ei = bestCut + 1;
            totalLoss += (unsigned int)minLoss;
        }
    }
    bool revert = (int)totalLoss > 0;
    for (int i = 0; i < P && !revert; i++)
        if (parts[i].isOpt && parts[i].ps + parts[i].si < 0) revert = true;
    if (revert)
        for (auto &p : parts) p.isOpt = 0;
}

}  // namespace

int preprocess(spk_system *s, const double *a, const int *ia, const int *ja, int n, int P,
               char uplo, int flb, const int *starts, const int *ends, int on_dev,
               double *ph) {
    cudaStream_t st = s->stream;
    if (n <= 0 || P <= 0) {
        set_error(SPK_ERR_ARG, "invalid size: n=%d nthreads=%d", n, P);
        return SPK_ERR_ARG;
    }
    if (P > n) {
        set_error(SPK_ERR_ARG, "nthreads=%d exceeds the %d rows (empty partitions)", P, n);
        return SPK_ERR_ARG;
    }
    char up = (uplo == 'l' || uplo == 'L') ? 'L' : ((uplo == 'u' || uplo == 'U') ? 'U' : 0);
    if (!up) {
        set_error(SPK_ERR_ARG, "uplo must be 'U' or 'L' (got '%c')", uplo);
        return SPK_ERR_ARG;
    }
    s->built = 0;
    s->lean = 0;
    // values derived from the previous matrix for the batched solves
    s->ell_valf.release();
    s->rdiagf.release();
    s->diag.release();
    s->anorm = 0.0;
    s->ell_reach = -1;
    PhaseClock clk(ph, st);
    const double prep_t0 = now_s();

    // ---- input: upload (host pointers) and mirror ('L')
    int nnz = 0;
    if (on_dev) SPK_CUDA(cudaMemcpy(&nnz, ia + n, sizeof(int), cudaMemcpyDeviceToHost));
    else nnz = ia[n];
    int ia0 = 0;
    if (on_dev) SPK_CUDA(cudaMemcpy(&ia0, ia, sizeof(int), cudaMemcpyDeviceToHost));
    else ia0 = ia[0];
    if (nnz <= 0 || ia0 != 0) {
        set_error(SPK_ERR_INPUT, "ia must start at 0 and end at nnz > 0 (ia[0]=%d, ia[n]=%d)", ia0, nnz);
        return SPK_ERR_INPUT;
    }
    s->n = n; s->nnz = nnz; s->P = P; s->uplo = up; s->flb = flb;
    // padded: the solver stages CSR slices in 16-byte granules that may extend
    // up to 3 elements past the last nonzero
    SPK_TRY(s->ua.alloc(nnz + 16));
    SPK_TRY(s->uia.alloc(n + 16));
    SPK_TRY(s->uja.alloc(nnz + 16));
    SPK_CUDA(cudaMemsetAsync(s->ua.p + nnz, 0, 16 * sizeof(double), st));
    SPK_CUDA(cudaMemsetAsync(s->uja.p + nnz, 0, 16 * sizeof(int), st));
    {
        DBuf<double> la(st); DBuf<int> lia(st), lja(st);
        const double *src_a = a; const int *src_ia = ia, *src_ja = ja;
        if (!on_dev) {
            if (up == 'L') {
                SPK_TRY(la.alloc(nnz));
                SPK_TRY(lia.alloc(n + 1));
                SPK_TRY(lja.alloc(nnz));
            }
            double *dst_a = (up == 'U') ? s->ua.p : la.p;
            int *dst_ia = (up == 'U') ? s->uia.p : lia.p;
            int *dst_ja = (up == 'U') ? s->uja.p : lja.p;
            SPK_CUDA(cudaMemcpyAsync(dst_a, a, sizeof(double) * nnz, cudaMemcpyHostToDevice, st));
            SPK_CUDA(cudaMemcpyAsync(dst_ia, ia, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st));
            SPK_CUDA(cudaMemcpyAsync(dst_ja, ja, sizeof(int) * nnz, cudaMemcpyHostToDevice, st));
            src_a = dst_a; src_ia = dst_ia; src_ja = dst_ja;
        } else if (up == 'U') {
            SPK_CUDA(cudaMemcpyAsync(s->ua.p, a, sizeof(double) * nnz, cudaMemcpyDeviceToDevice, st));
            SPK_CUDA(cudaMemcpyAsync(s->uia.p, ia, sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice, st));
            SPK_CUDA(cudaMemcpyAsync(s->uja.p, ja, sizeof(int) * nnz, cudaMemcpyDeviceToDevice, st));
        }
        if (up == 'L') {
            k_mirror<<<std::min(blocks_for(nnz), 148 * 16), 256, 0, st>>>(n, nnz, src_ia, src_ja, src_a,
                                                                          s->uia.p, s->uja.p, s->ua.p);
            SPK_CUDA(cudaGetLastError());
        }
        SPK_CUDA(cudaStreamSynchronize(st));
    }
    const int *uia = s->uia.p, *uja = s->uja.p;
    const double *ua = s->ua.p;
    {
        DBuf<unsigned long long> err(st);
        SPK_TRY(err.alloc(1));
        SPK_CUDA(cudaMemsetAsync(err.p, 0xff, sizeof(unsigned long long), st));
        k_validate<<<blocks_for(n), 256, 0, st>>>(n, uia, uja, err.p);
        SPK_CUDA(cudaGetLastError());
        unsigned long long e = 0;
        SPK_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(e), cudaMemcpyDeviceToHost, st));
        SPK_CUDA(cudaStreamSynchronize(st));
        if (e != ~0ull) {
            long long row = (long long)(e >> 3);
            int code = (int)(e & 7);
            if (up == 'L') row = n - 1 - row;
            static const char *what[] = {"", "empty row", "diagonal not in place",
                                         "columns unsorted, repeated or out of range"};
            set_error(SPK_ERR_INPUT, "malformed CSR at row %lld: %s", row, what[code]);
            return SPK_ERR_INPUT;
        }
    }

    // ---- matrixPartitioning (matrix_partitioning.c:18-36)
    std::vector<Part> &parts = s->parts;
    parts.assign(P, Part{});
    if (starts && ends) {
        // caller bounds are in the caller's row order: 'L' partition t, rows
        // [starts[t], ends[t]) of L, is partition P-1-t of the mirror J L J
        const bool lower = uplo == 'L' || uplo == 'l';
        for (int t = 0; t < P; t++) {
            const int c = lower ? P - 1 - t : t;
            parts[t].ps = lower ? n - ends[c] : starts[c];
            parts[t].pe = lower ? n - starts[c] : ends[c];
        }
        for (int t = 0; t < P; t++) {
            bool ok = parts[t].pe > parts[t].ps && (t == 0 ? parts[t].ps == 0 : parts[t].ps == parts[t - 1].pe);
            if (!ok || (t == P - 1 && parts[t].pe != n)) {
                set_error(SPK_ERR_ARG, "caller partitions must be nonempty, contiguous and cover [0, n)");
                return SPK_ERR_ARG;
            }
        }
    } else {
        int k = n / P, left = n % P;
        for (int t = 0; t < P; t++) {
            parts[t].ps = k * t;
            parts[t].pe = k * t + k;
        }
        parts[P - 1].pe += left;
    }
    std::vector<int> hps(P), hpe(P);
    for (int t = 0; t < P; t++) {
        Part &p = parts[t];
        p.num = p.pe - p.ps;
        p.startsD = p.ps; p.endsD = p.pe;
        p.startsR = n + p.ps; p.endsR = n + p.pe;
        hps[t] = p.ps; hpe[t] = p.pe;
    }
    SPK_TRY(to_device(s->d_ps, hps, st));
    SPK_TRY(to_device(s->d_pe, hpe, st));
    const int *dps = s->d_ps.p, *dpe = s->d_pe.p;

    // ---- dependents, interval ends, first dependent rows
    SPK_TRY(s->dep.alloc(n));
    SPK_CUDA(cudaMemsetAsync(s->dep.p, 0, sizeof(int) * n, st));
    DBuf<int> d_maxIR(st), d_minDR(st), d_hasDep(st);
    {
        std::vector<int> init_max(P), init_min(P);
        for (int t = 0; t < P; t++) { init_max[t] = hps[t] - 1; init_min[t] = hpe[t]; }
        SPK_TRY(to_device(d_maxIR, init_max, st));
        SPK_TRY(to_device(d_minDR, init_min, st));
        SPK_TRY(d_hasDep.alloc(P));
        SPK_CUDA(cudaMemsetAsync(d_hasDep.p, 0, sizeof(int) * P, st));
    }
    clk.lap(0);  // preprocessD (partitioning + upload)
    k_dependents<<<blocks_for(n), 256, 0, st>>>(n, P, dps, dpe, uia, uja, s->dep.p, d_maxIR.p, d_hasDep.p);
    k_min_dependent<<<blocks_for(n), 256, 0, st>>>(n, P, dps, s->dep.p, d_minDR.p);
    SPK_CUDA(cudaGetLastError());
    std::vector<int> hmax, hmin, hdep;
    SPK_TRY(to_host(hmax, d_maxIR.p, P, st));
    SPK_TRY(to_host(hmin, d_minDR.p, P, st));
    SPK_TRY(to_host(hdep, d_hasDep.p, P, st));
    s->redNec = 0;
    for (int t = 0; t < P; t++) {
        parts[t].hasDep = (char)hdep[t];
        parts[t].maxIR = hmax[t];
        parts[t].minDR = hmin[t];
        if (hdep[t]) s->redNec = 1;
    }
    clk.lap(1);  // setDependents

    // ---- preprocessS_PSTRSV3 (ops.c:214-373)
    s->totalArea = 0;
    int nk = 0;
    DBuf<int> d_mapR_all(st);
    std::vector<int> colCount(P, 0);
    if (s->redNec) {
        std::vector<char> refl(P, 0);
        for (int t = 1; t < P; t++)
            if (parts[t].minDR < parts[t].pe) refl[t] = 1;
        DBuf<char> d_refl(st);
        SPK_TRY(to_device(d_refl, refl, st));
        DBuf<int> cnt(st), off(st);
        SPK_TRY(cnt.alloc(n + 1));
        SPK_TRY(off.alloc(n + 1));
        SPK_CUDA(cudaMemsetAsync(cnt.p + n, 0, sizeof(int), st));
        k_coupling_keys<<<blocks_for(n), 256, 0, st>>>(n, P, dps, dpe, d_minDR.p, d_refl.p, uia, uja,
                                                       cnt.p, nullptr, nullptr);
        SPK_CUDA(cudaGetLastError());
        SPK_TRY(exclusive_scan(cnt.p, off.p, n + 1, st));
        int nkeys = 0;
        SPK_CUDA(cudaMemcpyAsync(&nkeys, off.p + n, sizeof(int), cudaMemcpyDeviceToHost, st));
        SPK_CUDA(cudaStreamSynchronize(st));
        DBuf<unsigned long long> keys(st), sorted(st), uniq(st);
        DBuf<int> nuniq(st);
        SPK_TRY(keys.alloc(nkeys));
        SPK_TRY(sorted.alloc(nkeys));
        SPK_TRY(uniq.alloc(nkeys));
        SPK_TRY(nuniq.alloc(1));
        if (nkeys) {
            k_coupling_keys<<<blocks_for(n), 256, 0, st>>>(n, P, dps, dpe, d_minDR.p, d_refl.p, uia, uja,
                                                           cnt.p, off.p, keys.p);
            SPK_CUDA(cudaGetLastError());
            int tbits = 1;
            while ((1 << tbits) < P) tbits++;
            size_t tmp = 0;
            SPK_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp, keys.p, sorted.p, nkeys, 0, 32 + tbits, st));
            DBuf<unsigned char> tb(st);
            SPK_TRY(tb.alloc(tmp));
            SPK_CUDA(cub::DeviceRadixSort::SortKeys(tb.p, tmp, keys.p, sorted.p, nkeys, 0, 32 + tbits, st));
            size_t tmp2 = 0;
            SPK_CUDA(cub::DeviceSelect::Unique(nullptr, tmp2, sorted.p, uniq.p, nuniq.p, nkeys, st));
            DBuf<unsigned char> tb2(st);
            SPK_TRY(tb2.alloc(tmp2));
            SPK_CUDA(cub::DeviceSelect::Unique(tb2.p, tmp2, sorted.p, uniq.p, nuniq.p, nkeys, st));
            SPK_CUDA(cudaMemcpyAsync(&nk, nuniq.p, sizeof(int), cudaMemcpyDeviceToHost, st));
            SPK_CUDA(cudaStreamSynchronize(st));
        }
        DBuf<int> d_cc(st);
        SPK_TRY(d_cc.alloc(P));
        SPK_CUDA(cudaMemsetAsync(d_cc.p, 0, sizeof(int) * P, st));
        SPK_TRY(d_mapR_all.alloc(nk));
        if (nk) {
            k_count_cols<<<blocks_for(nk), 256, 0, st>>>(nk, uniq.p, d_cc.p, d_mapR_all.p);
            SPK_CUDA(cudaGetLastError());
        }
        SPK_TRY(to_host(colCount, d_cc.p, P, st));

        long long endsPrev = 0;
        for (int t = 0; t < P; t++) {
            Part &p = parts[t];
            if (t == 0) {
                p.ei = p.maxIR - p.ps + 1;
                p.si = p.ei;
                p.startsS = p.endsS = 0;
                endsPrev = 0;
                continue;
            }
            long long cc = 0, rc = 0;
            if (refl[t]) {
                p.hasRefl = 1;
                cc = colCount[t];
                if (cc > 0) p.hasS = 1;
                p.nColsS = (int)cc;
                p.nRowsS = std::max(1 + p.maxIR - p.minDR, 0);
                rc = p.nRowsS;
                p.si = p.minDR - p.ps;
                p.ei = (p.maxIR < p.minDR) ? p.si + 1 : p.maxIR - p.ps + 1;
            } else {
                p.ei = p.maxIR - p.ps + 1;
                p.si = p.ei;
            }
            p.startsS = endsPrev;
            p.endsS = p.startsS + (long long)(int)(cc * rc);
            endsPrev = p.endsS;
            s->totalArea += cc * rc;
        }
        s->totalArea += 40 - (s->totalArea % 40);

        if (flb) {
            std::vector<int> hsi(P), hei(P);
            for (int t = 0; t < P; t++) { hsi[t] = parts[t].si; hei[t] = parts[t].ei; }
            DBuf<int> d_si(st), d_ei(st), d_cnt9(st);
            SPK_TRY(to_device(d_si, hsi, st));
            SPK_TRY(to_device(d_ei, hei, st));
            SPK_TRY(d_cnt9.alloc((size_t)P * kLB));
            SPK_CUDA(cudaMemsetAsync(d_cnt9.p, 0, sizeof(int) * P * kLB, st));
            k_lb_counts<<<blocks_for(n), 256, 0, st>>>(n, P, dps, dpe, d_si.p, d_ei.p, uia, uja, d_cnt9.p);
            SPK_CUDA(cudaGetLastError());
            std::vector<int> c9;
            SPK_TRY(to_host(c9, d_cnt9.p, (size_t)P * kLB, st));
            int ia01[2] = {0, 0};
            SPK_CUDA(cudaMemcpy(ia01, uia, 2 * sizeof(int), cudaMemcpyDeviceToHost));
            std::vector<int> row0(ia01[1] - ia01[0]);
            if (!row0.empty())
                SPK_CUDA(cudaMemcpy(row0.data(), uja, row0.size() * sizeof(int), cudaMemcpyDeviceToHost));
            load_balance(parts, c9, row0);
        }
        if (s->totalArea * (long long)sizeof(double) * 3 > kMemSize) {
            set_error(SPK_ERR_TOO_LARGE,
                      "Error: The estimated size of Matrix S is beyond boundaries! (%lld spike entries)",
                      s->totalArea);
            return SPK_ERR_TOO_LARGE;
        }
    }
    clk.lap(2);  // preprocessS (intervals, spike sizes, load balance)

    // ---- per-partition device metadata
    std::vector<PartDev> hpd(P);
    {
        int sm = 0;
        for (int t = 0; t < P; t++) {
            Part &p = parts[t];
            p.sMapR = sm;
            sm += p.nColsS;
            p.eMapR = sm;
        }
        s->nMapR = sm;
    }
    for (int t = 0; t < P; t++) {
        const Part &p = parts[t];
        PartDev &d = hpd[t];
        d.ps = p.ps; d.pe = p.pe; d.si = p.si; d.ei = p.ei;
        d.minDR = p.minDR; d.nRowsS = p.nRowsS; d.nColsS = p.nColsS; d.sMapR = p.sMapR;
        d.startsS = p.startsS;
        d.flags = ((p.hasRefl || p.isOpt) ? 1 : 0) | (p.hasRefl ? 2 : 0) | (p.hasS ? 4 : 0);
        d.pad = 0;
    }
    DBuf<PartDev> d_pd(st);
    SPK_TRY(to_device(d_pd, hpd, st));

    // ---- D and R_new pools
    {
        DBuf<int> nD(st), nR(st), oR(st);
        SPK_TRY(nD.alloc(n + 1));
        SPK_TRY(nR.alloc(n + 1));
        SPK_TRY(oR.alloc(n + 1));
        SPK_TRY(s->ID.alloc(2 * (size_t)n + 1));
        SPK_CUDA(cudaMemsetAsync(d_hasDep.p, 0, sizeof(int) * P, st));
        k_dr_counts<<<blocks_for(n + 1), 256, 0, st>>>(n, P, d_pd.p, dps, uia, uja, nD.p, nR.p, d_hasDep.p);
        SPK_CUDA(cudaGetLastError());
        SPK_TRY(exclusive_scan(nD.p, s->ID.p, n + 1, st));
        SPK_TRY(exclusive_scan(nR.p, oR.p, n + 1, st));
        int nDtot = 0, nRtot = 0;
        SPK_CUDA(cudaMemcpyAsync(&nDtot, s->ID.p + n, sizeof(int), cudaMemcpyDeviceToHost, st));
        SPK_CUDA(cudaMemcpyAsync(&nRtot, oR.p + n, sizeof(int), cudaMemcpyDeviceToHost, st));
        SPK_CUDA(cudaStreamSynchronize(st));
        s->nDpool = (long long)nDtot + nRtot;
        SPK_TRY(s->D.alloc(s->nDpool));
        SPK_TRY(s->JD.alloc(s->nDpool));
        k_add_offset<<<blocks_for(n + 1), 256, 0, st>>>(n + 1, oR.p, nDtot, s->ID.p + n);  // ID[n+r]
        k_dr_scatter<<<blocks_for(n), 256, 0, st>>>(n, P, d_pd.p, dps, uia, uja, ua, s->ID.p, s->D.p, s->JD.p);
        SPK_CUDA(cudaGetLastError());
        std::vector<int> hd2;
        SPK_TRY(to_host(hd2, d_hasDep.p, P, st));
        for (int t = 0; t < P; t++)
            if (hd2[t]) parts[t].hasDep = 1;
    }

    // ---- D0 | D1 | D2 pool
    {
        std::vector<Seg> segs;
        int row = 0;
        const int NEG = -2147483647 - 1, POS = 2147483647;
        if (s->redNec) {
            for (int t = 1; t < P; t++) {
                Part &p = parts[t];
                if (!p.hasRefl) continue;
                p.sD0 = row;
                int nr = p.ei - p.si;
                segs.push_back(Seg{row, nr, p.ps + p.si, p.si, p.ei, p.si, 0});
                row += nr;
                p.eD0 = row;
            }
            for (int t = 0; t < P; t++) {
                Part &p = parts[t];
                if (p.hasRefl || p.isOpt) {
                    p.sD1 = row;
                    int lo = p.ps + p.si, hi = p.pe;
                    if (lo < hi) { segs.push_back(Seg{row, hi - lo, lo, NEG, POS, p.si, 0}); row += hi - lo; }
                    else { segs.push_back(Seg{row, 1, 0, 0, 0, 0, 1}); row += 1; }
                    p.eD1 = row;
                }
            }
            for (int t = 0; t < P; t++) {
                Part &p = parts[t];
                if (p.hasRefl || p.isOpt) {
                    p.sD2 = row;
                    if (p.ei > 0) { segs.push_back(Seg{row, p.ei, p.ps, NEG, p.ei, 0, 0}); row += p.ei; }
                    else { segs.push_back(Seg{row, 1, 0, 0, 0, 0, 1}); row += 1; }
                    p.eD2 = row;
                }
            }
        }
        s->nIT2rows = row;
        SPK_TRY(s->IT2.alloc(row + 1));
        if (row == 0) {
            SPK_CUDA(cudaMemsetAsync(s->IT2.p, 0, sizeof(int), st));
            s->nT2 = 0;
            SPK_TRY(s->T2.alloc(1));
            SPK_TRY(s->JT2.alloc(1));
        } else {
            DBuf<Seg> d_segs(st);
            SPK_TRY(to_device(d_segs, segs, st));
            DBuf<int> cnt(st);
            SPK_TRY(cnt.alloc(row + 1));
            k_t2_counts<<<blocks_for(row + 1), 256, 0, st>>>(row, d_segs.p, (int)segs.size(), s->ID.p, s->JD.p, cnt.p);
            SPK_CUDA(cudaGetLastError());
            SPK_TRY(exclusive_scan(cnt.p, s->IT2.p, row + 1, st));
            int tot = 0;
            SPK_CUDA(cudaMemcpyAsync(&tot, s->IT2.p + row, sizeof(int), cudaMemcpyDeviceToHost, st));
            SPK_CUDA(cudaStreamSynchronize(st));
            s->nT2 = tot;
            SPK_TRY(s->T2.alloc(tot));
            SPK_TRY(s->JT2.alloc(tot));
            k_t2_scatter<<<blocks_for(row), 256, 0, st>>>(row, d_segs.p, (int)segs.size(), s->ID.p, s->JD.p,
                                                          s->D.p, s->IT2.p, s->T2.p, s->JT2.p);
            SPK_CUDA(cudaGetLastError());
        }
    }
    clk.lap(3);  // preprocessR (D, R_new, D0/D1/D2 extraction)

    // ---- mapR (preprocessMappings_PSTRSV3, ops.c:860-886)
    SPK_TRY(s->mapR.alloc(s->nMapR));
    if (s->nMapR) {
        if (s->nMapR != nk) {
            set_error(SPK_ERR_STATE, "internal: mapR size %d != distinct coupling columns %d", s->nMapR, nk);
            return SPK_ERR_STATE;
        }
        SPK_CUDA(cudaMemcpyAsync(s->mapR.p, d_mapR_all.p, sizeof(int) * nk, cudaMemcpyDeviceToDevice, st));
    }
    clk.lap(4);

    // ---- dense R -> S
    SPK_TRY(s->S.alloc(std::max<long long>(s->totalArea, 1)));
    SPK_CUDA(cudaMemsetAsync(s->S.p, 0, sizeof(double) * std::max<long long>(s->totalArea, 1), st));
    if (s->redNec) {
        k_scatter_rdense<<<blocks_for(n), 256, 0, st>>>(n, P, d_pd.p, dps, s->ID.p, s->JD.p, s->D.p,
                                                        s->mapR.p, s->S.p);
        SPK_CUDA(cudaGetLastError());
    }
    clk.lap(5);  // produceCompressedR

    // ---- spike sweep
    {
        std::vector<int> plist, sd0(P);
        int maxcc = 0;
        for (int t = 0; t < P; t++) {
            sd0[t] = parts[t].sD0;
            if (parts[t].hasS && parts[t].nRowsS > 0) {
                plist.push_back(t);
                maxcc = std::max(maxcc, parts[t].nColsS);
            }
        }
        if (!plist.empty()) {
            DBuf<int> d_pl(st), d_sd0(st);
            SPK_TRY(to_device(d_pl, plist, st));
            SPK_TRY(to_device(d_sd0, sd0, st));
            int bs = std::min(256, ((maxcc + 31) / 32) * 32);
            k_spike_sweep<<<(int)plist.size(), bs, 0, st>>>(d_pl.p, d_pd.p, d_sd0.p, s->IT2.p, s->JT2.p,
                                                            s->T2.p, s->S.p);
            SPK_CUDA(cudaGetLastError());
        }
    }
    clk.lap(6);  // produceS

    // ---- reduced system
    {
        DBuf<int> f(st), redIdx(st);
        SPK_TRY(f.alloc(n + 1));
        SPK_TRY(redIdx.alloc(n + 1));
        k_flags<<<blocks_for(n + 1), 256, 0, st>>>(n, s->dep.p, f.p);
        SPK_TRY(exclusive_scan(f.p, redIdx.p, n + 1, st));
        int nRed = 0;
        SPK_CUDA(cudaMemcpyAsync(&nRed, redIdx.p + n, sizeof(int), cudaMemcpyDeviceToHost, st));
        SPK_CUDA(cudaStreamSynchronize(st));
        s->nRed = nRed;
        SPK_TRY(s->mapRedX.alloc(nRed));
        k_reduced_ids<<<blocks_for(n), 256, 0, st>>>(n, redIdx.p, s->dep.p, s->mapRedX.p);
        SPK_TRY(s->d_lvl.alloc(P + 1));
        k_level_offsets<<<blocks_for(P + 1), 256, 0, st>>>(P, dps, redIdx.p, n, s->d_lvl.p);
        SPK_CUDA(cudaGetLastError());
        int rss = 0;
        if (P >= 2) SPK_CUDA(cudaMemcpy(&rss, redIdx.p + parts[P - 1].ps, sizeof(int), cudaMemcpyDeviceToHost));
        s->rss = rss;
        SPK_TRY(s->IT.alloc(rss + 1));
        if (rss > 0) {
            DBuf<int> cnt(st);
            SPK_TRY(cnt.alloc(rss + 1));
            k_reduced_rows<<<blocks_for(rss + 1), 256, 0, st>>>(rss, P, dps, d_pd.p, s->mapRedX.p, s->S.p,
                                                                s->mapR.p, s->dep.p, cnt.p, nullptr, nullptr,
                                                                nullptr);
            SPK_CUDA(cudaGetLastError());
            SPK_TRY(exclusive_scan(cnt.p, s->IT.p, rss + 1, st));
            int nT = 0;
            SPK_CUDA(cudaMemcpyAsync(&nT, s->IT.p + rss, sizeof(int), cudaMemcpyDeviceToHost, st));
            SPK_CUDA(cudaStreamSynchronize(st));
            s->nT = nT;
            SPK_TRY(s->T.alloc(nT));
            SPK_TRY(s->JT.alloc(nT));
            if (nT)
                k_reduced_rows<<<blocks_for(rss), 256, 0, st>>>(rss, P, dps, d_pd.p, s->mapRedX.p, s->S.p,
                                                                s->mapR.p, s->dep.p, cnt.p, s->IT.p, s->T.p,
                                                                s->JT.p);
            SPK_CUDA(cudaGetLastError());
        } else {
            SPK_CUDA(cudaMemsetAsync(s->IT.p, 0, sizeof(int), st));
            s->nT = 0;
            SPK_TRY(s->T.alloc(1));
            SPK_TRY(s->JT.alloc(1));
        }
        s->nnzRed = (int)(s->nT + nRed);
    }
    SPK_CUDA(cudaStreamSynchronize(st));
    clk.lap(7);  // produceReducedSystem
    s->prep_ms[0] = (now_s() - prep_t0) * 1e3;

    SPK_TRY(solve_prepare(s));
    s->built = 1;
    return SPK_OK;
}

}  // namespace spk
