// Spike solve for sm_100a (the per-call hot path of spike_pstrsv_solve,
// src/spike_pstrsv.c:149-239), on the upper-triangular CSR U.
//
//   phase 1  D1 y = b          rows [ps+si, pe) of each split block, entries with
//                              column < pe (the block-local part of the rows)
//   phase 2  reduced system    gather y at the dependents, unit-upper solve
//                              partition level by partition level, scatter
//   phase 3+4                  rows [ps, ps+ei) (split) or [ps, pe) (unsplit) by
//                              back substitution over the FULL rows: the entries
//                              at columns >= the segment end read the fixed x of
//                              phases 1-2, which is exactly b - R_new x followed
//                              by the D2 (or D) solve of the reference, fused
//
// Each segment is one warp's sequential job, processed bottom-up in tiles of
// 32 rows: lanes own rows, contributions from rows below the tile are
// accumulated in parallel, and the in-tile triangle is resolved with one
// broadcast per row from a per-warp coefficient tile in shared memory.
#include <algorithm>
#include <cstdio>
#include <ctime>

#include "spk_internal.cuh"

namespace spk {

namespace {

constexpr int kWarps = 4;    // warps per CTA of the segment solver
constexpr int kWin = 256;    // rows of recently solved x kept in shared memory per warp

inline double now_s() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

inline int blocks_for(long long n, int bs = 256) { return (int)((n + bs - 1) / bs); }

// Back substitution over rows [lo, hi) of U for each task, one warp per task.
// FULL = false: entries at columns >= hi are ignored (the block-local D1 solve).
// FULL = true:  entries at columns >= hi use xfix (the coupled D2/D solve).
template <bool FULL>
__global__ void __launch_bounds__(kWarps * 32)
k_segment_solve(const SolveTask *__restrict__ tasks, int ntasks, const int *__restrict__ ia,
                const int *__restrict__ ja, const double *__restrict__ a,
                const double *__restrict__ rhs, const double *__restrict__ xfix,
                double *__restrict__ xout) {
    __shared__ double coef[kWarps][32][32];  // [tile column i][lane row]
    __shared__ double win[kWarps][kWin];     // x of the last kWin solved rows, by row mod kWin
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int task = blockIdx.x * kWarps + wid;
    if (task >= ntasks) return;
    const int lo = tasks[task].lo, hi = tasks[task].hi;
    double(*C)[32] = coef[wid];
    double *W = win[wid];
    for (int top = hi; top > lo; top -= 32) {
        const int r0 = max(lo, top - 32), nr = top - r0;
#pragma unroll
        for (int i = 0; i < 32; i++) C[i][lane] = 0.0;
        __syncwarp();
        double acc = 0.0, rd = 0.0;
        if (lane < nr) {
            const int r = r0 + lane;
            const int b = ia[r], e = ia[r + 1];
            acc = rhs[r];
            rd = 1.0 / a[b];
            for (int q = b + 1; q < e; q++) {
                const int c = ja[q];
                const double v = a[q];
                if (c < top) {
                    C[c - r0][lane] = v;
                } else if (c < hi) {
                    const double xc = (c < top + kWin) ? W[c & (kWin - 1)] : xout[c];
                    acc = fma(-v, xc, acc);
                } else if (FULL) {
                    acc = fma(-v, xfix[c], acc);
                }
            }
        }
        __syncwarp();
        double myx = 0.0;
        for (int i = nr - 1; i >= 0; i--) {
            const double xi = __shfl_sync(0xffffffffu, acc * rd, i);
            if (lane == i) myx = xi;
            acc = fma(-C[i][lane], xi, acc);
        }
        if (lane < nr) {
            xout[r0 + lane] = myx;
            W[(r0 + lane) & (kWin - 1)] = myx;
        }
        __syncwarp();
    }
}

__global__ void k_copy_ranges(const SolveTask *__restrict__ ranges, int nranges,
                              const double *__restrict__ src, double *__restrict__ dst) {
    for (int k = blockIdx.y; k < nranges; k += gridDim.y) {
        const int lo = ranges[k].lo, hi = ranges[k].hi;
        for (int i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += gridDim.x * blockDim.x)
            dst[i] = src[i];
    }
}

__global__ void k_reverse(int n, const double *__restrict__ src, double *__restrict__ dst) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = src[n - 1 - i];
}

// produceReducedY + __usol2 + updateX (ops.c:1152-1177, 1247-1262) in one CTA:
// gather, then the unit-upper solve level by level (a level is one partition's
// dependents; its rows only reference later partitions), then scatter.
__global__ void __launch_bounds__(1024)
k_reduced_solve(int nRed, int rss, const int *__restrict__ mapRedX, const int *__restrict__ IT,
                const int *__restrict__ JT, const double *__restrict__ T, const int *__restrict__ lvl,
                const int *__restrict__ lvl_list, int nlvl, double *__restrict__ red,
                double *__restrict__ xbuf) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    for (int i = tid; i < nRed; i += blockDim.x) red[i] = xbuf[mapRedX[i]];
    __syncthreads();
    for (int li = 0; li < nlvl; li++) {
        const int t = lvl_list[li];
        const int k0 = lvl[t], k1 = min(lvl[t + 1], rss);
        for (int k = k0 + warp; k < k1; k += nwarps) {
            double sum = 0.0;
            for (int j = IT[k] + lane; j < IT[k + 1]; j += 32) sum = fma(T[j], red[JT[j]], sum);
#pragma unroll
            for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
            if (lane == 0) red[k] -= sum;
        }
        __syncthreads();
    }
    for (int i = tid; i < rss; i += blockDim.x) xbuf[mapRedX[i]] = red[i];
}

// b[r] -= R_new x for the rows of blocks with dependences (spike_pstrsv.c:213-215),
// used only when the caller asks for the reference's clobbered right-hand side.
__global__ void k_clobber_rhs(int n, int rev, const int *__restrict__ ID, const int *__restrict__ JD,
                              const double *__restrict__ D, const double *__restrict__ xu,
                              double *__restrict__ b) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    double sum = 0.0;
    for (int q = ID[n + r]; q < ID[n + r + 1]; q++) sum += D[q] * xu[JD[q]];
    if (ID[n + r + 1] > ID[n + r]) {
        const int o = rev ? n - 1 - r : r;
        b[o] = -sum + b[o];
    }
}

template <typename T>
int upload(DBuf<T> &d, const std::vector<T> &h) {
    SPK_TRY(d.alloc(h.size()));
    if (!h.empty()) SPK_CUDA(cudaMemcpy(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return SPK_OK;
}

}  // namespace

int solve_prepare(spk_system *s) {
    const int P = s->P;
    std::vector<SolveTask> t1, t2, c2;
    for (int t = 0; t < P; t++) {
        const Part &p = s->parts[t];
        const bool split = s->redNec && (p.hasRefl || p.isOpt);
        if (split) {
            // D1 rows [ps+si, pe); a cut before the block (si < 0) adds a row of the
            // previous block that no row of this block depends on, so it is skipped.
            const int lo = p.ps + std::max(p.si, 0);
            if (lo < p.pe) t1.push_back(SolveTask{lo, p.pe});
            if (p.ei > 0) t2.push_back(SolveTask{p.ps, p.ps + p.ei});
            const int keep = p.ps + std::max(p.ei, 0);
            if (keep < p.pe) c2.push_back(SolveTask{keep, p.pe});
        } else {
            t2.push_back(SolveTask{p.ps, p.pe});
        }
    }
    // longest segments first so that they start in the first wave
    auto longer = [](const SolveTask &x, const SolveTask &y) { return (x.hi - x.lo) > (y.hi - y.lo); };
    std::stable_sort(t1.begin(), t1.end(), longer);
    std::stable_sort(t2.begin(), t2.end(), longer);
    s->ntasks1 = (int)t1.size();
    s->ntasks2 = (int)t2.size();
    s->ncopy2 = (int)c2.size();
    SPK_TRY(upload(s->d_tasks1, t1));
    SPK_TRY(upload(s->d_tasks2, t2));
    SPK_TRY(upload(s->d_copy2, c2));

    // reduced levels holding entries, in descending partition order
    std::vector<int> lvl(P + 1), IT;
    SPK_CUDA(cudaMemcpy(lvl.data(), s->d_lvl.p, sizeof(int) * (P + 1), cudaMemcpyDeviceToHost));
    IT.resize(s->rss + 1);
    SPK_CUDA(cudaMemcpy(IT.data(), s->IT.p, sizeof(int) * (s->rss + 1), cudaMemcpyDeviceToHost));
    s->lvl_nonempty.clear();
    for (int t = P - 2; t >= 1; t--) {
        const int k0 = std::min(lvl[t], s->rss), k1 = std::min(lvl[t + 1], s->rss);
        if (k1 > k0 && IT[k1] > IT[k0]) s->lvl_nonempty.push_back(t);
    }
    s->nlvl = (int)s->lvl_nonempty.size();
    SPK_TRY(upload(s->d_lvl_list, s->lvl_nonempty));

    SPK_TRY(s->xbuf.alloc(s->n));
    SPK_TRY(s->red.alloc(std::max(s->nRed, 1)));
    if (s->uplo == 'L') {
        SPK_TRY(s->rhs_u.alloc(s->n));
        SPK_TRY(s->xout_u.alloc(s->n));
    }
    return SPK_OK;
}

int solve(spk_system *s, const double *b, double *x, cudaStream_t st, double *ph) {
    if (!s->built) {
        set_error(SPK_ERR_STATE, "no preprocessed system");
        return SPK_ERR_STATE;
    }
    const int n = s->n;
    const double *rhs = b;
    double *xf = x;
    double t0 = 0;
    auto lap = [&](int slot) {
        if (!ph) return;
        cudaStreamSynchronize(st);
        double t1 = now_s();
        ph[slot] += t1 - t0;
        t0 = t1;
    };
    if (ph) { cudaStreamSynchronize(st); t0 = now_s(); }
    if (s->uplo == 'L') {
        k_reverse<<<std::min(blocks_for(n), 148 * 8), 256, 0, st>>>(n, b, s->rhs_u.p);
        rhs = s->rhs_u.p;
        xf = s->xout_u.p;
    }
    lap(0);
    const int *ia = s->uia.p, *ja = s->uja.p;
    const double *a = s->ua.p;
    if (s->redNec) {
        if (s->ntasks1)
            k_segment_solve<false><<<(s->ntasks1 + kWarps - 1) / kWarps, kWarps * 32, 0, st>>>(
                s->d_tasks1.p, s->ntasks1, ia, ja, a, rhs, nullptr, s->xbuf.p);
        SPK_CUDA(cudaGetLastError());
        lap(1);
        if (s->nRed)
            k_reduced_solve<<<1, 1024, 0, st>>>(s->nRed, s->rss, s->mapRedX.p, s->IT.p, s->JT.p, s->T.p,
                                                s->d_lvl.p, s->d_lvl_list.p, s->nlvl, s->red.p, s->xbuf.p);
        SPK_CUDA(cudaGetLastError());
        lap(2);
        if (s->ntasks2)
            k_segment_solve<true><<<(s->ntasks2 + kWarps - 1) / kWarps, kWarps * 32, 0, st>>>(
                s->d_tasks2.p, s->ntasks2, ia, ja, a, rhs, s->xbuf.p, xf);
        if (s->ncopy2)
            k_copy_ranges<<<dim3(8, std::min(s->ncopy2, 4096)), 256, 0, st>>>(s->d_copy2.p, s->ncopy2,
                                                                            s->xbuf.p, xf);
        SPK_CUDA(cudaGetLastError());
        lap(3);
    } else {
        lap(1);
        lap(2);
        k_segment_solve<true><<<(s->ntasks2 + kWarps - 1) / kWarps, kWarps * 32, 0, st>>>(
            s->d_tasks2.p, s->ntasks2, ia, ja, a, rhs, s->xbuf.p, xf);
        SPK_CUDA(cudaGetLastError());
        lap(3);
    }
    if (s->uplo == 'L') {
        k_reverse<<<std::min(blocks_for(n), 148 * 8), 256, 0, st>>>(n, xf, x);
        SPK_CUDA(cudaGetLastError());
    }
    lap(4);
    return SPK_OK;
}

int clobber_rhs(spk_system *s, const double *x, double *b, cudaStream_t st) {
    // x in the caller's order; R_new works on U's order
    const double *xu = x;
    if (s->uplo == 'L') {
        k_reverse<<<std::min(blocks_for(s->n), 148 * 8), 256, 0, st>>>(s->n, x, s->xout_u.p);
        xu = s->xout_u.p;
    }
    k_clobber_rhs<<<blocks_for(s->n), 256, 0, st>>>(s->n, s->uplo == 'L', s->ID.p, s->JD.p, s->D.p, xu, b);
    SPK_CUDA(cudaGetLastError());
    return SPK_OK;
}

}  // namespace spk
