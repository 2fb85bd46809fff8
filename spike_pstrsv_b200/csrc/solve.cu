// Spike solve for sm_100a (the per-call hot path of spike_pstrsv_solve,
// src/spike_pstrsv.c:149-239), on the upper-triangular CSR U.
//
//   phase 1  D1 y = b          rows [ps+si, pe) of each split block, entries with
//                              column < pe (the block-local part of the rows)
//   phase 2  reduced system    gather y at the dependents, unit-upper solve
//                              partition level by partition level, scatter
//   phase 3+4                  rows [ps, ps+ei) (split) or [ps, pe) (unsplit) by
//                              back substitution over the FULL rows: entries at
//                              columns >= ps+ei read the fixed x of phases 1-2,
//                              which is exactly b - R_new x followed by the D2
//                              (or D) solve of the reference, fused
//
// Truncation.  For rows [si, ei) of a split block, x - y = -S x_c exactly, with S
// the block's spike (D0^{-1} R, computed bit-exactly at preprocessing) and x_c the
// coupling unknowns.  A spike row whose absolute sum is <= tau moves x by at most
// tau * ||x||_inf.  With tau = 2^-60 (the default, below FP64 resolution) phase 4
// copies y for the leading rows whose spike rows are all negligible instead of
// recomputing them, and the reduced solve drops reduced rows (= spike rows at the
// dependents) that are negligible.  tau < 0 disables both (exact mode).
//
// Segment solver.  One warp per segment (one warp per CTA so that the segments
// spread evenly over the SMs), bottom-up in tiles of 32 rows.  Each tile's CSR
// slice (values and column indices) is staged into shared memory by the TMA
// bulk-copy engine (cp.async.bulk + mbarrier), one tile ahead of the tile being
// solved.  Lanes own rows: the contributions of already-solved rows are
// accumulated in parallel, and the in-tile triangle is resolved with one warp
// broadcast per row from a coefficient tile in shared memory.  The reversal of
// uplo='L' (x_L[i] = x_U[n-1-i]) is folded into the right-hand-side loads and
// the solution stores.
#include <algorithm>
#include <cstdio>
#include <ctime>

#include "spk_internal.cuh"

namespace spk {

namespace {

constexpr int kWin = 128;       // rows of recently solved x kept in shared memory
constexpr int kCap = 640;       // staged nonzeros per tile (32 rows); larger tiles read global memory
constexpr int kCapV = kCap + 2; // + alignment slack (16-byte granules of doubles)
constexpr int kCapC = kCap + 8; // + alignment slack (16-byte granules of ints)
constexpr long long kWaitCycles = 1ll << 32;  // ~2 s at B200 clocks: bound of every barrier wait

inline double now_s() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

inline int blocks_for(long long n, int bs = 256) { return (int)((n + bs - 1) / bs); }

// ---- TMA bulk copy + mbarrier primitives (PTX ISA 8.x, sm_90+) -------------------

__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// ---- segment solver -------------------------------------------------------------

struct TileStage {
    int s0v, s0c;   // first staged value / column element (aligned down)
    int direct;     // 1: tile read from global memory (too many nonzeros to stage)
};

struct SegSmem {
    alignas(16) double v[2][kCapV];
    alignas(16) int c[2][kCapC];
    alignas(16) double coef[32][32];  // [tile column i][lane row l] = a(l, i) / a(i, i)
    double rdv[32];                   // 1 / diagonal of the tile's rows
    double win[kWin];                 // x of the last kWin solved rows, by row mod kWin
    alignas(8) unsigned long long bar[2];
};

struct SegArgs {
    const SegTask *tasks;
    int ntasks;
    const int *ia;
    const int *ja;
    const double *a;
    int n;
    const double *rhs;   // right-hand side in the caller's order
    const double *xfix;  // U-order x of phases 1-2 (FULL mode)
    double *xout;        // output
    int rev_in;          // rhs[i] holds row n-1-i of U
    int rev_out;         // xout is stored in the caller's order with reversal
    int *err;
};

// Issue (lane 0) the bulk copies staging tile [r0, top): values and columns of
// nonzeros ia[r0] .. ia[top], widened to 16-byte granules.
__device__ __forceinline__ void stage_tile(const SegArgs &A, SegSmem &S, int slot, int r0, int top,
                                           TileStage &ts) {
    const int e0 = A.ia[r0], e1 = A.ia[top];
    ts.direct = (e1 - e0) > kCap;
    ts.s0v = e0 & ~1;
    ts.s0c = e0 & ~3;
    if (ts.direct) return;
    const int endv = (e1 + 1) & ~1, endc = (e1 + 3) & ~3;
    const unsigned bv = (unsigned)(endv - ts.s0v) * 8u, bc = (unsigned)(endc - ts.s0c) * 4u;
    fence_proxy_async();
    mbar_arrive_expect_tx(&S.bar[slot], bv + bc);
    bulk_g2s(S.v[slot], A.a + ts.s0v, bv, &S.bar[slot]);
    bulk_g2s(S.c[slot], A.ja + ts.s0c, bc, &S.bar[slot]);
}

// x at a column below the current tile: solved in this task (shared window or
// xout) when c < hi_ext; else the fixed phase 1-2 value (FULL) or nothing (!FULL).
template <bool FULL>
__device__ __forceinline__ double solved_x(const SegArgs &A, const SegSmem &S, int c, int top, int hi_ext) {
    if (c < hi_ext) {
        if (c < top + kWin) return S.win[c & (kWin - 1)];
        return A.xout[A.rev_out ? A.n - 1 - c : c];
    }
    return FULL ? A.xfix[c] : 0.0;
}

// Solve rows [lo, hi) of the task bottom-up.  Columns >= hi_ext take xfix
// (FULL) or are skipped (!FULL).  Solved rows are written to xout and to the
// shared window.  Returns false after a timed-out wait.
template <bool FULL>
__device__ bool solve_range(const SegArgs &A, SegSmem &S, unsigned &phase, int lo, int hi, int hi_ext) {
    const int lane = threadIdx.x & 31;
    if (hi <= lo) return true;
    const int ntiles = (hi - lo + 31) / 32;
    TileStage cur;
    if (lane == 0) stage_tile(A, S, 0, max(lo, hi - 32), hi, cur);
    cur.direct = __shfl_sync(0xffffffffu, cur.direct, 0);
    cur.s0v = __shfl_sync(0xffffffffu, cur.s0v, 0);
    cur.s0c = __shfl_sync(0xffffffffu, cur.s0c, 0);
    const int n = A.n;
    // right-hand side of the first tile
    double rhs_next = 0.0;
    {
        const int r = max(lo, hi - 32) + lane;
        if (r < hi) rhs_next = A.rhs[A.rev_in ? n - 1 - r : r];
    }
    for (int it = 0; it < ntiles; it++) {
        const int top = hi - 32 * it;
        const int r0 = max(lo, top - 32), nr = top - r0;
        const int slot = it & 1;
        // stage the next tile (its slot was released at the end of tile it-1)
        TileStage nxt = cur;
        if (it + 1 < ntiles) {
            const int top1 = r0, r01 = max(lo, top1 - 32);
            if (lane == 0) stage_tile(A, S, slot ^ 1, r01, top1, nxt);
            nxt.direct = __shfl_sync(0xffffffffu, nxt.direct, 0);
            nxt.s0v = __shfl_sync(0xffffffffu, nxt.s0v, 0);
            nxt.s0c = __shfl_sync(0xffffffffu, nxt.s0c, 0);
        }
        const double rhs_cur = rhs_next;
        if (it + 1 < ntiles) {
            const int r = max(lo, r0 - 32) + lane;
            rhs_next = (r < r0) ? A.rhs[A.rev_in ? n - 1 - r : r] : 0.0;
        }
        // wait for this tile's slice
        const bool direct = cur.direct;
        if (!direct) {
            const long long t0 = clock64();
            while (!mbar_try_wait(&S.bar[slot], (phase >> slot) & 1u)) {
                if (clock64() - t0 > kWaitCycles) {
                    if (lane == 0) atomicExch(A.err, 1);
                    return false;
                }
            }
            phase ^= 1u << slot;
        }
        __syncwarp();
        const double *vb = direct ? A.a : S.v[slot];
        const int *cb = direct ? A.ja : S.c[slot];
        const int ov = direct ? 0 : cur.s0v, oc = direct ? 0 : cur.s0c;
        // row bounds, diagonal reciprocal and right-hand side
        int b = 0, e = 0;
        double acc = 0.0, rd = 0.0;
        if (lane < nr) {
            const int r = r0 + lane;
            b = A.ia[r];
            e = A.ia[r + 1];
            rd = 1.0 / vb[b - ov];
            acc = rhs_cur;
        }
        S.rdv[lane] = rd;
        __syncwarp();
        // in-tile entries (columns r < c < top come first in the sorted row):
        // coefficient a(r, c) / a(c, c) into column c - r0 of the tile
        int q = b + 1;
        for (; q < e; q++) {
            const int c = cb[q - oc];
            if (c >= top) break;
            S.coef[c - r0][lane] = vb[q - ov] * S.rdv[c - r0];
        }
        const int q_in_end = q;
        // entries at solved rows below the tile, four independent partial sums
        double p0 = 0.0, p1 = 0.0, p2 = 0.0, p3 = 0.0;
        for (; q + 3 < e; q += 4) {
            const int c0 = cb[q - oc], c1 = cb[q + 1 - oc], c2 = cb[q + 2 - oc], c3 = cb[q + 3 - oc];
            const double v0 = vb[q - ov], v1 = vb[q + 1 - ov], v2 = vb[q + 2 - ov], v3 = vb[q + 3 - ov];
            p0 = fma(v0, solved_x<FULL>(A, S, c0, top, hi_ext), p0);
            p1 = fma(v1, solved_x<FULL>(A, S, c1, top, hi_ext), p1);
            p2 = fma(v2, solved_x<FULL>(A, S, c2, top, hi_ext), p2);
            p3 = fma(v3, solved_x<FULL>(A, S, c3, top, hi_ext), p3);
        }
        for (; q < e; q++) p0 = fma(vb[q - ov], solved_x<FULL>(A, S, cb[q - oc], top, hi_ext), p0);
        acc -= (p0 + p1) + (p2 + p3);
        __syncwarp();
        // in-tile triangle: step i broadcasts lane i's final accumulator
        double myx = 0.0;
#pragma unroll
        for (int i = 31; i >= 0; i--) {
            if (i < nr) {
                const double ci = S.coef[i][lane];
                const double ai = __shfl_sync(0xffffffffu, acc, i);
                if (lane == i) myx = ai * rd;
                acc = fma(-ci, ai, acc);
            }
        }
        // leave the coefficient tile zero for the next tile
        for (int q2 = b + 1; q2 < q_in_end; q2++) S.coef[cb[q2 - oc] - r0][lane] = 0.0;
        if (lane < nr) {
            const int r = r0 + lane;
            A.xout[A.rev_out ? n - 1 - r : r] = myx;
            S.win[r & (kWin - 1)] = myx;
        }
        __syncwarp();
        cur = nxt;
    }
    return true;
}

// Copy rows [lo, hi) of the U-order src into xout (and the shared window).
__device__ void copy_rows(const SegArgs &A, SegSmem &S, int lo, int hi) {
    const int lane = threadIdx.x & 31;
    for (int r = lo + lane; r < hi; r += 32) {
        const double v = A.xfix[r];
        A.xout[A.rev_out ? A.n - 1 - r : r] = v;
        if (r < lo + kWin) S.win[r & (kWin - 1)] = v;
    }
    __syncwarp();
}

template <bool FULL>
__global__ void __launch_bounds__(32) k_segment_solve(SegArgs A) {
    __shared__ SegSmem S;
    const int task = blockIdx.x;
    if (task >= A.ntasks) return;
    const int lane = threadIdx.x;
    if (lane == 0) {
        mbar_init(&S.bar[0], 1);
        mbar_init(&S.bar[1], 1);
        fence_mbar_init();
    }
#pragma unroll
    for (int i = 0; i < 32; i++) S.coef[i][lane] = 0.0;
    __syncwarp();
    unsigned phase = 0u;  // bit k: parity of the next completion of stage k
    const SegTask t = A.tasks[task];
    // rows [hi, tail) keep the phase-1 values
    if (FULL && t.tail > t.hi) copy_rows(A, S, t.hi, t.tail);
    if (t.skip_hi > t.skip_lo) {
        if (!solve_range<FULL>(A, S, phase, t.skip_hi, t.hi, t.hi)) return;
        copy_rows(A, S, t.skip_lo, t.skip_hi);
        solve_range<FULL>(A, S, phase, t.lo, t.skip_lo, t.hi);
    } else {
        solve_range<FULL>(A, S, phase, t.lo, t.hi, t.hi);
    }
}

__global__ void k_reverse(int n, const double *__restrict__ src, double *__restrict__ dst) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = src[n - 1 - i];
}

// produceReducedY + __usol2 + updateX (ops.c:1152-1177, 1247-1262) in one CTA, on
// the kept reduced rows: rows[] lists them level by level (a level is one
// partition's dependents; its rows only reference later partitions), levels in
// descending partition order, lvl_off[] delimiting the levels.  Dropped rows keep
// y, so the gather/scatter only touches the kept rows and their columns.
__global__ void __launch_bounds__(1024)
k_reduced_solve(const int *__restrict__ rows, const int *__restrict__ lvl_off, int nlvl,
                const int *__restrict__ mapRedX, const int *__restrict__ IT, const int *__restrict__ JT,
                const double *__restrict__ T, double *__restrict__ xbuf) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int li = 0; li < nlvl; li++) {
        for (int q = lvl_off[li] + warp; q < lvl_off[li + 1]; q += nwarps) {
            const int k = rows[q];
            double sum = 0.0;
            for (int j = IT[k] + lane; j < IT[k + 1]; j += 32) sum = fma(T[j], xbuf[mapRedX[JT[j]]], sum);
#pragma unroll
            for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
            if (lane == 0) xbuf[mapRedX[k]] -= sum;
        }
        __syncthreads();
    }
}

// Absolute row sums of the dense spikes: first significant row per block
// (everything above it is negligible) and the kept reduced rows.
__global__ void k_first_significant(int nlist, const int *__restrict__ plist, const long long *__restrict__ startsS,
                                    const int *__restrict__ nRowsS, const int *__restrict__ nColsS,
                                    const double *__restrict__ S, double tau, int *__restrict__ first) {
    const int t = plist[blockIdx.y];
    const int rc = nRowsS[t], cc = nColsS[t];
    const double *X = S + startsS[t];
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rc; r += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < cc; j++) s += fabs(X[(long long)r * cc + j]);
        if (s > tau) atomicMin(&first[t], r);
    }
}

__global__ void k_reduced_keep(int rss, const int *__restrict__ IT, const double *__restrict__ T, double tau,
                               int *__restrict__ keep) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= rss) return;
    double s = 0.0;
    for (int j = IT[k]; j < IT[k + 1]; j++) s += fabs(T[j]);
    keep[k] = (IT[k + 1] > IT[k]) && (s > tau);
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
    const double tau = s->trunc_tol;
    // first significant spike row per split block (rows above it: x = y)
    std::vector<int> first(P, 0);
    {
        std::vector<int> plist, nr(P), nc(P);
        std::vector<long long> ss(P);
        for (int t = 0; t < P; t++) {
            const Part &p = s->parts[t];
            nr[t] = p.nRowsS;
            nc[t] = p.nColsS;
            ss[t] = p.startsS;
            first[t] = p.nRowsS;
            if (p.hasS && p.nRowsS > 0) plist.push_back(t);
        }
        if (tau >= 0 && !plist.empty()) {
            DBuf<int> d_pl, d_nr, d_nc, d_first;
            DBuf<long long> d_ss;
            SPK_TRY(upload(d_pl, plist));
            SPK_TRY(upload(d_nr, nr));
            SPK_TRY(upload(d_nc, nc));
            SPK_TRY(upload(d_ss, ss));
            SPK_TRY(upload(d_first, first));
            dim3 grid(8, (unsigned)plist.size());
            k_first_significant<<<grid, 256, 0, s->stream>>>((int)plist.size(), d_pl.p, d_ss.p, d_nr.p, d_nc.p,
                                                              s->S.p, tau, d_first.p);
            SPK_CUDA(cudaGetLastError());
            SPK_CUDA(cudaStreamSynchronize(s->stream));
            SPK_CUDA(cudaMemcpy(first.data(), d_first.p, sizeof(int) * P, cudaMemcpyDeviceToHost));
        } else {
            for (int t = 0; t < P; t++) first[t] = 0;
        }
    }
    std::vector<SegTask> t1, t2;
    long long rows1 = 0, rows2 = 0;
    for (int t = 0; t < P; t++) {
        const Part &p = s->parts[t];
        const bool split = s->redNec && (p.hasRefl || p.isOpt);
        if (split) {
            // D1 rows [ps+si, pe); a cut before the block (si < 0) adds a row of the
            // previous block that no row of this block depends on, so it is skipped.
            const int lo = p.ps + std::max(p.si, 0);
            if (lo < p.pe) {
                t1.push_back(SegTask{lo, p.pe, 0, 0, p.pe});
                rows1 += p.pe - lo;
            }
            const int hi = p.ps + std::max(p.ei, 0);
            SegTask k{p.ps, hi, 0, 0, p.pe};
            if (p.hasS && p.nRowsS > 0 && first[t] > 0) {
                k.skip_lo = p.ps + p.si;
                k.skip_hi = std::min(p.ps + p.si + first[t], hi);
            }
            rows2 += (hi - p.ps) - (k.skip_hi - k.skip_lo);
            t2.push_back(k);
        } else {
            t2.push_back(SegTask{p.ps, p.pe, 0, 0, p.pe});
            rows2 += p.pe - p.ps;
        }
    }
    // longest segments first so that they start in the first wave
    auto longer = [](const SegTask &x, const SegTask &y) {
        return (x.hi - x.lo - (x.skip_hi - x.skip_lo)) > (y.hi - y.lo - (y.skip_hi - y.skip_lo));
    };
    std::stable_sort(t1.begin(), t1.end(), longer);
    std::stable_sort(t2.begin(), t2.end(), longer);
    s->ntasks1 = (int)t1.size();
    s->ntasks2 = (int)t2.size();
    s->rows_phase1 = rows1;
    s->rows_phase4 = rows2;
    SPK_TRY(upload(s->d_tasks1, t1));
    SPK_TRY(upload(s->d_tasks2, t2));

    // kept reduced rows, grouped by level in descending partition order
    std::vector<int> lvl(P + 1);
    SPK_CUDA(cudaMemcpy(lvl.data(), s->d_lvl.p, sizeof(int) * (P + 1), cudaMemcpyDeviceToHost));
    std::vector<int> keep(std::max(s->rss, 1), 0);
    if (s->rss > 0) {
        DBuf<int> d_keep;
        SPK_TRY(d_keep.alloc(s->rss));
        k_reduced_keep<<<blocks_for(s->rss), 256, 0, s->stream>>>(s->rss, s->IT.p, s->T.p,
                                                                 tau >= 0 ? tau : -1.0, d_keep.p);
        SPK_CUDA(cudaGetLastError());
        SPK_CUDA(cudaStreamSynchronize(s->stream));
        SPK_CUDA(cudaMemcpy(keep.data(), d_keep.p, sizeof(int) * s->rss, cudaMemcpyDeviceToHost));
    }
    std::vector<int> rows, off{0};
    for (int t = P - 2; t >= 1; t--) {
        const int k0 = std::min(lvl[t], s->rss), k1 = std::min(lvl[t + 1], s->rss);
        const size_t before = rows.size();
        for (int k = k0; k < k1; k++)
            if (keep[k]) rows.push_back(k);
        if (rows.size() > before) off.push_back((int)rows.size());
    }
    s->nlvl = (int)off.size() - 1;
    s->nkept = (int)rows.size();
    SPK_TRY(upload(s->d_red_rows, rows));
    SPK_TRY(upload(s->d_red_off, off));

    SPK_TRY(s->xbuf.alloc(s->n));
    if (s->uplo == 'L') SPK_TRY(s->xout_u.alloc(s->n));
    SPK_TRY(s->d_err.alloc(1));
    SPK_CUDA(cudaMemset(s->d_err.p, 0, sizeof(int)));
    return SPK_OK;
}

int solve(spk_system *s, const double *b, double *x, cudaStream_t st, double *ph) {
    if (!s->built) {
        set_error(SPK_ERR_STATE, "no preprocessed system");
        return SPK_ERR_STATE;
    }
    double t0 = 0;
    auto lap = [&](int slot) {
        if (!ph) return;
        cudaStreamSynchronize(st);
        double t1 = now_s();
        ph[slot] += t1 - t0;
        t0 = t1;
    };
    if (ph) { cudaStreamSynchronize(st); t0 = now_s(); }
    lap(0);
    const bool prof = s->profiling && s->ev[0][0];
    const int ring = (int)(s->ev_next % spk_system::kEvRing);
    if (prof) {
        if (s->ev_pending[ring]) SPK_TRY(collect_event_set(s, ring));
        cudaEventRecord(s->ev[ring][0], st);
    }
    SegArgs A;
    A.ia = s->uia.p;
    A.ja = s->uja.p;
    A.a = s->ua.p;
    A.n = s->n;
    A.rhs = b;
    A.rev_in = s->uplo == 'L';
    A.err = s->d_err.p;
    if (s->redNec && s->ntasks1) {
        A.tasks = s->d_tasks1.p;
        A.ntasks = s->ntasks1;
        A.xfix = nullptr;
        A.xout = s->xbuf.p;
        A.rev_out = 0;
        k_segment_solve<false><<<s->ntasks1, 32, 0, st>>>(A);
        SPK_CUDA(cudaGetLastError());
        s->launches++;
    }
    if (prof) cudaEventRecord(s->ev[ring][1], st);
    lap(1);
    if (s->redNec && s->nkept) {
        k_reduced_solve<<<1, 1024, 0, st>>>(s->d_red_rows.p, s->d_red_off.p, s->nlvl, s->mapRedX.p, s->IT.p,
                                            s->JT.p, s->T.p, s->xbuf.p);
        SPK_CUDA(cudaGetLastError());
        s->launches++;
    }
    if (prof) cudaEventRecord(s->ev[ring][2], st);
    lap(2);
    A.tasks = s->d_tasks2.p;
    A.ntasks = s->ntasks2;
    A.xfix = s->xbuf.p;
    A.xout = x;
    A.rev_out = s->uplo == 'L';
    k_segment_solve<true><<<s->ntasks2, 32, 0, st>>>(A);
    SPK_CUDA(cudaGetLastError());
    s->launches++;
    if (prof) {
        cudaEventRecord(s->ev[ring][3], st);
        s->ev_pending[ring] = 1;
        s->ev_next++;
    }
    lap(3);
    return SPK_OK;
}

int collect_event_set(spk_system *s, int k) {
    SPK_CUDA(cudaEventSynchronize(s->ev[k][3]));
    for (int p = 0; p < 3; p++) {
        float ms = 0;
        SPK_CUDA(cudaEventElapsedTime(&ms, s->ev[k][p], s->ev[k][p + 1]));
        s->phase_ms[p] += ms;
    }
    s->ev_pending[k] = 0;
    s->profiled_solves++;
    return SPK_OK;
}

int collect_phase_times(spk_system *s) {
    for (int k = 0; k < spk_system::kEvRing; k++)
        if (s->ev_pending[k]) SPK_TRY(collect_event_set(s, k));
    return SPK_OK;
}

int check_device_error(spk_system *s) {
    int e = 0;
    SPK_CUDA(cudaMemcpy(&e, s->d_err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        SPK_CUDA(cudaMemset(s->d_err.p, 0, sizeof(int)));
        set_error(SPK_ERR_TIMEOUT, "a bounded wait in the segment solver gave up");
        return SPK_ERR_TIMEOUT;
    }
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
