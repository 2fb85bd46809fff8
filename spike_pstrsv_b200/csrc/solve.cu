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
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <mutex>

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

// After a timed-out barrier wait: give the bulk copy still addressed to this
// CTA's shared memory (parity `parity` of barrier `bar`) a second bounded period
// to land, so that the CTA does not exit while a copy writes into its shared
// memory.  Returns either way (a copy that never lands cannot be cancelled).
__device__ __noinline__ void drain_copy(unsigned long long *bar, unsigned parity) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > (1ll << 32)) return;
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

constexpr int kCapR = 34;        // staged 1/diagonal values per tile (+ alignment slack)

struct TileStage {
    int s0v, s0c, s0r;  // first staged value / column / reciprocal element (aligned down)
    int direct;         // 1: values and columns read from global memory (too many nonzeros)
};

struct SegSmem {
    alignas(16) double v[2][kCapV];
    alignas(16) int c[2][kCapC];
    alignas(16) double rd[2][kCapR];  // 1 / diagonal of the tile's rows
    alignas(16) double coef[32][32];  // [tile column i][lane row l] = a(l, i) / a(i, i)
    double win[kWin];                 // x of the last kWin solved rows, by row mod kWin
    alignas(8) unsigned long long bar[2];
};

struct SegArgs {
    const SegTask *tasks;
    int ntasks;
    const int *ia;
    const int *ja;
    const double *a;
    const double *rdiag;  // 1 / diagonal per row of U (padded for 16-byte granules)
    const double *ell_val;  // sliced ELL of U's off-diagonals over absolute 32-row tiles
    const int *ell_col;
    const int *ell_ptr;     // tile j occupies entries [ell_ptr[j], ell_ptr[j+1]); slot k of row 32j+l at +32k+l
    int n;
    const double *rhs;    // right-hand side in the caller's order
    const double *xfix;   // U-order x of phases 1-2 (FULL mode)
    double *xout;         // output
    int rev_in;           // rhs[i] holds row n-1-i of U
    int rev_out;          // xout is stored in the caller's order with reversal
    int *err;
    int fail_entry;       // test hook: take the timed-out-wait exit before any copy
};

// Lane 0: stage tile [r0, top) whose nonzeros are [e0, e1): the reciprocals of
// its diagonal and, unless the tile is too large, its values and column
// indices, each widened to 16-byte granules.
__device__ __forceinline__ void stage_tile(const SegArgs &A, SegSmem &S, int slot, int r0, int top, int e0,
                                           int e1, TileStage &ts) {
    ts.direct = (e1 - e0) > kCap;
    ts.s0v = e0 & ~1;
    ts.s0c = e0 & ~3;
    ts.s0r = r0 & ~1;
    const unsigned br = (unsigned)(((top + 1) & ~1) - ts.s0r) * 8u;
    unsigned bv = 0, bc = 0;
    if (!ts.direct) {
        bv = (unsigned)(((e1 + 1) & ~1) - ts.s0v) * 8u;
        bc = (unsigned)(((e1 + 3) & ~3) - ts.s0c) * 4u;
    }
    fence_proxy_async();
    mbar_arrive_expect_tx(&S.bar[slot], br + bv + bc);
    bulk_g2s(S.rd[slot], A.rdiag + ts.s0r, br, &S.bar[slot]);
    if (!ts.direct) {
        bulk_g2s(S.v[slot], A.a + ts.s0v, bv, &S.bar[slot]);
        bulk_g2s(S.c[slot], A.ja + ts.s0c, bc, &S.bar[slot]);
    }
}

__device__ __forceinline__ void bcast_stage(TileStage &t) {
    t.direct = __shfl_sync(0xffffffffu, t.direct, 0);
    t.s0v = __shfl_sync(0xffffffffu, t.s0v, 0);
    t.s0c = __shfl_sync(0xffffffffu, t.s0c, 0);
    t.s0r = __shfl_sync(0xffffffffu, t.s0r, 0);
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
// shared window.  Row pointers are prefetched two tiles ahead and the
// right-hand side one tile ahead, in registers; the tile's CSR slice and
// diagonal reciprocals are staged one tile ahead by the bulk-copy engine.
// Returns false after a timed-out wait.
template <bool FULL>
__device__ bool solve_range(const SegArgs &A, SegSmem &S, unsigned &phase, int lo, int hi, int hi_ext) {
    const unsigned FULLMASK = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    if (hi <= lo) return true;
    const int n = A.n;
    const int ntiles = (hi - lo + 31) / 32;
    // tile k covers rows [r0_k, top_k): top_0 = hi, top_{k+1} = r0_k, r0_k = max(lo, top_k - 32)
    int top = hi, r0 = max(lo, hi - 32);
    int top1 = r0, r01 = max(lo, r0 - 32);
    auto load_ia = [&](int rr0, int rtop) {
        const int r = rr0 + lane;
        return A.ia[r < rtop ? r : rtop];
    };
    auto load_rhs = [&](int rr0, int rtop) {
        const int r = rr0 + lane;
        return r < rtop ? A.rhs[A.rev_in ? n - 1 - r : r] : 0.0;
    };
    int ia_top = A.ia[hi];                                 // ia[top] of the current tile
    int ia_c = load_ia(r0, top);                           // ia[r0 + lane] of the current tile
    int ia_n = ntiles > 1 ? load_ia(r01, top1) : 0;        // the next tile's
    double rhs_c = load_rhs(r0, top);
    TileStage cur;
    {
        const int e0 = __shfl_sync(FULLMASK, ia_c, 0);
        if (lane == 0) stage_tile(A, S, 0, r0, top, e0, ia_top, cur);
        bcast_stage(cur);
    }
    for (int it = 0; it < ntiles; it++) {
        const int slot = it & 1;
        const int nr = top - r0;
        // prefetch: right-hand side of tile it+1, row pointers of tile it+2;
        // stage tile it+1 (its slot was released at the end of tile it-1)
        int top2 = 0, r02 = 0, ia_nn = 0;
        double rhs_n = 0.0;
        TileStage nxt = cur;
        if (it + 1 < ntiles) {
            rhs_n = load_rhs(r01, top1);
            if (it + 2 < ntiles) {
                top2 = r01;
                r02 = max(lo, r01 - 32);
                ia_nn = load_ia(r02, top2);
            }
            const int e0 = __shfl_sync(FULLMASK, ia_n, 0);
            const int e1 = __shfl_sync(FULLMASK, ia_c, 0);  // ia[top1] = ia[r0]
            if (lane == 0) stage_tile(A, S, slot ^ 1, r01, top1, e0, e1, nxt);
            bcast_stage(nxt);
        }
        // row bounds of this tile
        int b = ia_c;
        int e = __shfl_down_sync(FULLMASK, ia_c, 1);
        if (lane == nr - 1) e = ia_top;
        if (lane >= nr) b = e = 0;
        // wait for this tile's slice
        {
            const long long t0 = clock64();
            while (!mbar_try_wait(&S.bar[slot], (phase >> slot) & 1u)) {
                if (clock64() - t0 > kWaitCycles) {
                    drain_copy(&S.bar[slot], (phase >> slot) & 1u);
                    if (it + 1 < ntiles) drain_copy(&S.bar[slot ^ 1], (phase >> (slot ^ 1)) & 1u);
                    if (lane == 0) atomicExch(A.err, 1);
                    return false;
                }
            }
            phase ^= 1u << slot;
        }
        const bool direct = cur.direct;
        const double *vb = direct ? A.a : S.v[slot];
        const int *cb = direct ? A.ja : S.c[slot];
        const int ov = direct ? 0 : cur.s0v, oc = direct ? 0 : cur.s0c;
        const double *rdt = S.rd[slot] - 0;
        const int orr = cur.s0r;
        const double rd = lane < nr ? rdt[r0 + lane - orr] : 0.0;
        double acc = rhs_c;
        // entries after the diagonal: in-tile columns (r < c < top) give the
        // coefficient a(r, c) / a(c, c); solved columns below the tile are summed
        double p[4] = {0.0, 0.0, 0.0, 0.0};
        unsigned mask = 0u;
        for (int q = b + 1; q < e; q += 4) {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int qq = q + k;
                if (qq < e) {
                    const int c = cb[qq - oc];
                    const double v = vb[qq - ov];
                    if (c < top) {
                        S.coef[c - r0][lane] = v * rdt[c - orr];
                        mask |= 1u << (c - r0);
                    } else {
                        p[k] = fma(v, solved_x<FULL>(A, S, c, top, hi_ext), p[k]);
                    }
                }
            }
        }
        acc -= (p[0] + p[1]) + (p[2] + p[3]);
        __syncwarp();
        // in-tile triangle: step i broadcasts lane i's (final) accumulator.  Lane
        // i's row has no entries left of its diagonal, so its accumulator does
        // not change after its own step.
        if (nr == 32) {
#pragma unroll
            for (int i = 31; i >= 0; i--) {
                const double ci = S.coef[i][lane];
                const double ai = __shfl_sync(FULLMASK, acc, i);
                acc = fma(-ci, ai, acc);
            }
        } else {
            for (int i = nr - 1; i >= 0; i--) {
                const double ci = S.coef[i][lane];
                const double ai = __shfl_sync(FULLMASK, acc, i);
                acc = fma(-ci, ai, acc);
            }
        }
        const double myx = acc * rd;
        // leave the coefficient tile zero for the next tile
        while (mask) {
            const int i = __ffs(mask) - 1;
            S.coef[i][lane] = 0.0;
            mask &= mask - 1u;
        }
        if (lane < nr) {
            const int r = r0 + lane;
            A.xout[A.rev_out ? n - 1 - r : r] = myx;
            S.win[r & (kWin - 1)] = myx;
        }
        __syncwarp();
        // advance
        ia_top = __shfl_sync(FULLMASK, ia_c, 0);
        ia_c = ia_n;
        ia_n = ia_nn;
        rhs_c = rhs_n;
        top = top1;
        r0 = r01;
        top1 = top2;
        r01 = r02;
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
    if (A.fail_entry) {
        if (lane == 0) atomicExch(A.err, 1);
        return;
    }
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

// ---- tile solver on the sliced-ELL layout -----------------------------------------
//
// Same algorithm as the CSR segment solver, on absolute 32-row tiles: tile j =
// rows [32j, 32j+32); a task covers its tiles from the one holding hi-1 down to
// the one holding lo, with the rows outside [lo, hi) masked.  The tile's slots
// are contiguous (32 x width values and columns, 128/256-byte aligned), so each
// tile is one set of bulk copies with no alignment slack, lanes read their slots
// conflict-free, and every lane runs the same number of slot steps.
//
// K right-hand sides are solved together (column-major, leading dimensions ldb /
// ldx, n for the internal buffers): the matrix slice is read once, each lane
// keeps K accumulators, and a chain step broadcasts K independent values, so a
// step costs about the latency of one.  T is the arithmetic/storage type of the
// matrix and internal vectors (double, or float for the mixed-precision solve);
// the right-hand side is read as FP64 and converted, the output type is TO.

constexpr int kEllCap = 20;  // staged slots per row; wider tiles are read from global memory

template <int K, typename T>
struct TileCfg {
    static constexpr int kWinR = K == 1 ? 128 : 64;           // solved rows kept per right-hand side
    static constexpr int kChunk = K == 1 ? 8 : (K <= 4 ? 4 : 2);  // slots per load-first chunk
    static constexpr int kPart = K == 1 ? 4 : 1;               // partial sums per right-hand side
};

template <int K, typename T>
struct TileSmemK {
    alignas(128) T v[2][kEllCap * 32];
    alignas(128) int c[2][kEllCap * 32];
    alignas(128) T rd[2][32];        // 1 / diagonal of the tile's rows
    alignas(16) T coef[33][32];      // [tile column i][lane row l] = a(l, i) / a(i, i); row 32: scratch
    T win[K][TileCfg<K, T>::kWinR];  // x of the last solved rows, by row mod kWinR
    alignas(8) unsigned long long bar[2];
};

struct TileArgs {
    const SegTask *tasks;
    int ntasks;
    const void *ell_val;  // T
    const int *ell_col;
    const int *ell_ptr;
    const void *rdiag;    // T, padded to whole tiles
    int n;
    const double *rhs;    // caller order, column-major
    long long ldb;
    int rev_in;
    const void *xfix;     // T, U order, column-major with leading dimension n (FULL mode)
    void *xout;           // TO
    long long ldx;
    int rev_out;
    int acc;              // right-hand-side-parallel phase 3+4: xout += x (needs couplings within the window)
    int *err;
    int fail_entry;       // test hook: take the timed-out-wait exit before any copy
};

// Lane 0: stage tile j (entries [e0, e1)): its diagonal reciprocals and its first
// kEllCap slots of values and columns.
template <typename T, typename S_>
__device__ __forceinline__ void stage_ell(const TileArgs &A, S_ &S, int slot, int j, int e0, int e1) {
    const unsigned ne = (unsigned)min(e1 - e0, kEllCap * 32);
    fence_proxy_async();
    mbar_arrive_expect_tx(&S.bar[slot], 32u * sizeof(T) + ne * (unsigned)(sizeof(T) + 4));
    bulk_g2s(S.rd[slot], (const T *)A.rdiag + 32ll * j, 32u * sizeof(T), &S.bar[slot]);
    if (ne) {
        bulk_g2s(S.v[slot], (const T *)A.ell_val + e0, ne * (unsigned)sizeof(T), &S.bar[slot]);
        bulk_g2s(S.c[slot], A.ell_col + e0, ne * 4u, &S.bar[slot]);
    }
}

template <bool FULL, int K, typename T, typename TO>
__device__ bool tile_range(const TileArgs &A, TileSmemK<K, T> &S, unsigned &phase, int lo, int hi, int hi_ext) {
    using C = TileCfg<K, T>;
    constexpr int W = C::kWinR, CH = C::kChunk, NP = C::kPart;
    const unsigned FULLMASK = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    if (hi <= lo) return true;
    const int n = A.n;
    const T *evg = (const T *)A.ell_val;
    const T *xfix = (const T *)A.xfix;
    TO *xout = (TO *)A.xout;
    const int jt = (hi - 1) >> 5, jb = lo >> 5;
    const int ntiles = jt - jb + 1;
    auto load_rhs = [&](int j, T (&r)[K]) {
        const int row = 32 * j + lane;
        const bool ok = row >= lo && row < hi;
        const long long o = A.rev_in ? n - 1 - row : row;
#pragma unroll
        for (int k = 0; k < K; k++) r[k] = ok ? (T)A.rhs[k * A.ldb + o] : T(0);
    };
    int p_hi = A.ell_ptr[jt + 1], p_lo = A.ell_ptr[jt];
    int p_next = ntiles > 1 ? A.ell_ptr[jt - 1] : 0;
    T rhs_c[K];
    load_rhs(jt, rhs_c);
    if (lane == 0) stage_ell<T>(A, S, 0, jt, p_lo, p_hi);
    for (int it = 0; it < ntiles; it++) {
        const int j = jt - it;
        const int slot = it & 1;
        const int row0 = 32 * j;
        const int a0 = max(lo, row0), a1 = min(hi, row0 + 32);
        // stage tile j-1, prefetch its right-hand side and the pointer of tile j-2
        int p_next2 = 0;
        T rhs_n[K];
#pragma unroll
        for (int k = 0; k < K; k++) rhs_n[k] = T(0);
        if (it + 1 < ntiles) {
            if (lane == 0) stage_ell<T>(A, S, slot ^ 1, j - 1, p_next, p_lo);
            load_rhs(j - 1, rhs_n);
            if (it + 2 < ntiles) p_next2 = A.ell_ptr[j - 2];
        }
        {
            const long long t0 = clock64();
            while (!mbar_try_wait(&S.bar[slot], (phase >> slot) & 1u)) {
                if (clock64() - t0 > kWaitCycles) {
                    drain_copy(&S.bar[slot], (phase >> slot) & 1u);
                    if (it + 1 < ntiles) drain_copy(&S.bar[slot ^ 1], (phase >> (slot ^ 1)) & 1u);
                    if (lane == 0) atomicExch(A.err, 1);
                    return false;
                }
            }
            phase ^= 1u << slot;
        }
        const int width = (p_hi - p_lo) >> 5;
        const int nst = min(width, kEllCap);  // staged slots; the rest are read from global memory
        const T *rdt = S.rd[slot];
        const int row = row0 + lane;
        const bool act = row >= a0 && row < a1;
        const T rd = rdt[lane];
        T acc[K];
        T pacc[K][NP];
#pragma unroll
        for (int k = 0; k < K; k++) {
            acc[k] = act ? rhs_c[k] : T(0);
#pragma unroll
            for (int p = 0; p < NP; p++) pacc[k][p] = T(0);
        }
        bool slow = false;
        // Slots in chunks: all loads of a chunk are issued before its shared
        // stores (the stores may alias the staged buffers, so loads cannot move
        // past them).  In-tile columns store a(r, c) / a(c, c) into the
        // coefficient tile (others into the scratch row); columns inside the
        // shared window are summed; columns beyond the window or past hi_ext are
        // flagged for the slow pass.
        if (act) {
            const T *vs = S.v[slot];
            const int *cs = S.c[slot];
            const T *vg = evg + p_lo;
            const int *cg = A.ell_col + p_lo;
            auto chunk = [&](const int (&cr)[CH], const T (&vr)[CH]) {
                int ci[CH];
                T rr[CH], wr[CH][K];
#pragma unroll
                for (int u = 0; u < CH; u++) {
                    ci[u] = cr[u] < a1 ? cr[u] - row0 : 32;
                    rr[u] = rdt[ci[u] & 31];
#pragma unroll
                    for (int k = 0; k < K; k++) wr[u][k] = S.win[k][cr[u] & (W - 1)];
                }
#pragma unroll
                for (int u = 0; u < CH; u++) {
                    S.coef[ci[u]][lane] = vr[u] * rr[u];
                    const bool in_win = ci[u] == 32 && cr[u] < hi_ext && cr[u] < a1 + W;
#pragma unroll
                    for (int k = 0; k < K; k++)
                        pacc[k][u % NP] = in_win ? fma(vr[u], wr[u][k], pacc[k][u % NP]) : pacc[k][u % NP];
                    slow = slow || (ci[u] == 32 && !in_win && (FULL || cr[u] < hi_ext));
                }
            };
            // staged slots (the common case: the tile's width fits the stage); a
            // loop of its own, so that its loads are shared-memory loads only
            for (int k0 = 0; k0 < nst; k0 += CH) {
                int cr[CH];
                T vr[CH];
#pragma unroll
                for (int u = 0; u < CH; u++) {
                    const int k = k0 + u;
                    cr[u] = k < nst ? cs[k * 32 + lane] : row;  // no-op slot: zero into the row's own position
                    vr[u] = k < nst ? vs[k * 32 + lane] : T(0);
                }
                chunk(cr, vr);
            }
            // slots beyond the stage, from global memory
            for (int k0 = nst; k0 < width; k0 += CH) {
                int cr[CH];
                T vr[CH];
#pragma unroll
                for (int u = 0; u < CH; u++) {
                    const int k = k0 + u;
                    cr[u] = k < width ? cg[k * 32 + lane] : row;
                    vr[u] = k < width ? vg[k * 32 + lane] : T(0);
                }
                chunk(cr, vr);
            }
        }
        if (__any_sync(FULLMASK, slow) && act) {
            // columns solved long ago (beyond the window) or fixed by phases 1-2
            for (int k = 0; k < width; k++) {
                const int c = k < nst ? S.c[slot][k * 32 + lane] : A.ell_col[p_lo + k * 32 + lane];
                const T v = k < nst ? S.v[slot][k * 32 + lane] : evg[p_lo + k * 32 + lane];
                if (c < a1) continue;
                if (c < hi_ext) {
                    if (c >= a1 + W) {
                        const long long o = A.rev_out ? n - 1 - c : c;
#pragma unroll
                        for (int q = 0; q < K; q++) pacc[q][0] = fma(v, (T)xout[q * A.ldx + o], pacc[q][0]);
                    }
                } else if (FULL) {
#pragma unroll
                    for (int q = 0; q < K; q++) pacc[q][0] = fma(v, xfix[(long long)q * n + c], pacc[q][0]);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < K; k++) {
            if constexpr (NP == 4)
                acc[k] -= (pacc[k][0] + pacc[k][1]) + (pacc[k][2] + pacc[k][3]);
            else
                acc[k] -= pacc[k][0];
        }
        __syncwarp();
        // in-tile triangle over the active rows (bottom-up); a lane's accumulators
        // are final after its own step
        const int i_hi = a1 - 1 - row0, i_lo = a0 - row0;
        if (i_hi == 31 && i_lo == 0 && K == 1) {
            // blocks of four rows (i, i-1, i-2, i-3): the four accumulators are
            // broadcast together, every lane resolves the block's four unknowns from
            // the in-block coefficients (uniform loads) and applies all four columns;
            // a lane's own coefficients for columns at or below its row are zero, so
            // lanes inside the block come out with their final values too
#pragma unroll
            for (int i = 31; i >= 3; i -= 4) {
                const T c0 = S.coef[i][lane], c1 = S.coef[i - 1][lane];
                const T c2 = S.coef[i - 2][lane], c3 = S.coef[i - 3][lane];
                const T u10 = S.coef[i][i - 1];
                const T u20 = S.coef[i][i - 2], u21 = S.coef[i - 1][i - 2];
                const T u30 = S.coef[i][i - 3], u31 = S.coef[i - 1][i - 3], u32 = S.coef[i - 2][i - 3];
                const T b0 = __shfl_sync(FULLMASK, acc[0], i), b1 = __shfl_sync(FULLMASK, acc[0], i - 1);
                const T b2 = __shfl_sync(FULLMASK, acc[0], i - 2), b3 = __shfl_sync(FULLMASK, acc[0], i - 3);
                const T a1 = fma(-u10, b0, b1);
                const T a2 = fma(-u21, a1, fma(-u20, b0, b2));
                const T a3 = fma(-u32, a2, fma(-u31, a1, fma(-u30, b0, b3)));
                T t = fma(-c0, b0, acc[0]);
                t = fma(-c1, a1, t);
                t = fma(-c2, a2, t);
                acc[0] = fma(-c3, a3, t);
            }
        } else if (i_hi == 31 && i_lo == 0) {
#pragma unroll
            for (int i = 31; i >= 0; i--) {
                const T ci = S.coef[i][lane];
#pragma unroll
                for (int k = 0; k < K; k++) {
                    const T ai = __shfl_sync(FULLMASK, acc[k], i);
                    acc[k] = fma(-ci, ai, acc[k]);
                }
            }
        } else {
            for (int i = i_hi; i >= i_lo; i--) {
                const T ci = S.coef[i][lane];
#pragma unroll
                for (int k = 0; k < K; k++) {
                    const T ai = __shfl_sync(FULLMASK, acc[k], i);
                    acc[k] = fma(-ci, ai, acc[k]);
                }
            }
        }
        // leave the coefficient tile zero for the next tile
#pragma unroll
        for (int i = 0; i < 32; i++) S.coef[i][lane] = T(0);
        if (act) {
            const long long o = A.rev_out ? n - 1 - row : row;
#pragma unroll
            for (int k = 0; k < K; k++) {
                const T xv = acc[k] * rd;
                xout[k * A.ldx + o] = (TO)xv;
                S.win[k][row & (W - 1)] = xv;
            }
        }
        __syncwarp();
        p_hi = p_lo;
        p_lo = p_next;
        p_next = p_next2;
#pragma unroll
        for (int k = 0; k < K; k++) rhs_c[k] = rhs_n[k];
    }
    return true;
}

// Copy rows [lo, hi) of the phase-1 values into the output and the window.
template <int K, typename T, typename TO>
__device__ void tile_copy_rows(const TileArgs &A, TileSmemK<K, T> &S, int lo, int hi) {
    constexpr int W = TileCfg<K, T>::kWinR;
    const int lane = threadIdx.x & 31;
    const T *xfix = (const T *)A.xfix;
    TO *xout = (TO *)A.xout;
    for (int r0 = lo; r0 < hi; r0 += 32 * 8) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            T v[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int r = r0 + 32 * u + lane;
                v[u] = r < hi ? xfix[(long long)k * A.n + r] : T(0);
            }
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int r = r0 + 32 * u + lane;
                if (r < hi) {
                    xout[k * A.ldx + (A.rev_out ? A.n - 1 - r : r)] = (TO)v[u];
                    if (r < lo + W) S.win[k][r & (W - 1)] = v[u];
                }
            }
        }
    }
    __syncwarp();
}

template <bool FULL, int K, typename T, typename TO>
__device__ __forceinline__ void tile_task(const TileArgs &A, int task) {
    __shared__ TileSmemK<K, T> S;
    if (task >= A.ntasks) return;
    const int lane = threadIdx.x;
    if (A.fail_entry) {
        if (lane == 0) atomicExch(A.err, 1);
        return;
    }
    if (lane == 0) {
        mbar_init(&S.bar[0], 1);
        mbar_init(&S.bar[1], 1);
        fence_mbar_init();
    }
#pragma unroll
    for (int i = 0; i < 33; i++) S.coef[i][lane] = T(0);
    __syncwarp();
    unsigned phase = 0u;
    const SegTask t = A.tasks[task];
    if (FULL && t.tail > t.hi) tile_copy_rows<K, T, TO>(A, S, t.hi, t.tail);
    if (t.skip_hi > t.skip_lo) {
        if (!tile_range<FULL, K, T, TO>(A, S, phase, t.skip_hi, t.hi, t.hi)) return;
        tile_copy_rows<K, T, TO>(A, S, t.skip_lo, t.skip_hi);
        tile_range<FULL, K, T, TO>(A, S, phase, t.lo, t.skip_lo, t.hi);
    } else {
        tile_range<FULL, K, T, TO>(A, S, phase, t.lo, t.hi, t.hi);
    }
}

template <bool FULL, int K, typename T, typename TO>
__global__ void __launch_bounds__(32) k_tile_solve(TileArgs A) {
    tile_task<FULL, K, T, TO>(A, blockIdx.x);
}

// Many systems in one launch: block b solves task work[b].y of the system
// whose arguments are args[work[b].x] (a flat work list, longest tasks first).
template <bool FULL, int K, typename T, typename TO>
__global__ void __launch_bounds__(32) k_tile_multi(const TileArgs *__restrict__ args, const int2 *__restrict__ work) {
    const int2 w = work[blockIdx.x];
    const TileArgs A = args[w.x];
    tile_task<FULL, K, T, TO>(A, w.y);
}

// ---- right-hand-side-parallel tile solver (batches of up to 32) -----------------
//
// Lane k owns right-hand side k and walks the rows of the task bottom-up; the
// row's slots are warp-uniform broadcast loads and there is no cross-lane
// dependency (no chain broadcast).
//
// * A 129-row window in shared memory, indexed [row mod 128][lane], holds x of
//   the solved rows and, for the tile being solved, its right-hand sides
//   (written there, coalesced along rows, before the tile's first row; row r's
//   slot then turns from b_r into x_r).  Writing tile rows row0..row0+31 evicts
//   rows row0+128.., so the window answers for columns c < row0 + 128 (at least
//   r + 97); farther columns of the task read the output in global memory.
//   Window row 128 is zero (padding slots point there).
// * The next tile's slots are bulk-copied (slot-major, as stored) while the
//   current tile is solved, then transposed to row-major so that a row's slots
//   are a few 16-byte broadcast loads.  A tile whose columns all fall inside
//   the window (the common case) stores window offsets instead of columns and
//   runs the branch-free path, unrolled for its width class (4, 8, 16 slots)
//   with the next row's slots loaded ahead.
// * The next tile's right-hand sides are loaded into registers while the
//   current tile is solved.  Lanes k >= nk idle (no global access).

constexpr int kRhsWin = 128;  // window rows (power of two)
constexpr int kRhsCap = 16;   // transposed slots per row; wider tiles run the general path
constexpr int kRhsLd = 33;    // window row stride (elements)

template <typename T>
struct RhsSmem {
    alignas(128) T v[kRhsCap * 32];   // next tile, slot-major
    alignas(128) int c[kRhsCap * 32];
    alignas(128) T rdn[32];
    alignas(16) int rc[33][kRhsCap];  // current tile, row l at l + 1: window offsets (fast) or columns (-1: padding)
    alignas(16) T rv[33][kRhsCap];
    T rv0[33];  // fast tiles: coefficient of column row + 1 (taken out of rc/rv), row l at l + 1
    T rd[32];
    T win[kRhsWin + 1][kRhsLd];
    alignas(8) unsigned long long bar;
};

template <typename T>
__device__ __forceinline__ void stage_rhs_tile(const TileArgs &A, RhsSmem<T> &S, int j, int e0, int e1) {
    const unsigned ne = (unsigned)min(e1 - e0, kRhsCap * 32);
    fence_proxy_async();
    mbar_arrive_expect_tx(&S.bar, 32u * sizeof(T) + ne * (unsigned)(sizeof(T) + 4));
    bulk_g2s(S.rdn, (const T *)A.rdiag + 32ll * j, 32u * sizeof(T), &S.bar);
    if (ne) {
        bulk_g2s(S.v, (const T *)A.ell_val + e0, ne * (unsigned)sizeof(T), &S.bar);
        bulk_g2s(S.c, A.ell_col + e0, ne * 4u, &S.bar);
    }
}

// Right-hand sides of tile row row0 + lane for the rows in [a0, a1) (other
// lanes load row a0 and their values go unused; columns k >= nk repeat column
// nk - 1).  Unconditional and kept as loaded (FP64), so that the loads stay in
// flight until the next tile consumes them.
__device__ __forceinline__ void load_rhs_tile(const TileArgs &A, int row0, int a0, int a1, int nk, double (&nb)[32]) {
    int row = row0 + (threadIdx.x & 31);
    if (row < a0 || row >= a1) row = a0;
    const long long o = A.rev_in ? A.n - 1 - row : row;
    const double *src = A.rhs + o;
#pragma unroll
    for (int k = 0; k < 32; k++) nb[k] = src[min(k, nk - 1) * A.ldb];
}

// x of column c > r for lane's right-hand side: window below wlim, the task's
// output below hi_ext, the phase-1 values (FULL) or zero beyond.
template <bool FULL, typename T, typename TO>
__device__ __forceinline__ T rhs_x(const TileArgs &A, const RhsSmem<T> &S, int c, int wlim, int hi_ext, bool act) {
    const int lane = threadIdx.x & 31;
    if (c < wlim) return S.win[c & (kRhsWin - 1)][lane];
    if (!act) return T(0);
    if (c < hi_ext) return (T)((const TO *)A.xout)[lane * A.ldx + (A.rev_out ? A.n - 1 - c : c)];
    return FULL ? ((const T *)A.xfix)[(long long)lane * A.n + c] : T(0);
}

template <int W, typename T>
__device__ __forceinline__ void rhs_row_slots(const RhsSmem<T> &S, int lp1, int (&ci)[W], T (&cv)[W]) {
#pragma unroll
    for (int i = 0; i < W; i += 4) {
        const int4 c4 = *reinterpret_cast<const int4 *>(&S.rc[lp1][i]);
        ci[i] = c4.x;
        ci[i + 1] = c4.y;
        ci[i + 2] = c4.z;
        ci[i + 3] = c4.w;
    }
    if constexpr (sizeof(T) == 8) {
#pragma unroll
        for (int i = 0; i < W; i += 2) {
            const double2 v2 = *reinterpret_cast<const double2 *>(&S.rv[lp1][i]);
            cv[i] = v2.x;
            cv[i + 1] = v2.y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < W; i += 4) {
            const float4 v4 = *reinterpret_cast<const float4 *>(&S.rv[lp1][i]);
            cv[i] = v4.x;
            cv[i + 1] = v4.y;
            cv[i + 2] = v4.z;
            cv[i + 3] = v4.w;
        }
    }
}

// One row of a fast tile in registers: slot offsets and values, the window
// values they point at, b (the row's own window slot), the coefficient of the
// column row + 1 and 1/diagonal.
template <int W, typename T>
struct RhsRow {
    int ci[W];
    T cv[W];
    T xv[W];
    T b, v0, rd;
};

// Issue the loads of row r (tile row l).  The window loads run before x of row
// r + 1 is stored: that column is the separate v0 term, every other column is
// at least r + 2 and already in the window.
template <int W, typename T>
__device__ __forceinline__ void rhs_fetch(const RhsSmem<T> &S, int l, int r, RhsRow<W, T> &R) {
    const int lane = threadIdx.x & 31;
    const T *wf = &S.win[0][0];
    rhs_row_slots<W, T>(S, l + 1, R.ci, R.cv);
#pragma unroll
    for (int i = 0; i < W; i++) R.xv[i] = wf[R.ci[i] + lane];
    R.b = wf[(r & (kRhsWin - 1)) * kRhsLd + lane];
    R.v0 = S.rv0[l + 1];
    R.rd = S.rd[l & 31];
}

// x_r from the fetched row and x_{r+1} (register); stores it in the window.
template <int W, typename T>
__device__ __forceinline__ T rhs_finish(RhsSmem<T> &S, int r, const RhsRow<W, T> &R, T xnext) {
    const int lane = threadIdx.x & 31;
    T p[4] = {R.b, T(0), T(0), T(0)};
#pragma unroll
    for (int i = 0; i < W; i++) p[i & 3] = fma(-R.cv[i], R.xv[i], p[i & 3]);
    const T x = (((p[1] + p[2]) + p[3]) + fma(-R.v0, xnext, p[0])) * R.rd;
    S.win[r & (kRhsWin - 1)][lane] = x;
    return x;
}

// Rows a1-1 .. a0 of a tile whose slots are window offsets (branch-free),
// software-pipelined one row ahead; two rows per trip so the register sets
// alternate instead of being copied.
template <int W, typename T>
__device__ __forceinline__ void rhs_rows_fast(RhsSmem<T> &S, int row0, int a0, int a1, int wlim) {
    const int lane = threadIdx.x & 31;
    T xnext = a1 < wlim ? S.win[a1 & (kRhsWin - 1)][lane] : T(0);
    RhsRow<W, T> A, B;
    rhs_fetch<W, T>(S, a1 - 1 - row0, a1 - 1, A);
    int r = a1 - 1;
    for (; r - 1 >= a0; r -= 2) {
        rhs_fetch<W, T>(S, r - 1 - row0, r - 1, B);
        xnext = rhs_finish<W, T>(S, r, A, xnext);
        rhs_fetch<W, T>(S, r - 2 - row0, r - 2, A);  // row a0 - 1 at most: the spare row 0 / zero slots
        xnext = rhs_finish<W, T>(S, r - 1, B, xnext);
    }
    if (r >= a0) rhs_finish<W, T>(S, r, A, xnext);
}

// Rows a1-1 .. a0 of any tile: columns (slots >= kRhsCap from global memory),
// window / output / phase-1 lookups per slot.
template <bool FULL, typename T, typename TO>
__device__ void rhs_rows_general(const TileArgs &A, RhsSmem<T> &S, int row0, int a0, int a1, int width, int p_lo,
                                 int wlim, int hi_ext, bool act) {
    const int lane = threadIdx.x & 31;
    const int nst = min(width, kRhsCap);
    const T *vg = (const T *)A.ell_val + p_lo;
    const int *cg = A.ell_col + p_lo;
    for (int r = a1 - 1; r >= a0; r--) {
        const int l = r - row0;
        T *wr = &S.win[r & (kRhsWin - 1)][lane];
        T p0 = *wr, p1 = T(0);
        for (int q = 0; q < width; q++) {
            const int c = q < nst ? S.rc[l + 1][q] : cg[q * 32 + l];
            const T v = q < nst ? S.rv[l + 1][q] : vg[q * 32 + l];
            if (c > r) {
                if (q & 1) p1 = fma(-v, rhs_x<FULL, T, TO>(A, S, c, wlim, hi_ext, act), p1);
                else p0 = fma(-v, rhs_x<FULL, T, TO>(A, S, c, wlim, hi_ext, act), p0);
            }
        }
        *wr = (p0 + p1) * S.rd[l];
    }
}

template <bool FULL, typename T, typename TO>
__device__ bool rhs_range(const TileArgs &A, RhsSmem<T> &S, unsigned &phase, int lo, int hi, int hi_ext, int halo_end,
                          int nk) {
    const int lane = threadIdx.x & 31;
    if (hi <= lo) return true;
    const bool act = lane < nk;
    const int n = A.n;
    TO *xout = (TO *)A.xout;
    const int jt = (hi - 1) >> 5, jb = lo >> 5;
    const int ntiles = jt - jb + 1;
    int p_hi = A.ell_ptr[jt + 1], p_lo = A.ell_ptr[jt];
    int p_next = ntiles > 1 ? A.ell_ptr[jt - 1] : 0;
    __syncwarp();
    if (lane == 0) stage_rhs_tile<T>(A, S, jt, p_lo, p_hi);
    double nb[32];
    load_rhs_tile(A, 32 * jt, max(lo, 32 * jt), hi, nk, nb);
    for (int it = 0; it < ntiles; it++) {
        const int j = jt - it;
        const int row0 = 32 * j;
        const int row = row0 + lane;
        const int a0 = max(lo, row0), a1 = min(hi, row0 + 32);
        const bool mine = row >= a0 && row < a1;
        if (mine) {
            T *w = S.win[row & (kRhsWin - 1)];
#pragma unroll
            for (int k = 0; k < 32; k++) w[k] = (T)nb[k];
        }
        {
            const long long t0 = clock64();
            while (!mbar_try_wait(&S.bar, phase)) {
                if (clock64() - t0 > kWaitCycles) {
                    drain_copy(&S.bar, phase);
                    if (lane == 0) atomicExch(A.err, 1);
                    return false;
                }
            }
            phase ^= 1u;
        }
        // transpose the staged tile to row-major (lane = row)
        const int width = (p_hi - p_lo) >> 5;
        const int nst = min(width, kRhsCap);
        const int wlim = min(row0 + kRhsWin, FULL ? halo_end : hi_ext);
        int cl[kRhsCap];
        T vl[kRhsCap];
        bool local = true;
#pragma unroll
        for (int q = 0; q < kRhsCap; q++) {
            cl[q] = q < nst ? S.c[q * 32 + lane] : -1;
            vl[q] = q < nst ? S.v[q * 32 + lane] : T(0);
            if (cl[q] == row || (!FULL && cl[q] >= hi_ext)) cl[q] = -1;  // padding; phase 1: no coupling
            if (mine && cl[q] >= wlim) local = false;
        }
        const bool fast = __all_sync(0xffffffffu, local) && width <= kRhsCap;
        T v0 = T(0);
        if (fast) {
#pragma unroll
            for (int q = 0; q < kRhsCap; q++)
                if (cl[q] == row + 1) {
                    v0 = vl[q];
                    cl[q] = -1;
                    vl[q] = T(0);
                }
        }
        S.rv0[lane + 1] = v0;
#pragma unroll
        for (int q = 0; q < kRhsCap; q += 4) {
            int4 o;
            int *op = &o.x;
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int c = cl[q + u];
                op[u] = fast ? (c < 0 ? kRhsWin * kRhsLd : (c & (kRhsWin - 1)) * kRhsLd) : c;
            }
            *reinterpret_cast<int4 *>(&S.rc[lane + 1][q]) = o;
        }
        if constexpr (sizeof(T) == 8) {
#pragma unroll
            for (int q = 0; q < kRhsCap; q += 2)
                *reinterpret_cast<double2 *>(&S.rv[lane + 1][q]) = make_double2(vl[q], vl[q + 1]);
        } else {
#pragma unroll
            for (int q = 0; q < kRhsCap; q += 4)
                *reinterpret_cast<float4 *>(&S.rv[lane + 1][q]) = make_float4(vl[q], vl[q + 1], vl[q + 2], vl[q + 3]);
        }
        S.rd[lane] = S.rdn[lane];
        __syncwarp();
        int p_next2 = 0;
        if (it + 1 < ntiles) {
            if (lane == 0) stage_rhs_tile<T>(A, S, j - 1, p_next, p_lo);
            if (it + 2 < ntiles) p_next2 = A.ell_ptr[j - 2];
            load_rhs_tile(A, row0 - 32, max(lo, row0 - 32), row0, nk, nb);
        }
        double xold[32];  // acc: the tile's current output, loaded while the rows are solved
        if (FULL && A.acc) {
            const long long o = A.rev_out ? n - 1 - (mine ? row : a0) : (mine ? row : a0);
#pragma unroll
            for (int k = 0; k < 32; k++) xold[k] = ((const double *)A.xout)[min(k, nk - 1) * A.ldx + o];
        }
        if (fast) {
            if (width <= 4) rhs_rows_fast<4, T>(S, row0, a0, a1, wlim);
            else if (width <= 8) rhs_rows_fast<8, T>(S, row0, a0, a1, wlim);
            else rhs_rows_fast<16, T>(S, row0, a0, a1, wlim);
        } else {
            rhs_rows_general<FULL, T, TO>(A, S, row0, a0, a1, width, p_lo, wlim, hi_ext, act);
        }
        __syncwarp();
        if (mine) {
            const long long o = A.rev_out ? n - 1 - row : row;
            const T *w = S.win[row & (kRhsWin - 1)];
#pragma unroll
            for (int k = 0; k < 32; k++)
                if (k < nk) xout[k * A.ldx + o] = (FULL && A.acc) ? (TO)(xold[k] + (double)w[k]) : (TO)w[k];
        }
        __syncwarp();
        p_hi = p_lo;
        p_lo = p_next;
        p_next = p_next2;
    }
    return true;
}

// Phase-1 values of rows [lo, hi) (the rows above a task, which its couplings
// read) into the window.
template <typename T>
__device__ void rhs_load_halo(const TileArgs &A, RhsSmem<T> &S, int lo, int hi, int nk) {
    const int lane = threadIdx.x & 31;
    const T *xfix = (const T *)A.xfix;
    for (int r0 = lo; r0 < hi; r0 += 32) {
        const int r = r0 + lane;
        const bool ok = r < hi;
        T v[32];
#pragma unroll
        for (int k = 0; k < 32; k++) v[k] = (ok && k < nk) ? xfix[(long long)k * A.n + r] : T(0);
        if (ok) {
            T *w = S.win[r & (kRhsWin - 1)];
#pragma unroll
            for (int k = 0; k < 32; k++) w[k] = v[k];
        }
    }
    __syncwarp();
}

// Copy rows [lo, hi) of the phase-1 values into the output and the window, 32
// rows (lane = row) by all right-hand sides per step, loads ahead of stores.
template <typename T, typename TO>
__device__ void rhs_copy_rows(const TileArgs &A, RhsSmem<T> &S, int lo, int hi, int nk) {
    const int lane = threadIdx.x & 31;
    const T *xfix = (const T *)A.xfix;
    TO *xout = (TO *)A.xout;
    for (int r0 = lo; r0 < hi; r0 += 32) {
        const int r = r0 + lane;
        const bool ok = r < hi;
        T v[32];
        double old[32];
        const long long o = A.rev_out ? A.n - 1 - (ok ? r : lo) : (ok ? r : lo);
#pragma unroll
        for (int k = 0; k < 32; k++) v[k] = (ok && k < nk) ? xfix[(long long)k * A.n + r] : T(0);
        if (A.acc) {
#pragma unroll
            for (int k = 0; k < 32; k++) old[k] = ((const double *)A.xout)[min(k, nk - 1) * A.ldx + o];
        }
        if (ok) {
#pragma unroll
            for (int k = 0; k < 32; k++)
                if (k < nk) xout[k * A.ldx + o] = A.acc ? (TO)(old[k] + (double)v[k]) : (TO)v[k];
            if (r < lo + kRhsWin) {
                T *w = S.win[r & (kRhsWin - 1)];
#pragma unroll
                for (int k = 0; k < 32; k++) w[k] = v[k];
            }
        }
    }
    __syncwarp();
}

template <bool FULL, typename T, typename TO>
__global__ void __launch_bounds__(32) k_rhs_solve(TileArgs A, int nk) {
    __shared__ RhsSmem<T> S;
    const int task = blockIdx.x;
    if (task >= A.ntasks) return;
    const int lane = threadIdx.x;
    if (A.fail_entry) {
        if (lane == 0) atomicExch(A.err, 1);
        return;
    }
    if (lane == 0) {
        mbar_init(&S.bar, 1);
        fence_mbar_init();
    }
    S.win[kRhsWin][lane] = T(0);
#pragma unroll
    for (int q = 0; q < kRhsCap; q += 4) *reinterpret_cast<int4 *>(&S.rc[0][q]) = make_int4(0, 0, 0, 0);
    if (lane < kRhsCap) S.rv[0][lane] = T(0);
    if (lane == 0) S.rv0[0] = T(0);
    __syncwarp();
    unsigned phase = 0u;
    const SegTask t = A.tasks[task];
    // phase 3+4: the rows above the task (3 tiles) come from the phase-1 values
    const int halo_end = FULL ? min(A.n, t.hi + kRhsWin - 32) : t.hi;
    if (FULL) rhs_load_halo<T>(A, S, t.hi, halo_end, nk);
    if (FULL && t.tail > t.hi) rhs_copy_rows<T, TO>(A, S, t.hi, t.tail, nk);
    if (t.skip_hi > t.skip_lo) {
        if (!rhs_range<FULL, T, TO>(A, S, phase, t.skip_hi, t.hi, t.hi, halo_end, nk)) return;
        rhs_copy_rows<T, TO>(A, S, t.skip_lo, t.skip_hi, nk);
        rhs_range<FULL, T, TO>(A, S, phase, t.lo, t.skip_lo, t.hi, halo_end, nk);
    } else {
        rhs_range<FULL, T, TO>(A, S, phase, t.lo, t.hi, t.hi, halo_end, nk);
    }
}

// sliced-ELL construction: widths per tile, then slots (padding: value 0, column = row)
__global__ void k_ell_width(int n, const int *__restrict__ ia, int *__restrict__ width) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int len = r < n ? ia[r + 1] - ia[r] - 1 : 0;
    int w = len;
#pragma unroll
    for (int o = 16; o; o >>= 1) w = max(w, __shfl_xor_sync(0xffffffffu, w, o));
    if ((threadIdx.x & 31) == 0 && (r >> 5) < (n + 31) / 32) width[r >> 5] = w * 32;
}

__global__ void k_ell_fill(int n, int ntiles, const int *__restrict__ ia, const int *__restrict__ ja,
                           const double *__restrict__ a, const int *__restrict__ ptr, double *__restrict__ ev,
                           int *__restrict__ ec) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = r >> 5, l = r & 31;
    if (j >= ntiles) return;
    const int width = (ptr[j + 1] - ptr[j]) >> 5;
    const int b = r < n ? ia[r] + 1 : 0, len = r < n ? ia[r + 1] - ia[r] - 1 : 0;
    const int self = r < n ? r : n - 1;
    for (int k = 0; k < width; k++) {
        const long long o = (long long)ptr[j] + 32 * k + l;
        if (k < len) {
            ev[o] = a[b + k];
            ec[o] = ja[b + k];
        } else {
            ev[o] = 0.0;
            ec[o] = self;
        }
    }
}

// ---- internal spikes for coupled blocks the reference gives no spike --------------
//
// For rows [ps, rl] of a block (rl = its last coupling row), x - y = -W x_c with
// W = D^{-1} R over the block's rows [ps, rl] (D: entries at columns <= rl; R:
// entries at the coupling columns >= pe, compressed to the distinct ones).  Rows
// whose W row sums to <= tau keep the block-local value in phase 4.  One thread
// per coupling column sweeps the rows bottom-up; W lives in a scratch matrix.

__global__ void k_aux_sweep(int ps, int rl, int pe, const int *__restrict__ ia, const int *__restrict__ ja,
                            const double *__restrict__ a, const int *__restrict__ cols, int ncols,
                            double *__restrict__ W) {
    for (int j = threadIdx.x; j < ncols; j += blockDim.x) {
        const int cj = cols[j];
        for (int r = rl; r >= ps; r--) {
            const int b = ia[r], e = ia[r + 1];
            // coupling entry (r, cj), if any: binary search in the row's sorted columns
            int lo = b, hi = e;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (ja[mid] < cj) lo = mid + 1; else hi = mid;
            }
            double acc = (lo < e && ja[lo] == cj) ? a[lo] : 0.0;
            for (int q = b + 1; q < e; q++) {
                const int c = ja[q];
                if (c > rl) break;
                acc -= a[q] * W[(long long)(c - ps) * ncols + j];
            }
            W[(long long)(r - ps) * ncols + j] = acc / a[b];
        }
    }
}

__global__ void k_aux_first(int rows, int ncols, const double *__restrict__ W, double tau, int *__restrict__ first) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    double s = 0.0;
    for (int j = 0; j < ncols; j++) s += fabs(W[(long long)r * ncols + j]);
    if (s > tau) atomicMin(first, r);
}

// max(m, v) for norms that must not lose a NaN: once either operand is NaN the
// result is NaN (fmax would drop it and let a failed solve look converged)
__device__ __forceinline__ double nanmax(double m, double v) { return (v > m || v != v) ? v : m; }

// ---- batched solve support --------------------------------------------------------

// Reduced solve on the kept rows for K right-hand sides stored in T with FP64
// accumulation (same level structure as k_reduced_solve).  With FP32 storage and
// an FP64 scratch `red` ([K][nred]), the reduced unknowns are gathered into it,
// every level is solved and stored in FP64, and they are rounded to T once, on
// the way back: the coupled boundary system stays FP64 throughout.
template <int K>
constexpr int red_threads() { return K >= 16 ? 512 : 1024; }  // K >= 16: registers for the K sums

template <int K, typename T>
__device__ __forceinline__ void reduced_body(const int *__restrict__ rows, const int *__restrict__ lvl_off, int nlvl,
                                             const int *__restrict__ mapRedX, const int *__restrict__ IT,
                                             const int *__restrict__ JT, const double *__restrict__ Tv,
                                             T *__restrict__ xbuf, int n, double *__restrict__ red, int nred) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    if (red) {
        for (long long e = threadIdx.x; e < (long long)K * nred; e += blockDim.x) {
            const int k = (int)(e / nred), i = (int)(e % nred);
            red[e] = (double)xbuf[(long long)k * n + mapRedX[i]];
        }
        __syncthreads();
        for (int li = 0; li < nlvl; li++) {
            for (int q = lvl_off[li] + warp; q < lvl_off[li + 1]; q += nwarps) {
                const int kr = rows[q];
                double sum[K];
#pragma unroll
                for (int k = 0; k < K; k++) sum[k] = 0.0;
                for (int j = IT[kr] + lane; j < IT[kr + 1]; j += 32) {
                    const int c = JT[j];
#pragma unroll
                    for (int k = 0; k < K; k++) sum[k] = fma(Tv[j], red[(long long)k * nred + c], sum[k]);
                }
#pragma unroll
                for (int k = 0; k < K; k++) {
#pragma unroll
                    for (int o = 16; o; o >>= 1) sum[k] += __shfl_xor_sync(0xffffffffu, sum[k], o);
                }
                if (lane == 0) {
#pragma unroll
                    for (int k = 0; k < K; k++) red[(long long)k * nred + kr] -= sum[k];
                }
            }
            __syncthreads();
        }
        for (long long e = threadIdx.x; e < (long long)K * nred; e += blockDim.x) {
            const int k = (int)(e / nred), i = (int)(e % nred);
            xbuf[(long long)k * n + mapRedX[i]] = (T)red[e];
        }
        return;
    }
    for (int li = 0; li < nlvl; li++) {
        for (int q = lvl_off[li] + warp; q < lvl_off[li + 1]; q += nwarps) {
            const int kr = rows[q];
            double sum[K];
#pragma unroll
            for (int k = 0; k < K; k++) sum[k] = 0.0;
            for (int j = IT[kr] + lane; j < IT[kr + 1]; j += 32) {
                const int c = mapRedX[JT[j]];
#pragma unroll
                for (int k = 0; k < K; k++) sum[k] = fma(Tv[j], (double)xbuf[(long long)k * n + c], sum[k]);
            }
#pragma unroll
            for (int k = 0; k < K; k++) {
#pragma unroll
                for (int o = 16; o; o >>= 1) sum[k] += __shfl_xor_sync(0xffffffffu, sum[k], o);
            }
            if (lane == 0) {
                const long long r = mapRedX[kr];
#pragma unroll
                for (int k = 0; k < K; k++) xbuf[k * (long long)n + r] = (T)((double)xbuf[k * (long long)n + r] - sum[k]);
            }
        }
        __syncthreads();
    }
}

template <int K, typename T>
__global__ void __launch_bounds__(red_threads<K>())
k_reduced_solve_k(const int *__restrict__ rows, const int *__restrict__ lvl_off, int nlvl,
                  const int *__restrict__ mapRedX, const int *__restrict__ IT, const int *__restrict__ JT,
                  const double *__restrict__ Tv, T *__restrict__ xbuf, int n, double *__restrict__ red, int nred) {
    reduced_body<K, T>(rows, lvl_off, nlvl, mapRedX, IT, JT, Tv, xbuf, n, red, nred);
}

// Reduced solves of many systems: block b takes the system of args[list[b]].
struct RedArgs {
    const int *rows, *lvl_off;
    int nlvl;
    const int *mapRedX, *IT, *JT;
    const double *Tv;
    void *xbuf;  // T
    int n;
    double *red;  // FP64 reduced unknowns of an FP32 batch ([K][nred]), or null
    int nred;
};

template <int K, typename T>
__global__ void __launch_bounds__(red_threads<K>()) k_reduced_multi(const RedArgs *__restrict__ args) {
    const RedArgs A = args[blockIdx.x];
    reduced_body<K, T>(A.rows, A.lvl_off, A.nlvl, A.mapRedX, A.IT, A.JT, A.Tv, (T *)A.xbuf, A.n, A.red, A.nred);
}

// R = B - A X in FP64 on the ELL copy (plus the diagonal), in the caller's order
// (rev: caller row i is U row n-1-i).  One thread per row; a warp covers a tile.
template <int K>
__device__ __forceinline__ void residual_row(int r, int n, const int *__restrict__ ptr, const double *__restrict__ ev,
                                             const int *__restrict__ ec, const double *__restrict__ diag,
                                             const double *__restrict__ X, long long ldx,
                                             const double *__restrict__ B, long long ldb, double *__restrict__ R,
                                             long long ldr, int rev) {
    if (r >= n) return;
    const int j = r >> 5;
    const int w = (ptr[j + 1] - ptr[j]) >> 5;
    const long long base = ptr[j] + (r & 31);
    const long long orow = rev ? n - 1 - r : r;
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = diag[r] * X[k * ldx + orow];
    for (int q = 0; q < w; q++) {
        const int c = ec[base + 32ll * q];
        const double v = ev[base + 32ll * q];
        const long long oc = rev ? n - 1 - c : c;
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] = fma(v, X[k * ldx + oc], acc[k]);
    }
#pragma unroll
    for (int k = 0; k < K; k++) R[k * ldr + orow] = B[k * ldb + orow] - acc[k];
}

template <int K>
__global__ void k_residual(int n, const int *__restrict__ ptr, const double *__restrict__ ev,
                           const int *__restrict__ ec, const double *__restrict__ diag,
                           const double *__restrict__ X, long long ldx, const double *__restrict__ B,
                           long long ldb, double *__restrict__ R, long long ldr, int rev) {
    residual_row<K>(blockIdx.x * blockDim.x + threadIdx.x, n, ptr, ev, ec, diag, X, ldx, B, ldb, R, ldr, rev);
}

// Residuals (and, with `norms`, per-column max |R|, |X|, |B|) and X += D of many
// systems: block b covers rows 256 * work[b].y .. of the system args[work[b].x].
struct VecArgs {
    int n, rev;
    const int *ptr;
    const double *ev;
    const int *ec;
    const double *diag;
    double *X;
    long long ldx;
    const double *B;
    long long ldb;
    double *R;  // residual (ld n)
    const double *D;  // correction (ld n)
    unsigned long long *norms;  // 3 per column
};

template <int K>
__global__ void __launch_bounds__(256) k_residual_multi(const VecArgs *__restrict__ args, const int2 *__restrict__ work,
                                                       int with_norms) {
    const int2 w = work[blockIdx.x];
    const VecArgs &A = args[w.x];
    const int r = w.y * 256 + threadIdx.x;
    residual_row<K>(r, A.n, A.ptr, A.ev, A.ec, A.diag, A.X, A.ldx, A.B, A.ldb, A.R, A.n, A.rev);
    if (!with_norms) return;
    const long long o = A.rev ? A.n - 1 - (long long)min(r, A.n - 1) : min(r, A.n - 1);
#pragma unroll
    for (int k = 0; k < K; k++) {
        double mr = 0, mx = 0, mb = 0;
        if (r < A.n) {
            mr = fabs(A.R[k * (long long)A.n + o]);
            mx = fabs(A.X[k * A.ldx + o]);
            mb = fabs(A.B[k * A.ldb + o]);
        }
#pragma unroll
        for (int s = 16; s; s >>= 1) {
            mr = nanmax(mr, __shfl_xor_sync(0xffffffffu, mr, s));
            mx = nanmax(mx, __shfl_xor_sync(0xffffffffu, mx, s));
            mb = nanmax(mb, __shfl_xor_sync(0xffffffffu, mb, s));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMax(&A.norms[3 * k + 0], __double_as_longlong(mr));
            atomicMax(&A.norms[3 * k + 1], __double_as_longlong(mx));
            atomicMax(&A.norms[3 * k + 2], __double_as_longlong(mb));
        }
    }
}

template <int K>
__global__ void __launch_bounds__(256) k_axpy_multi(const VecArgs *__restrict__ args, const int2 *__restrict__ work) {
    const int2 w = work[blockIdx.x];
    const VecArgs &A = args[w.x];
    const int r = w.y * 256 + threadIdx.x;
    if (r >= A.n) return;
#pragma unroll
    for (int k = 0; k < K; k++) A.X[k * A.ldx + r] += A.D[k * (long long)A.n + r];
}

// R = B - A X for up to 32 right-hand sides with lane = right-hand side
// (FP64).  A block of kResWarps warps walks a chunk of kResChunk tiles
// top-down (U order).  Each tile's X rows enter a 128-row shared window
// ([row mod 128][lane]; it holds the tile and the 96 rows above, which its
// couplings read), its B rows a 32 x 33 tile that turns into R, its slots a
// slot-major copy; thread (warp w, lane l) moves rows row0 + l of columns
// 8w .. 8w+7 (coalesced along rows) and the next tile's values are loaded into
// registers while the current tile is computed.  The warps split the tile's
// rows.  Columns beyond the window (couplings wider than 96 rows) and slots
// beyond kResCap read global memory.  With norms != nullptr it also folds
// max |R|, max |X|, max |B| per right-hand side into norms[3k..3k+2] (as
// k_norms).
constexpr int kResWarps = 4;
constexpr int kResChunk = 32;  // tiles per block
constexpr int kResCap = 16;    // staged slots per row
constexpr int kResCols = 32 / kResWarps;

struct ResSmem {
    double win[kRhsWin][33];
    double bt[32][33];
    double v[kResCap * 32];
    int c[kResCap * 32];
    double dg[32];
    unsigned long long nrm[kResWarps][3][32];
};

struct ResTile {
    double x[kResCols], b[kResCols];
    double v[kResCap * 32 / (32 * kResWarps)];
    int c[kResCap * 32 / (32 * kResWarps)];
    double dg;
};

__global__ void __launch_bounds__(32 * kResWarps)
k_rhs_residual(int n, int nk, const int *__restrict__ ptr, const double *__restrict__ ev, const int *__restrict__ ec,
               const double *__restrict__ diag, const double *__restrict__ X, long long ldx,
               const double *__restrict__ B, long long ldb, double *__restrict__ R, long long ldr, int rev,
               unsigned long long *__restrict__ norms) {
    extern __shared__ __align__(16) unsigned char res_raw[];
    ResSmem &S = *reinterpret_cast<ResSmem *>(res_raw);
    constexpr int NT = 32 * kResWarps, NS = kResCap * 32 / NT;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ntiles = (n + 31) >> 5;
    const int jb = blockIdx.x * kResChunk, je = min(ntiles, jb + kResChunk);  // tiles [jb, je)
    if (jb >= je) return;
    const int k0 = warp * kResCols;
    auto orow = [&](int r) -> long long { return rev ? (long long)n - 1 - r : r; };
    // halo: X rows [hi, hi + 96) above the chunk
    {
        const int hi = min(n, 32 * je), he = min(n, hi + kRhsWin - 32);
        for (int r = hi + lane; r < he; r += 32)
#pragma unroll
            for (int u = 0; u < kResCols; u++)
                if (k0 + u < nk) S.win[r & (kRhsWin - 1)][k0 + u] = X[(k0 + u) * ldx + orow(r)];
    }
    auto fetch = [&](int j, ResTile &T) {
        const int r = min(32 * j + lane, n - 1);
        const long long o = orow(r);
#pragma unroll
        for (int u = 0; u < kResCols; u++) {
            const int k = min(k0 + u, nk - 1);
            T.x[u] = X[k * ldx + o];
            T.b[u] = B[k * ldb + o];
        }
        const int p0 = ptr[j], ne = min(ptr[j + 1] - p0, kResCap * 32);
#pragma unroll
        for (int i = 0; i < NS; i++) {
            const int e = tid + NT * i;
            T.v[i] = e < ne ? ev[p0 + e] : 0.0;
            T.c[i] = e < ne ? ec[p0 + e] : 0;
        }
        T.dg = diag[min(32 * j + lane, n - 1)];
    };
    ResTile cur;
    fetch(je - 1, cur);
    double mr = 0, mx = 0, mb = 0;
    for (int j = je - 1; j >= jb; j--) {
        const int row0 = 32 * j, rows = min(32, n - row0);
        // current tile into shared memory
        if (lane < rows) {
            double *w = S.win[(row0 + lane) & (kRhsWin - 1)];
#pragma unroll
            for (int u = 0; u < kResCols; u++) {
                w[k0 + u] = cur.x[u];
                S.bt[lane][k0 + u] = cur.b[u];
            }
        }
#pragma unroll
        for (int i = 0; i < NS; i++) {
            S.v[tid + NT * i] = cur.v[i];
            S.c[tid + NT * i] = cur.c[i];
        }
        if (warp == 0) S.dg[lane] = cur.dg;
        const int p0 = ptr[j], width = (ptr[j + 1] - p0) >> 5, nst = min(width, kResCap);
        bool local = width <= kResCap;
#pragma unroll
        for (int i = 0; i < NS; i++) local = local && cur.c[i] < row0 + kRhsWin;
        local = __syncthreads_and(local);
        if (j > jb) fetch(j - 1, cur);
        if (local) {
            // every column inside the window: branch-free slot loop
            const double *wf = &S.win[0][0] + lane;
            for (int l = warp; l < rows; l += kResWarps) {
                const int r = row0 + l;
                double a[4] = {0.0, 0.0, 0.0, 0.0};
                int q = 0;
                for (; q + 4 <= width; q += 4) {
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int c = S.c[(q + u) * 32 + l];
                        a[u] = fma(S.v[(q + u) * 32 + l], wf[(c & (kRhsWin - 1)) * 33], a[u]);
                    }
                }
                for (; q < width; q++) {
                    const int c = S.c[q * 32 + l];
                    a[0] = fma(S.v[q * 32 + l], wf[(c & (kRhsWin - 1)) * 33], a[0]);
                }
                const double xr = wf[(r & (kRhsWin - 1)) * 33];
                const double b = S.bt[l][lane];
                const double res = b - fma(S.dg[l], xr, (a[0] + a[1]) + (a[2] + a[3]));
                S.bt[l][lane] = res;
                mr = nanmax(mr, fabs(res));
                mx = nanmax(mx, fabs(xr));
                mb = nanmax(mb, fabs(b));
            }
        } else
        for (int l = warp; l < rows; l += kResWarps) {
            const int r = row0 + l;
            double a0 = 0.0, a1 = 0.0;
            int q = 0;
            for (; q + 2 <= nst; q += 2) {
                const int c0 = S.c[q * 32 + l], c1 = S.c[(q + 1) * 32 + l];
                const double v0 = S.v[q * 32 + l], v1 = S.v[(q + 1) * 32 + l];
                const double x0 = c0 < row0 + kRhsWin ? S.win[c0 & (kRhsWin - 1)][lane]
                                                      : (lane < nk ? X[lane * ldx + orow(c0)] : 0.0);
                const double x1 = c1 < row0 + kRhsWin ? S.win[c1 & (kRhsWin - 1)][lane]
                                                      : (lane < nk ? X[lane * ldx + orow(c1)] : 0.0);
                a0 = fma(v0, x0, a0);
                a1 = fma(v1, x1, a1);
            }
            for (; q < width; q++) {
                const int c = q < nst ? S.c[q * 32 + l] : ec[p0 + 32 * q + l];
                const double v = q < nst ? S.v[q * 32 + l] : ev[p0 + 32 * q + l];
                const double x = c < row0 + kRhsWin ? S.win[c & (kRhsWin - 1)][lane]
                                                    : (lane < nk ? X[lane * ldx + orow(c)] : 0.0);
                a0 = fma(v, x, a0);
            }
            const double xr = S.win[r & (kRhsWin - 1)][lane];
            const double b = S.bt[l][lane];
            const double res = b - fma(S.dg[l], xr, a0 + a1);
            S.bt[l][lane] = res;
            mr = nanmax(mr, fabs(res));
            mx = nanmax(mx, fabs(xr));
            mb = nanmax(mb, fabs(b));
        }
        __syncthreads();
        if (lane < rows) {
            const long long o = orow(row0 + lane);
#pragma unroll
            for (int u = 0; u < kResCols; u++)
                if (k0 + u < nk) R[(k0 + u) * ldr + o] = S.bt[lane][k0 + u];
        }
        __syncthreads();  // before the next tile rewrites bt, the slots and the window
    }
    if (norms) {
        S.nrm[warp][0][lane] = __double_as_longlong(mr);
        S.nrm[warp][1][lane] = __double_as_longlong(mx);
        S.nrm[warp][2][lane] = __double_as_longlong(mb);
        __syncthreads();
        if (warp == 0 && lane < nk) {
#pragma unroll
            for (int w = 0; w < 3; w++) {
                unsigned long long m = 0;
#pragma unroll
                for (int u = 0; u < kResWarps; u++) m = max(m, S.nrm[u][w][lane]);
                atomicMax(&norms[3 * lane + w], m);
            }
        }
    }
}

// Largest distance from a tile's first row to a column of its slots.
__global__ void k_ell_reach(int ntiles, const int *__restrict__ ptr, const int *__restrict__ col, int *__restrict__ out) {
    const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (j >= ntiles) return;
    int m = 0;
    for (int e = ptr[j] + (threadIdx.x & 31); e < ptr[j + 1]; e += 32) m = max(m, col[e] - 32 * j);
#pragma unroll
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// Per right-hand side: max |R|, max |X|, max |B| (bit patterns of non-negative
// doubles order like the values, so an integer max is exact).
__global__ void k_norms(int n, int nrhs, const double *__restrict__ R, long long ldr, const double *__restrict__ X,
                        long long ldx, const double *__restrict__ B, long long ldb,
                        unsigned long long *__restrict__ out) {
    const int k = blockIdx.y;
    double mr = 0, mx = 0, mb = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        mr = nanmax(mr, fabs(R[k * ldr + i]));
        mx = nanmax(mx, fabs(X[k * ldx + i]));
        mb = nanmax(mb, fabs(B[k * ldb + i]));
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        mr = nanmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
        mx = nanmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        mb = nanmax(mb, __shfl_xor_sync(0xffffffffu, mb, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&out[3 * k + 0], __double_as_longlong(mr));
        atomicMax(&out[3 * k + 1], __double_as_longlong(mx));
        atomicMax(&out[3 * k + 2], __double_as_longlong(mb));
    }
}

// X += D (D column-major with leading dimension n)
__global__ void k_axpy(int n, int nrhs, const double *__restrict__ D, double *__restrict__ X, long long ldx) {
    const int k = blockIdx.y;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        X[k * ldx + i] += D[k * (long long)n + i];
}

__global__ void k_to_float(long long count, const double *__restrict__ src, float *__restrict__ dst) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}

__global__ void k_diag_rowsum(int n, const int *__restrict__ ia, const double *__restrict__ a,
                              double *__restrict__ diag, unsigned long long *__restrict__ anorm) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    double s = 0.0;
    if (r < n) {
        diag[r] = a[ia[r]];
        for (int q = ia[r]; q < ia[r + 1]; q++) s += fabs(a[q]);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) s = fmax(s, __shfl_xor_sync(0xffffffffu, s, o));
    if ((threadIdx.x & 31) == 0) atomicMax(anorm, __double_as_longlong(s));
}

__global__ void k_reciprocal_diag(int n, const int *__restrict__ ia, const double *__restrict__ a,
                                  double *__restrict__ rdiag) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) rdiag[r] = 1.0 / a[ia[r]];
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
    if (h.empty()) return SPK_OK;
    if (d.on_stream) SPK_CUDA(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, d.ord));
    else SPK_CUDA(cudaMemcpy(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return SPK_OK;
}

}  // namespace

// Internal spikes (no counterpart in the reference): coupled blocks the
// reference gives no spike, whose phase-4 range would otherwise not be
// truncated, get the spike of their coupling columns (a one-CTA sweep per
// block); aux_first[t] >= 0: rows [ps, ps + aux_first[t]) keep y.
int aux_spikes(spk_system *s, std::vector<int> &aux_first) {
    const int P = s->P;
    const double tau = s->trunc_tol;
    aux_first.assign(P, -1);
    std::vector<int> hia(s->n + 1);
    bool have_ia = false;
    for (int t = 0; t < P; t++) {
        const Part &p = s->parts[t];
        const bool split = p.hasRefl || p.isOpt;
        const bool banded_trunc = split && p.hasS && p.nRowsS > 0;
        const int rl = p.maxIR;  // last row with a coupling column
        if (banded_trunc || rl < p.ps || rl + 1 - p.ps < 256 || p.pe >= s->n) continue;
        if (!have_ia) {
            SPK_CUDA(cudaMemcpy(hia.data(), s->uia.p, sizeof(int) * (s->n + 1), cudaMemcpyDeviceToHost));
            have_ia = true;
        }
        // distinct coupling columns of rows [ps, rl]
        const int e0 = hia[p.ps], e1 = hia[rl + 1];
        std::vector<int> hja(e1 - e0);
        SPK_CUDA(cudaMemcpy(hja.data(), s->uja.p + e0, sizeof(int) * (e1 - e0), cudaMemcpyDeviceToHost));
        std::vector<int> cols;
        for (int c : hja)
            if (c >= p.pe) cols.push_back(c);
        std::sort(cols.begin(), cols.end());
        cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
        if (cols.empty() || cols.size() > 1024) continue;
        const int rows = rl + 1 - p.ps, nc = (int)cols.size();
        DBuf<int> d_cols(s->stream), d_first(s->stream);
        DBuf<double> W(s->stream);
        SPK_TRY(upload(d_cols, cols));
        SPK_TRY(W.alloc((size_t)rows * nc));
        SPK_TRY(d_first.alloc(1));
        SPK_CUDA(cudaMemcpyAsync(d_first.p, &rows, sizeof(int), cudaMemcpyHostToDevice, s->stream));
        k_aux_sweep<<<1, ((nc + 31) / 32) * 32, 0, s->stream>>>(p.ps, rl, p.pe, s->uia.p, s->uja.p, s->ua.p,
                                                                d_cols.p, nc, W.p);
        k_aux_first<<<blocks_for(rows), 256, 0, s->stream>>>(rows, nc, W.p, tau, d_first.p);
        SPK_CUDA(cudaGetLastError());
        SPK_CUDA(cudaStreamSynchronize(s->stream));  // the stream does not sync with cudaMemcpy
        int f = rows;
        SPK_CUDA(cudaMemcpy(&f, d_first.p, sizeof(int), cudaMemcpyDeviceToHost));
        aux_first[t] = f;
    }
    return SPK_OK;
}

bool aux_candidates(const spk_system *s) {
    for (int t = 0; t < s->P; t++) {
        const Part &p = s->parts[t];
        const bool banded_trunc = (p.hasRefl || p.isOpt) && p.hasS && p.nRowsS > 0;
        const int rl = p.maxIR;
        if (!(banded_trunc || rl < p.ps || rl + 1 - p.ps < 256 || p.pe >= s->n)) return true;
    }
    return false;
}

// The segment task lists of the partition solve from the first significant
// spike rows and the internal spikes.
int build_seg_tasks(spk_system *s, const std::vector<int> &first, const std::vector<int> &aux_first) {
    const int P = s->P;
    std::vector<SegTask> t1, t2;
    long long rows1 = 0, rows2 = 0;
    for (int t = 0; t < P; t++) {
        const Part &p = s->parts[t];
        if (aux_first[t] >= 0) {
            // block-local y over the whole block in phase 1; phase 4 recomputes rows
            // [ps + aux_first, last coupling row] and keeps y elsewhere
            t1.push_back(SegTask{p.ps, p.pe, 0, 0, p.pe});
            rows1 += p.pe - p.ps;
            const int hi = p.maxIR + 1;
            SegTask k{p.ps, hi, p.ps, p.ps + std::min(aux_first[t], hi - p.ps), p.pe};
            rows2 += (hi - p.ps) - (k.skip_hi - k.skip_lo);
            t2.push_back(k);
            continue;
        }
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
    return SPK_OK;
}

int solve_prepare(spk_system *s) {
    const int P = s->P;
    const double tau = s->trunc_tol;
    auto wall_ms = []() {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch())
            .count();
    };
    double lap = wall_ms();
    auto mark = [&](int slot) {
        const double t = wall_ms();
        s->prep_ms[slot] = t - lap;
        lap = t;
    };
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
            DBuf<int> d_pl(s->stream), d_nr(s->stream), d_nc(s->stream), d_first(s->stream);
            DBuf<long long> d_ss(s->stream);
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
    // internal spikes: computed here only when the partition solve is the
    // default one (no chain plan, below); with chains they wait for the first
    // partition-path use (partition_ensure), as only those solves read them
    s->first_sig = first;
    std::vector<int> aux_first(P, -1);
    s->aux_pending = tau >= 0 && s->redNec && aux_candidates(s);
    mark(1);  // first significant spike rows
    SPK_TRY(build_seg_tasks(s, first, aux_first));

    // kept reduced rows, grouped by level in descending partition order
    std::vector<int> lvl(P + 1);
    SPK_CUDA(cudaMemcpy(lvl.data(), s->d_lvl.p, sizeof(int) * (P + 1), cudaMemcpyDeviceToHost));
    std::vector<int> keep(std::max(s->rss, 1), 0);
    if (s->rss > 0) {
        DBuf<int> d_keep(s->stream);
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
    mark(2);  // task lists, reduced levels, buffers
    // 1 / diagonal of U, padded to whole 32-row tiles (staged 256 bytes per tile)
    const int ntiles = (s->n + 31) / 32;
    SPK_TRY(s->rdiag.alloc(32ll * ntiles + 32));
    SPK_CUDA(cudaMemset(s->rdiag.p, 0, sizeof(double) * (32ll * ntiles + 32)));
    k_reciprocal_diag<<<blocks_for(s->n), 256, 0, s->stream>>>(s->n, s->uia.p, s->ua.p, s->rdiag.p);
    SPK_CUDA(cudaGetLastError());
    // sliced ELL of the off-diagonals; kept when padding stays within 2x the off-diagonals
    {
        DBuf<int> width(s->stream);
        SPK_TRY(width.alloc(ntiles + 1));
        SPK_CUDA(cudaMemsetAsync(width.p, 0, sizeof(int) * (ntiles + 1), s->stream));
        k_ell_width<<<blocks_for(32ll * ntiles), 256, 0, s->stream>>>(s->n, s->uia.p, width.p);
        SPK_CUDA(cudaGetLastError());
        std::vector<int> hw(ntiles + 1);
        SPK_CUDA(cudaStreamSynchronize(s->stream));
        SPK_CUDA(cudaMemcpy(hw.data(), width.p, sizeof(int) * ntiles, cudaMemcpyDeviceToHost));
        std::vector<int> ptr(ntiles + 1, 0);
        long long tot = 0;
        for (int j = 0; j < ntiles; j++) {
            ptr[j] = (int)std::min<long long>(tot, 2147483647ll);
            tot += hw[j];
        }
        const long long offdiag = (long long)s->nnz - s->n;
        const char *no_ell = getenv("SPK_DISABLE_ELL");  // test hook: force the CSR segment solver
        s->ell_ok = tot < 2147483647ll && tot <= 2 * std::max<long long>(offdiag, 1) + 32ll * ntiles &&
                    !(no_ell && no_ell[0] == '1');
        if (s->ell_ok) {
            ptr[ntiles] = (int)tot;
            SPK_TRY(upload(s->ell_ptr, ptr));
            SPK_TRY(s->ell_val.alloc(std::max<long long>(tot, 1)));
            SPK_TRY(s->ell_col.alloc(std::max<long long>(tot, 1)));
            k_ell_fill<<<blocks_for(32ll * ntiles), 256, 0, s->stream>>>(s->n, ntiles, s->uia.p, s->uja.p, s->ua.p,
                                                                         s->ell_ptr.p, s->ell_val.p, s->ell_col.p);
            SPK_CUDA(cudaGetLastError());
        } else {
            s->ell_val.release();
            s->ell_col.release();
            s->ell_ptr.release();
        }
        s->ell_entries = s->ell_ok ? tot : 0;
    }
    SPK_CUDA(cudaStreamSynchronize(s->stream));
    SPK_TRY(s->d_err.alloc(1));
    SPK_CUDA(cudaMemset(s->d_err.p, 0, sizeof(int)));
    mark(3);  // 1/diagonal, sliced ELL
    SPK_TRY(chain_prepare(s));
    if (!s->chain_ok) SPK_TRY(partition_ensure(s));
    mark(4);  // chain layout, spikes and plans (or the internal spikes without chains)
    return SPK_OK;
}

// Internal spikes and the task lists that use them, before the first solve on
// the partition path (a no-op once done, or when no block needs them).
int partition_ensure(spk_system *s) {
    if (!s->aux_pending) return SPK_OK;
    std::vector<int> aux_first;
    SPK_TRY(aux_spikes(s, aux_first));
    SPK_TRY(build_seg_tasks(s, s->first_sig, aux_first));
    s->aux_pending = 0;
    return SPK_OK;
}

namespace {

// One Spike solve of K right-hand sides with the tile solver: phase 1 into the
// U-order work buffer (T, leading dimension n), the kept reduced rows, phase 3+4
// into xo (FP64, caller order).
template <int K, typename T>
int launch_tiles(spk_system *s, const double *rhs, long long ldb, double *xo, long long ldx, T *work,
                 cudaStream_t st, bool prof, int ring) {
    TileArgs A{};
    A.ell_val = sizeof(T) == 8 ? (const void *)s->ell_val.p : (const void *)s->ell_valf.p;
    A.ell_col = s->ell_col.p;
    A.ell_ptr = s->ell_ptr.p;
    A.rdiag = sizeof(T) == 8 ? (const void *)s->rdiag.p : (const void *)s->rdiagf.p;
    A.n = s->n;
    A.rhs = rhs;
    A.ldb = ldb;
    A.rev_in = s->uplo == 'L';
    A.err = s->d_err.p;
    A.fail_entry = s->dbg_fail_waits > 0;
    if (s->redNec && s->ntasks1) {
        A.tasks = s->d_tasks1.p;
        A.ntasks = s->ntasks1;
        A.xfix = nullptr;
        A.xout = work;
        A.ldx = s->n;
        A.rev_out = 0;
        k_tile_solve<false, K, T, T><<<s->ntasks1, 32, 0, st>>>(A);
        SPK_CUDA(cudaGetLastError());
        s->launches++;
    }
    if (prof) cudaEventRecord(s->ev[ring][1], st);
    if (s->redNec && s->nkept) {
        k_reduced_solve_k<K, T><<<1, red_threads<K>(), 0, st>>>(s->d_red_rows.p, s->d_red_off.p, s->nlvl, s->mapRedX.p,
                                                     s->IT.p, s->JT.p, s->T.p, work, s->n,
                                                     sizeof(T) == 4 ? s->red_scratch : nullptr, s->nRed);
        SPK_CUDA(cudaGetLastError());
        s->launches++;
    }
    if (prof) cudaEventRecord(s->ev[ring][2], st);
    A.tasks = s->d_tasks2.p;
    A.ntasks = s->ntasks2;
    A.xfix = work;
    A.xout = xo;
    A.ldx = ldx;
    A.rev_out = s->uplo == 'L';
    k_tile_solve<true, K, T, double><<<s->ntasks2, 32, 0, st>>>(A);
    SPK_CUDA(cudaGetLastError());
    s->launches++;
    return SPK_OK;
}

template <typename T>
int launch_tiles_k(spk_system *s, int K, const double *rhs, long long ldb, double *xo, long long ldx, T *work,
                   cudaStream_t st) {
    switch (K) {
        case 1: return launch_tiles<1, T>(s, rhs, ldb, xo, ldx, work, st, false, 0);
        case 2: return launch_tiles<2, T>(s, rhs, ldb, xo, ldx, work, st, false, 0);
        case 4: return launch_tiles<4, T>(s, rhs, ldb, xo, ldx, work, st, false, 0);
        case 8: return launch_tiles<8, T>(s, rhs, ldb, xo, ldx, work, st, false, 0);
        case 16: return launch_tiles<16, T>(s, rhs, ldb, xo, ldx, work, st, false, 0);
    }
    set_error(SPK_ERR_ARG, "unsupported batch width %d", K);
    return SPK_ERR_ARG;
}

// One Spike solve of nk <= 32 right-hand sides with the right-hand-side-parallel
// solver; work holds 32 columns (leading dimension n).
template <typename T>
int launch_rhs(spk_system *s, int nk, const double *rhs, long long ldb, double *xo, long long ldx, T *work,
               cudaStream_t st, bool acc = false) {
    TileArgs A{};
    A.ell_val = sizeof(T) == 8 ? (const void *)s->ell_val.p : (const void *)s->ell_valf.p;
    A.ell_col = s->ell_col.p;
    A.ell_ptr = s->ell_ptr.p;
    A.rdiag = sizeof(T) == 8 ? (const void *)s->rdiag.p : (const void *)s->rdiagf.p;
    A.n = s->n;
    A.rhs = rhs;
    A.ldb = ldb;
    A.rev_in = s->uplo == 'L';
    A.err = s->d_err.p;
    A.fail_entry = s->dbg_fail_waits > 0;
    if (s->redNec && s->ntasks1) {
        A.tasks = s->d_tasks1.p;
        A.ntasks = s->ntasks1;
        A.xout = work;
        A.ldx = s->n;
        k_rhs_solve<false, T, T><<<s->ntasks1, 32, 0, st>>>(A, nk);
        SPK_CUDA(cudaGetLastError());
        s->launches++;
    }
    if (s->redNec && s->nkept) {
        k_reduced_solve_k<32, T><<<1, red_threads<32>(), 0, st>>>(s->d_red_rows.p, s->d_red_off.p, s->nlvl, s->mapRedX.p,
                                                      s->IT.p, s->JT.p, s->T.p, work, s->n,
                                                      sizeof(T) == 4 ? s->red_scratch : nullptr, s->nRed);
        SPK_CUDA(cudaGetLastError());
        s->launches++;
    }
    A.tasks = s->d_tasks2.p;
    A.ntasks = s->ntasks2;
    A.xfix = work;
    A.xout = xo;
    A.ldx = ldx;
    A.rev_out = s->uplo == 'L';
    A.acc = acc;
    k_rhs_solve<true, T, double><<<s->ntasks2, 32, 0, st>>>(A, nk);
    SPK_CUDA(cudaGetLastError());
    s->launches++;
    return SPK_OK;
}

// Coupling reach of the ELL copy (computed once).
int ensure_reach(spk_system *s) {
    if (s->ell_reach >= 0) return SPK_OK;
    DBuf<int> d;
    SPK_TRY(d.alloc(1));
    SPK_CUDA(cudaMemsetAsync(d.p, 0, sizeof(int), s->stream));
    const int ntiles = (s->n + 31) >> 5;
    k_ell_reach<<<(ntiles + 7) / 8, 256, 0, s->stream>>>(ntiles, s->ell_ptr.p, s->ell_col.p, d.p);
    SPK_CUDA(cudaGetLastError());
    int h = 0;
    SPK_CUDA(cudaStreamSynchronize(s->stream));
    SPK_CUDA(cudaMemcpy(&h, d.p, sizeof(int), cudaMemcpyDeviceToHost));
    s->ell_reach = h;
    return SPK_OK;
}

int ensure_work(spk_system *s, size_t bytes) {
    if (s->work.n >= bytes) return SPK_OK;
    return s->work.alloc(bytes);
}

// float copies of the ELL values and diagonal reciprocals (mixed-precision solve)
int ensure_fp32(spk_system *s) {
    if (s->ell_valf.p) return SPK_OK;
    const long long ne = std::max<long long>(s->ell_entries, 1), nr = s->rdiag.n;
    SPK_TRY(s->ell_valf.alloc(ne));
    SPK_TRY(s->rdiagf.alloc(nr));
    k_to_float<<<1184, 256, 0, s->stream>>>(s->ell_entries, s->ell_val.p, s->ell_valf.p);
    k_to_float<<<1184, 256, 0, s->stream>>>(nr, s->rdiag.p, s->rdiagf.p);
    SPK_CUDA(cudaGetLastError());
    SPK_CUDA(cudaStreamSynchronize(s->stream));
    return SPK_OK;
}

// FP64 diagonal and ||A||_inf for residuals
int ensure_residual(spk_system *s) {
    if (s->diag.p) return SPK_OK;
    SPK_TRY(s->diag.alloc(s->n));
    DBuf<unsigned long long> an;
    SPK_TRY(an.alloc(1));
    SPK_CUDA(cudaMemsetAsync(an.p, 0, sizeof(unsigned long long), s->stream));
    k_diag_rowsum<<<blocks_for(s->n), 256, 0, s->stream>>>(s->n, s->uia.p, s->ua.p, s->diag.p, an.p);
    SPK_CUDA(cudaGetLastError());
    unsigned long long h = 0;
    SPK_CUDA(cudaStreamSynchronize(s->stream));
    SPK_CUDA(cudaMemcpy(&h, an.p, sizeof(h), cudaMemcpyDeviceToHost));
    memcpy(&s->anorm, &h, sizeof(double));
    SPK_TRY(s->d_norms.alloc(3 * 32));
    return SPK_OK;
}

template <int K>
void launch_residual(spk_system *s, const double *X, long long ldx, const double *B, long long ldb, double *R,
                     long long ldr, cudaStream_t st) {
    k_residual<K><<<blocks_for(s->n), 256, 0, st>>>(s->n, s->ell_ptr.p, s->ell_val.p, s->ell_col.p, s->diag.p, X, ldx,
                                                     B, ldb, R, ldr, s->uplo == 'L');
}

// max for scaled residuals that keeps a NaN (std::max would drop it)
inline double worst_of(double w, double v) { return (v > w || v != v) ? v : w; }

// R = B - A X (FP64) for K right-hand sides; with norms, also the per-column
// max |R|, |X|, |B| in d_norms (read back by scaled_residual).
int residual(spk_system *s, int K, const double *X, long long ldx, const double *B, long long ldb, double *R,
             long long ldr, cudaStream_t st, bool norms) {
    if (norms) SPK_CUDA(cudaMemsetAsync(s->d_norms.p, 0, sizeof(unsigned long long) * 3 * K, st));
    // the fixed-width kernels cover 1, 2, 4, 8 and 16 columns; other widths (the
    // chain path batches any count up to 32) take the any-width kernel, which
    // touches only columns < K
    if (K > 16 || (K & (K - 1)) != 0) {
        SPK_CUDA(cudaFuncSetAttribute(k_rhs_residual, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sizeof(ResSmem)));
        const int ntiles = (s->n + 31) >> 5;
        const int blocks = (ntiles + kResChunk - 1) / kResChunk;
        k_rhs_residual<<<blocks, 32 * kResWarps, sizeof(ResSmem), st>>>(
            s->n, K, s->ell_ptr.p, s->ell_val.p, s->ell_col.p, s->diag.p, X, ldx, B, ldb, R, ldr, s->uplo == 'L',
            norms ? s->d_norms.p : nullptr);
        SPK_CUDA(cudaGetLastError());
        return SPK_OK;
    }
    switch (K) {
        case 1: launch_residual<1>(s, X, ldx, B, ldb, R, ldr, st); break;
        case 2: launch_residual<2>(s, X, ldx, B, ldb, R, ldr, st); break;
        case 4: launch_residual<4>(s, X, ldx, B, ldb, R, ldr, st); break;
        case 8: launch_residual<8>(s, X, ldx, B, ldb, R, ldr, st); break;
        case 16: launch_residual<16>(s, X, ldx, B, ldb, R, ldr, st); break;
        default:
            set_error(SPK_ERR_ARG, "residual of %d columns", K);
            return SPK_ERR_ARG;
    }
    SPK_CUDA(cudaGetLastError());
    if (norms) {
        k_norms<<<dim3(64, K), 256, 0, st>>>(s->n, K, R, ldr, X, ldx, B, ldb, s->d_norms.p);
        SPK_CUDA(cudaGetLastError());
    }
    return SPK_OK;
}

// max over the K right-hand sides of ||R||_inf / (||A||_inf ||X||_inf + ||B||_inf),
// from the norms residual() left in d_norms
int scaled_residual(spk_system *s, int K, cudaStream_t st, double *out) {
    unsigned long long h[96];
    SPK_CUDA(cudaMemcpyAsync(h, s->d_norms.p, sizeof(unsigned long long) * 3 * K, cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaStreamSynchronize(st));
    double worst = 0.0;
    for (int k = 0; k < K; k++) {
        double nr, nx, nb;
        memcpy(&nr, &h[3 * k], 8);
        memcpy(&nx, &h[3 * k + 1], 8);
        memcpy(&nb, &h[3 * k + 2], 8);
        const double den = s->anorm * nx + nb;
        worst = worst_of(worst, den > 0 ? nr / den : nr);
    }
    *out = worst;
    return SPK_OK;
}

}  // namespace

// diag and ||A|| for the residuals (read from the CSR, which spk_compact releases)
int residual_prepare(spk_system *s) { return ensure_residual(s); }

int solve(spk_system *s, const double *b, double *x, cudaStream_t st, double *ph) {
    if (!s->built) {
        set_error(SPK_ERR_STATE, "no preprocessed system");
        return SPK_ERR_STATE;
    }
    if (!(s->chain_ok && (!ph || s->lean))) SPK_TRY(partition_ensure(s));  // the partition path below
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
    if (s->chain_ok && (!ph || s->lean)) {  // a compacted system has no other path (no phase times)
        SPK_TRY(chain_solve(s, b, x, st, prof, ring));
    } else if (s->ell_ok && !ph) {
        SPK_TRY((launch_tiles<1, double>(s, b, s->n, x, s->n, s->xbuf.p, st, prof, ring)));
    } else {
        // CSR segment solver (or the timed legacy path, which times the phases)
        SegArgs A;
        A.ia = s->uia.p;
        A.ja = s->uja.p;
        A.a = s->ua.p;
        A.rdiag = s->rdiag.p;
        A.n = s->n;
        A.rhs = b;
        A.rev_in = s->uplo == 'L';
        A.err = s->d_err.p;
        A.fail_entry = s->dbg_fail_waits > 0;
        TileArgs TA{};
        TA.ell_val = s->ell_val.p;
        TA.ell_col = s->ell_col.p;
        TA.ell_ptr = s->ell_ptr.p;
        TA.rdiag = s->rdiag.p;
        TA.n = s->n;
        TA.rhs = b;
        TA.ldb = s->n;
        TA.rev_in = s->uplo == 'L';
        TA.err = s->d_err.p;
        TA.fail_entry = s->dbg_fail_waits > 0;
        if (s->redNec && s->ntasks1) {
            A.tasks = TA.tasks = s->d_tasks1.p;
            A.ntasks = TA.ntasks = s->ntasks1;
            A.xfix = nullptr;
            TA.xfix = nullptr;
            A.xout = s->xbuf.p;
            TA.xout = s->xbuf.p;
            TA.ldx = s->n;
            A.rev_out = TA.rev_out = 0;
            if (s->ell_ok) k_tile_solve<false, 1, double, double><<<s->ntasks1, 32, 0, st>>>(TA);
            else k_segment_solve<false><<<s->ntasks1, 32, 0, st>>>(A);
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
        A.tasks = TA.tasks = s->d_tasks2.p;
        A.ntasks = TA.ntasks = s->ntasks2;
        A.xfix = s->xbuf.p;
        TA.xfix = s->xbuf.p;
        A.xout = x;
        TA.xout = x;
        TA.ldx = s->n;
        A.rev_out = TA.rev_out = s->uplo == 'L';
        if (s->ell_ok) k_tile_solve<true, 1, double, double><<<s->ntasks2, 32, 0, st>>>(TA);
        else k_segment_solve<true><<<s->ntasks2, 32, 0, st>>>(A);
        SPK_CUDA(cudaGetLastError());
        s->launches++;
    }
    if (prof) {
        cudaEventRecord(s->ev[ring][3], st);
        s->ev_pending[ring] = 1;
        s->ev_next++;
    }
    lap(3);
    return SPK_OK;
}

// Batched solve of nrhs right-hand sides (device, column-major).  mode 0: FP64
// solves in groups of 32 (right-hand-side-parallel solver) and 16/8/4/2/1 (tile
// solver).  mode 1: FP32 tile solves with FP64
// residuals R = B - A X and FP64 correction updates X += solve32(R), iterated
// until the scaled residual is <= tol (tol < 0: exactly maxit corrections, no
// host synchronisation).
int solve_batch(spk_system *s, int nrhs, const double *B, long long ldb, double *X, long long ldx, int mode,
                double tol, int maxit, cudaStream_t st, int *iters, double *resid) {
    if (!s->built) {
        set_error(SPK_ERR_STATE, "no preprocessed system");
        return SPK_ERR_STATE;
    }
    if (nrhs <= 0 || ldb < s->n || ldx < s->n || (mode != 0 && mode != 1)) {
        set_error(SPK_ERR_ARG, "invalid batch arguments (nrhs=%d, ldb=%lld, ldx=%lld, mode=%d)", nrhs, ldb, ldx, mode);
        return SPK_ERR_ARG;
    }
    if (!s->ell_ok) {
        if (mode != 0) {
            set_error(SPK_ERR_ARG, "the mixed-precision batch needs the sliced-ELL layout");
            return SPK_ERR_ARG;
        }
        for (int k = 0; k < nrhs; k++) SPK_TRY(solve(s, B + k * ldb, X + k * ldx, st, nullptr));
        if (iters) *iters = 0;
        return SPK_OK;
    }
    const long long n = s->n;
    int max_it = 0;
    double worst = 0.0;
    // work columns (up to 32 x n, FP64 or FP32), residual and correction columns
    // (32 x n FP64 each): from the caller's workspace when one is set, else the
    // system's own buffers, grown on demand
    const bool need_r = mode == 1 || resid, need_d = mode == 1;
    const size_t col_bytes = ((size_t)32 * n * sizeof(double) + 255) / 256 * 256;
    char *work_p = nullptr;
    double *rbuf_p = nullptr, *dbuf_p = nullptr;
    if (mode == 1) {
        SPK_TRY(ensure_fp32(s));
        SPK_TRY(ensure_reach(s));
    }
    if (need_r) SPK_TRY(ensure_residual(s));
    // FP32 batches: the FP64 reduced unknowns (32 columns), after the other blocks
    const size_t red_bytes = mode == 1 ? (size_t)32 * s->nRed * sizeof(double) : 0;
    if (s->ext_ws) {
        const size_t need = col_bytes * (1 + need_r + need_d) + red_bytes;
        if (s->ext_ws_bytes < need) {
            set_error(SPK_ERR_TOO_LARGE, "workspace of %zu bytes is below the %zu this batch needs", s->ext_ws_bytes,
                      need);
            return SPK_ERR_TOO_LARGE;
        }
        work_p = s->ext_ws;
        if (need_r) rbuf_p = (double *)(s->ext_ws + col_bytes);
        if (need_d) dbuf_p = (double *)(s->ext_ws + 2 * col_bytes);
    } else {
        if (need_r && s->rbuf.n < (size_t)(32 * n)) SPK_TRY(s->rbuf.alloc(32 * n));
        if (need_d && s->dbuf.n < (size_t)(32 * n)) SPK_TRY(s->dbuf.alloc(32 * n));
        rbuf_p = s->rbuf.p;
        dbuf_p = s->dbuf.p;
    }
    auto work_for = [&](size_t bytes) -> int {
        if (s->ext_ws) return SPK_OK;
        SPK_TRY(ensure_work(s, bytes));
        work_p = s->work.p;
        return SPK_OK;
    };
    // The right-hand-side-parallel solver runs one warp per task along the task's
    // rows; it pays off once the tasks fill the GPU (two per SM).  With fewer
    // tasks the tile solver (rows of a tile across the lanes) has the shorter path.
    int dev = 0, sms = 148;
    SPK_CUDA(cudaGetDevice(&dev));
    SPK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const bool wide_ok = std::min(s->redNec ? s->ntasks1 : s->ntasks2, s->ntasks2) >= 2 * sms;
    int dev0 = 0, sms0 = 148;
    SPK_CUDA(cudaGetDevice(&dev0));
    SPK_CUDA(cudaDeviceGetAttribute(&sms0, cudaDevAttrMultiProcessorCount, dev0));
    const bool part_wide = std::min(s->redNec ? s->ntasks1 : s->ntasks2, s->ntasks2) >= 2 * sms0;
    // FP64: the chain kernel (faster than the partition kernels at every partition
    // count measured); FP32 + refinement: the chain kernel when the partitions give
    // too few tasks to fill the GPU
    const char *cb = getenv("SPK_CHAIN_BATCH");  // 1: always the chain kernels, 0: never
    const bool use_chain =
        s->chain_ok && (s->lean || (s->batch_path >= 0 ? s->batch_path == 1
                                                       : (cb ? cb[0] == '1' : (mode == 0 || !part_wide))));
    if (!use_chain) SPK_TRY(partition_ensure(s));
    if (use_chain) {
        // the chain tasks fill the GPU whatever the partition count: every group
        // of up to 32 columns is one right-hand-side-parallel chain solve (used
        // when the partitions alone give too few tasks to fill the GPU)
        for (int g = 0; g < nrhs;) {
            const int K = std::min(nrhs - g, 32);
            const double *Bg = B + g * ldb;
            double *Xg = X + g * ldx;
            if (mode == 0) {
                SPK_TRY(chain_solve_rhs(s, 0, K, Bg, ldb, Xg, ldx, st));
                if (resid) {
                    SPK_TRY(residual(s, K, Xg, ldx, Bg, ldb, rbuf_p, n, st, true));
                    double r = 0;
                    SPK_TRY(scaled_residual(s, K, st, &r));
                    worst = worst_of(worst, r);
                }
            } else {
                SPK_TRY(chain_solve_rhs(s, 1, K, Bg, ldb, Xg, ldx, st));
                int it = 0;
                double r = -1.0;
                for (;; it++) {
                    const bool check = tol >= 0 || (resid && it == maxit);
                    if (tol < 0 && it == maxit && !resid) break;
                    SPK_TRY(residual(s, K, Xg, ldx, Bg, ldb, rbuf_p, n, st, check));
                    if (check) {
                        SPK_TRY(scaled_residual(s, K, st, &r));
                        if ((tol >= 0 && r <= tol) || it == maxit) break;
                    }
                    if (it == maxit) break;
                    SPK_TRY(chain_solve_rhs(s, 1, K, rbuf_p, n, dbuf_p, n, st));
                    k_axpy<<<dim3(148, K), 256, 0, st>>>(s->n, K, dbuf_p, Xg, ldx);
                    SPK_CUDA(cudaGetLastError());
                }
                max_it = std::max(max_it, it);
                if (!(r < 0)) worst = worst_of(worst, r);
            }
            g += K;
        }
        if (iters) *iters = max_it;
        if (resid) *resid = worst;
        if (resid || (mode != 0 && tol >= 0)) SPK_TRY(check_device_error(s));
        return SPK_OK;
    }
    for (int g = 0; g < nrhs;) {
        const int left = nrhs - g;
        // 17..32 columns: one right-hand-side-parallel pass (work holds 32 columns);
        // fewer (or few tasks): the tile solver in power-of-two groups
        const int K = (wide_ok && left > 16) ? std::min(left, 32)
                                             : left >= 16 ? 16 : left >= 8 ? 8 : left >= 4 ? 4 : left >= 2 ? 2 : 1;
        const bool rhs_path = K > 16;
        const long long wcols = rhs_path ? 32 : K;
        const double *Bg = B + g * ldb;
        double *Xg = X + g * ldx;
        if (mode == 0) {
            SPK_TRY(work_for(sizeof(double) * wcols * n));
            if (rhs_path)
                SPK_TRY(launch_rhs<double>(s, K, Bg, ldb, Xg, ldx, (double *)work_p, st));
            else
                SPK_TRY(launch_tiles_k<double>(s, K, Bg, ldb, Xg, ldx, (double *)work_p, st));
            if (resid) {
                SPK_TRY(residual(s, K, Xg, ldx, Bg, ldb, rbuf_p, n, st, true));
                double r = 0;
                SPK_TRY(scaled_residual(s, K, st, &r));
                worst = worst_of(worst, r);
            }
        } else {
            // FP32 work columns, then the FP64 reduced unknowns (a lent
            // workspace holds them after its column blocks)
            const size_t fbytes = (sizeof(float) * wcols * n + 255) / 256 * 256;
            const bool red64 = s->redNec && s->nkept;
            SPK_TRY(work_for(fbytes + (red64 ? red_bytes : 0)));
            float *wk = (float *)work_p;
            s->red_scratch = !red64 ? nullptr
                             : s->ext_ws ? (double *)(s->ext_ws + col_bytes * (1 + need_r + need_d))
                                         : (double *)(work_p + fbytes);
            struct ClearRed {
                spk_system *s;
                ~ClearRed() { s->red_scratch = nullptr; }
            } clear_red{s};
            auto solve32 = [&](const double *rhs, long long ld, double *xo, long long ldo) {
                return rhs_path ? launch_rhs<float>(s, K, rhs, ld, xo, ldo, wk, st)
                               : launch_tiles_k<float>(s, K, rhs, ld, xo, ldo, wk, st);
            };
            SPK_TRY(solve32(Bg, ldb, Xg, ldx));
            int it = 0;
            double r = -1.0;
            for (;; it++) {
                const bool check = tol >= 0 || (resid && it == maxit);
                if (tol < 0 && it == maxit && !resid) break;
                SPK_TRY(residual(s, K, Xg, ldx, Bg, ldb, rbuf_p, n, st, check));
                if (check) {
                    SPK_TRY(scaled_residual(s, K, st, &r));
                    if ((tol >= 0 && r <= tol) || it == maxit) break;
                }
                if (it == maxit) break;
                if (rhs_path && s->ell_reach < kRhsWin) {
                    // correction added in place by phase 3+4 (no coupling leaves the window)
                    SPK_TRY(launch_rhs<float>(s, K, rbuf_p, n, Xg, ldx, wk, st, true));
                } else {
                    SPK_TRY(solve32(rbuf_p, n, dbuf_p, n));
                    k_axpy<<<dim3(148, K), 256, 0, st>>>(s->n, K, dbuf_p, Xg, ldx);
                    SPK_CUDA(cudaGetLastError());
                }
            }
            max_it = std::max(max_it, it);
            if (!(r < 0)) worst = worst_of(worst, r);
        }
        g += K;
    }
    if (iters) *iters = max_it;
    if (resid) *resid = worst;
    // a call that waited for its residuals reports a failed device wait too
    if (resid || (mode != 0 && tol >= 0)) SPK_TRY(check_device_error(s));
    return SPK_OK;
}

// ---- allocation-free batched solve -------------------------------------------------
//
// The phase-1 work columns live in a fixed array compiled into the library
// instead of the per-system buffer that solve_batch grows on demand, so a call
// allocates nothing.  Groups shrink to fit (K * n <= kStaticScratch).  Every
// work entry a solve reads is written earlier in the same solve (phase 1 rows
// and the reduced rows), so nothing in the scratch has to start at zero.  One
// scratch per device: solves whose work overlaps on the GPU race on it.

constexpr long long kStaticScratch = 1ll << 19;  // FP64 values (4 MiB)
static __device__ __align__(256) double g_static_scratch[kStaticScratch];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
double *g_static_ptr[kMaxDevices];

// Device address of the scratch on the current device, looked up once per
// device (the lookup may load the library's device code on that device).
int static_scratch(double **out) {
    int dev = 0;
    SPK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error(SPK_ERR_ARG, "device %d is beyond the %d devices the static scratch table covers", dev,
                  kMaxDevices);
        return SPK_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p) {
            set_error(SPK_ERR_CUDA, "cudaGetSymbolAddress of the static scratch failed on device %d: %s", dev,
                      cudaGetErrorString(e));
            return SPK_ERR_CUDA;
        }
        g_static_ptr[dev] = (double *)p;
    }
    *out = g_static_ptr[dev];
    return SPK_OK;
}
}  // namespace

int solve_batch_static(spk_system *s, int nrhs, const double *B, long long ldb, double *X, long long ldx,
                       cudaStream_t st) {
    if (!s->built) {
        set_error(SPK_ERR_STATE, "no preprocessed system");
        return SPK_ERR_STATE;
    }
    if (s->lean) {
        set_error(SPK_ERR_STATE, "the system was compacted (spk_compact): the static batched solve needs its partition pools");
        return SPK_ERR_STATE;
    }
    const long long n = s->n;
    if (nrhs <= 0 || ldb < n || ldx < n) {
        set_error(SPK_ERR_ARG, "invalid batch arguments (nrhs=%d, ldb=%lld, ldx=%lld)", nrhs, ldb, ldx);
        return SPK_ERR_ARG;
    }
    if (!s->ell_ok) {
        set_error(SPK_ERR_ARG, "the allocation-free solve needs the sliced-ELL layout (this system uses the CSR "
                               "solver)");
        return SPK_ERR_ARG;
    }
    if (n > kStaticScratch) {
        set_error(SPK_ERR_TOO_LARGE,
                  "system of %lld rows exceeds the allocation-free solve's static scratch of %lld FP64 values",
                  n, kStaticScratch);
        return SPK_ERR_TOO_LARGE;
    }
    double *work = nullptr;
    SPK_TRY(static_scratch(&work));
    // the same choice as solve_batch: the right-hand-side-parallel solver only
    // when the tasks fill the GPU (two per SM), else tile groups of up to 16
    int dev = 0, sms = 148;
    SPK_CUDA(cudaGetDevice(&dev));
    SPK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const bool wide_ok = std::min(s->redNec ? s->ntasks1 : s->ntasks2, s->ntasks2) >= 2 * sms;
    for (int g = 0; g < nrhs;) {
        const int left = nrhs - g;
        int K = wide_ok ? 32 : 16;
        while (K > 1 && (K > left || K * n > kStaticScratch)) K >>= 1;
        const double *Bg = B + g * ldb;
        double *Xg = X + g * ldx;
        if (K == 32)
            SPK_TRY(launch_rhs<double>(s, K, Bg, ldb, Xg, ldx, work, st));
        else
            SPK_TRY(launch_tiles_k<double>(s, K, Bg, ldb, Xg, ldx, work, st));
        g += K;
    }
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
        s->dbg_fail_waits = 0;  // the test hook (spk_debug_set "fail_waits") ends once reported
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

// ---- many systems in one captured launch sequence (spk_group) --------------------
//
// Every system's right-hand sides are split into width classes K in
// {16, 8, 4, 2, 1} ("virtual systems": one system, K columns).  Per class, one
// k_tile_multi launch runs the phase-1 tasks of all its virtual systems from a
// flat work list (longest tasks first), one k_reduced_multi launch their
// reduced solves (a block per virtual system), one k_tile_multi launch their
// phase 3+4 tasks; FP32 + refinement adds k_residual_multi and k_axpy_multi
// over flat row-block lists.  The whole sequence is captured once into a CUDA
// graph and replayed by spk_group_solve.

namespace spk {
namespace {

constexpr int kGroupK[5] = {16, 8, 4, 2, 1};

struct GroupVS {
    spk_system *s;
    int sys;  // index in the group
    int K, col0;
    const double *B;
    long long ldb;
    double *X;
    long long ldx;
    char *work;
    double *R, *D;
    double *red;  // FP32 batches: the FP64 reduced unknowns ([K][nRed])
};

struct GroupClass {
    int K = 0;
    DBuf<TileArgs> a1, a4, c1, c4;  // solve and correction-solve arguments (phase 1, phase 3+4)
    DBuf<int2> w1, w4, vw;
    DBuf<RedArgs> red, cred;
    DBuf<VecArgs> va;
    int n1 = 0, n4 = 0, nred = 0, nvw = 0;
    std::vector<int> vs;  // virtual systems of the class
};

}  // namespace
}  // namespace spk

struct spk_group {
    int mode = 0, iters = 0;
    std::vector<spk_system *> sys;
    std::vector<spk::GroupVS> vs;
    spk::GroupClass cls[5];
    spk::DBuf<char> pool;
    spk::DBuf<unsigned long long> norms;
    long long norm_cols = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long kernels = 0;
};

namespace spk {
namespace {

TileArgs make_args(const GroupVS &v, bool fp32, bool phase4, const double *rhs, long long ldb, double *xo,
                   long long ldx) {
    spk_system *s = v.s;
    TileArgs A{};
    A.ell_val = fp32 ? (const void *)s->ell_valf.p : (const void *)s->ell_val.p;
    A.ell_col = s->ell_col.p;
    A.ell_ptr = s->ell_ptr.p;
    A.rdiag = fp32 ? (const void *)s->rdiagf.p : (const void *)s->rdiag.p;
    A.n = s->n;
    A.rhs = rhs;
    A.ldb = ldb;
    A.rev_in = s->uplo == 'L';
    A.err = s->d_err.p;
    if (!phase4) {
        A.tasks = s->d_tasks1.p;
        A.ntasks = s->ntasks1;
        A.xout = v.work;
        A.ldx = s->n;
    } else {
        A.tasks = s->d_tasks2.p;
        A.ntasks = s->ntasks2;
        A.xfix = v.work;
        A.xout = xo;
        A.ldx = ldx;
        A.rev_out = s->uplo == 'L';
    }
    return A;
}

template <typename T>
int upload_vec(DBuf<T> &d, const std::vector<T> &h) {
    SPK_TRY(d.alloc(std::max<size_t>(h.size(), 1)));
    if (!h.empty()) SPK_CUDA(cudaMemcpy(d.p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
    return SPK_OK;
}

// Work lists and argument tables of one class.
int build_class(spk_group *g, GroupClass &c, const std::vector<std::vector<SegTask>> &t1,
                const std::vector<std::vector<SegTask>> &t4) {
    const bool fp32 = g->mode == 1;
    std::vector<TileArgs> a1, a4, c1, c4;
    std::vector<RedArgs> red, cred;
    std::vector<VecArgs> va;
    std::vector<std::pair<long long, int2>> w1, w4;
    std::vector<int2> vw;
    for (size_t i = 0; i < c.vs.size(); i++) {
        const GroupVS &v = g->vs[c.vs[i]];
        spk_system *s = v.s;
        a1.push_back(make_args(v, fp32, false, v.B, v.ldb, nullptr, 0));
        a4.push_back(make_args(v, fp32, true, v.B, v.ldb, v.X, v.ldx));
        if (fp32) {
            c1.push_back(make_args(v, true, false, v.R, s->n, nullptr, 0));
            c4.push_back(make_args(v, true, true, v.R, s->n, v.D, s->n));
        }
        if (s->redNec && s->ntasks1)
            for (int t = 0; t < s->ntasks1; t++) {
                const SegTask &q = t1[v.sys][t];
                w1.push_back({(long long)(q.hi - q.lo), make_int2((int)i, t)});
            }
        for (int t = 0; t < s->ntasks2; t++) {
            const SegTask &q = t4[v.sys][t];
            w4.push_back({(long long)(q.hi - q.lo) + (q.tail - q.hi), make_int2((int)i, t)});
        }
        if (s->redNec && s->nkept) {
            RedArgs r{s->d_red_rows.p, s->d_red_off.p, s->nlvl, s->mapRedX.p, s->IT.p, s->JT.p, s->T.p, v.work,
                      s->n, fp32 ? v.red : nullptr, s->nRed};
            red.push_back(r);
            cred.push_back(r);
        }
        VecArgs a{};
        a.n = s->n;
        a.rev = s->uplo == 'L';
        a.ptr = s->ell_ptr.p;
        a.ev = s->ell_val.p;
        a.ec = s->ell_col.p;
        a.diag = s->diag.p;
        a.X = v.X;
        a.ldx = v.ldx;
        a.B = v.B;
        a.ldb = v.ldb;
        a.R = v.R;
        a.D = v.D;
        a.norms = g->norms.p + 3ll * (v.col0);
        va.push_back(a);
        for (int b = 0; b * 256 < s->n; b++) vw.push_back(make_int2((int)i, b));
    }
    auto sorted = [](std::vector<std::pair<long long, int2>> &w) {
        std::stable_sort(w.begin(), w.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
        std::vector<int2> o;
        for (auto &e : w) o.push_back(e.second);
        return o;
    };
    SPK_TRY(upload_vec(c.a1, a1));
    SPK_TRY(upload_vec(c.a4, a4));
    if (fp32) {
        SPK_TRY(upload_vec(c.c1, c1));
        SPK_TRY(upload_vec(c.c4, c4));
    }
    const std::vector<int2> s1 = sorted(w1), s4 = sorted(w4);
    SPK_TRY(upload_vec(c.w1, s1));
    SPK_TRY(upload_vec(c.w4, s4));
    c.n1 = (int)s1.size();
    c.n4 = (int)s4.size();
    // reduced solves: one argument block per virtual system that has a reduced system
    SPK_TRY(upload_vec(c.red, red));
    SPK_TRY(upload_vec(c.cred, cred));
    c.nred = (int)red.size();
    SPK_TRY(upload_vec(c.va, va));
    SPK_TRY(upload_vec(c.vw, vw));
    c.nvw = (int)vw.size();
    return SPK_OK;
}

template <int K, typename T>
void enqueue_solve(spk_group *g, GroupClass &c, bool correction, cudaStream_t st) {
    const TileArgs *p1 = correction ? c.c1.p : c.a1.p;
    const TileArgs *p4 = correction ? c.c4.p : c.a4.p;
    if (c.n1) {
        k_tile_multi<false, K, T, T><<<c.n1, 32, 0, st>>>(p1, c.w1.p);
        g->kernels++;
    }
    if (c.nred) {
        k_reduced_multi<K, T><<<c.nred, red_threads<K>(), 0, st>>>(c.red.p);
        g->kernels++;
    }
    if (c.n4) {
        k_tile_multi<true, K, T, double><<<c.n4, 32, 0, st>>>(p4, c.w4.p);
        g->kernels++;
    }
}

template <int K>
void enqueue_class(spk_group *g, GroupClass &c, cudaStream_t st) {
    if (g->mode == 0) {
        enqueue_solve<K, double>(g, c, false, st);
        return;
    }
    enqueue_solve<K, float>(g, c, false, st);
    for (int it = 0; it < g->iters; it++) {
        k_residual_multi<K><<<c.nvw, 256, 0, st>>>(c.va.p, c.vw.p, 0);
        enqueue_solve<K, float>(g, c, true, st);
        k_axpy_multi<K><<<c.nvw, 256, 0, st>>>(c.va.p, c.vw.p);
        g->kernels += 2;
    }
}

void enqueue_all(spk_group *g, cudaStream_t st) {
    for (auto &c : g->cls) {
        if (c.vs.empty()) continue;
        switch (c.K) {
            case 16: enqueue_class<16>(g, c, st); break;
            case 8: enqueue_class<8>(g, c, st); break;
            case 4: enqueue_class<4>(g, c, st); break;
            case 2: enqueue_class<2>(g, c, st); break;
            default: enqueue_class<1>(g, c, st); break;
        }
    }
}

}  // namespace
}  // namespace spk

using namespace spk;

extern "C" {

int spk_group_destroy(spk_group *g) {
    if (!g) return SPK_OK;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return SPK_OK;
}

int spk_group_create(spk_group **out, int count, spk_system *const *systems, const int *nrhs,
                     const double *const *B, const long long *ldb, double *const *X, const long long *ldx, int mode,
                     int iters, void *stream) {
    if (!out || count <= 0 || !systems || !nrhs || !B || !ldb || !X || !ldx || (mode != 0 && mode != 1) ||
        iters < 0) {
        set_error(SPK_ERR_ARG, "invalid group arguments (count=%d, mode=%d, iters=%d)", count, mode, iters);
        return SPK_ERR_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    spk_group *g = new spk_group();
    g->mode = mode;
    g->iters = mode == 1 ? iters : 0;
    auto fail = [&](int rc) {
        spk_group_destroy(g);
        return rc;
    };
    std::vector<std::vector<SegTask>> t1(count), t4(count);
    long long cols = 0, pool_bytes = 0;
    for (int i = 0; i < count; i++) {
        spk_system *s = systems[i];
        if (!s || !s->built || !s->ell_ok || nrhs[i] <= 0 || ldb[i] < s->n || ldx[i] < s->n || !B[i] || !X[i]) {
            set_error(SPK_ERR_ARG, "group member %d: needs a preprocessed system on the sliced-ELL layout, nrhs > 0 "
                                   "and leading dimensions >= n", i);
            return fail(SPK_ERR_ARG);
        }
        if (s->lean) {
            set_error(SPK_ERR_STATE, "group member %d was compacted (spk_compact): groups need the partition pools", i);
            return fail(SPK_ERR_STATE);
        }
        if (const int rc = partition_ensure(s); rc != SPK_OK) return fail(rc);
        if (mode == 1) {
            int rc = ensure_fp32(s);
            if (rc == SPK_OK) rc = ensure_residual(s);
            if (rc != SPK_OK) return fail(rc);
        } else if (!s->diag.p) {
            const int rc = ensure_residual(s);
            if (rc != SPK_OK) return fail(rc);
        }
        t1[i].resize(s->ntasks1);
        t4[i].resize(s->ntasks2);
        if (s->ntasks1 && cudaMemcpy(t1[i].data(), s->d_tasks1.p, sizeof(SegTask) * s->ntasks1,
                                     cudaMemcpyDeviceToHost) != cudaSuccess)
            return fail(SPK_ERR_CUDA);
        if (cudaMemcpy(t4[i].data(), s->d_tasks2.p, sizeof(SegTask) * s->ntasks2, cudaMemcpyDeviceToHost) !=
            cudaSuccess)
            return fail(SPK_ERR_CUDA);
        g->sys.push_back(s);
        // width classes: binary decomposition of nrhs in pieces of at most 16
        int left = nrhs[i], col = 0;
        while (left > 0) {
            int K = 16;
            while (K > left) K >>= 1;
            GroupVS v{};
            v.s = s;
            v.sys = i;
            v.K = K;
            v.col0 = (int)cols;
            v.B = B[i] + col * ldb[i];
            v.ldb = ldb[i];
            v.X = X[i] + col * ldx[i];
            v.ldx = ldx[i];
            const long long kn = (long long)K * s->n;
            v.work = (char *)(intptr_t)pool_bytes;  // offsets until the pool exists
            pool_bytes += ((kn * (mode == 1 ? 4 : 8)) + 255) / 256 * 256;
            if (mode == 1) {
                v.R = (double *)(intptr_t)pool_bytes;
                pool_bytes += (kn * 8 + 255) / 256 * 256;
                v.D = (double *)(intptr_t)pool_bytes;
                pool_bytes += (kn * 8 + 255) / 256 * 256;
                v.red = (double *)(intptr_t)pool_bytes;
                pool_bytes += ((long long)K * s->nRed * 8 + 255) / 256 * 256;
            }
            g->vs.push_back(v);
            cols += K;
            col += K;
            left -= K;
        }
    }
    if (g->pool.alloc(std::max<long long>(pool_bytes, 256)) != SPK_OK) return fail(SPK_ERR_NOMEM);
    if (g->norms.alloc(3 * cols) != SPK_OK) return fail(SPK_ERR_NOMEM);
    g->norm_cols = cols;
    for (auto &v : g->vs) {
        v.work = g->pool.p + (intptr_t)v.work;
        if (mode == 1) {
            v.R = (double *)(g->pool.p + (intptr_t)v.R);
            v.D = (double *)(g->pool.p + (intptr_t)v.D);
            v.red = (double *)(g->pool.p + (intptr_t)v.red);
        }
    }
    for (int c = 0; c < 5; c++) g->cls[c].K = kGroupK[c];
    for (int i = 0; i < (int)g->vs.size(); i++)
        for (int c = 0; c < 5; c++)
            if (g->vs[i].K == kGroupK[c]) g->cls[c].vs.push_back(i);
    for (auto &c : g->cls) {
        if (c.vs.empty()) continue;
        const int rc = build_class(g, c, t1, t4);
        if (rc != SPK_OK) return fail(rc);
    }
    // capture the launch sequence
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        (void)cudaGetLastError();  // not sticky: clear it for the caller's next checks
        set_error(SPK_ERR_CUDA, "cudaStreamBeginCapture failed (a legacy default stream cannot be captured)");
        return fail(SPK_ERR_CUDA);
    }
    enqueue_all(g, st);
    cudaError_t e = cudaStreamEndCapture(st, &g->graph);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        set_error(SPK_ERR_CUDA, "group graph capture failed: %s", cudaGetErrorString(e));
        return fail(SPK_ERR_CUDA);
    }
    *out = g;
    return SPK_OK;
}

int spk_group_solve(spk_group *g, void *stream) {
    if (!g || !g->exec) {
        set_error(SPK_ERR_ARG, "null group");
        return SPK_ERR_ARG;
    }
    SPK_CUDA(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
    return SPK_OK;
}

int spk_group_residual(spk_group *g, void *stream, double *worst) {
    if (!g || !worst) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    // residuals into the R buffers of FP32 groups, or a scratch pool for FP64 groups
    DBuf<double> scratch;
    if (g->mode == 0) {
        long long maxkn = 0;
        for (auto &v : g->vs) maxkn += (long long)v.K * v.s->n;
        SPK_TRY(scratch.alloc(std::max<long long>(maxkn, 1)));
        long long off = 0;
        for (auto &c : g->cls) {
            if (c.vs.empty()) continue;
            std::vector<VecArgs> va(c.vs.size());
            SPK_CUDA(cudaMemcpy(va.data(), c.va.p, sizeof(VecArgs) * va.size(), cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < va.size(); i++) {
                va[i].R = scratch.p + off;
                off += (long long)va[i].n * c.K;
            }
            SPK_CUDA(cudaMemcpy(c.va.p, va.data(), sizeof(VecArgs) * va.size(), cudaMemcpyHostToDevice));
        }
    }
    SPK_CUDA(cudaMemsetAsync(g->norms.p, 0, sizeof(unsigned long long) * 3 * g->norm_cols, st));
    for (auto &c : g->cls) {
        if (c.vs.empty()) continue;
        switch (c.K) {
            case 16: k_residual_multi<16><<<c.nvw, 256, 0, st>>>(c.va.p, c.vw.p, 1); break;
            case 8: k_residual_multi<8><<<c.nvw, 256, 0, st>>>(c.va.p, c.vw.p, 1); break;
            case 4: k_residual_multi<4><<<c.nvw, 256, 0, st>>>(c.va.p, c.vw.p, 1); break;
            case 2: k_residual_multi<2><<<c.nvw, 256, 0, st>>>(c.va.p, c.vw.p, 1); break;
            default: k_residual_multi<1><<<c.nvw, 256, 0, st>>>(c.va.p, c.vw.p, 1); break;
        }
        SPK_CUDA(cudaGetLastError());
    }
    std::vector<unsigned long long> h(3 * g->norm_cols);
    SPK_CUDA(cudaMemcpyAsync(h.data(), g->norms.p, sizeof(unsigned long long) * h.size(), cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaStreamSynchronize(st));
    double w = 0.0;
    for (auto &v : g->vs)
        for (int k = 0; k < v.K; k++) {
            double nr, nx, nb;
            memcpy(&nr, &h[3 * (v.col0 + k)], 8);
            memcpy(&nx, &h[3 * (v.col0 + k) + 1], 8);
            memcpy(&nb, &h[3 * (v.col0 + k) + 2], 8);
            const double den = v.s->anorm * nx + nb;
            w = worst_of(w, den > 0 ? nr / den : nr);
        }
    *worst = w;
    for (auto *s : g->sys) SPK_TRY(check_device_error(s));
    return SPK_OK;
}

long long spk_group_info(const spk_group *g, const char *name) {
    if (!g || !name) return -1;
    if (!strcmp(name, "kernels")) return g->kernels;
    if (!strcmp(name, "virtual_systems")) return (long long)g->vs.size();
    if (!strcmp(name, "columns")) return g->norm_cols;
    long long items = 0;
    for (auto &c : g->cls) items += c.n1 + c.n4;
    if (!strcmp(name, "task_items")) return items;
    if (!strcmp(name, "pool_bytes")) return (long long)g->pool.n;
    return -1;
}

}  // extern "C"
