// Chain solver: the default one-right-hand-side FP64 solve of
// spike_pstrsv_solve (src/spike_pstrsv.c:149-239) when spike truncation is on.
//
// Decomposition.  The rows of U are cut into chains [a, q) of a few thousand
// rows, aligned to 32-row tiles and independent of the caller's partition count
// (the partitions still define every piece of reference state; only the solve's
// task decomposition differs).  For a chain, x - y = -S x_c exactly, where y is
// the chain-local solution (columns >= q taken as zero), x_c the true values of
// the columns >= q and S = D_chain^{-1} R_chain the chain's spike: the same
// identity the reference's phases 1-4 rest on (src/spike_pstrsv.c:194-229), with
// the chain in the role of a partition.  Preprocessing computes every chain's
// spike exactly (k_chain_spike) and finds f, the first row from the top whose
// spike row has an absolute sum above tau (2^-60 by default, below FP64
// resolution relative to ||x||_inf).  Rows [a, f) of y are final.
//
//   phase 1   every chain solves [a, q) with zero coupling and stores rows [a, f)
//   phase 4   every chain with f < q re-solves [f, q), reading the columns >= q
//             from x (rows that phase 1 of the chain below stored)
//
// Valid when every chain but the top one keeps its first `reach` rows (f >= a +
// reach, reach = the widest column distance): then phase 4 only reads final
// values.  Preprocessing doubles the chain length until that holds, and falls
// back to the partition-based solve otherwise.
//
// Kernel.  One warp per task, lane = row of a 32-row tile, tiles bottom-up.  The
// matrix is stored for this solver as a sliced ELL of ROW-SCALED off-diagonals
// a(r,c)/a(r,r) (so x_r = b_r/a(r,r) - sum v'(r,c) x_c) with 8-bit column
// offsets c - r, per tile slot-pair-major (values: one 16-byte copy per lane per
// two slots; offsets: one 4-byte copy per lane per four slots).  Each tile is
// staged into shared memory by cp.async one tile ahead; every lane copies and
// reads only its own row, so a stage needs no barrier.  Shared memory also holds
// the solved-row window (gathers of far columns) and a per-lane column of
// in-tile coefficients: coef[i][lane] = v'(row0+lane, row0+i) is written and
// read by its own lane only, so the in-tile triangle needs no barrier beyond the
// warp shuffles that broadcast each solved row.
//
// Memory per solve (banded workload, 16 off-diagonals per row): 16 x 9 B of
// matrix + 8 B 1/diagonal + 8 B b + 8 B x per row in phase 1, the same per
// re-solved row in phase 4.  No scratch vector: phase 1 writes final rows
// straight into x.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <set>
#include <type_traits>
#include <utility>
#include <vector>

#include "spk_internal.cuh"

namespace spk {

namespace {

constexpr unsigned kFull = 0xffffffffu;

// Checked builds (-DSPK_DEVICE_CHECKS): every index of the chain kernels is
// bounds-checked; a failed check records (code, block, index) in g_chain_check
// (first one kept) and the access uses index 0 instead.  Off by default.
#ifdef SPK_DEVICE_CHECKS
__device__ unsigned long long g_chain_check;
__device__ __noinline__ long long chk_fail(int code, long long i) {
    atomicCAS(&g_chain_check, 0ull,
              ((unsigned long long)code << 48) | ((unsigned long long)(blockIdx.x & 0xffffff) << 24) |
                  (unsigned long long)(i & 0xffffff));
    return 0;
}
#define CK(i, n, code) \
    (((unsigned long long)(long long)(i) < (unsigned long long)(long long)(n)) ? (long long)(i) : chk_fail((code), (long long)(i)))
#else
#define CK(i, n, code) (i)
#endif

inline int nblocks(long long n, int bs = 256) { return (int)((n + bs - 1) / bs); }

// The dynamic shared memory a kernel may take, raised once per kernel and device
// to the device's opt-in maximum.  Launches of the same kernel for systems of
// different sizes come from several host threads (the serving loop's workers);
// setting the attribute to each launch's own size would race with the launches
// of other threads.
template <typename K>
int allow_smem(K kern) {
    static std::mutex mu;
    static std::set<std::pair<int, const void *>> done;
    int dev = 0;
    SPK_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(mu);
    const auto key = std::make_pair(dev, (const void *)kern);
    if (done.count(key)) return SPK_OK;
    int mx = 0;
    SPK_CUDA(cudaDeviceGetAttribute(&mx, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    SPK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    done.insert(key);
    return SPK_OK;
}

// ---- layout construction -----------------------------------------------------------

// Per 32-row tile: the widest row (off-diagonal count) and, over all rows, the
// widest column distance (last column - row; columns are sorted).
__global__ void k_chain_scan(int n, const int *__restrict__ ia, const int *__restrict__ ja, int *__restrict__ width,
                             int *__restrict__ reach) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    int len = 0, dist = 0;
    if (r < n) {
        const int b = ia[r], e = ia[r + 1];
        len = e - b - 1;
        dist = len > 0 ? ja[e - 1] - r : 0;
    }
    int w = len, d = dist;
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        w = max(w, __shfl_xor_sync(kFull, w, o));
        d = max(d, __shfl_xor_sync(kFull, d, o));
    }
    if ((threadIdx.x & 31) == 0 && (r >> 5) < (n + 31) / 32) {
        width[r >> 5] = w;
        atomicMax(reach, d);
    }
}

// Slots of tile j = rows 32j..32j+31: slot k of lane l holds value
// val[ptr_j + (k>>1)*64 + 2l + (k&1)] and offset byte off[ptr_j + (k>>2)*128 +
// 4l + (k&3)]; padding: value 0, offset 0 (column = the row itself).
__global__ void k_chain_fill(int n, int ntiles, const int *__restrict__ ia, const int *__restrict__ ja,
                             const double *__restrict__ a, const int *__restrict__ ptr, double *__restrict__ val,
                             unsigned char *__restrict__ off) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = r >> 5, l = r & 31;
    if (j >= ntiles) return;
    const int w = (ptr[j + 1] - ptr[j]) >> 5;
    const long long base = ptr[j];
    int b = 0, len = 0;
    double rd = 0.0;
    if (r < n) {
        b = ia[r];
        len = ia[r + 1] - b - 1;
        rd = 1.0 / a[b];
    }
    for (int k = 0; k < w; k++) {
        const long long vo = base + (k >> 1) * 64 + 2 * l + (k & 1);
        const long long oo = base + (k >> 2) * 128 + 4 * l + (k & 3);
        if (k < len) {
            val[vo] = a[b + 1 + k] * rd;
            off[oo] = (unsigned char)(ja[b + 1 + k] - r);
        } else {
            val[vo] = 0.0;
            off[oo] = 0;
        }
    }
}

// ---- spikes of the chains -------------------------------------------------------------
//
// One warp per chain [a, q); lane owns spike columns lane + 32 cc (cc < C), i.e.
// the unit responses to x at columns q + lane + 32 cc.  A ring of reach + 1 rows
// in shared memory ([slot][32 C]) holds the spike rows the recurrence still
// reads; rows [q, q + reach) start as unit vectors, and every row r < q is
// X_r = -sum_k v'(r, r + off_k) X_{r + off_k}.  Each lane reads only its own
// columns, so the ring needs no barrier.  f = the smallest row whose absolute
// row sum exceeds tau (q when none).

struct SpikeArgs {
    const int2 *chains;  // [a, q)
    int nchains;
    const double *val;
    const unsigned *off;  // offset bytes as 32-bit words
    const int *ptr;
    int reach;
    double tau;
    int *first;
    long long nval, nptr;  // element counts (bounds of the checked build)
};

template <int C>
__global__ void __launch_bounds__(32) k_chain_spike(SpikeArgs A) {
    extern __shared__ double ring[];  // [(reach + 1) * 32 * C]
    const int lane = threadIdx.x;
    const int2 ch = A.chains[blockIdx.x];
    const int a = ch.x, q = ch.y;
    const int R = A.reach + 1;
    // slot(q - 1) = 0, slot(q + j) = j + 1
    for (int s = 0; s < R; s++) {
#pragma unroll
        for (int cc = 0; cc < C; cc++) {
            const int col = lane + 32 * cc;
            ring[s * 32 * C + col] = (s >= 1 && col == s - 1) ? 1.0 : 0.0;
        }
    }
    int first = q;
    int sr = 0;  // slot of the current row
    for (int r = q - 1; r >= a; r--) {
        const int j = r >> 5, l = r & 31;
        const int p0 = A.ptr[CK(j, A.nptr, 1)];
        const int w = (A.ptr[CK(j + 1, A.nptr, 2)] - p0) >> 5;
        double acc[C][2];
#pragma unroll
        for (int cc = 0; cc < C; cc++) acc[cc][0] = acc[cc][1] = 0.0;
        for (int k0 = 0; k0 < w; k0 += 4) {
            const unsigned ow = __ldg(A.off + CK(((p0 + (k0 >> 2) * 128) >> 2) + l, A.nval / 4, 3));
            const double2 va = __ldg((const double2 *)A.val + CK((p0 + (k0 >> 1) * 64) / 2 + l, A.nval / 2, 4));
            const double2 vb = __ldg((const double2 *)A.val + CK((p0 + ((k0 >> 1) + 1) * 64) / 2 + l, A.nval / 2, 5));
            const double v4[4] = {va.x, va.y, vb.x, vb.y};
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int o = (ow >> (8 * u)) & 0xff;
                int cs = sr + o;
                cs -= cs >= R ? R : 0;
#pragma unroll
                for (int cc = 0; cc < C; cc++)
                    acc[cc][u & 1] = fma(-v4[u], ring[CK(cs * 32 * C + lane + 32 * cc, R * 32 * C, 6)], acc[cc][u & 1]);
            }
        }
        double s = 0.0;
#pragma unroll
        for (int cc = 0; cc < C; cc++) {
            const double x = acc[cc][0] + acc[cc][1];
            ring[CK(sr * 32 * C + lane + 32 * cc, R * 32 * C, 7)] = x;
            s += fabs(x);
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
        if (!(s <= A.tau)) first = r;  // NaN counts as significant
        sr = sr == 0 ? R - 1 : sr - 1;
    }
    if (lane == 0) A.first[blockIdx.x] = first;
}

// ---- the solve kernel -----------------------------------------------------------------

struct ChainArgs {
    const ChainTask *tasks;
    const double *val;
    const unsigned *off;
    const int *ptr;
    const double *rd;   // 1 / diagonal, padded to whole tiles
    int n;
    const double *b;    // caller order
    double *x;          // caller order
    int rev;            // uplo 'L': caller row i is U row n-1-i
    int mask;           // window rows - 1 (power of two >= reach + 32)
    int reach;          // widest column distance
    int sw;             // slots of the widest tile (stage size)
    long long nval, nptr, nrd;  // element counts (bounds of the checked build)
    int *err;
    int fail_entry;     // test hook: report a failed wait and return (spk_debug_set "fail_waits")
};

// cp.async (sm_80+): per-thread asynchronous global -> shared copies, tracked
// by commit groups (no register scoreboard, so a tile in flight never stalls
// the tile being solved)
__device__ __forceinline__ void cpa16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cpa8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cpa4(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// tiles staged in shared memory per task: the one solved + NS - 1 in flight (NS is
// a template parameter of the solve kernel, 2 or 3: s->ch_stages)

// One staged tile (sw = the widest tile's slots, a multiple of 4).  Lane l
// copies (and later reads) only its own row: value pairs v[(k/2)*32 + l],
// offset words o[(k/4)*32 + l], rd[l], b[l].
struct ChainStage {
    double2 *v;   // [16 sw]
    double *rd;   // [32]
    double *b;    // [32]
    unsigned *o;  // [8 sw]
};

__host__ __device__ __forceinline__ int chain_stage_bytes(int sw) { return 288 * sw + 512; }

__device__ __forceinline__ ChainStage chain_stage(unsigned char *base, int s, int sw) {
    unsigned char *p = base + (size_t)s * chain_stage_bytes(sw);
    ChainStage S;
    S.v = (double2 *)p;
    S.rd = (double *)(p + 256 * sw);
    S.b = S.rd + 32;
    S.o = (unsigned *)(p + 256 * sw + 512);
    return S;
}

template <int W>
__device__ __forceinline__ void stage_tile(const ChainArgs &A, const ChainStage &S, int j, int wq, int p0, int lo,
                                           int hi, int lane) {
    const double2 *vp = (const double2 *)A.val;
#pragma unroll
    for (int k = 0; k < W / 2; k++)
        if (2 * k < wq) cpa16(&S.v[CK(32 * k + lane, 16 * A.sw, 10)], vp + CK(p0 / 2 + 32 * k + lane, A.nval / 2, 11));
#pragma unroll
    for (int k = 0; k < W / 4; k++)
        if (4 * k < wq) cpa4(&S.o[CK(32 * k + lane, 8 * A.sw, 12)], A.off + CK((p0 >> 2) + 32 * k + lane, A.nval / 4, 13));
    const int r = 32 * j + lane;
    if (r >= lo && r < hi) {
        cpa8(&S.rd[lane], A.rd + CK(r, A.nrd, 14));
        cpa8(&S.b[lane], A.b + CK(A.rev ? A.n - 1 - r : r, A.n, 15));
    }
}

template <int W>
__device__ __forceinline__ void solve_tile(const ChainArgs &A, const ChainStage &S, int wq, int j,
                                           const ChainTask &t, double *coef, unsigned *msk, double *win, int lane) {
    const int row0 = 32 * j, r = row0 + lane;
    const bool act = r >= t.lo && r < t.hi;
    double acc = act ? S.b[lane] * S.rd[lane] : 0.0;
    double p[4] = {0.0, 0.0, 0.0, 0.0};
    unsigned mask = 0u;  // bit i: this row has the in-tile column row0 + i
    // In-tile columns go into the lane's coefficient column (and its mask),
    // far columns multiply the window value at their row.  Groups of eight
    // slots are branch-free (slots past the tile's width are dead), so the
    // loads of a group overlap.
#pragma unroll
    for (int g = 0; g < W / 8 + (W % 8 ? 1 : 0); g++) {
        if (8 * g < wq) {
            unsigned ow[2] = {0u, 0u};
            double2 v2[4];
#pragma unroll
            for (int h = 0; h < 2; h++)
                if (8 * g + 4 * h < W) ow[h] = S.o[CK(32 * (2 * g + h) + lane, 8 * A.sw, 16)];
#pragma unroll
            for (int h = 0; h < 4; h++)
                if (8 * g + 2 * h < W) v2[h] = S.v[CK(32 * (4 * g + h) + lane, 16 * A.sw, 17)];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int k = 8 * g + u;
                if (k < W) {
                    const int o = (int)((ow[u >> 2] >> (8 * (u & 3))) & 0xff);
                    const bool live = act && k < wq && o > 0;  // offset 0: padding
                    const int d = lane + o;
                    const double v = (u & 1) ? v2[u >> 1].y : v2[u >> 1].x;
                    if (live && d < 32) {
                        coef[d * 32 + lane] = v;
                        mask |= 1u << d;
                    }
                    if (live && d >= 32) p[u & 3] = fma(v, win[(row0 + d) & A.mask], p[u & 3]);
                }
            }
        }
    }
    acc -= (p[0] + p[1]) + (p[2] + p[3]);
    msk[lane] = mask;
    __syncwarp();  // the block coefficients and masks below are other lanes'
    // In-tile triangle, bottom-up, four rows per step: the four accumulators are
    // broadcast together, every lane resolves the block's four unknowns from the
    // block's six coefficients and applies all four columns.  Coefficients are
    // read under the masks (a column no row of this tile set holds an older
    // tile's value and is never used), so nothing is cleared between tiles.
#pragma unroll
    for (int i = 31; i >= 3; i -= 4) {
        const uint4 mq = *reinterpret_cast<const uint4 *>(msk + i - 3);  // rows i-3 .. i
        auto cf = [&](bool has, int col, int row) { return has ? coef[col * 32 + row] : 0.0; };
        const double c0 = cf((mask >> i) & 1u, i, lane), c1 = cf((mask >> (i - 1)) & 1u, i - 1, lane);
        const double c2 = cf((mask >> (i - 2)) & 1u, i - 2, lane), c3 = cf((mask >> (i - 3)) & 1u, i - 3, lane);
        const double u10 = cf((mq.z >> i) & 1u, i, i - 1);
        const double u20 = cf((mq.y >> i) & 1u, i, i - 2), u21 = cf((mq.y >> (i - 1)) & 1u, i - 1, i - 2);
        const double u30 = cf((mq.x >> i) & 1u, i, i - 3), u31 = cf((mq.x >> (i - 1)) & 1u, i - 1, i - 3);
        const double u32 = cf((mq.x >> (i - 2)) & 1u, i - 2, i - 3);
        const double b0 = __shfl_sync(kFull, acc, i), b1 = __shfl_sync(kFull, acc, i - 1);
        const double b2 = __shfl_sync(kFull, acc, i - 2), b3 = __shfl_sync(kFull, acc, i - 3);
        const double a1 = fma(-u10, b0, b1);
        const double a2 = fma(-u21, a1, fma(-u20, b0, b2));
        const double a3 = fma(-u32, a2, fma(-u31, a1, fma(-u30, b0, b3)));
        const double t01 = fma(-c1, a1, fma(-c0, b0, acc));
        acc = fma(-c3, a3, fma(-c2, a2, t01));
    }
    if (act) {
        win[r & A.mask] = acc;
        if (r >= t.st_lo && r < t.st_hi) A.x[CK(A.rev ? A.n - 1 - r : r, A.n, 18)] = acc;
    }
    __syncwarp();  // window rows and coefficient reads done before the next tile
}

// PRE: phase 4 (the window starts with x of rows [hi, hi + window)); else
// phase 1 (it starts at zero: zero coupling beyond the chain).
template <bool PRE, int W, int NS>
__global__ void __launch_bounds__(32) k_chain_solve(ChainArgs A) {
    constexpr int kChainStages = NS;
    extern __shared__ __align__(16) unsigned char smc[];
    ChainStage stg[kChainStages];
#pragma unroll
    for (int s = 0; s < kChainStages; s++) stg[s] = chain_stage(smc, s, A.sw);
    double *coef = (double *)(smc + kChainStages * chain_stage_bytes(A.sw));  // [32 columns][32 lanes]
    unsigned *msk = (unsigned *)(coef + 32 * 32);                             // [32] in-tile column masks
    double *win = coef + 32 * 32 + 16;                                        // [mask + 1]
    const int lane = threadIdx.x;
    if (A.fail_entry) {
        if (lane == 0) atomicExch(A.err, 1);
        return;
    }
    const ChainTask t = A.tasks[blockIdx.x];
    for (int k = lane; k <= A.mask; k += 32) {
        const int r = t.hi + k;
        double v = 0.0;
        if (PRE && r < A.n && k < A.reach) v = A.x[CK(A.rev ? A.n - 1 - r : r, A.n, 19)];  // the coupling rows only
        win[r & A.mask] = v;
    }
    __syncwarp();
    const int jt = (t.hi - 1) >> 5, jb = t.lo >> 5;
    // slot counts of the tiles, 32 at a time: lane l holds tile (base - l)'s
    auto ptr_pair = [&](int base, int &p0, int &p1) {
        const int jj = base - lane;
        p0 = jj >= jb ? __ldg(A.ptr + CK(jj, A.nptr, 20)) : 0;
        p1 = jj >= jb ? __ldg(A.ptr + CK(jj + 1, A.nptr, 21)) : 0;
    };
    int pbase = jt, pa, pb;
    ptr_pair(pbase, pa, pb);
    auto tile_ptr = [&](int jj, int &p0, int &wq) {
        if (pbase - jj >= 32) {  // uniform: the next 32 tiles' pointers
            pbase -= 32;
            ptr_pair(pbase, pa, pb);
        }
        p0 = __shfl_sync(kFull, pa, pbase - jj);
        wq = (__shfl_sync(kFull, pb, pbase - jj) - p0) >> 5;
    };
    int wq_st[kChainStages];
#pragma unroll
    for (int s = 0; s < kChainStages - 1; s++) {
        const int jj = jt - s;
        if (jj >= jb) {
            int p0;
            tile_ptr(jj, p0, wq_st[s]);
            stage_tile<W>(A, stg[s], jj, wq_st[s], p0, t.lo, t.hi, lane);
        }
        cpa_commit();
    }
    for (int j0 = jt; j0 >= jb; j0 -= kChainStages) {
#pragma unroll
        for (int s = 0; s < kChainStages; s++) {
            const int j = j0 - s;
            if (j >= jb) {
                const int sl = (s + kChainStages - 1) % kChainStages;  // stage of tile j - (NS - 1)
                const int jl = j - (kChainStages - 1);
                if (jl >= jb) {
                    int p0;
                    tile_ptr(jl, p0, wq_st[sl]);
                    stage_tile<W>(A, stg[sl], jl, wq_st[sl], p0, t.lo, t.hi, lane);
                }
                cpa_commit();
                cpa_wait<kChainStages - 1>();  // this tile's copies have landed (own lane's)
                solve_tile<W>(A, stg[s], wq_st[s], j, t, coef, msk, win, lane);
            }
        }
    }
    cpa_wait<0>();
}

size_t chain_smem_bytes(const spk_system *s) {
    return (size_t)s->ch_stages * chain_stage_bytes(s->ch_sw) + sizeof(double) * (32 * 32 + 16 + s->ch_win);
}

template <bool PRE>
int launch_chain(spk_system *s, const ChainTask *tasks, int ntasks, const double *b, double *x, cudaStream_t st) {
    if (ntasks <= 0) return SPK_OK;
    ChainArgs A;
    A.tasks = tasks;
    A.val = s->ch_val.p;
    A.off = (const unsigned *)s->ch_off.p;
    A.ptr = s->ch_ptr.p;
    A.rd = s->rdiag.p;
    A.n = s->n;
    A.b = b;
    A.x = x;
    A.rev = s->uplo == 'L';
    A.mask = s->ch_win - 1;
    A.reach = s->ch_reach;
    A.sw = s->ch_sw;
    A.nval = (long long)s->ch_val.n;
    A.nptr = (long long)s->ch_ptr.n;
    A.nrd = (long long)s->rdiag.n;
    A.err = s->d_err.p;
    A.fail_entry = s->dbg_fail_waits > 0;
    auto go = [&](auto kern) -> int {
        SPK_TRY(allow_smem(kern));
        kern<<<ntasks, 32, chain_smem_bytes(s), st>>>(A);
        SPK_CUDA(cudaGetLastError());
        return SPK_OK;
    };
    if (s->ch_stages == 2) {
        switch (s->ch_width) {
            case 4: SPK_TRY(go(k_chain_solve<PRE, 4, 2>)); break;
            case 8: SPK_TRY(go(k_chain_solve<PRE, 8, 2>)); break;
            case 16: SPK_TRY(go(k_chain_solve<PRE, 16, 2>)); break;
            case 32: SPK_TRY(go(k_chain_solve<PRE, 32, 2>)); break;
            default: SPK_TRY(go(k_chain_solve<PRE, 64, 2>)); break;
        }
    } else {
        switch (s->ch_width) {
            case 4: SPK_TRY(go(k_chain_solve<PRE, 4, 3>)); break;
            case 8: SPK_TRY(go(k_chain_solve<PRE, 8, 3>)); break;
            case 16: SPK_TRY(go(k_chain_solve<PRE, 16, 3>)); break;
            case 32: SPK_TRY(go(k_chain_solve<PRE, 32, 3>)); break;
            default: SPK_TRY(go(k_chain_solve<PRE, 64, 3>)); break;
        }
    }
    s->launches++;
    return SPK_OK;
}

// ---- many right-hand sides --------------------------------------------------------------
//
// The same chains and tasks, up to 32 right-hand sides per pass.  A block of
// one or two warps walks one task bottom-up and shares its staged tiles; warp
// w owns right-hand sides [RPW w, RPW (w+1)) of the pass (RPW = 16 in FP64, 32
// in FP32) and a window of its own: [WR][9 vectors of 16 bytes] (row r at r mod
// WR, WR = reach + 32), eight vectors of right-hand sides and one of padding.
// Lane (q, kv) = (lane / 8, lane % 8) solves the row at place q of each group of
// four rows for the 16-byte vector kv of right-hand sides (2 FP64 or 4 FP32),
// so a quarter warp reads one window row as 128 contiguous bytes (no bank
// conflicts) and every load, address and slot weight serves a whole vector.
//
// A row's coefficients at offsets inside its own group (at most three, fixed
// by the row's place, row mod 4) are kept apart at preprocessing: the slot
// values the kernel reads have them zeroed, and near[row][0..3] holds them in
// the order the in-group chain applies them.  So the slot sums of the four rows
// read only rows of earlier groups and run side by side; the chain then hands
// each place's values to the lanes below it by shuffles (three steps).
//
// A tile (32 rows) is staged by cp.async one tile ahead: slot values, offset
// bytes and 1/diag; the row loop turns a slot's offset into its column's window
// row.  Right-hand sides and near coefficients are read straight into
// registers a group ahead of use; solved rows go to X from the row loop (one
// warp) or through a transpose of the tile (lane = row, two warps).

template <typename T>
struct RhsArgs {
    const ChainTask *tasks;
    const T *val;          // row-scaled values in T, chain layout, in-group coefficients zeroed
    const T *near;         // [rows][4] in-group coefficients in order of use
    const unsigned *off;
    const int *ptr;
    const T *rd;           // 1 / diagonal in T
    int n;
    const double *B;       // caller order, column-major
    long long ldb;
    double *X;             // caller order, column-major (FP64 output)
    long long ldx;
    int rev;
    int nk;                // right-hand sides in this pass (<= 32)
    int wr;                // window rows (reach + 32)
    int reach;             // widest column distance
    int sw;                // slots of the widest tile
    long long nval, nptr, nrd, nnear;  // element counts (bounds of the checked build)
    int *err;
    int fail_entry;
};

// Shared-memory vector loads and stores by 32-bit address (volatile with a
// memory clobber, so that the compiler keeps them in order with the other
// accesses of the window; the hardware schedule is left to the assembler).
__device__ __forceinline__ double2 lds_v(unsigned a, double2) {
    double2 v;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ float4 lds_v(unsigned a, float4) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ void sts_v(unsigned a, double2 v) {
    asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(a), "d"(v.x), "d"(v.y) : "memory");
}
__device__ __forceinline__ void sts_v(unsigned a, float4 v) {
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(a), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w) : "memory");
}

constexpr int kRowBytes = 144;  // a window row: 8 vectors of right-hand sides + 1 of padding

template <typename T>
struct RhsStage {
    T *v;         // [32 sw] as copied: pair (k/2)*32 + l holds slots k, k+1 of row l
    unsigned *o;  // [8 sw]  offset words (k/4)*32 + l
    T *rd;        // [32]
};

__host__ __device__ __forceinline__ int rhs_stage_bytes(int sw, int tsize) {
    return 32 * sw * tsize + 32 * sw + 32 * 8;
}

template <typename T>
__device__ __forceinline__ RhsStage<T> rhs_stage(unsigned char *base, int sw) {
    RhsStage<T> S;
    S.v = (T *)base;
    S.o = (unsigned *)(base + 32 * sw * sizeof(T));
    S.rd = (T *)(base + 32 * sw * sizeof(T) + 32 * sw);
    return S;
}

// cp.async of tile j: warp w copies the slot pairs k with k % nw == w (lane =
// row); warp 0 also 1/diag of the task's rows.
template <typename T, int W>
__device__ __forceinline__ void rhs_stage_tile(const RhsArgs<T> &A, const RhsStage<T> &S, int j, int p0, int wq,
                                               int lo, int hi, int lane, int w, int nw) {
#pragma unroll
    for (int k = 0; k < W / 2; k++) {
        if (k % nw == w && 2 * k < wq) {
            T *dst = S.v + CK(64 * k + 2 * lane, 32 * A.sw - 1, 30);
            const T *src = A.val + CK(p0 + 64 * k + 2 * lane, A.nval - 1, 31);
            if (sizeof(T) == 8) cpa16(dst, src);
            else cpa8(dst, src);
        }
    }
#pragma unroll
    for (int k = 0; k < W / 4; k++)
        if (k % nw == w && 4 * k < wq)
            cpa4(S.o + CK(32 * k + lane, 8 * A.sw, 32), A.off + CK((p0 >> 2) + 32 * k + lane, A.nval / 4, 33));
    const int r = 32 * j + lane;
    if (w == 0 && r >= lo && r < hi) {
        if (sizeof(T) == 8) cpa8(S.rd + lane, A.rd + CK(r, A.nrd, 34));
        else cpa4(S.rd + lane, A.rd + CK(r, A.nrd, 34));
    }
}

// The batched kernel's slot values and near coefficients (one thread per row
// of the chain layout, padding rows of the last tile included): a row at place
// p = 3 - (row mod 4) of its group of four has its coefficients at offsets
// 1..p moved out of the slots into near[row] = {coef at offset p, p-1, p-2, 0}
// (zero where the offset would be below 1): step d of the in-group chain applies
// entry d, the coefficient of the row at place d.
__global__ void k_chain_near(long long rows, const int *ptr, const double *val, const unsigned *off, double *valb,
                             double *near) {
    const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const long long j = r >> 5;
    const int l = (int)(r & 31);
    const int p0 = ptr[j], wq = (ptr[j + 1] - p0) >> 5;
    const int p = 3 - (l & 3);
    double n1 = 0.0, n2 = 0.0, n3 = 0.0;
    for (int k = 0; k < wq; k++) {
        const long long e = (long long)p0 + 64 * (k >> 1) + 2 * l + (k & 1);
        const unsigned ow = off[(p0 >> 2) + 32 * (k >> 2) + l];
        const int o = (int)((ow >> (8 * (k & 3))) & 0xff);
        double v = val[e];
        if (o >= 1 && o <= p) {
            n1 += o == 1 ? v : 0.0;
            n2 += o == 2 ? v : 0.0;
            n3 += o == 3 ? v : 0.0;
            v = 0.0;
        }
        valb[e] = v;
    }
    double *nr = near + 4 * r;
    nr[0] = p == 1 ? n1 : (p == 2 ? n2 : (p == 3 ? n3 : 0.0));
    nr[1] = p == 2 ? n1 : (p == 3 ? n2 : 0.0);
    nr[2] = p == 3 ? n1 : 0.0;
    nr[3] = 0.0;
}

template <typename T, int W, bool PRE>
__global__ void __launch_bounds__(64) k_chain_rhs(RhsArgs<T> A) {
    using V2 = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
    using VT = typename std::conditional<sizeof(T) == 8, double2, float4>::type;  // 16 bytes
    constexpr int V = 16 / (int)sizeof(T);  // right-hand sides per lane
    constexpr int RPW = 8 * V;              // right-hand sides per warp
    extern __shared__ __align__(16) unsigned char smr[];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
    const int q = lane >> 3, kv = lane & 7;  // place in the group of four, vector of right-hand sides
    if (A.fail_entry) {
        if (tid == 0) atomicExch(A.err, 1);
        return;
    }
    const int WR = A.wr;
    const int sb = rhs_stage_bytes(A.sw, sizeof(T));
    unsigned char *winb = smr + 2 * sb + w * WR * kRowBytes;  // this warp's window
    const unsigned wbase = (unsigned)__cvta_generic_to_shared(winb) + 16u * kv;  // this lane's vector
#ifdef SPK_DEVICE_CHECKS
    const unsigned wb = (unsigned)(WR * kRowBytes);
#endif
    const ChainTask t = A.tasks[blockIdx.x];
    const int n = A.n;
    const int c0 = RPW * w;
    const int nkw = max(0, min(RPW, A.nk - c0));
    // window: the coupling rows above the task (phase 4: x from phase 1; phase
    // 1: zero); farther rows start at zero, so that no stale value is ever read
    for (int e = lane; e < WR * RPW; e += 32) {
        const int i = e / RPW, k = e % RPW;
        const int r = t.hi + i;
        const bool ok = PRE && r < n && i < A.reach && k < nkw;
        const long long o = A.rev ? (long long)n - 1 - r : r;
        T *wr = (T *)(winb + (r % WR) * kRowBytes);
        wr[k] = ok ? (T)A.X[(long long)(c0 + k) * A.ldx + CK(o, n, 36)] : T(0);
    }
    // this lane's right-hand sides b[r][c0 + V kv + e] (0 outside the task or past nk)
    auto bload = [&](int r, double *bv) {
        const bool in = r >= t.lo && r < t.hi;
        const long long o = A.rev ? (long long)n - 1 - r : r;
#pragma unroll
        for (int e = 0; e < V; e++) {
            const int c = V * kv + e;
            bv[e] = (in && c < nkw) ? A.B[(long long)(c0 + c) * A.ldb + CK(o, n, 35)] : 0.0;
        }
    };
    const int jt = (t.hi - 1) >> 5, jb = t.lo >> 5;
    // this lane's row's in-group coefficients (0 outside the task)
    auto nload = [&](int r, T *c) {
        if (r >= t.lo && r < t.hi) {
            const VT *np = reinterpret_cast<const VT *>(A.near + CK(4ll * r, A.nnear - 3, 46));
            const VT u0 = np[0];
            c[0] = reinterpret_cast<const T *>(&u0)[0];
            c[1] = reinterpret_cast<const T *>(&u0)[1];
            if (sizeof(T) == 8) {
                const VT u1 = np[1];
                c[2] = reinterpret_cast<const T *>(&u1)[0];
            } else {
                c[2] = reinterpret_cast<const T *>(&u0)[2];
            }
        } else {
            c[0] = c[1] = c[2] = T(0);
        }
    };
    double bn[V];  // the next group's right-hand sides and coefficients (loaded a group ahead of use)
    T cn[3];
    {
        const int r0 = ((t.hi - 1 - 32 * jt) | 3) + 32 * jt - q;
        bload(r0, bn);
        nload(r0, cn);
    }
    auto tile_ptr = [&](int jj, int &p0, int &wq) {
        p0 = __ldg(A.ptr + CK(jj, A.nptr, 37));
        wq = (__ldg(A.ptr + CK(jj + 1, A.nptr, 38)) - p0) >> 5;
    };
    int p0n, wqn;
    tile_ptr(jt, p0n, wqn);
    rhs_stage_tile<T, W>(A, rhs_stage<T>(smr, A.sw), jt, p0n, wqn, t.lo, t.hi, lane, w, nw);
    cpa_commit();
    int wq_cur = wqn;
    if (jt - 1 >= jb) tile_ptr(jt - 1, p0n, wqn);
    for (int j = jt, it = 0; j >= jb; j--, it++) {
        const RhsStage<T> S = rhs_stage<T>(smr + (it & 1) * sb, A.sw);
        const int wq = wq_cur;
        __syncthreads();  // every warp is done with the other buffer
        if (j - 1 >= jb) {
            rhs_stage_tile<T, W>(A, rhs_stage<T>(smr + ((it + 1) & 1) * sb, A.sw), j - 1, p0n, wqn, t.lo, t.hi, lane,
                                 w, nw);
            wq_cur = wqn;
            if (j - 2 >= jb) tile_ptr(j - 2, p0n, wqn);
        }
        cpa_commit();
        cpa_wait<1>();
        __syncthreads();  // tile j has landed, every thread's copies
        const int row0 = 32 * j;
        const int base = row0 % WR;
        auto slot_of = [&](int i) {
            const int v = base + i;
            return v >= WR ? v - WR : v;
        };
        const int a0 = max(t.lo, row0), a1 = min(t.hi, row0 + 32);
        // groups of four rows, top first; lane (q, kv) solves the row at place q
        // for its V right-hand sides; rows below a0 are computed but not stored
        for (int top = (a1 - 1 - row0) | 3; top >= a0 - row0; top -= 4) {
            const int i = top - q;
            double bv[V];
#pragma unroll
            for (int e = 0; e < V; e++) bv[e] = bn[e];
            bload(row0 + i - 4, bn);
            T c3[3] = {cn[0], cn[1], cn[2]};
            nload(row0 + i - 4, cn);
            const T rd = S.rd[i];
            T acc[4][V];
#pragma unroll
            for (int e = 0; e < V; e++) {
                acc[0][e] = acc[1][e] = acc[2][e] = acc[3][e] = T(0);
            }
            const int si = slot_of(i);  // window row of this lane's row
#pragma unroll
            for (int g = 0; g < (W + 7) / 8; g++) {
                if (8 * g < wq) {
                    // eight slots (four in a half-filled group: the tile's slot
                    // count is a multiple of four): offsets, window loads, sums
                    constexpr int NS = W < 8 ? W : 8;
                    const bool full = 8 * g + 8 <= wq;
                    unsigned ow[2];
                    ow[0] = S.o[CK(64 * g + i, 8 * A.sw, 47)];
                    ow[1] = (NS > 4 && full) ? S.o[CK(64 * g + 32 + i, 8 * A.sw, 47)] : 0u;
                    VT xv[8];
#pragma unroll
                    for (int u = 0; u < NS; u++) {
                        if (u < 4 || full) {
                            int v = si + (int)((ow[u >> 2] >> (8 * (u & 3))) & 0xff);
                            v -= v >= WR ? WR : 0;
                            xv[u] = lds_v(wbase + CK((unsigned)(v * kRowBytes), wb, 42), VT{});
                        }
                    }
#pragma unroll
                    for (int hh = 0; hh < NS / 2; hh++) {
                        if (hh < 2 || full) {
                            const V2 vv = *reinterpret_cast<const V2 *>(S.v + CK(64 * (4 * g + hh) + 2 * i, 32 * A.sw - 1, 41));
                            const T *xa = reinterpret_cast<const T *>(&xv[2 * hh]);
                            const T *xb = reinterpret_cast<const T *>(&xv[2 * hh + 1]);
#pragma unroll
                            for (int e = 0; e < V; e++) {
                                acc[(2 * hh) & 3][e] = fma(vv.x, xa[e], acc[(2 * hh) & 3][e]);
                                acc[(2 * hh + 1) & 3][e] = fma(vv.y, xb[e], acc[(2 * hh + 1) & 3][e]);
                            }
                        }
                    }
                }
            }
            VT xr;
            T *x = reinterpret_cast<T *>(&xr);
#pragma unroll
            for (int e = 0; e < V; e++) x[e] = (T)bv[e] * rd - ((acc[0][e] + acc[1][e]) + (acc[2][e] + acc[3][e]));
            // the in-group chain: step d hands place d's values to the lanes
            // below it; rows at or above a1 (a task's first group only) keep
            // their window value, the group's lowest row is always below a1
            const unsigned ad = wbase + (unsigned)(slot_of(i) * kRowBytes);
            const int r = row0 + i;
            const bool first = row0 + top >= a1;
#pragma unroll
            for (int d = 0; d < 3; d++) {
                if (first && q == d && r >= a1) xr = lds_v(ad, VT{});
                VT bd;
                T *bdt = reinterpret_cast<T *>(&bd);
                const T *xs = reinterpret_cast<const T *>(&xr);
#pragma unroll
                for (int e = 0; e < V; e++) bdt[e] = __shfl_sync(0xffffffffu, xs[e], kv + 8 * d);
                if (q > d) {
#pragma unroll
                    for (int e = 0; e < V; e++) x[e] = fma(-c3[d], bdt[e], x[e]);
                }
            }
            if (r >= a0 && r < a1) {
                sts_v(ad, xr);
                // one warp: x straight from the row loop (four rows of a column
                // per 32-byte sector); two warps share the load/store path, and
                // the tile's transpose below keeps their stores coalesced
                if (nw == 1 && r >= t.st_lo && r < t.st_hi) {
                    const long long o = A.rev ? (long long)n - 1 - r : r;
#pragma unroll
                    for (int e = 0; e < V; e++)
                        if (V * kv + e < nkw)
                            A.X[(long long)(c0 + V * kv + e) * A.ldx + CK(o, n, 44)] = (double)x[e];
                }
            }
        }
        if (nw > 1) {
            __syncwarp();
            // x rows of this tile out (lane = row), one 16-byte vector per load
            const int r = row0 + lane;
            if (r >= a0 && r < a1 && r >= t.st_lo && r < t.st_hi) {
                const long long o = A.rev ? (long long)n - 1 - r : r;
                const unsigned ar = (unsigned)__cvta_generic_to_shared(winb) + (unsigned)(slot_of(lane) * kRowBytes);
                for (int k0 = 0; k0 < nkw; k0 += V) {
                    const VT val = lds_v(ar + 16u * (k0 / V), VT{});
                    const T *vt = reinterpret_cast<const T *>(&val);
#pragma unroll
                    for (int e = 0; e < V; e++)
                        if (k0 + e < nkw) A.X[(long long)(c0 + k0 + e) * A.ldx + CK(o, n, 44)] = (double)vt[e];
                }
            }
        }
    }
    cpa_wait<0>();
}

size_t rhs_smem_bytes(const spk_system *s, int tsize, int nw) {
    return 2 * (size_t)rhs_stage_bytes(s->ch_sw, tsize) + (size_t)nw * kRowBytes * (s->ch_reach + 32);
}

template <typename T, bool PRE>
int launch_chain_rhs(spk_system *s, const ChainTask *tasks, int ntasks, int nk, const double *B, long long ldb,
                     double *X, long long ldx, cudaStream_t st) {
    if (ntasks <= 0) return SPK_OK;
    const bool f64 = sizeof(T) == 8;
    RhsArgs<T> A;
    A.tasks = tasks;
    A.val = f64 ? (const T *)(const void *)s->ch_valb.p : (const T *)(const void *)s->ch_valbf.p;
    A.near = f64 ? (const T *)(const void *)s->ch_near.p : (const T *)(const void *)s->ch_nearf.p;
    A.off = (const unsigned *)s->ch_off.p;
    A.ptr = s->ch_ptr.p;
    A.rd = f64 ? (const T *)(const void *)s->rdiag.p : (const T *)(const void *)s->rdiagf.p;
    A.n = s->n;
    A.B = B;
    A.ldb = ldb;
    A.X = X;
    A.ldx = ldx;
    A.rev = s->uplo == 'L';
    A.nk = nk;
    A.wr = s->ch_reach + 32;
    A.reach = s->ch_reach;
    A.sw = s->ch_sw;
    A.nval = (long long)s->ch_val.n;
    A.nptr = (long long)s->ch_ptr.n;
    A.nrd = (long long)(f64 ? s->rdiag.n : s->rdiagf.n);
    A.nnear = (long long)s->ch_near.n;
    A.err = s->d_err.p;
    A.fail_entry = s->dbg_fail_waits > 0;
    const int rpw = 8 * (16 / (int)sizeof(T));  // right-hand sides per warp
    const int nw = (nk + rpw - 1) / rpw;
    const size_t smem = rhs_smem_bytes(s, sizeof(T), nw);
    auto go = [&](auto kern) -> int {
        SPK_TRY(allow_smem(kern));
        kern<<<ntasks, 32 * nw, smem, st>>>(A);
        SPK_CUDA(cudaGetLastError());
        return SPK_OK;
    };
    switch (s->ch_width) {
        case 4: SPK_TRY(go(k_chain_rhs<T, 4, PRE>)); break;
        case 8: SPK_TRY(go(k_chain_rhs<T, 8, PRE>)); break;
        case 16: SPK_TRY(go(k_chain_rhs<T, 16, PRE>)); break;
        case 32: SPK_TRY(go(k_chain_rhs<T, 32, PRE>)); break;
        default: SPK_TRY(go(k_chain_rhs<T, 64, PRE>)); break;
    }
    s->launches++;
    return SPK_OK;
}

template <typename T>
int upload_vec(DBuf<T> &d, const std::vector<T> &h) {
    SPK_TRY(d.alloc(h.size()));
    if (h.empty()) return SPK_OK;
    if (d.on_stream) SPK_CUDA(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, d.ord));
    else SPK_CUDA(cudaMemcpy(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return SPK_OK;
}

int spike_firsts(spk_system *s, const std::vector<int2> &chains, std::vector<int> &first) {
    DBuf<int2> d_ch(s->stream);
    DBuf<int> d_first(s->stream);
    SPK_TRY(upload_vec(d_ch, chains));
    SPK_TRY(d_first.alloc(chains.size()));
    SpikeArgs A;
    A.chains = d_ch.p;
    A.nchains = (int)chains.size();
    A.val = s->ch_val.p;
    A.off = (const unsigned *)s->ch_off.p;
    A.ptr = s->ch_ptr.p;
    A.reach = s->ch_reach;
    A.tau = s->trunc_tol;
    A.first = d_first.p;
    A.nval = (long long)s->ch_val.n;
    A.nptr = (long long)s->ch_ptr.n;
    const int C = s->ch_reach <= 32 ? 1 : (s->ch_reach <= 64 ? 2 : 4);
    const int smem = (int)sizeof(double) * (s->ch_reach + 1) * 32 * C;
    switch (C) {
        case 1:
            SPK_TRY(allow_smem(k_chain_spike<1>));
            k_chain_spike<1><<<A.nchains, 32, smem, s->stream>>>(A);
            break;
        case 2:
            SPK_TRY(allow_smem(k_chain_spike<2>));
            k_chain_spike<2><<<A.nchains, 32, smem, s->stream>>>(A);
            break;
        default:
            SPK_TRY(allow_smem(k_chain_spike<4>));
            k_chain_spike<4><<<A.nchains, 32, smem, s->stream>>>(A);
            break;
    }
    SPK_CUDA(cudaGetLastError());
    first.assign(chains.size(), 0);
    SPK_CUDA(cudaStreamSynchronize(s->stream));
    SPK_CUDA(cudaMemcpy(first.data(), d_first.p, sizeof(int) * chains.size(), cudaMemcpyDeviceToHost));
    return SPK_OK;
}

__global__ void k_chain_to_float(long long n, const double *__restrict__ a, float *__restrict__ b) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

// The batched kernel's slot values and near coefficients (FP64, and FP32 when
// fp32), made on the first batched solve that needs them.
int chain_batch_values(spk_system *s, int fp32) {
    if (!s->ch_valb.p) {
        const long long rows = 32ll * ((long long)s->ch_ptr.n - 1);
        SPK_TRY(s->ch_valb.alloc(s->ch_val.n));
        SPK_TRY(s->ch_near.alloc(std::max(4 * rows, 4ll)));
        k_chain_near<<<(unsigned)((rows + 255) / 256), 256, 0, s->stream>>>(
            rows, s->ch_ptr.p, s->ch_val.p, (const unsigned *)s->ch_off.p, s->ch_valb.p, s->ch_near.p);
        SPK_CUDA(cudaGetLastError());
        SPK_CUDA(cudaStreamSynchronize(s->stream));
    }
    if (fp32 && !s->ch_valbf.p) {
        SPK_TRY(s->ch_valbf.alloc(s->ch_valb.n));
        SPK_TRY(s->ch_nearf.alloc(s->ch_near.n));
        if (!s->rdiagf.p) {
            SPK_TRY(s->rdiagf.alloc(s->rdiag.n));
            k_chain_to_float<<<1184, 256, 0, s->stream>>>((long long)s->rdiag.n, s->rdiag.p, s->rdiagf.p);
        }
        k_chain_to_float<<<1184, 256, 0, s->stream>>>((long long)s->ch_valb.n, s->ch_valb.p, s->ch_valbf.p);
        k_chain_to_float<<<1184, 256, 0, s->stream>>>((long long)s->ch_near.n, s->ch_near.p, s->ch_nearf.p);
        SPK_CUDA(cudaGetLastError());
        SPK_CUDA(cudaStreamSynchronize(s->stream));
    }
    return SPK_OK;
}

void chain_release(spk_system *s) {
    s->chain_ok = 0;
    s->batch_path = -1;
    s->ch_val.release();
    s->ch_valb.release();
    s->ch_valbf.release();
    s->ch_near.release();
    s->ch_nearf.release();
    s->ch_off.release();
    s->ch_ptr.release();
    s->d_ctasks1.release();
    s->d_ctasks4.release();
    s->cp_batch.release();
    s->cp_host.release();
    s->host_plan_tried = 0;
    if (s->pipe_exec) cudaGraphExecDestroy(s->pipe_exec);
    s->pipe_exec = nullptr;
    s->pipe_b = s->pipe_db = nullptr;
    s->pipe_x = s->pipe_dx = nullptr;
    s->pipe_K = 0;
    s->h_ctasks1.clear();
    s->h_ctasks4.clear();
    s->nctasks1 = s->nctasks4 = 0;
    s->ch_rows1 = s->ch_rows4 = 0;
    s->ch_count = 0;
    s->ch_len = 0;
}

}  // namespace

int chain_occupancy(spk_system *s, int *occ);
int chain_rhs_occupancy(spk_system *s, int *occ);
int build_plan(spk_system *s, long long len, int reach, ChainPlan *extra);

// Build the chain layout, the chains' spikes and the two task lists; leaves
// chain_ok = 0 (the partition-based solve) when truncation is off, the layout
// does not apply (column distance > 128, more than 64 off-diagonals in a row),
// or no chain length up to the limit keeps every chain's first rows final.
int chain_prepare(spk_system *s) {
    chain_release(s);
    const char *dis = getenv("SPK_DISABLE_CHAIN");  // test hook: force the partition-based solve
    if (s->trunc_tol < 0 || (dis && dis[0] == '1') || s->n < 64) return SPK_OK;
    const int n = s->n, ntiles = (n + 31) / 32;
    std::vector<int> hw(ntiles);
    int reach = 0;
    {
        DBuf<int> width(s->stream), d_reach(s->stream);
        SPK_TRY(width.alloc(ntiles));
        SPK_TRY(d_reach.alloc(1));
        SPK_CUDA(cudaMemsetAsync(d_reach.p, 0, sizeof(int), s->stream));
        k_chain_scan<<<nblocks(32ll * ntiles), 256, 0, s->stream>>>(n, s->uia.p, s->uja.p, width.p, d_reach.p);
        SPK_CUDA(cudaGetLastError());
        SPK_CUDA(cudaStreamSynchronize(s->stream));
        SPK_CUDA(cudaMemcpy(hw.data(), width.p, sizeof(int) * ntiles, cudaMemcpyDeviceToHost));
        SPK_CUDA(cudaMemcpy(&reach, d_reach.p, sizeof(int), cudaMemcpyDeviceToHost));
    }
    int wmax = 0;
    std::vector<int> ptr(ntiles + 1, 0);
    long long tot = 0;
    for (int j = 0; j < ntiles; j++) {
        const int wq = (hw[j] + 3) & ~3;
        wmax = std::max(wmax, wq);
        ptr[j] = (int)std::min<long long>(tot, 2147483647ll);
        tot += 32ll * wq;
    }
    if (reach < 1 || reach > 128 || wmax > 64 || tot >= 2147483647ll) return SPK_OK;
    ptr[ntiles] = (int)tot;
    s->ch_width = wmax <= 4 ? 4 : (wmax <= 8 ? 8 : (wmax <= 16 ? 16 : (wmax <= 32 ? 32 : 64)));
    s->ch_sw = (wmax + 7) & ~7;  // stages hold whole groups of eight slots
    // two stages (one tile in flight) measured as fast as three on the banded
    // workload and leave room for more resident tasks when tiles are wide
    s->ch_stages = 2;
    if (const char *e = getenv("SPK_CHAIN_STAGES")) s->ch_stages = atoi(e) == 3 ? 3 : 2;
    s->ch_reach = reach;
    int win = 64;
    while (win < reach + 32) win <<= 1;
    s->ch_win = win;
    SPK_TRY(upload_vec(s->ch_ptr, ptr));
    SPK_TRY(s->ch_val.alloc(std::max<long long>(tot, 2)));
    SPK_TRY(s->ch_off.alloc(std::max<long long>(tot, 4)));
    k_chain_fill<<<nblocks(32ll * ntiles), 256, 0, s->stream>>>(n, ntiles, s->uia.p, s->uja.p, s->ua.p,
                                                                 s->ch_ptr.p, s->ch_val.p, s->ch_off.p);
    SPK_CUDA(cudaGetLastError());

    // chain length: as many chains as the solve kernel keeps resident on the
    // GPU at once (one wave), at least 1024 rows; doubled until valid
    int dev = 0, sms = 148, occ = 8;
    SPK_CUDA(cudaGetDevice(&dev));
    SPK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    SPK_TRY(chain_occupancy(s, &occ));
    // (seven per SM at most: with more, phase 1 gains nothing and phase 4 grows)
    long long len = 32ll * ((n / (sms * (long long)std::min(std::max(occ, 1), 7)) + 31) / 32);
    len = std::max<long long>(len, 1024);
    if (const char *e = getenv("SPK_CHAIN_ROWS")) len = std::max(32ll, 32ll * ((atoll(e) + 31) / 32));
    SPK_TRY(build_plan(s, len, reach, nullptr));
    if (!s->chain_ok) return SPK_OK;
    // the batched kernel keeps fewer tasks resident (a wider window): its own
    // chains, as many as it keeps resident
    int occb = 4;
    SPK_TRY(chain_rhs_occupancy(s, &occb));
    long long lenb = 32ll * ((n / (sms * (long long)std::max(occb, 1)) + 31) / 32);
    lenb = std::max<long long>(lenb, s->ch_len);
    if (const char *e = getenv("SPK_CHAIN_BATCH_ROWS")) lenb = std::max(32ll, 32ll * ((atoll(e) + 31) / 32));
    if (lenb > s->ch_len) SPK_TRY(build_plan(s, lenb, reach, &s->cp_batch));
    return SPK_OK;
}

// Chains of `len` rows (doubled up to three times until every chain keeps its
// first `reach` rows, never fewer than 8 chains): their spikes, the two task
// lists (row order: the pipelined and sharded solves launch them by row range).
// extra == nullptr: the plain solve's plan (sets chain_ok, or releases everything
// when no length is valid); else a second plan (left unbuilt, so that the plain
// plan's tasks are used, when no length short of the plain one is valid).
int build_plan(spk_system *s, long long len, int reach, ChainPlan *extra) {
    const int n = s->n;
    const long long max_len = std::min<long long>(8 * len, std::max<long long>(len, 32ll * ((n / 8 + 31) / 32)));
    for (; len <= max_len; len *= 2) {
        if (extra && len == s->ch_len) break;  // the same chains as the plain solve
        std::vector<int2> chains;
        for (long long a = 0; a < n; a += len)
            chains.push_back(make_int2((int)a, (int)std::min<long long>(a + len, n)));
        std::vector<int> first;
        SPK_TRY(spike_firsts(s, chains, first));
        bool ok = true;
        for (size_t c = 1; c < chains.size() && ok; c++)
            ok = first[c] >= std::min(chains[c].x + reach, chains[c].y);
        if (!ok) continue;
        std::vector<ChainTask> t1, t4;
        long long rows1 = 0, rows4 = 0;
        for (size_t c = 0; c < chains.size(); c++) {
            const int a = chains[c].x, q = chains[c].y, f = first[c];
            t1.push_back(ChainTask{a, q, a, f});
            rows1 += q - a;
            if (f < q) {
                t4.push_back(ChainTask{f, q, f, q});
                rows4 += q - f;
            }
        }
        if (extra) {
            SPK_TRY(upload_vec(extra->d1, t1));
            SPK_TRY(upload_vec(extra->d4, t4));
            extra->h1 = t1;
            extra->h4 = t4;
            extra->len = (int)len;
            return SPK_OK;
        }
        s->h_ctasks1 = t1;
        s->h_ctasks4 = t4;
        SPK_TRY(upload_vec(s->d_ctasks1, t1));
        SPK_TRY(upload_vec(s->d_ctasks4, t4));
        s->nctasks1 = (int)t1.size();
        s->nctasks4 = (int)t4.size();
        s->ch_rows1 = rows1;
        s->ch_rows4 = rows4;
        s->ch_count = (int)chains.size();
        s->ch_len = (int)len;
        s->chain_ok = 1;
        return SPK_OK;
    }
    if (extra) {
        extra->release();  // the plain solve's tasks are used
        return SPK_OK;
    }
    chain_release(s);
    return SPK_OK;
}

// Resident blocks per SM of the phase-1 solve kernel (its shared memory bounds it).
int chain_occupancy(spk_system *s, int *occ) {
    const size_t smem = chain_smem_bytes(s);
    auto q = [&](auto kern) -> int {
        SPK_TRY(allow_smem(kern));
        SPK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, 32, smem));
        return SPK_OK;
    };
    const bool two = s->ch_stages == 2;
    switch (s->ch_width) {
        case 4: return two ? q(k_chain_solve<false, 4, 2>) : q(k_chain_solve<false, 4, 3>);
        case 8: return two ? q(k_chain_solve<false, 8, 2>) : q(k_chain_solve<false, 8, 3>);
        case 16: return two ? q(k_chain_solve<false, 16, 2>) : q(k_chain_solve<false, 16, 3>);
        case 32: return two ? q(k_chain_solve<false, 32, 2>) : q(k_chain_solve<false, 32, 3>);
        default: return two ? q(k_chain_solve<false, 64, 2>) : q(k_chain_solve<false, 64, 3>);
    }
}

// Resident blocks per SM of the batched (FP64) chain kernel.
int chain_rhs_occupancy(spk_system *s, int *occ) {
    const size_t smem = rhs_smem_bytes(s, sizeof(double), 2);
    auto q = [&](auto kern) -> int {
        SPK_TRY(allow_smem(kern));
        SPK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, 64, smem));
        return SPK_OK;
    };
    switch (s->ch_width) {
        case 4: return q(k_chain_rhs<double, 4, false>);
        case 8: return q(k_chain_rhs<double, 8, false>);
        case 16: return q(k_chain_rhs<double, 16, false>);
        case 32: return q(k_chain_rhs<double, 32, false>);
        default: return q(k_chain_rhs<double, 64, false>);
    }
}

// One solve of host arrays b and x through the chain path with the copies
// overlapped: the rows are cut into chunks of whole chains (U order), each with
// a stream of its own.  Chunk k's right-hand side is copied in on s->st_in; its
// phase 1 starts on its stream once that copy has landed (chunks run side by
// side: a chain is a serial walk, so one chunk alone leaves most SMs idle);
// its phase 4 waits for phase 1 of chunk k+1 (it reads the first rows of the
// chain below); its x is copied out on s->st_out once its phase 4 is done.  One
// cudaMemcpyAsync per chunk and direction; overlap needs page-locked b and x
// (pageable memory gives the same result with the copies serialised).
int chain_pipeline(spk_system *s, const double *b, double *x, double *db, double *dx, int K);

int chain_solve_host(spk_system *s, const double *b, double *x, double *db, double *dx) {
    // After the last copy lands, one chain still has to be solved before its rows
    // can leave: the pipeline takes chains of at most 2,048 rows (built once,
    // on the first host-array solve) to shorten that tail.
    if (!s->host_plan_tried) {
        s->host_plan_tried = 1;
        long long len = 2048;
        if (const char *e = getenv("SPK_PIPELINE_ROWS")) len = std::max(32ll, 32ll * ((atoll(e) + 31) / 32));
        if (len < s->ch_len) SPK_TRY(build_plan(s, len, s->ch_reach, &s->cp_host));
    }
    const int nch = (int)(s->cp_host.len > 0 ? s->cp_host.h1.size() : s->h_ctasks1.size());
    int K = 16;
    if (const char *e = getenv("SPK_PIPELINE_CHUNKS")) K = std::max(1, atoi(e));
    K = std::min(K, std::max(nch, 1));
    if (!s->st_in) {
        SPK_CUDA(cudaStreamCreateWithFlags(&s->st_in, cudaStreamNonBlocking));
        SPK_CUDA(cudaStreamCreateWithFlags(&s->st_out, cudaStreamNonBlocking));
    }
    while ((int)s->pipe_st.size() < K) {
        cudaStream_t q;
        SPK_CUDA(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
        s->pipe_st.push_back(q);
    }
    while ((int)s->pipe_ev.size() < 3 * K + 1) {
        cudaEvent_t e;
        SPK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        s->pipe_ev.push_back(e);
    }
    // the same page-locked b and x (and device copies, chunk count) as the last
    // call: replay the pipeline captured then; the second such call captures it
    const bool same = s->pipe_b == b && s->pipe_x == x && s->pipe_db == db && s->pipe_dx == dx && s->pipe_K == K;
    if (same && s->pipe_exec) {
        SPK_CUDA(cudaGraphLaunch(s->pipe_exec, s->stream));
        SPK_CUDA(cudaStreamSynchronize(s->stream));
        return SPK_OK;
    }
    if (!same) {
        if (s->pipe_exec) cudaGraphExecDestroy(s->pipe_exec);
        s->pipe_exec = nullptr;
        s->pipe_b = b;
        s->pipe_x = x;
        s->pipe_db = db;
        s->pipe_dx = dx;
        s->pipe_K = K;
    }
    auto locked = [](const void *p) {
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return at.type == cudaMemoryTypeHost;
    };
    const bool capture = same && !s->pipe_nograph && locked(b) && locked(x);
    if (capture) SPK_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = chain_pipeline(s, b, x, db, dx, K);
    if (capture) {
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(s->stream, &g);
        cudaGraphExec_t ex = nullptr;
        if (rc == SPK_OK && e == cudaSuccess) e = cudaGraphInstantiate(&ex, g, 0);
        if (g) cudaGraphDestroy(g);
        if (rc != SPK_OK) return rc;
        if (e == cudaSuccess) {
            s->pipe_exec = ex;
            SPK_CUDA(cudaGraphLaunch(ex, s->stream));
        } else {
            cudaGetLastError();
            s->pipe_nograph = 1;  // not capturable here: the direct pipeline from now on
            SPK_TRY(chain_pipeline(s, b, x, db, dx, K));
        }
    } else {
        SPK_TRY(rc);
    }
    SPK_CUDA(cudaStreamSynchronize(s->stream));
    return SPK_OK;
}

// The pipeline's copies and launches, forked from and joined back to the
// system's stream (nothing here synchronizes: it may be captured).
int chain_pipeline(spk_system *s, const double *b, double *x, double *db, double *dx, int K) {
    const ChainPlan &hp = s->cp_host;
    const bool own = hp.len > 0;
    const std::vector<ChainTask> &T1 = own ? hp.h1 : s->h_ctasks1, &T4 = own ? hp.h4 : s->h_ctasks4;
    const ChainTask *D1 = own ? hp.d1.p : s->d_ctasks1.p, *D4 = own ? hp.d4.p : s->d_ctasks4.p;
    const int n = s->n, nch = (int)T1.size(), n4 = (int)T4.size();
    cudaEvent_t *ev_in = s->pipe_ev.data(), *ev_p1 = ev_in + K, *ev_done = ev_in + 2 * K, *ev_start = ev_in + 3 * K;
    const bool rev = s->uplo == 'L';
    // chunk k: chains [c0(k), c0(k+1)), U rows [A(k), Q(k)), phase-4 tasks [t0(k), t0(k+1))
    std::vector<int> c0(K + 1), t0(K + 1, 0);
    for (int k = 0; k <= K; k++) c0[k] = (int)((long long)nch * k / K);
    {
        int t = 0;
        for (int k = 0; k < K; k++) {
            t0[k] = t;
            const int qend = T1[c0[k + 1] - 1].hi;
            while (t < n4 && T4[t].hi <= qend) t++;
        }
        t0[K] = n4;
    }
    auto lo_rows = [&](int k, int &lo, int &cnt) {
        const int A = T1[c0[k]].lo, Q = T1[c0[k + 1] - 1].hi;
        lo = rev ? n - Q : A;
        cnt = Q - A;
    };
    // everything starts after the work already queued on the system's stream
    SPK_CUDA(cudaEventRecord(ev_start[0], s->stream));
    SPK_CUDA(cudaStreamWaitEvent(s->st_in, ev_start[0], 0));
    SPK_CUDA(cudaStreamWaitEvent(s->st_out, ev_start[0], 0));
    for (int k = 0; k < K; k++) {
        int lo, cnt;
        lo_rows(k, lo, cnt);
        SPK_CUDA(cudaMemcpyAsync(db + lo, b + lo, sizeof(double) * cnt, cudaMemcpyHostToDevice, s->st_in));
        SPK_CUDA(cudaEventRecord(ev_in[k], s->st_in));
    }
    // chunk k's phase 1 on stream k; phase 4 of chunk k-1 (which reads the first
    // rows of chunk k) right behind it on the same stream: streams share the
    // device's hardware queues, and a launch queued behind one it does not
    // depend on would wait for it
    for (int k = 0; k <= K; k++) {
        if (k < K) {
            cudaStream_t q = s->pipe_st[k];
            SPK_CUDA(cudaStreamWaitEvent(q, ev_in[k], 0));
            SPK_TRY(launch_chain<false>(s, D1 + c0[k], c0[k + 1] - c0[k], db, dx, q));
            SPK_CUDA(cudaEventRecord(ev_p1[k], q));
        }
        if (k > 0) {
            const int j = k - 1;
            cudaStream_t q = s->pipe_st[k < K ? k : K - 1];
            if (k < K) SPK_CUDA(cudaStreamWaitEvent(q, ev_p1[j], 0));
            SPK_TRY(launch_chain<true>(s, D4 + t0[j], t0[j + 1] - t0[j], db, dx, q));
            SPK_CUDA(cudaEventRecord(ev_done[j], q));
            int lo, cnt;
            lo_rows(j, lo, cnt);
            SPK_CUDA(cudaStreamWaitEvent(s->st_out, ev_done[j], 0));
            SPK_CUDA(cudaMemcpyAsync(x + lo, dx + lo, sizeof(double) * cnt, cudaMemcpyDeviceToHost, s->st_out));
        }
    }
    // the system's stream continues after the whole solve
    SPK_CUDA(cudaEventRecord(ev_start[0], s->st_out));
    SPK_CUDA(cudaStreamWaitEvent(s->stream, ev_start[0], 0));
    return SPK_OK;
}

// Up to 32 right-hand sides (device, column-major) through the chain path:
// phase 1 then phase 4 of the right-hand-side-parallel chain kernel, in T
// (double, or float with the FP32 copy of the values).  X is FP64.
int chain_solve_rhs(spk_system *s, int fp32, int nk, const double *B, long long ldb, double *X, long long ldx,
                    cudaStream_t st) {
    if (nk < 1 || nk > 32) {
        set_error(SPK_ERR_ARG, "chain batch of %d columns (1..32)", nk);
        return SPK_ERR_ARG;
    }
    const ChainPlan &bp = s->cp_batch;
    const bool own = bp.len > 0;  // the batched kernel's own chains
    const ChainTask *t1 = own ? bp.d1.p : s->d_ctasks1.p, *t4 = own ? bp.d4.p : s->d_ctasks4.p;
    const int n1 = own ? (int)bp.h1.size() : s->nctasks1, n4 = own ? (int)bp.h4.size() : s->nctasks4;
    SPK_TRY(chain_batch_values(s, fp32));
    if (fp32) {
        SPK_TRY((launch_chain_rhs<float, false>(s, t1, n1, nk, B, ldb, X, ldx, st)));
        SPK_TRY((launch_chain_rhs<float, true>(s, t4, n4, nk, B, ldb, X, ldx, st)));
    } else {
        SPK_TRY((launch_chain_rhs<double, false>(s, t1, n1, nk, B, ldb, X, ldx, st)));
        SPK_TRY((launch_chain_rhs<double, true>(s, t4, n4, nk, B, ldb, X, ldx, st)));
    }
    return SPK_OK;
}

// The tasks of one phase whose chains lie in U rows [row_lo, row_hi): phase 1
// tasks start at their chain's first row, phase 4 tasks end at its last row.
int chain_phase(spk_system *s, int phase, int row_lo, int row_hi, const double *b, double *x, cudaStream_t st) {
    const std::vector<ChainTask> &v = phase == 1 ? s->h_ctasks1 : s->h_ctasks4;
    int i0 = 0, i1 = 0;
    for (i0 = 0; i0 < (int)v.size() && (phase == 1 ? v[i0].lo : v[i0].hi - 1) < row_lo; i0++) {}
    for (i1 = i0; i1 < (int)v.size() && (phase == 1 ? v[i1].hi : v[i1].hi) <= row_hi; i1++) {}
    if (phase == 1) return launch_chain<false>(s, s->d_ctasks1.p + i0, i1 - i0, b, x, st);
    return launch_chain<true>(s, s->d_ctasks4.p + i0, i1 - i0, b, x, st);
}

// The first failed check of a checked build (0: none, or not a checked build).
long long chain_device_check() {
#ifdef SPK_DEVICE_CHECKS
    unsigned long long v = 0;
    if (cudaMemcpyFromSymbol(&v, g_chain_check, sizeof(v)) != cudaSuccess) return -1;
    return (long long)v;
#else
    return 0;
#endif
}

// One solve through the chain path: phase 1 then phase 4 on stream st.
int chain_solve(spk_system *s, const double *b, double *x, cudaStream_t st, bool prof, int ring) {
    SPK_TRY(launch_chain<false>(s, s->d_ctasks1.p, s->nctasks1, b, x, st));
    if (prof) {
        cudaEventRecord(s->ev[ring][1], st);
        cudaEventRecord(s->ev[ring][2], st);
    }
    SPK_TRY(launch_chain<true>(s, s->d_ctasks4.p, s->nctasks4, b, x, st));
    return SPK_OK;
}

// Tuning knobs of a system solved by chains (spk_tune).  A changed plan or stage
// count drops the captured host-array pipeline (it holds the old launches); the
// caller keeps the system's solves off the GPU meanwhile (the device is
// synchronized before task lists are replaced).
int chain_tune(spk_system *s, const char *name, long long v) {
    if (!s->chain_ok) {
        set_error(SPK_ERR_STATE, "spk_tune needs a system solved by chains");
        return SPK_ERR_STATE;
    }
    auto drop_pipeline = [&]() {
        if (s->pipe_exec) cudaGraphExecDestroy(s->pipe_exec);
        s->pipe_exec = nullptr;
        s->pipe_b = s->pipe_db = nullptr;
        s->pipe_x = s->pipe_dx = nullptr;
        s->pipe_K = 0;
    };
    if (!strcmp(name, "stages")) {  // tiles staged by the one-right-hand-side kernel
        if (v != 2 && v != 3) {
            set_error(SPK_ERR_ARG, "stages must be 2 or 3 (got %lld)", v);
            return SPK_ERR_ARG;
        }
        SPK_CUDA(cudaDeviceSynchronize());
        s->ch_stages = (int)v;
        drop_pipeline();
        return SPK_OK;
    }
    if (!strcmp(name, "batch_path")) {  // 1 chain kernels, 0 partition kernels, -1 automatic
        if (v < -1 || v > 1 || (v == 0 && s->lean)) {
            set_error(SPK_ERR_ARG, "batch_path must be -1, 0 or 1 (0 needs the partition pools: not compacted)");
            return SPK_ERR_ARG;
        }
        s->batch_path = (int)v;
        return SPK_OK;
    }
    const bool plain = !strcmp(name, "rows");
    if (!plain && strcmp(name, "batch_rows")) {
        set_error(SPK_ERR_ARG, "unknown tuning knob '%s' (rows, batch_rows, stages, batch_path)", name);
        return SPK_ERR_ARG;
    }
    // rows per chain task, whole tiles; build_plan doubles the length (at most
    // three times) until every chain keeps its first rows final
    if (v < 32 || v > s->n) {
        set_error(SPK_ERR_ARG, "%s must be in [32, n] (got %lld)", name, v);
        return SPK_ERR_ARG;
    }
    const long long len = 32ll * ((v + 31) / 32);
    ChainPlan fresh;
    const int keep_len = s->ch_len;
    s->ch_len = 0;  // so that build_plan builds the extra plan even at the plain length
    const int rc = build_plan(s, len, s->ch_reach, &fresh);
    s->ch_len = keep_len;
    SPK_TRY(rc);
    if (!fresh.len) {
        set_error(SPK_ERR_ARG, "no chain length from %lld rows keeps every chain's first rows final", len);
        return SPK_ERR_ARG;
    }
    SPK_CUDA(cudaDeviceSynchronize());
    if (!plain) {
        s->cp_batch.release();
        s->cp_batch.d1.p = fresh.d1.p, s->cp_batch.d1.n = fresh.d1.n, fresh.d1.p = nullptr;
        s->cp_batch.d4.p = fresh.d4.p, s->cp_batch.d4.n = fresh.d4.n, fresh.d4.p = nullptr;
        s->cp_batch.h1.swap(fresh.h1);
        s->cp_batch.h4.swap(fresh.h4);
        s->cp_batch.len = fresh.len;
        return SPK_OK;
    }
    // the plain plan: keep the batched solve on its own chains (it used the plain
    // ones when it had no plan of its own)
    if (!s->cp_batch.len) {
        ChainPlan old;
        old.h1 = s->h_ctasks1;
        old.h4 = s->h_ctasks4;
        SPK_TRY(upload_vec(old.d1, old.h1));
        SPK_TRY(upload_vec(old.d4, old.h4));
        old.len = s->ch_len;
        s->cp_batch.d1.p = old.d1.p, s->cp_batch.d1.n = old.d1.n, old.d1.p = nullptr;
        s->cp_batch.d4.p = old.d4.p, s->cp_batch.d4.n = old.d4.n, old.d4.p = nullptr;
        s->cp_batch.h1.swap(old.h1);
        s->cp_batch.h4.swap(old.h4);
        s->cp_batch.len = old.len;
    }
    s->d_ctasks1.release();
    s->d_ctasks4.release();
    s->d_ctasks1.p = fresh.d1.p, s->d_ctasks1.n = fresh.d1.n, fresh.d1.p = nullptr;
    s->d_ctasks4.p = fresh.d4.p, s->d_ctasks4.n = fresh.d4.n, fresh.d4.p = nullptr;
    long long rows1 = 0, rows4 = 0;
    for (const ChainTask &t : fresh.h1) rows1 += t.hi - t.lo;
    for (const ChainTask &t : fresh.h4) rows4 += t.hi - t.lo;
    s->h_ctasks1.swap(fresh.h1);
    s->h_ctasks4.swap(fresh.h4);
    s->nctasks1 = (int)s->h_ctasks1.size();
    s->nctasks4 = (int)s->h_ctasks4.size();
    s->ch_rows1 = rows1;
    s->ch_rows4 = rows4;
    s->ch_count = s->nctasks1;
    s->ch_len = fresh.len;
    drop_pipeline();
    return SPK_OK;
}

}  // namespace spk
