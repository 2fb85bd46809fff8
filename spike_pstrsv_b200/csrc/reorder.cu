// Partition-aware reordering ahead of the Spike preprocessing: the role of the
// reference's matrixReordering (src/matrix_reordering.c:83-305) with its helpers
// matrixAnalysis (:307-356), matrixSymmetrization (:29-80) and matrixDuplication
// (:18-27), under the same names and signatures.
//
// The reference partitions the graph of A + A^T into nthreads parts with METIS
// k-way (METIS_PartGraphKway, communication-volume objective; METIS 5 API, the
// version is not pinned by the reference), numbers the rows part by part
// (original order inside a part, :152-172), applies that symmetric permutation
// to the full matrix, keeps the requested triangle and hands the part sizes to
// the next preprocessing as caller-set partitions (IS_MATRIX_PARTITIONED).
// METIS is not part of this library, so the partitioner is a bandwidth-driven
// one: a reverse Cuthill-McKee ordering of the same graph (per connected
// component from a pseudo-peripheral node found by the George-Liu iteration
// started at the component's lightest node,
// neighbours taken in increasing degree, ties by index), cut into nthreads
// contiguous ranges of nearly equal nonzero count; part k is range k.  Rows
// that are close in an RCM order are close in the matrix, so a part touches only
// the parts beside it: for the triangle that the Spike solve runs on, a block
// couples to the next block alone, through the rows at the boundary.  The rows
// are renumbered in the RCM order (grouped by part, the band kept inside each
// part; the reference keeps a METIS part's rows in their original order).
// The steps after that are the reference's: the permuted matrix as CSR with
// sorted columns (:174-190, mkl_dcsrcoo job 2), the upper or lower triangle
// (:192-264), the partition bounds from the part sizes (:266-276).  The
// reference's matrixReordering given the RCM-ordered matrix and these
// contiguous parts produces the same arrays.
//
// The O(nnz) steps run on the GPU with one 64-bit key per entry and a CUB radix
// sort over the bits the keys use: the graph (both orientations of every
// off-diagonal entry, sorted, repeats removed), and after the ordering the
// permuted triangle (every entry renumbered, sorted by (row, column), the other
// triangle dropped, row pointers by binary search).  The ordering itself runs
// on the host: breadth-first search is sequential.  spk_reorder_plan builds the
// same graph on the host, for planning without a GPU.
#include <cub/cub.cuh>

#include <algorithm>
#include <cctype>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "spk_internal.cuh"

namespace spk {
namespace {

using I64 = long long;

int check_csr(int n, const int *ia, const int *ja) {
    if (n <= 0 || !ia || !ja) {
        set_error(SPK_ERR_ARG, "reordering: n must be positive and ia, ja non-null (n=%d)", n);
        return SPK_ERR_ARG;
    }
    if (ia[0] != 0) {
        set_error(SPK_ERR_INPUT, "reordering: ia[0] = %d, expected 0 (0-based CSR)", ia[0]);
        return SPK_ERR_INPUT;
    }
    for (int r = 0; r < n; ++r) {
        if (ia[r + 1] < ia[r]) {
            set_error(SPK_ERR_INPUT, "reordering: row pointers decrease at row %d", r);
            return SPK_ERR_INPUT;
        }
        for (int k = ia[r]; k < ia[r + 1]; ++k)
            if (ja[k] < 0 || ja[k] >= n) {
                set_error(SPK_ERR_INPUT, "reordering: column %d of row %d out of range [0, %d)", ja[k], r, n);
                return SPK_ERR_INPUT;
            }
    }
    return SPK_OK;
}

// Pattern of A + A^T without the diagonal: rows sorted, no repeats.
struct Graph {
    std::vector<I64> p;
    std::vector<int> j;
    int deg(int v) const { return (int)(p[v + 1] - p[v]); }
};

void symmetric_pattern(int n, const int *ia, const int *ja, Graph &g) {
    std::vector<I64> tp(n + 1, 0);
    for (int r = 0; r < n; ++r)
        for (int k = ia[r]; k < ia[r + 1]; ++k)
            if (ja[k] != r) tp[ja[k] + 1]++;
    for (int c = 0; c < n; ++c) tp[c + 1] += tp[c];
    std::vector<int> tj(tp[n]);
    {
        std::vector<I64> cur(tp.begin(), tp.end() - 1);
        for (int r = 0; r < n; ++r)  // rows in increasing order: every row of A^T comes out sorted
            for (int k = ia[r]; k < ia[r + 1]; ++k)
                if (ja[k] != r) tj[cur[ja[k]]++] = r;
    }
    g.p.assign(n + 1, 0);
    g.j.clear();
    g.j.reserve(2 * tp[n]);
    std::vector<int> row;
    for (int r = 0; r < n; ++r) {
        row.assign(ja + ia[r], ja + ia[r + 1]);
        if (!std::is_sorted(row.begin(), row.end())) std::sort(row.begin(), row.end());
        size_t x = 0;
        I64 y = tp[r];
        int last = -1;
        while (x < row.size() || y < tp[r + 1]) {
            int v = (y >= tp[r + 1] || (x < row.size() && row[x] <= tj[y])) ? row[x++] : tj[y++];
            if (v == r || v == last) continue;
            g.j.push_back(v);
            last = v;
        }
        g.p[r + 1] = (I64)g.j.size();
    }
}

// Breadth-first search from root; nodes in visit order and the start of every
// level.  Visited marks are stamps, so no clearing between searches.
struct Levels {
    std::vector<int> nodes;
    std::vector<size_t> start;
};

struct Stamps {
    std::vector<unsigned> s;
    unsigned mark = 0;
    explicit Stamps(int n) : s(n, 0) {}
    unsigned next() {
        if (++mark == UINT_MAX) {
            std::fill(s.begin(), s.end(), 0u);
            mark = 1;
        }
        return mark;
    }
};

void bfs(const Graph &g, int root, Stamps &st, Levels &out) {
    const unsigned m = st.next();
    out.nodes.clear();
    out.start.clear();
    out.nodes.push_back(root);
    st.s[root] = m;
    size_t lo = 0;
    while (lo < out.nodes.size()) {
        out.start.push_back(lo);
        const size_t hi = out.nodes.size();
        for (size_t q = lo; q < hi; ++q) {
            const int v = out.nodes[q];
            for (I64 k = g.p[v]; k < g.p[v + 1]; ++k) {
                const int u = g.j[k];
                if (st.s[u] != m) {
                    st.s[u] = m;
                    out.nodes.push_back(u);
                }
            }
        }
        lo = hi;
    }
}

inline bool lighter(const Graph &g, int x, int y) {  // degree, then index
    const int dx = g.deg(x), dy = g.deg(y);
    return dx != dy ? dx < dy : x < y;
}

// George-Liu: from the lightest node of the component, move to the lightest
// node of the last breadth-first level while that lengthens the level structure.
// (Starting at the component's first node instead saves one search but left
// wider bands, e.g. 149 against 103 rows on a scrambled banded matrix.)
int pseudo_peripheral(const Graph &g, int s0, Stamps &st) {
    Levels lv, lx;
    bfs(g, s0, st, lv);
    int r = s0;
    for (int v : lv.nodes)
        if (lighter(g, v, r)) r = v;
    if (r != s0) bfs(g, r, st, lv);
    for (int it = 0; it < 32; ++it) {
        int x = -1;
        for (size_t q = lv.start.back(); q < lv.nodes.size(); ++q)
            if (x < 0 || lighter(g, lv.nodes[q], x)) x = lv.nodes[q];
        bfs(g, x, st, lx);
        if (lx.start.size() <= lv.start.size()) break;
        r = x;
        std::swap(lv, lx);
    }
    return r;
}

// Reverse Cuthill-McKee order of the graph (order[q] = node at position q).
void rcm(const Graph &g, int n, std::vector<int> &order) {
    order.clear();
    order.reserve(n);
    std::vector<char> placed(n, 0);
    Stamps st(n);
    for (int s0 = 0; s0 < n; ++s0) {
        if (placed[s0]) continue;
        const int root = g.deg(s0) == 0 ? s0 : pseudo_peripheral(g, s0, st);
        size_t head = order.size();
        order.push_back(root);
        placed[root] = 1;
        while (head < order.size()) {
            const int v = order[head++];
            const size_t first = order.size();
            for (I64 k = g.p[v]; k < g.p[v + 1]; ++k) {
                const int u = g.j[k];
                if (!placed[u]) {
                    placed[u] = 1;
                    order.push_back(u);
                }
            }
            std::sort(order.begin() + first, order.end(), [&](int x, int y) { return lighter(g, x, y); });
        }
    }
    std::reverse(order.begin(), order.end());
}

// Cut the order into nparts contiguous ranges of nearly equal weight (row
// nonzeros of A), every range non-empty; part[v] = range of node v.
void cut(int n, const int *ia, const std::vector<int> &order, int nparts, std::vector<int> &part) {
    I64 total = 0;
    for (int v = 0; v < n; ++v) total += std::max(1, ia[v + 1] - ia[v]);
    std::vector<int> bound(nparts + 1);
    bound[0] = 0;
    bound[nparts] = n;
    I64 acc = 0;
    int q = 0;
    for (int k = 1; k < nparts; ++k) {
        while (q < n && acc * nparts < total * k) {
            const int v = order[q++];
            acc += std::max(1, ia[v + 1] - ia[v]);
        }
        bound[k] = std::min(std::max(q, bound[k - 1] + 1), n - (nparts - k));
    }
    part.assign(n, 0);
    for (int k = 0; k < nparts; ++k)
        for (int p = bound[k]; p < bound[k + 1]; ++p) part[order[p]] = k;
}

int check_plan_args(int n, const int *ia, const int *ja, int nparts) {
    SPK_TRY(check_csr(n, ia, ja));
    if (nparts <= 0 || nparts > n || nparts > SPK_MAX_EXPORTED_PARTS) {
        set_error(SPK_ERR_ARG, "reordering: %d parts for %d rows (1..min(n, %d))", nparts, n,
                  SPK_MAX_EXPORTED_PARTS);
        return SPK_ERR_ARG;
    }
    return SPK_OK;
}

// The partitioner on a graph built by the caller (host or GPU pattern: the same
// sorted, repeat-free rows).
void plan_on(const Graph &g, int n, const int *ia, int nparts, std::vector<int> &order, std::vector<int> &part) {
    rcm(g, n, order);
    cut(n, ia, order, nparts, part);
}

// --------------------------------------------------------------------------
// GPU: permute every entry, sort by (row, column), keep one triangle
// --------------------------------------------------------------------------

// One warp per row: key = new row << 32 | new column for entries of the kept
// triangle, (n << 32) for the others, which sorts them after every kept entry.
__global__ void k_permute_keys(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                               const int *__restrict__ iperm, int upper, unsigned long long *__restrict__ keys,
                               int *__restrict__ idx, unsigned long long *__restrict__ kept) {
    const int lane = threadIdx.x & 31;
    const I64 w0 = ((I64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const I64 nw = ((I64)gridDim.x * blockDim.x) >> 5;
    const unsigned long long drop = (unsigned long long)(unsigned)n << 32;
    unsigned long long cnt = 0;
    for (I64 r = w0; r < n; r += nw) {
        const int rn = iperm[r];
        const int e = ia[r + 1];
        for (int k = ia[r] + lane; k < e; k += 32) {
            const int cn = iperm[ja[k]];
            const bool keep = upper ? cn >= rn : cn <= rn;
            keys[k] = keep ? (((unsigned long long)(unsigned)rn << 32) | (unsigned)cn) : drop;
            idx[k] = k;
            cnt += keep;
        }
    }
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0 && cnt) atomicAdd(kept, cnt);
}

// ip[r] = first sorted key of row r (binary search), r = 0..n; ip[n] = kept.
__global__ void k_row_ptr(int n, const unsigned long long *__restrict__ keys, I64 kept, int *__restrict__ ip) {
    for (I64 r = (I64)blockIdx.x * blockDim.x + threadIdx.x; r <= n; r += (I64)gridDim.x * blockDim.x) {
        const unsigned long long t = (unsigned long long)r << 32;
        I64 lo = 0, hi = kept;
        while (lo < hi) {
            const I64 mid = (lo + hi) >> 1;
            if (keys[mid] < t) lo = mid + 1;
            else hi = mid;
        }
        ip[r] = (int)lo;
    }
}

__global__ void k_gather_entries(I64 kept, const unsigned long long *__restrict__ keys, const int *__restrict__ idx,
                                 const double *__restrict__ a, double *__restrict__ ao, int *__restrict__ jo) {
    for (I64 k = (I64)blockIdx.x * blockDim.x + threadIdx.x; k < kept; k += (I64)gridDim.x * blockDim.x) {
        ao[k] = a[idx[k]];
        jo[k] = (int)(unsigned)(keys[k] & 0xffffffffull);
    }
}

// Pattern of A + A^T on the GPU: both orientations of every off-diagonal entry
// as keys row << 32 | column (diagonal entries: n << 32, sorted last), radix
// sort, unique.  One warp per row.
__global__ void k_sym_keys(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                           unsigned long long *__restrict__ keys) {
    const int lane = threadIdx.x & 31;
    const I64 w0 = ((I64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const I64 nw = ((I64)gridDim.x * blockDim.x) >> 5;
    const unsigned long long drop = (unsigned long long)(unsigned)n << 32;
    for (I64 r = w0; r < n; r += nw) {
        const int e = ia[r + 1];
        for (int k = ia[r] + lane; k < e; k += 32) {
            const unsigned c = (unsigned)ja[k];
            const bool off = c != (unsigned)r;
            keys[2 * (I64)k] = off ? (((unsigned long long)r << 32) | c) : drop;
            keys[2 * (I64)k + 1] = off ? (((unsigned long long)c << 32) | (unsigned)r) : drop;
        }
    }
}

// p[r] = first key of row r (binary search), r = 0..n; p[n] = count.
__global__ void k_row_ptr64(int n, const unsigned long long *__restrict__ keys, I64 count, I64 *__restrict__ p) {
    for (I64 r = (I64)blockIdx.x * blockDim.x + threadIdx.x; r <= n; r += (I64)gridDim.x * blockDim.x) {
        const unsigned long long t = (unsigned long long)r << 32;
        I64 lo = 0, hi = count;
        while (lo < hi) {
            const I64 mid = (lo + hi) >> 1;
            if (keys[mid] < t) lo = mid + 1;
            else hi = mid;
        }
        p[r] = lo;
    }
}

__global__ void k_key_cols(I64 count, const unsigned long long *__restrict__ keys, int *__restrict__ j) {
    for (I64 k = (I64)blockIdx.x * blockDim.x + threadIdx.x; k < count; k += (I64)gridDim.x * blockDim.x)
        j[k] = (int)(unsigned)(keys[k] & 0xffffffffull);
}

template <typename T>
T *host_alloc(size_t count) {
    void *p = nullptr;
    if (posix_memalign(&p, 64, std::max<size_t>(count, 1) * sizeof(T)) != 0) return nullptr;
    return (T *)p;
}

int grid_for(I64 work, int threads) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const I64 want = (work + threads - 1) / threads;
    return (int)std::max<I64>(1, std::min<I64>(want, (I64)sms * 16));
}

int row_bits_for(int n) {
    int b = 1;
    while (b < 31 && (1u << b) <= (unsigned)n) ++b;
    return b;
}

// The graph of the partitioner (pattern of A + A^T without the diagonal) built
// on the GPU from the host CSR; the same rows as symmetric_pattern.
int symmetric_pattern_gpu(int n, const int *ia, const int *ja, Graph &g) {
    const I64 nnz = ia[n];
    cudaStream_t st = nullptr;
    SPK_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    int rc = SPK_OK;
    {
        DBuf<int> d_ia(st), d_ja(st), d_j(st);
        DBuf<unsigned long long> d_keys(st), d_sorted(st), d_uniq(st);
        DBuf<I64> d_p(st), d_count(st);
        DBuf<unsigned char> d_tmp(st);
        auto run = [&]() -> int {
            SPK_TRY(d_ia.alloc(n + 1));
            SPK_TRY(d_ja.alloc(nnz));
            SPK_TRY(d_keys.alloc(2 * nnz));
            SPK_CUDA(cudaMemcpyAsync(d_ia.p, ia, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st));
            SPK_CUDA(cudaMemcpyAsync(d_ja.p, ja, sizeof(int) * nnz, cudaMemcpyHostToDevice, st));
            k_sym_keys<<<grid_for((I64)n * 32, 256), 256, 0, st>>>(n, d_ia.p, d_ja.p, d_keys.p);
            SPK_CUDA(cudaGetLastError());
            d_ja.release();
            SPK_TRY(d_sorted.alloc(2 * nnz));
            const int end_bit = 32 + row_bits_for(n);
            size_t t1 = 0, t2 = 0;
            SPK_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, t1, d_keys.p, d_sorted.p, 2 * nnz, 0, end_bit, st));
            SPK_CUDA(cub::DeviceSelect::Unique(nullptr, t2, d_sorted.p, d_keys.p, d_count.p, 2 * nnz, st));
            SPK_TRY(d_tmp.alloc(std::max(t1, t2)));
            SPK_TRY(d_count.alloc(1));
            SPK_CUDA(cub::DeviceRadixSort::SortKeys(d_tmp.p, t1, d_keys.p, d_sorted.p, 2 * nnz, 0, end_bit, st));
            SPK_CUDA(cub::DeviceSelect::Unique(d_tmp.p, t2, d_sorted.p, d_keys.p, d_count.p, 2 * nnz, st));
            I64 count = 0;
            SPK_CUDA(cudaMemcpyAsync(&count, d_count.p, sizeof(I64), cudaMemcpyDeviceToHost, st));
            SPK_CUDA(cudaStreamSynchronize(st));
            // unique keys in d_keys; the diagonal's key (row n), if any, is last
            d_sorted.release();
            d_tmp.release();
            SPK_TRY(d_p.alloc(n + 1));
            k_row_ptr64<<<grid_for((I64)n + 1, 256), 256, 0, st>>>(n, d_keys.p, count, d_p.p);
            SPK_CUDA(cudaGetLastError());
            g.p.assign(n + 1, 0);
            SPK_CUDA(cudaMemcpyAsync(g.p.data(), d_p.p, sizeof(I64) * (n + 1), cudaMemcpyDeviceToHost, st));
            SPK_CUDA(cudaStreamSynchronize(st));
            const I64 edges = g.p[n];  // entries of rows < n: the diagonal's key excluded
            SPK_TRY(d_j.alloc(edges));
            if (edges) {
                k_key_cols<<<grid_for(edges, 256), 256, 0, st>>>(edges, d_keys.p, d_j.p);
                SPK_CUDA(cudaGetLastError());
            }
            g.j.resize(edges);
            if (edges) SPK_CUDA(cudaMemcpyAsync(g.j.data(), d_j.p, sizeof(int) * edges, cudaMemcpyDeviceToHost, st));
            SPK_CUDA(cudaStreamSynchronize(st));
            return SPK_OK;
        };
        rc = run();
    }
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    return rc;
}

// The triangle of P A P^T (P: row i of the result is row perm[i] of A) as a new
// host CSR with sorted columns.
int permute_triangle(int n, const double *a, const int *ia, const int *ja, const std::vector<int> &iperm,
                     bool upper, double **ao_h, int **ia_h, int **ja_h) {
    const I64 nnz = ia[n];
    cudaStream_t st = nullptr;
    SPK_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    int rc = SPK_OK;
    double *ao = nullptr;
    int *io = nullptr, *jo = nullptr;
    {
        DBuf<int> d_ia(st), d_ja(st), d_iperm(st), d_idx(st), d_idx2(st), d_ip(st), d_jo(st);
        DBuf<double> d_a(st), d_ao(st);
        DBuf<unsigned long long> d_keys(st), d_keys2(st), d_kept(st);
        DBuf<unsigned char> d_tmp(st);
        auto run = [&]() -> int {
            SPK_TRY(d_ia.alloc(n + 1));
            SPK_TRY(d_ja.alloc(nnz));
            SPK_TRY(d_a.alloc(nnz));
            SPK_TRY(d_iperm.alloc(n));
            SPK_TRY(d_keys.alloc(nnz));
            SPK_TRY(d_keys2.alloc(nnz));
            SPK_TRY(d_idx.alloc(nnz));
            SPK_TRY(d_idx2.alloc(nnz));
            SPK_TRY(d_kept.alloc(1));
            SPK_CUDA(cudaMemcpyAsync(d_ia.p, ia, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st));
            SPK_CUDA(cudaMemcpyAsync(d_ja.p, ja, sizeof(int) * nnz, cudaMemcpyHostToDevice, st));
            SPK_CUDA(cudaMemcpyAsync(d_a.p, a, sizeof(double) * nnz, cudaMemcpyHostToDevice, st));
            SPK_CUDA(cudaMemcpyAsync(d_iperm.p, iperm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
            SPK_CUDA(cudaMemsetAsync(d_kept.p, 0, sizeof(unsigned long long), st));
            k_permute_keys<<<grid_for((I64)n * 32, 256), 256, 0, st>>>(n, d_ia.p, d_ja.p, d_iperm.p, upper ? 1 : 0,
                                                                      d_keys.p, d_idx.p, d_kept.p);
            SPK_CUDA(cudaGetLastError());
            // rows need the bits of n (the dropped entries' row), columns 32 bits
            const int end_bit = 32 + row_bits_for(n);
            size_t tmp = 0;
            SPK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, d_keys.p, d_keys2.p, d_idx.p, d_idx2.p, nnz, 0,
                                                     end_bit, st));
            SPK_TRY(d_tmp.alloc(tmp));
            SPK_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp.p, tmp, d_keys.p, d_keys2.p, d_idx.p, d_idx2.p, nnz, 0,
                                                     end_bit, st));
            unsigned long long kept = 0;
            SPK_CUDA(cudaMemcpyAsync(&kept, d_kept.p, sizeof(kept), cudaMemcpyDeviceToHost, st));
            SPK_CUDA(cudaStreamSynchronize(st));
            d_tmp.release();
            d_keys.release();
            d_idx.release();
            d_ja.release();
            SPK_TRY(d_ip.alloc(n + 1));
            SPK_TRY(d_ao.alloc(kept));
            SPK_TRY(d_jo.alloc(kept));
            k_row_ptr<<<grid_for((I64)n + 1, 256), 256, 0, st>>>(n, d_keys2.p, (I64)kept, d_ip.p);
            SPK_CUDA(cudaGetLastError());
            if (kept) {
                k_gather_entries<<<grid_for((I64)kept, 256), 256, 0, st>>>((I64)kept, d_keys2.p, d_idx2.p, d_a.p,
                                                                          d_ao.p, d_jo.p);
                SPK_CUDA(cudaGetLastError());
            }
            ao = host_alloc<double>(kept);
            jo = host_alloc<int>(kept);
            io = host_alloc<int>(n + 1);
            if (!ao || !jo || !io) {
                set_error(SPK_ERR_NOMEM, "reordering: host allocation of %llu entries failed", kept);
                return SPK_ERR_NOMEM;
            }
            SPK_CUDA(cudaMemcpyAsync(io, d_ip.p, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, st));
            if (kept) {
                SPK_CUDA(cudaMemcpyAsync(ao, d_ao.p, sizeof(double) * kept, cudaMemcpyDeviceToHost, st));
                SPK_CUDA(cudaMemcpyAsync(jo, d_jo.p, sizeof(int) * kept, cudaMemcpyDeviceToHost, st));
            }
            SPK_CUDA(cudaStreamSynchronize(st));
            return SPK_OK;
        };
        rc = run();
    }
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (rc != SPK_OK) {
        free(ao);
        free(io);
        free(jo);
        return rc;
    }
    *ao_h = ao;
    *ia_h = io;
    *ja_h = jo;
    return SPK_OK;
}

// The triangle of a host CSR (no permutation), for matrixAnalysis without a file.
int host_triangle(int n, const double *a, const int *ia, const int *ja, bool upper, double **ao, int **io, int **jo) {
    I64 kept = 0;
    for (int r = 0; r < n; ++r)
        for (int k = ia[r]; k < ia[r + 1]; ++k) kept += upper ? ja[k] >= r : ja[k] <= r;
    double *av = host_alloc<double>(kept);
    int *iv = host_alloc<int>(n + 1), *jv = host_alloc<int>(kept);
    if (!av || !iv || !jv) {
        free(av);
        free(iv);
        free(jv);
        set_error(SPK_ERR_NOMEM, "reordering: host allocation failed");
        return SPK_ERR_NOMEM;
    }
    I64 q = 0;
    iv[0] = 0;
    for (int r = 0; r < n; ++r) {
        for (int k = ia[r]; k < ia[r + 1]; ++k)
            if (upper ? ja[k] >= r : ja[k] <= r) {
                av[q] = a[k];
                jv[q] = ja[k];
                ++q;
            }
        iv[r + 1] = (int)q;
    }
    *ao = av;
    *io = iv;
    *jo = jv;
    return SPK_OK;
}

void set_bounds(const std::vector<int> &sizes) {
    int s = 0;
    for (size_t t = 0; t < sizes.size(); ++t) {
        partition_numRows[t] = sizes[t];
        partition_starts[t] = s;
        partition_ends[t] = s + sizes[t];
        s += sizes[t];
    }
}

}  // namespace

// Reorder the full matrix (*a, *ia, *ja) into nparts partitions and keep one
// triangle; see matrixReordering below.  Status-returning form.
int reorder(double **a, int **ia, int **ja, int n, int nparts, char uplo, std::vector<int> *perm_out) {
    if (!a || !ia || !ja || !*a || !*ia || !*ja) {
        set_error(SPK_ERR_ARG, "reordering: null matrix");
        return SPK_ERR_ARG;
    }
    SPK_TRY(check_plan_args(n, *ia, *ja, nparts));
    std::vector<int> order, part;
    {
        Graph g;
        SPK_TRY(symmetric_pattern_gpu(n, *ia, *ja, g));
        plan_on(g, n, *ia, nparts, order, part);
    }
    // Rows in RCM order: the partitions are ranges of it, so the rows are grouped
    // by partition (src/matrix_reordering.c:152-172) and keep the narrow band
    // inside each one.  (The reference keeps the original order inside a METIS
    // part; inside an RCM range that order can be arbitrary - a scrambled input
    // stays scrambled - and the dense spikes of the next preprocessing grow with
    // the partition's width.)
    std::vector<int> sizes(nparts, 0), iperm(n);
    for (int v = 0; v < n; ++v) sizes[part[v]]++;
    const std::vector<int> &perm = order;
    for (int i = 0; i < n; ++i) iperm[perm[i]] = i;
    const char u = (char)toupper((unsigned char)uplo);
    double *ao = nullptr;
    int *io = nullptr, *jo = nullptr;
    SPK_TRY(permute_triangle(n, *a, *ia, *ja, iperm, u == 'U', &ao, &io, &jo));
    free(*a);
    free(*ia);
    free(*ja);
    *a = ao;
    *ia = io;
    *ja = jo;
    set_bounds(sizes);
    IS_MATRIX_PARTITIONED = 1;
    if (perm_out) *perm_out = perm;
    return SPK_OK;
}

}  // namespace spk

extern "C" {

// The partitioner alone, host code (no GPU; the graph is built on the host,
// where matrixReordering builds the same graph on the GPU): the RCM order and
// the part of every row.
int spk_reorder_plan(int n, const int *ia, const int *ja, int nparts, int *order, int *part) {
    SPK_TRY(spk::check_plan_args(n, ia, ja, nparts));
    std::vector<int> o, p;
    {
        spk::Graph g;
        spk::symmetric_pattern(n, ia, ja, g);
        spk::plan_on(g, n, ia, nparts, o, p);
    }
    if (order) std::copy(o.begin(), o.end(), order);
    if (part) std::copy(p.begin(), p.end(), part);
    return SPK_OK;
}

int spk_reorder(double **a, int **ia, int **ja, int n, int nparts, char uplo, int *perm) {
    std::vector<int> pv;
    SPK_TRY(spk::reorder(a, ia, ja, n, nparts, uplo, perm ? &pv : nullptr));
    if (perm) std::copy(pv.begin(), pv.end(), perm);
    return SPK_OK;
}

void matrixDuplication(int numRows, double *a, MKL_INT *ia, MKL_INT *ja, double **a_dup, MKL_INT **ia_dup,
                       MKL_INT **ja_dup) {
    const long long nnz = ia[numRows];
    *a_dup = spk::host_alloc<double>(nnz);
    *ja_dup = spk::host_alloc<int>(nnz);
    *ia_dup = spk::host_alloc<int>(numRows + 1);
    if (!*a_dup || !*ja_dup || !*ia_dup) {
        fprintf(stderr, "matrixDuplication: host allocation failed\n");
        return;
    }
    memcpy(*a_dup, a, sizeof(double) * nnz);
    memcpy(*ja_dup, ja, sizeof(int) * nnz);
    memcpy(*ia_dup, ia, sizeof(int) * (numRows + 1));
}

// A <- A + A^T with values summed (the reference: mkl_dcsradd with trans 'T',
// src/matrix_reordering.c:56-62); sorted columns in every row.
void matrixSymmetrization(double **a, MKL_INT **ia, MKL_INT **ja, int numRows) {
    const int n = numRows;
    if (spk::check_csr(n, *ia, *ja) != SPK_OK) {
        fprintf(stderr, "matrixSymmetrization: %s\n", spk_last_error());
        return;
    }
    const int *pi = *ia, *pj = *ja;
    const double *pa = *a;
    std::vector<long long> tp(n + 1, 0);
    for (int r = 0; r < n; ++r)
        for (int k = pi[r]; k < pi[r + 1]; ++k) tp[pj[k] + 1]++;
    for (int c = 0; c < n; ++c) tp[c + 1] += tp[c];
    std::vector<int> tj(tp[n]);
    std::vector<double> tv(tp[n]);
    {
        std::vector<long long> cur(tp.begin(), tp.end() - 1);
        for (int r = 0; r < n; ++r)
            for (int k = pi[r]; k < pi[r + 1]; ++k) {
                tj[cur[pj[k]]] = r;
                tv[cur[pj[k]]++] = pa[k];
            }
    }
    std::vector<std::pair<int, double>> row;
    std::vector<int> ci(n + 1, 0);
    std::vector<int> cj;
    std::vector<double> cv;
    cj.reserve(2 * tp[n]);
    cv.reserve(2 * tp[n]);
    for (int r = 0; r < n; ++r) {
        row.clear();
        for (int k = pi[r]; k < pi[r + 1]; ++k) row.emplace_back(pj[k], pa[k]);
        for (long long k = tp[r]; k < tp[r + 1]; ++k) row.emplace_back(tj[k], tv[k]);
        std::stable_sort(row.begin(), row.end(),
                         [](const std::pair<int, double> &x, const std::pair<int, double> &y) { return x.first < y.first; });
        for (size_t q = 0; q < row.size(); ++q) {
            if (q && row[q].first == row[q - 1].first) cv.back() += row[q].second;
            else {
                cj.push_back(row[q].first);
                cv.push_back(row[q].second);
            }
        }
        ci[r + 1] = (int)cj.size();
    }
    double *na = spk::host_alloc<double>(cv.size());
    int *ni = spk::host_alloc<int>(n + 1), *nj = spk::host_alloc<int>(cj.size());
    if (!na || !ni || !nj) {
        free(na);
        free(ni);
        free(nj);
        fprintf(stderr, "matrixSymmetrization: host allocation failed\n");
        return;
    }
    std::copy(cv.begin(), cv.end(), na);
    std::copy(cj.begin(), cj.end(), nj);
    std::copy(ci.begin(), ci.end(), ni);
    free(*a);
    free(*ia);
    free(*ja);
    *a = na;
    *ia = ni;
    *ja = nj;
}

// 1 when no entry of the requested triangle couples two of nthreads equal
// partitions (no reordering needed; the matrix is replaced by that triangle,
// re-read from matrixFileName as the reference does, or taken from memory when
// the name is NULL), else 0.  The partition globals are set as
// matrixPartitioning sets them (src/matrix_partitioning.c:18-36).
int matrixAnalysis(int numRows, int nthreads, double **a, MKL_INT **ia, MKL_INT **ja, const char uplo,
                   const char symm, const char *matrixFileName) {
    const int n = numRows;
    if (n <= 0 || nthreads <= 0 || nthreads > SPK_MAX_EXPORTED_PARTS) return 0;
    if (!IS_MATRIX_PARTITIONED) {
        const int k = n / nthreads;
        for (int t = 0; t < nthreads; ++t) {
            partition_numRows[t] = k;
            partition_starts[t] = k * t;
            partition_ends[t] = k * t + k;
        }
        partition_numRows[nthreads - 1] += n % nthreads;
        partition_ends[nthreads - 1] += n % nthreads;
    } else {
        IS_MATRIX_PARTITIONED = 0;
    }
    const bool upper = toupper((unsigned char)uplo) == 'U';
    for (int t = 0; t < nthreads; ++t) {
        const int ps = partition_starts[t], pe = partition_ends[t];
        for (int k = (*ia)[ps]; k < (*ia)[pe]; ++k)
            if (upper ? (*ja)[k] >= pe : (*ja)[k] < ps) return 0;
    }
    double *na = nullptr;
    int *ni = nullptr, *nj = nullptr;
    int m = n;
    const char u = (char)toupper((unsigned char)uplo);
    if (matrixFileName) {
        matrixMarketToCSR(matrixFileName, &na, &ni, &nj, &m, uplo, symm);
        if (!na) return 1;
    } else if (u != 'U' && u != 'L') {
        return 1;  // 'N': the matrix stays whole
    } else if (spk::host_triangle(n, *a, *ia, *ja, upper, &na, &ni, &nj) != SPK_OK) {
        return 1;
    }
    free(*a);
    free(*ia);
    free(*ja);
    *a = na;
    *ia = ni;
    *ja = nj;
    return 1;
}

// Replaces matrixReordering (src/matrix_reordering.c:83-305).  (*a, *ia, *ja):
// the full n x n matrix (host CSR, 0-based; arrays from malloc/posix_memalign,
// as matrixMarketToCSR returns them: they are freed and replaced).  When the
// equal partitions already decouple (matrixAnalysis) the matrix becomes its
// triangle and nothing is reordered.  Otherwise the rows are reordered for
// nthreads partitions (RCM ranges, above), the matrix becomes the upper
// (uplo 'U') or lower (any other uplo, as in the reference) triangle of the
// reordered matrix, partition_starts / ends / numRows hold the partition bounds
// and IS_MATRIX_PARTITIONED is 1, so the next spike_pstrsv_preproc with
// nthreads partitions uses them.  symm only matters for the re-read: the
// partitioner always works on the pattern of A + A^T.  Needs a GPU.
void matrixReordering(double **a, MKL_INT **ia, MKL_INT **ja, int numRows, int nthreads, const char uplo,
                      const char symm, const char *matrixFileName) {
    if (matrixAnalysis(numRows, nthreads, a, ia, ja, uplo, symm, matrixFileName)) return;
    if (spk::reorder(a, ia, ja, numRows, nthreads, uplo, nullptr) != SPK_OK)
        printf("Matrix Reordering is NOT successfull: %s\n", spk_last_error());
}

}  // extern "C"
