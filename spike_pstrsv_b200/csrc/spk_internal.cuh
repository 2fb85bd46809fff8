// Internal declarations shared by the sm_100a Spike triangular-solve library.
//
// Layout of one preprocessed system in HBM (all 0-based, int32 indices):
//   U      : the upper-triangular CSR the Spike algorithm runs on (the input for
//            uplo='U', the reversal mirror J L J for uplo='L').
//   pools  : the reference's preprocessing products, bit-identical to the
//            reference layout (spike_pstrsv_globals.h:13-55): D/ID/JD holding D
//            and R_new, T2/IT2/JT2 holding D0|D1|D2, mapR, dense spikes S,
//            reduced system T/IT/JT and mapReducedX.
//   solve  : per-partition task tables, reduced-level offsets and scratch
//            vectors used by the solve kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/spike_pstrsv.h"

namespace spk {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
void set_error(int code, const char *fmt, ...);
int last_error_code();

#define SPK_CUDA(call)                                                                  \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            ::spk::set_error(SPK_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,   \
                             cudaGetErrorString(e_));                                   \
            return SPK_ERR_CUDA;                                                        \
        }                                                                               \
    } while (0)

#define SPK_TRY(call)                     \
    do {                                  \
        int rc_ = (call);                 \
        if (rc_ != SPK_OK) return rc_;    \
    } while (0)

// ---------------------------------------------------------------------------
// device buffers
// ---------------------------------------------------------------------------
template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    // A scoped temporary used only on one stream is allocated and freed in that
    // stream's order (cudaMallocAsync / cudaFreeAsync): its release does not
    // wait for the whole device, as cudaFree does, while other threads' solves
    // run.  Host copies into it go through that stream.
    cudaStream_t ord = nullptr;
    bool on_stream = false;
    DBuf() = default;
    explicit DBuf(cudaStream_t s) : ord(s), on_stream(true) {}
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) {
            if (on_stream) cudaFreeAsync(p, ord);
            else cudaFree(p);
        }
        p = nullptr;
        n = 0;
    }
    int alloc(size_t count) {
        release();
        if (count == 0) count = 1;
        cudaError_t e = on_stream ? cudaMallocAsync((void **)&p, count * sizeof(T), ord)
                                  : cudaMalloc((void **)&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            set_error(SPK_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", count * sizeof(T),
                      cudaGetErrorString(e));
            return SPK_ERR_NOMEM;
        }
        n = count;
        return SPK_OK;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// ---------------------------------------------------------------------------
// one preprocessed system
// ---------------------------------------------------------------------------
struct Part {  // per-partition host metadata (reference names in comments)
    int ps, pe, num;            // partition_starts / partition_ends / partition_numRows
    int si, ei;                 // start_intervals / end_intervals
    int minDR, maxIR;           // first dependent row / last coupling row (global)
    char hasDep, hasRefl, hasS, isOpt;
    int nRowsS, nColsS;         // numRows_S / numCols_S
    long long startsS, endsS;   // starts_S / ends_S
    int sD0, eD0, sD1, eD1, sD2, eD2;
    int startsD, endsD, startsR, endsR;
    int sMapR, eMapR;
};

// One warp's job in the segment solver: rows [lo, hi) of U by back
// substitution, except rows [skip_lo, skip_hi), which take the phase-1 value,
// and rows [hi, tail), which are copied from the phase-1 values.
struct SegTask {
    int lo, hi;
    int skip_lo, skip_hi;
    int tail;
};

// One warp's job in the chain solver: rows [lo, hi) of U bottom-up (hi is a
// multiple of 32 or n), storing rows [st_lo, st_hi) into x.
struct ChainTask {
    int lo, hi;
    int st_lo, st_hi;
};

// A second chain decomposition of the same rows (the batched kernel's longer
// chains, the host-array pipeline's shorter ones): task lists on the device and
// the host (row order).
struct ChainPlan {
    DBuf<ChainTask> d1, d4;
    std::vector<ChainTask> h1, h4;
    int len = 0;  // 0: not built (the plain solve's chains are used)
    void release() {
        d1.release();
        d4.release();
        h1.clear();
        h4.clear();
        len = 0;
    }
};

// Truncation threshold on absolute spike-row sums (2^-60, below FP64 resolution
// relative to ||x||_inf); negative = exact mode (nothing dropped).
constexpr double kDefaultTruncTol = 8.673617379884035e-19;

}  // namespace spk

struct spk_system {
    int n = 0, nnz = 0, P = 0;
    char uplo = 'U';
    int flb = 1;
    int built = 0;
    int redNec = 0;
    int nRed = 0, rss = 0, nnzRed = 0;
    long long totalArea = 0;
    int nIT2rows = 0;
    long long nT = 0, nDpool = 0, nT2 = 0;
    int nMapR = 0;
    std::vector<spk::Part> parts;

    // working upper-triangular CSR
    spk::DBuf<double> ua;
    spk::DBuf<int> uia, uja;
    // reference-layout pools
    spk::DBuf<double> D, T2, S, T;
    spk::DBuf<int> ID, JD, IT2, JT2, mapR, dep, mapRedX, IT, JT;
    // solve support
    double trunc_tol = spk::kDefaultTruncTol;
    spk::DBuf<int> d_ps, d_pe, d_lvl;  // partition bounds; reduced row offset per partition
    spk::DBuf<spk::SegTask> d_tasks1, d_tasks2;
    int ntasks1 = 0, ntasks2 = 0;
    long long rows_phase1 = 0, rows_phase4 = 0;  // rows solved per call by phase 1 / phase 4
    spk::DBuf<double> xbuf, xout_u, rdiag;
    spk::DBuf<double> ell_val;  // sliced ELL of U's off-diagonals (32-row tiles)
    spk::DBuf<int> ell_col, ell_ptr;
    int ell_ok = 0;
    long long ell_entries = 0;
    // batched / mixed-precision solve support (allocated on first use)
    spk::DBuf<float> ell_valf, rdiagf;
    spk::DBuf<double> diag, rbuf, dbuf;
    spk::DBuf<char> work;
    spk::DBuf<unsigned long long> d_norms;
    double anorm = 0.0;
    int ell_reach = -1;
    spk::DBuf<double> stage_b, stage_x;  // device copies of host b / x for spk_solve
    char *ext_ws = nullptr;  // caller-lent device workspace for the batched solves (spk_set_workspace)
    size_t ext_ws_bytes = 0;  // largest column distance from a tile's first row (-1: not computed)
    // chain solver (default one-right-hand-side solve; chain.cu)
    int chain_ok = 0, ch_width = 0, ch_sw = 0, ch_reach = 0, ch_win = 0, ch_count = 0, ch_len = 0, ch_stages = 3;
    spk::DBuf<double> ch_val;          // row-scaled off-diagonals, sliced ELL
    spk::DBuf<double> ch_valb;         // batched solves: the same with in-group coefficients zeroed
    spk::DBuf<float> ch_valbf;         //   and its FP32 copy (made on first use)
    spk::DBuf<double> ch_near;         // batched solves: [rows][4] in-group coefficients
    spk::DBuf<float> ch_nearf;         //   and its FP32 copy
    spk::DBuf<unsigned char> ch_off;   // column offsets c - r (8 bits)
    spk::DBuf<int> ch_ptr;             // first slot of each 32-row tile
    spk::DBuf<spk::ChainTask> d_ctasks1, d_ctasks4;
    spk::ChainPlan cp_batch;  // the batched kernel's own chains (longer; built at preprocessing)
    spk::ChainPlan cp_host;   // the host-array pipeline's chains (shorter; built on first use)
    int batch_path = -1;      // spk_tune "batch_path": 1 chain kernels, 0 partition kernels, -1 automatic
    // wall milliseconds of the last preprocessing: the reference's steps, first
    // significant spike rows + internal spikes, reduced levels + buffers, the
    // sliced-ELL layout, the chain layout and plans (spk_debug_scalar "prep_us_*")
    double prep_ms[5] = {0, 0, 0, 0, 0};
    // first significant spike row per block; internal spikes not yet computed
    // (the partition solve's task lists are then untruncated on those blocks)
    std::vector<int> first_sig;
    int aux_pending = 0;
    int host_plan_tried = 0;
    int nctasks1 = 0, nctasks4 = 0;
    long long ch_rows1 = 0, ch_rows4 = 0;
    std::vector<spk::ChainTask> h_ctasks1, h_ctasks4;
    cudaStream_t st_in = nullptr, st_out = nullptr;  // copy streams of the pipelined host-array solve
    std::vector<cudaEvent_t> pipe_ev;
    std::vector<cudaStream_t> pipe_st;  // one per chunk of the pipelined solve
    // the pipeline captured as a graph, replayed while the caller keeps the same
    // page-locked b and x (and the same device copies and chunk count)
    cudaGraphExec_t pipe_exec = nullptr;
    const double *pipe_b = nullptr, *pipe_db = nullptr;
    double *pipe_x = nullptr, *pipe_dx = nullptr;
    int pipe_K = 0, pipe_nograph = 0;
    spk::DBuf<int> d_red_rows, d_red_off, d_err;  // kept reduced rows by level; device error flag
    int nlvl = 0, nkept = 0;
    int dbg_fail_waits = 0;  // test hook: solve kernels report a failed wait at entry (spk_debug_set)
    int lean = 0;  // spk_compact: only what the chain solves read is kept (partition paths refused)
    double *red_scratch = nullptr;  // FP64 reduced unknowns of the FP32 batched solve in flight
    // optional per-phase device timing (spk_set_profiling)
    int profiling = 0;
    static constexpr int kEvRing = 64;           // event sets in flight before a forced collection
    cudaEvent_t ev[kEvRing][4] = {};
    int ev_pending[kEvRing] = {};
    long long ev_next = 0;
    double phase_ms[3] = {0, 0, 0};
    long long profiled_solves = 0, launches = 0;
    cudaStream_t stream = nullptr;
    int own_stream = 0;
};

namespace spk {

int preprocess(spk_system *s, const double *a, const int *ia, const int *ja, int n, int P,
               char uplo, int flb, const int *starts, const int *ends, int ptr_on_device,
               double *phase_seconds);
int solve(spk_system *s, const double *b, double *x, cudaStream_t stream, double *phase_seconds);
int solve_batch(spk_system *s, int nrhs, const double *B, long long ldb, double *X, long long ldx, int mode,
                double tol, int maxit, cudaStream_t stream, int *iters, double *resid);
int solve_batch_static(spk_system *s, int nrhs, const double *B, long long ldb, double *X, long long ldx,
                       cudaStream_t st);
int solve_prepare(spk_system *s);
int residual_prepare(spk_system *s);
int chain_prepare(spk_system *s);
int chain_tune(spk_system *s, const char *name, long long v);
int partition_ensure(spk_system *s);
int chain_solve(spk_system *s, const double *b, double *x, cudaStream_t st, bool prof, int ring);
int chain_solve_host(spk_system *s, const double *b, double *x, double *db, double *dx);
long long chain_device_check();
int chain_phase(spk_system *s, int phase, int row_lo, int row_hi, const double *b, double *x, cudaStream_t st);
int chain_solve_rhs(spk_system *s, int fp32, int nk, const double *B, long long ldb, double *X, long long ldx,
                    cudaStream_t st);
int check_device_error(spk_system *s);
int collect_phase_times(spk_system *s);
int collect_event_set(spk_system *s, int k);

// pointer classification
int is_device_pointer(const void *p);

}  // namespace spk
