// Exported C ABI: the reference's five entry points and profiler globals
// (single resident system, as the reference's static arrays), and the
// handle-based spk_* extension.
#include <algorithm>
#include <cstdarg>
#include <ctime>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "spk_internal.cuh"

// ---- globals with the reference's names (src/spike_pstrsv_globals.h:53-79) ----
extern "C" {
char PSTRSV_VERBOSE = 0;
char FORCE_LOAD_BALANCE = 1;
char IS_MATRIX_PARTITIONED = 0;
char SPK_CLOBBER_B = 0;
char SPK_EXACT = 0;
MKL_INT partition_numRows[SPK_MAX_EXPORTED_PARTS];
MKL_INT partition_starts[SPK_MAX_EXPORTED_PARTS];
MKL_INT partition_ends[SPK_MAX_EXPORTED_PARTS];
MKL_INT numRowsReducedSystem = 0;
double memoryAlloc_timer_pstrsv3 = 0;
double preprocessD_timer_pstrsv3 = 0;
double preprocessR_timer_pstrsv3 = 0;
double setDependents_timer_pstrsv3 = 0;
double preprocessS_timer_pstrsv3 = 0;
double preprocessMappings_timer_pstrsv3 = 0;
double produceCompressedR_timer_pstrsv3 = 0;
double produceS_timer_pstrsv3 = 0;
double produceReducedSystem_timer_pstrsv3 = 0;
double init_vars_pstrsv3 = 0;
double reduced_solver_timer_pstrsv3 = 0;
double temp_timer[SPK_MAX_EXPORTED_PARTS];
double waitBefore_timer_pstrsv3[SPK_MAX_EXPORTED_PARTS];
double computeY_timer[SPK_MAX_EXPORTED_PARTS];
double solveIndependent_timer[SPK_MAX_EXPORTED_PARTS];
double subtract_Rx_timer[SPK_MAX_EXPORTED_PARTS];
double waitAfter_timer_pstrsv3[SPK_MAX_EXPORTED_PARTS];
double solveD2_timer[SPK_MAX_EXPORTED_PARTS];
double solveD_timer[SPK_MAX_EXPORTED_PARTS];
}

namespace spk {

namespace {
thread_local std::string g_err_msg;
thread_local int g_err_code = SPK_OK;
std::mutex g_legacy_mu;
spk_system *g_legacy = nullptr;
// device staging for host-pointer solves of the legacy API
DBuf<double> g_b, g_x;
}  // namespace

void set_error(int code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err_msg = buf;
    g_err_code = code;
}

int last_error_code() { return g_err_code; }

int is_device_pointer(const void *p) {
    cudaPointerAttributes attr;
    cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

int clobber_rhs(spk_system *s, const double *x, double *b, cudaStream_t st);

namespace {

int make_system(spk_system **out) {
    spk_system *s = new (std::nothrow) spk_system();
    if (!s) {
        set_error(SPK_ERR_NOMEM, "host allocation failed");
        return SPK_ERR_NOMEM;
    }
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete s;
        set_error(SPK_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
        return SPK_ERR_CUDA;
    }
    s->own_stream = 1;
    // preprocessing's scoped temporaries come from the device's default memory
    // pool in stream order: keep up to 256 MiB of it mapped between
    // synchronizations instead of returning it at each one
    int dev = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        unsigned long long keep = 256ull << 20;  // the attribute is a 64-bit unsigned value
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    *out = s;
    return SPK_OK;
}

// SPK_DEBUG_SYNC=1: report the first CUDA error of the teardown steps on stderr
static bool debug_sync() {
    static const bool on = [] {
        const char *e = getenv("SPK_DEBUG_SYNC");
        return e && e[0] == '1';
    }();
    return on;
}

static void debug_check(const char *where, const spk_system *s = nullptr) {
    if (!debug_sync()) return;
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess)
        fprintf(stderr, "spike_pstrsv debug: %s (n=%d chain=%d): %s\n", where, s ? s->n : -1, s ? s->chain_ok : -1,
                cudaGetErrorString(e));
}

void destroy_system(spk_system *s) {
    if (!s) return;
    debug_check("before teardown", s);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto &set : s->ev)
        for (auto &e : set)
            if (e) cudaEventDestroy(e);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    if (s->pipe_exec) cudaGraphExecDestroy(s->pipe_exec);
    for (cudaEvent_t e : s->pipe_ev) cudaEventDestroy(e);
    for (cudaStream_t q : s->pipe_st) cudaStreamDestroy(q);
    if (s->st_in) cudaStreamDestroy(s->st_in);
    if (s->st_out) cudaStreamDestroy(s->st_out);
    debug_check("after stream teardown", s);
    delete s;
    debug_check("after buffer release");
}

void export_partitions(const spk_system *s) {
    int P = s->P < SPK_MAX_EXPORTED_PARTS ? s->P : SPK_MAX_EXPORTED_PARTS;
    for (int t = 0; t < P; t++) {
        partition_starts[t] = s->parts[t].ps;
        partition_ends[t] = s->parts[t].pe;
        partition_numRows[t] = s->parts[t].num;
    }
    numRowsReducedSystem = s->nRed;
}

void report(const char *where) {
    if (g_err_code == SPK_ERR_TOO_LARGE)
        fprintf(stderr, "%s", "Error: The estimated size of Matrix S is beyond boundaries!\n");
    else
        fprintf(stderr, "spike_pstrsv (%s): %s\n", where, g_err_msg.c_str());
}

void reset_solve_timers(int P) {
    int n = P < SPK_MAX_EXPORTED_PARTS ? P : SPK_MAX_EXPORTED_PARTS;
    memset(temp_timer, 0, sizeof(double) * n);
    memset(waitBefore_timer_pstrsv3, 0, sizeof(double) * n);
    memset(computeY_timer, 0, sizeof(double) * n);
    memset(solveIndependent_timer, 0, sizeof(double) * n);
    memset(subtract_Rx_timer, 0, sizeof(double) * n);
    memset(waitAfter_timer_pstrsv3, 0, sizeof(double) * n);
    memset(solveD2_timer, 0, sizeof(double) * n);
    memset(solveD_timer, 0, sizeof(double) * n);
    reduced_solver_timer_pstrsv3 = 0;
    init_vars_pstrsv3 = 0;
}

// spike_pstrsv_preproc / _spike_pstrsv_preproc (spike_pstrsv.c:40-140)
void legacy_preproc(double *a, MKL_INT *ia, MKL_INT *ja, int n, int nthreads, char uplo, bool timed) {
    std::lock_guard<std::mutex> lk(g_legacy_mu);
    reset_solve_timers(nthreads > 0 ? nthreads : 1);  // initTimers_PSTRSV3 (ops.c:108-120)
    if (!g_legacy && make_system(&g_legacy) != SPK_OK) {
        report("preproc");
        return;
    }
    const int *starts = nullptr, *ends = nullptr;
    if (IS_MATRIX_PARTITIONED) {  // matrix_partitioning.c:23-35
        if (nthreads <= SPK_MAX_EXPORTED_PARTS) {
            starts = partition_starts;
            ends = partition_ends;
        }
        IS_MATRIX_PARTITIONED = 0;
    }
    int on_dev = is_device_pointer(a) && is_device_pointer(ia) && is_device_pointer(ja);
    double ph[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    g_legacy->trunc_tol = SPK_EXACT ? -1.0 : kDefaultTruncTol;
    int rc = preprocess(g_legacy, a, ia, ja, n, nthreads, uplo, FORCE_LOAD_BALANCE, starts, ends, on_dev,
                        timed ? ph : nullptr);
    if (rc != SPK_OK) {
        report("preproc");
        return;
    }
    if (timed) {
        preprocessD_timer_pstrsv3 += ph[0];
        setDependents_timer_pstrsv3 += ph[1];
        preprocessS_timer_pstrsv3 += ph[2];
        preprocessR_timer_pstrsv3 += ph[3];
        preprocessMappings_timer_pstrsv3 += ph[4];
        produceCompressedR_timer_pstrsv3 += ph[5];
        produceS_timer_pstrsv3 += ph[6];
        produceReducedSystem_timer_pstrsv3 += ph[7];
    }
    export_partitions(g_legacy);
    if (PSTRSV_VERBOSE) logPSTRSV3(nthreads);
}

// spike_pstrsv_solve / _spike_pstrsv_solve (spike_pstrsv.c:149-355)
void legacy_solve(char uplo, int m, double *b, double *x, int nthreads, bool timed) {
    std::lock_guard<std::mutex> lk(g_legacy_mu);
    spk_system *s = g_legacy;
    char up = (uplo == 'l' || uplo == 'L') ? 'L' : ((uplo == 'u' || uplo == 'U') ? 'U' : 0);
    if (!s || !s->built) {
        set_error(SPK_ERR_STATE, "spike_pstrsv_solve called before spike_pstrsv_preproc");
        report("solve");
        return;
    }
    if (m != s->n || nthreads != s->P || up != s->uplo) {
        set_error(SPK_ERR_STATE, "solve(m=%d, nthreads=%d, uplo=%c) does not match preproc(n=%d, nthreads=%d, uplo=%c)",
                  m, nthreads, uplo, s->n, s->P, s->uplo);
        report("solve");
        return;
    }
    cudaStream_t st = s->stream;
    double ph[5] = {0, 0, 0, 0, 0};
    int bd = is_device_pointer(b), xd = is_device_pointer(x);
    const double *db = b;
    double *dx = x;
    double t0 = 0;
    if (timed) {
        timespec ts;
        clock_gettime(CLOCK_MONOTONIC, &ts);
        t0 = ts.tv_sec + 1e-9 * ts.tv_nsec;
    }
    if (!bd && g_b.n < (size_t)m && g_b.alloc(m) != SPK_OK) { report("solve"); return; }
    if (!xd) {
        if (g_x.n < (size_t)m && g_x.alloc(m) != SPK_OK) { report("solve"); return; }
        dx = g_x.p;
    }
    if (!bd && !xd && !timed && !SPK_CLOBBER_B && s->chain_ok) {
        // host arrays: copies overlapped with the solve, chunk by chunk
        int rc = chain_solve_host(s, b, x, g_b.p, g_x.p);
        if (rc == SPK_OK) rc = check_device_error(s);
        if (rc != SPK_OK) report("solve");
        return;
    }
    if (!bd) {
        if (cudaMemcpyAsync(g_b.p, b, sizeof(double) * m, cudaMemcpyHostToDevice, st) != cudaSuccess) {
            set_error(SPK_ERR_CUDA, "copy of b to the device failed");
            report("solve");
            return;
        }
        db = g_b.p;
    }
    int rc = solve(s, db, dx, st, timed ? ph : nullptr);
    if (rc == SPK_OK && SPK_CLOBBER_B) {
        rc = clobber_rhs(s, dx, bd ? b : g_b.p, st);
        if (rc == SPK_OK && !bd)
            cudaMemcpyAsync(b, g_b.p, sizeof(double) * m, cudaMemcpyDeviceToHost, st);
    }
    if (rc == SPK_OK && !xd)
        cudaMemcpyAsync(x, dx, sizeof(double) * m, cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (rc == SPK_OK && e == cudaSuccess) rc = check_device_error(s);
    if (rc != SPK_OK || e != cudaSuccess) {
        if (e != cudaSuccess) set_error(SPK_ERR_CUDA, "solve: %s", cudaGetErrorString(e));
        report("solve");
        return;
    }
    if (timed) {
        timespec ts;
        clock_gettime(CLOCK_MONOTONIC, &ts);
        double total = ts.tv_sec + 1e-9 * ts.tv_nsec - t0;
        computeY_timer[0] += ph[1];
        reduced_solver_timer_pstrsv3 += ph[2];
        solveD2_timer[0] += ph[3];
        init_vars_pstrsv3 += total - ph[1] - ph[2] - ph[3];  // copies, reversals, launches
    }
}

}  // namespace
}  // namespace spk

using namespace spk;

extern "C" {

void spike_pstrsv_preproc(double *a, MKL_INT *ia, MKL_INT *ja, int n, int nthreads, const char uplo) {
    legacy_preproc(a, ia, ja, n, nthreads, uplo, false);
}

void _spike_pstrsv_preproc(double *a, MKL_INT *ia, MKL_INT *ja, int n, int nthreads, const char uplo) {
    legacy_preproc(a, ia, ja, n, nthreads, uplo, true);
}

void spike_pstrsv(const char uplo, int m, double *a, MKL_INT *ia, MKL_INT *ja, double *b, double *x,
                  int nthreads) {
    legacy_preproc(a, ia, ja, m, nthreads, uplo, false);
    legacy_solve(uplo, m, b, x, nthreads, false);
}

void spike_pstrsv_solve(const char uplo, int m, double *b, double *x, int nthreads) {
    legacy_solve(uplo, m, b, x, nthreads, false);
}

void _spike_pstrsv_solve(const char uplo, int m, double *b, double *x, int nthreads) {
    legacy_solve(uplo, m, b, x, nthreads, true);
}

void free_PSTRSV3(void) {
    std::lock_guard<std::mutex> lk(g_legacy_mu);
    destroy_system(g_legacy);
    g_legacy = nullptr;
    g_b.release();
    g_x.release();
}

// logPSTRSV3 (ops.c:1311-1332): the same text format, so log parsers keep working.
void logPSTRSV3(int nthreads) {
    spk_system *s = g_legacy;
    if (!s || !s->built) return;
    int P = nthreads < s->P ? nthreads : s->P;
    printf("* * * * * * * * * * * * * * * * * * * * * * \n");
    printf("* Matrix Information\t\t\t\t\t\t\n");
    printf("* ------------------\t\t\t\t\t\t\n");
    printf("* Reduced system size: %d x %d\t\t\t\t\n", s->nRed, s->nRed);
    printf("* Reduced system nnzs: %d \t\t\t\t\t\n", s->nnzRed);
    for (int t = 0; t < P; t++) {
        const Part &p = s->parts[t];
        printf("* S[%d] size: %d x %d\t\t\t\t\t\n", t, p.nRowsS, p.nColsS);
        printf("* isOptimized[%d]: %d\t\t\t\t\t\n", t, p.isOpt);
        printf("* hasReflection[%d]: %d\t\t\t\t\t\n", t, p.hasRefl);
        printf("* hasDependences[%d]: %d\t\t\t\t\n", t, p.hasDep);
        printf("* hasToCalculateS[%d]: %d\t\t\t\t\n", t, p.hasS);
        printf("* Intervals start[%d]: %d, end[%d]: %d\t\n", t, p.si, t, p.ei);
        printf("* Partition start[%d]: %d, end[%d]: %d\t\n", t, p.ps, t, p.pe);
    }
    printf("* * * * * * * * * * * * * * * * * * * * * * \n\n");
    fflush(stdout);
}

const char *spk_last_error(void) { return g_err_msg.c_str(); }
int spk_last_error_code(void) { return g_err_code; }

int spk_create(spk_system **out) {
    if (!out) {
        set_error(SPK_ERR_ARG, "null output pointer");
        return SPK_ERR_ARG;
    }
    return make_system(out);
}

int spk_destroy(spk_system *s) {
    destroy_system(s);
    return SPK_OK;
}

int spk_preproc(spk_system *s, const double *a, const int *ia, const int *ja, int n, int nparts, char uplo,
                int flb, const int *starts, const int *ends) {
    if (!s || !a || !ia || !ja) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    int on_dev = is_device_pointer(a) && is_device_pointer(ia) && is_device_pointer(ja);
    const int rc = preprocess(s, a, ia, ja, n, nparts, uplo, flb, starts, ends, on_dev, nullptr);
    debug_check("after preprocessing", s);
    return rc;
}

int spk_solve_device(spk_system *s, const double *b, double *x, void *stream) {
    if (!s || !b || !x) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    return solve(s, b, x, (cudaStream_t)stream, nullptr);
}

int spk_solve(spk_system *s, const double *b, double *x) {
    if (!s || !b || !x) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    if (!s->built) {
        set_error(SPK_ERR_STATE, "no preprocessed system");
        return SPK_ERR_STATE;
    }
    int n = s->n;
    int bd = is_device_pointer(b), xd = is_device_pointer(x);
    // host arrays go through device copies kept with the system (allocated once)
    const double *db = b;
    double *dx = x;
    if (!bd) {
        if (s->stage_b.n < (size_t)n) SPK_TRY(s->stage_b.alloc(n));
        db = s->stage_b.p;
    }
    if (!xd) {
        if (s->stage_x.n < (size_t)n) SPK_TRY(s->stage_x.alloc(n));
        dx = s->stage_x.p;
    }
    if (!bd && !xd && s->chain_ok) {
        SPK_TRY(chain_solve_host(s, b, x, s->stage_b.p, s->stage_x.p));
        debug_check("after the pipelined solve", s);
        const int rc = check_device_error(s);
        debug_check("after the error word", s);
        return rc;
    }
    if (!bd) SPK_CUDA(cudaMemcpyAsync(s->stage_b.p, b, sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
    SPK_TRY(solve(s, db, dx, s->stream, nullptr));
    if (!xd) SPK_CUDA(cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
    SPK_CUDA(cudaStreamSynchronize(s->stream));
    debug_check("after the partition solve", s);
    const int rc = check_device_error(s);
    debug_check("after the error word", s);
    return rc;
}

int spk_check(spk_system *s) {
    if (!s) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    SPK_CUDA(cudaStreamSynchronize(s->stream));
    return check_device_error(s);
}

int spk_solve_batch(spk_system *s, int nrhs, const double *B, long long ldb, double *X, long long ldx, int mode,
                    double tol, int maxit, void *stream, int *iters, double *resid) {
    if (!s || !B || !X) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    if (!is_device_pointer(B) || !is_device_pointer(X)) {
        set_error(SPK_ERR_ARG, "spk_solve_batch takes device arrays");
        return SPK_ERR_ARG;
    }
    return solve_batch(s, nrhs, B, ldb, X, ldx, mode, tol, maxit, (cudaStream_t)stream, iters, resid);
}

int spk_solve_batch_noalloc(spk_system *s, int nrhs, const double *B, long long ldb, double *X, long long ldx,
                            void *stream) {
    if (!s || !B || !X) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    if (!is_device_pointer(B) || !is_device_pointer(X)) {
        set_error(SPK_ERR_ARG, "spk_solve_batch_noalloc takes device arrays");
        return SPK_ERR_ARG;
    }
    return solve_batch_static(s, nrhs, B, ldb, X, ldx, (cudaStream_t)stream);
}

int spk_set_workspace(spk_system *s, void *dev_ptr, long long bytes) {
    if (!s || bytes < 0 || (dev_ptr && !is_device_pointer(dev_ptr)) || (!dev_ptr && bytes)) {
        set_error(SPK_ERR_ARG, "invalid workspace (pointer %p, %lld bytes)", dev_ptr, bytes);
        return SPK_ERR_ARG;
    }
    if (dev_ptr && ((uintptr_t)dev_ptr & 255)) {
        set_error(SPK_ERR_ARG, "workspace must be 256-byte aligned");
        return SPK_ERR_ARG;
    }
    s->ext_ws = (char *)dev_ptr;
    s->ext_ws_bytes = dev_ptr ? (size_t)bytes : 0;
    if (dev_ptr) {
        // the system's own batch buffers are no longer needed
        s->work.release();
        s->rbuf.release();
        s->dbuf.release();
    }
    return SPK_OK;
}

long long spk_workspace_bytes(const spk_system *s, int mode, int with_residual) {
    if (!s) return -1;
    const long long col = ((32ll * s->n * 8) + 255) / 256 * 256;
    // FP32 + refinement also keeps the reduced unknowns in FP64 (32 columns)
    const long long red = mode == 1 ? 32ll * s->nRed * 8 : 0;
    return col * (1 + (mode == 1 || with_residual) + (mode == 1)) + red;
}

int spk_set_profiling(spk_system *s, int on) {
    if (!s) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    if (on && !s->ev[0][0])
        for (auto &set : s->ev)
            for (auto &e : set) SPK_CUDA(cudaEventCreate(&e));
    s->profiling = on;
    return SPK_OK;
}

int spk_phase_times(spk_system *s, double *ms3, long long *solves) {
    if (!s || !ms3) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    SPK_TRY(collect_phase_times(s));
    for (int k = 0; k < 3; k++) {
        ms3[k] = s->phase_ms[k];
        s->phase_ms[k] = 0;
    }
    if (solves) *solves = s->profiled_solves;
    s->profiled_solves = 0;
    return SPK_OK;
}

int spk_set_truncation(spk_system *s, double tau) {
    if (!s) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    if (s->lean) {
        set_error(SPK_ERR_STATE, "the system was compacted (spk_compact): preprocess it again to change the truncation");
        return SPK_ERR_STATE;
    }
    s->trunc_tol = tau;
    if (s->built) return solve_prepare(s);
    return SPK_OK;
}

int spk_tune(spk_system *s, const char *name, long long value) {
    if (!s || !name) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    if (!s->built) {
        set_error(SPK_ERR_STATE, "spk_tune needs a preprocessed system");
        return SPK_ERR_STATE;
    }
    return spk::chain_tune(s, name, value);
}

int spk_compact(spk_system *s, long long *freed) {
    if (!s) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    if (!s->built || !s->chain_ok) {
        set_error(SPK_ERR_STATE, "spk_compact needs a preprocessed system solved by chains");
        return SPK_ERR_STATE;
    }
    if (s->lean) {
        if (freed) *freed = 0;
        return SPK_OK;
    }
    SPK_TRY(spk::residual_prepare(s));  // diag and ||A|| come from the CSR
    const long long before = spk_debug_scalar(s, "device_bytes");
    s->ua.release();
    s->uia.release();
    s->uja.release();
    s->D.release();
    s->T2.release();
    s->S.release();
    s->T.release();
    s->ID.release();
    s->JD.release();
    s->IT2.release();
    s->JT2.release();
    s->mapR.release();
    s->dep.release();
    s->mapRedX.release();
    s->IT.release();
    s->JT.release();
    s->d_ps.release();
    s->d_pe.release();
    s->d_lvl.release();
    s->d_tasks1.release();
    s->d_tasks2.release();
    s->xbuf.release();
    s->xout_u.release();
    s->d_red_rows.release();
    s->d_red_off.release();
    s->lean = 1;
    if (freed) *freed = before - spk_debug_scalar(s, "device_bytes");
    return SPK_OK;
}

spk_system *spk_legacy_system(void) { return g_legacy; }

long long spk_debug_scalar(const spk_system *s, const char *name) {
    if (!s || !name) return -1;
    if (!strcmp(name, "numRowsReducedSystem")) return s->nRed;
    if (!strcmp(name, "numNnzsReducedSystem")) return s->nnzRed;
    if (!strcmp(name, "reducedSystemSolverStart")) return s->rss;
    if (!strcmp(name, "isReducedSystemNecessary")) return s->redNec;
    if (!strcmp(name, "totalArea")) return s->totalArea;
    if (!strcmp(name, "n")) return s->n;
    if (!strcmp(name, "nnz")) return s->nnz;
    if (!strcmp(name, "P")) return s->P;
    if (!strcmp(name, "rows_phase1")) return s->rows_phase1;
    if (!strcmp(name, "launches")) return s->launches;
    if (!strcmp(name, "ell")) return s->ell_ok;
    if (!strcmp(name, "ell_entries")) return s->ell_entries;
    if (!strcmp(name, "launches_per_solve")) {
        if (s->chain_ok) return (s->nctasks1 ? 1 : 0) + (s->nctasks4 ? 1 : 0);
        return (s->redNec && s->ntasks1 ? 1 : 0) + (s->redNec && s->nkept ? 1 : 0) + 1;
    }
    if (!strcmp(name, "chain")) return s->chain_ok;
    if (!strcmp(name, "lean")) return s->lean;
    if (!strcmp(name, "device_check")) return chain_device_check();  // checked builds only
    if (!strcmp(name, "chains")) return s->ch_count;
    if (!strcmp(name, "chain_rows")) return s->ch_len;
    if (!strcmp(name, "chain_width")) return s->ch_width;
    if (!strcmp(name, "chain_reach")) return s->ch_reach;
    if (!strcmp(name, "chain_rows_phase1")) return s->ch_rows1;
    if (!strcmp(name, "chain_rows_phase4")) return s->ch_rows4;
    if (!strcmp(name, "chain_tasks_phase4")) return s->nctasks4;
    if (!strcmp(name, "chain_batch_rows")) return s->cp_batch.len ? s->cp_batch.len : s->ch_len;
    // wall microseconds of the last preprocessing, by part
    if (!strncmp(name, "prep_us_", 8)) {
        static const char *parts[5] = {"reference", "spikes", "tasks", "ell", "chains"};
        for (int i = 0; i < 5; ++i)
            if (!strcmp(name + 8, parts[i])) return (long long)(s->prep_ms[i] * 1e3);
    }
    // spk_tune's knobs under their own names
    if (!strcmp(name, "rows")) return s->ch_len;
    if (!strcmp(name, "batch_rows")) return s->cp_batch.len ? s->cp_batch.len : s->ch_len;
    if (!strcmp(name, "stages")) return s->ch_stages;
    if (!strcmp(name, "batch_path")) return s->batch_path;
    if (!strcmp(name, "chain_host_rows")) return s->cp_host.len ? s->cp_host.len : s->ch_len;
    if (!strcmp(name, "chain_bytes")) return (long long)(s->ch_val.bytes() + s->ch_off.bytes() + s->ch_ptr.bytes());
    if (!strcmp(name, "rows_phase4")) return s->rows_phase4;
    if (!strcmp(name, "kept_reduced_rows")) return s->nkept;
    if (!strcmp(name, "reduced_levels")) return s->nlvl;
    if (!strcmp(name, "device_bytes")) {
        long long b = 0;
        b += s->ua.bytes() + s->uia.bytes() + s->uja.bytes() + s->D.bytes() + s->ID.bytes() + s->JD.bytes();
        b += s->T2.bytes() + s->IT2.bytes() + s->JT2.bytes() + s->S.bytes() + s->T.bytes() + s->IT.bytes();
        b += s->JT.bytes() + s->mapR.bytes() + s->dep.bytes() + s->mapRedX.bytes() + s->xbuf.bytes();
        b += s->xout_u.bytes() + s->d_tasks1.bytes() + s->d_tasks2.bytes() + s->d_red_rows.bytes();
        b += s->rdiag.bytes() + s->ell_val.bytes() + s->ell_col.bytes() + s->ell_ptr.bytes();
        b += s->ell_valf.bytes() + s->rdiagf.bytes() + s->diag.bytes() + s->rbuf.bytes() + s->dbuf.bytes() + s->work.bytes();
        b += s->stage_b.bytes() + s->stage_x.bytes();
        b += s->ch_val.bytes() + s->ch_valb.bytes() + s->ch_valbf.bytes() + s->ch_near.bytes() + s->ch_nearf.bytes() + s->ch_off.bytes() + s->ch_ptr.bytes() + s->d_ctasks1.bytes() +
             s->d_ctasks4.bytes();
        return b;
    }
    return -1;
}

int spk_chain_phase(spk_system *s, int phase, int row_lo, int row_hi, const double *b, double *x, void *stream) {
    if (!s || !b || !x) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    if (!s->built || !s->chain_ok) {
        set_error(SPK_ERR_STATE, "spk_chain_phase needs a system solved by chains (default truncation, banded rows)");
        return SPK_ERR_STATE;
    }
    if ((phase != 1 && phase != 4) || row_lo < 0 || row_hi > s->n || row_lo > row_hi) {
        set_error(SPK_ERR_ARG, "invalid chain phase %d or row range [%d, %d)", phase, row_lo, row_hi);
        return SPK_ERR_ARG;
    }
    if (!is_device_pointer(b) || !is_device_pointer(x)) {
        set_error(SPK_ERR_ARG, "spk_chain_phase takes device arrays");
        return SPK_ERR_ARG;
    }
    return chain_phase(s, phase, row_lo, row_hi, b, x, (cudaStream_t)stream);
}

int spk_debug_set(spk_system *s, const char *name, long long value) {
    if (!s || !name) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    if (!strcmp(name, "fail_waits")) {
        s->dbg_fail_waits = value != 0;
        return SPK_OK;
    }
    set_error(SPK_ERR_ARG, "unknown debug setting '%s'", name);
    return SPK_ERR_ARG;
}

int spk_debug_array(const spk_system *s, const char *name, void *dst, long long cap, long long *count,
                    char *type) {
    if (!s || !name || !count || !type) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    const int P = s->P, n = s->n;
    // per-partition host metadata
    struct Field { const char *name; char ty; };
    auto part_field = [&](const Part &p, const char *nm, long long *q) -> int {
        if (!strcmp(nm, "partition_starts")) return p.ps;
        if (!strcmp(nm, "partition_ends")) return p.pe;
        if (!strcmp(nm, "partition_numRows")) return p.num;
        if (!strcmp(nm, "starts_D")) return p.startsD;
        if (!strcmp(nm, "ends_D")) return p.endsD;
        if (!strcmp(nm, "starts_R")) return p.startsR;
        if (!strcmp(nm, "ends_R")) return p.endsR;
        if (!strcmp(nm, "hasDependences")) return p.hasDep;
        if (!strcmp(nm, "hasReflections")) return p.hasRefl;
        if (!strcmp(nm, "hasToCalculateSs")) return p.hasS;
        if (!strcmp(nm, "isOptimizeds")) return p.isOpt;
        if (!strcmp(nm, "numRows_S")) return p.nRowsS;
        if (!strcmp(nm, "numCols_S")) return p.nColsS;
        if (!strcmp(nm, "start_intervals")) return p.si;
        if (!strcmp(nm, "end_intervals")) return p.ei;
        if (!strcmp(nm, "starts_D0")) return p.sD0;
        if (!strcmp(nm, "ends_D0")) return p.eD0;
        if (!strcmp(nm, "starts_D1")) return p.sD1;
        if (!strcmp(nm, "ends_D1")) return p.eD1;
        if (!strcmp(nm, "starts_D2")) return p.sD2;
        if (!strcmp(nm, "ends_D2")) return p.eD2;
        if (!strcmp(nm, "starts_mapR")) return p.sMapR;
        if (!strcmp(nm, "ends_mapR")) return p.eMapR;
        if (!strcmp(nm, "starts_S")) { *q = p.startsS; return 0; }
        if (!strcmp(nm, "ends_S")) { *q = p.endsS; return 0; }
        *q = -1;
        return -2147483647 - 1;
    };
    static const Field pfields[] = {
        {"partition_starts", 'i'}, {"partition_ends", 'i'}, {"partition_numRows", 'i'}, {"starts_D", 'i'},
        {"ends_D", 'i'}, {"starts_R", 'i'}, {"ends_R", 'i'}, {"hasDependences", 'c'},
        {"hasReflections", 'c'}, {"hasToCalculateSs", 'c'}, {"isOptimizeds", 'c'}, {"numRows_S", 'i'},
        {"numCols_S", 'i'}, {"start_intervals", 'i'}, {"end_intervals", 'i'}, {"starts_D0", 'i'},
        {"ends_D0", 'i'}, {"starts_D1", 'i'}, {"ends_D1", 'i'}, {"starts_D2", 'i'}, {"ends_D2", 'i'},
        {"starts_mapR", 'i'}, {"ends_mapR", 'i'}, {"starts_S", 'q'}, {"ends_S", 'q'}};
    for (const Field &f : pfields) {
        if (strcmp(f.name, name)) continue;
        *count = P;
        *type = f.ty;
        if (dst) {
            long long m = cap < P ? cap : P;
            for (long long t = 0; t < m; t++) {
                long long q = 0;
                int v = part_field(s->parts[t], name, &q);
                if (f.ty == 'i') ((int *)dst)[t] = v;
                else if (f.ty == 'c') ((char *)dst)[t] = (char)v;
                else ((long long *)dst)[t] = q;
            }
        }
        return SPK_OK;
    }
    const void *src = nullptr;
    long long cnt = 0;
    char ty = 'i';
    if (!strcmp(name, "D")) { src = s->D.p; cnt = s->nDpool; ty = 'd'; }
    else if (!strcmp(name, "JD")) { src = s->JD.p; cnt = s->nDpool; }
    else if (!strcmp(name, "ID")) { src = s->ID.p; cnt = 2LL * n + 1; }
    else if (!strcmp(name, "T2")) { src = s->T2.p; cnt = s->nT2; ty = 'd'; }
    else if (!strcmp(name, "JT2")) { src = s->JT2.p; cnt = s->nT2; }
    else if (!strcmp(name, "IT2")) { src = s->IT2.p; cnt = s->nIT2rows + 1; }
    else if (!strcmp(name, "mapR")) { src = s->mapR.p; cnt = s->nMapR; }
    else if (!strcmp(name, "S")) { src = s->S.p; cnt = s->totalArea; ty = 'd'; }
    else if (!strcmp(name, "mapReducedX")) { src = s->mapRedX.p; cnt = s->nRed; }
    else if (!strcmp(name, "T")) { src = s->T.p; cnt = s->nT; ty = 'd'; }
    else if (!strcmp(name, "JT")) { src = s->JT.p; cnt = s->nT; }
    else if (!strcmp(name, "IT")) { src = s->IT.p; cnt = s->rss + 1; }
    else if (!strcmp(name, "dependents")) { src = s->dep.p; cnt = n; }
    else if (!strcmp(name, "U_ia")) { src = s->uia.p; cnt = n + 1; }
    else if (!strcmp(name, "U_ja")) { src = s->uja.p; cnt = s->nnz; }
    else if (!strcmp(name, "U_a")) { src = s->ua.p; cnt = s->nnz; ty = 'd'; }
    else if (!strcmp(name, "chain_tasks1") || !strcmp(name, "chain_tasks4")) {
        // (lo, hi, st_lo, st_hi) per task, U order, host copies
        const std::vector<ChainTask> &v = name[11] == '1' ? s->h_ctasks1 : s->h_ctasks4;
        *count = 4LL * (long long)v.size();
        *type = 'i';
        if (dst) memcpy(dst, v.data(), sizeof(int) * (size_t)std::min<long long>(cap, *count));
        return SPK_OK;
    }
    else {
        set_error(SPK_ERR_ARG, "unknown array '%s'", name);
        return SPK_ERR_ARG;
    }
    *count = cnt;
    *type = ty;
    if (dst && cnt > 0 && src) {
        long long m = cap < cnt ? cap : cnt;
        size_t es = ty == 'd' ? 8 : 4;
        cudaStreamSynchronize(s->stream);
        SPK_CUDA(cudaMemcpy(dst, src, (size_t)m * es, cudaMemcpyDeviceToHost));
    }
    return SPK_OK;
}

}  // extern "C"
