// Serving loop: resident preprocessed systems, footprint admission with LRU
// eviction, and continuous batching of solve requests.
//
// The reference splits preprocessing (spike_pstrsv_preproc, src/spike_pstrsv.c:40-81)
// from solving (spike_pstrsv_solve, :149-239) but keeps a single global system.
// The server keeps many systems (spk_system handles) resident in HBM and serves
// solve requests against them:
//
// * Matrices are registered with spk_server_put_matrix (the server keeps a host
//   copy of the CSR arrays).  A matrix is preprocessed when a batch first needs
//   it; its device footprint (spk_debug_scalar "device_bytes", which grows when
//   the batched solves add their work buffers) counts against the HBM budget.
//   When admitting a matrix would exceed the budget, idle resident systems are
//   destroyed in least-recently-used order; a matrix that still does not fit
//   waits until running batches release theirs.
// * Requests (nrhs right-hand sides in host memory) queue per matrix.  Each of
//   nslots worker threads owns a CUDA stream and device/pinned staging buffers;
//   a free worker takes the matrix whose oldest request waited longest, packs up
//   to kBatchRhs right-hand sides of that matrix's queued requests into one
//   batch (requests that arrive while other batches run join the next batch of
//   their matrix), and runs copy-in, spk_solve_batch and copy-out on its
//   stream, so batches of different matrices overlap on the device.  One matrix
//   is in at most one batch at a time (its handle's work buffers are shared).
// * Each request records its latency (submit to result in host memory) and the
//   scaled residual of its batch, which must be <= 1e-12: FP32 + refinement
//   batches take one correction step and are solved again in FP64 if above it.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "spk_internal.cuh"

namespace {

constexpr int kBatchRhs = 32;
constexpr double kTol = 1e-12;  // scaled residual every served result must reach
constexpr int kIrSteps = 1;     // FP32 correction steps per batch (one reaches 1e-12 on well-conditioned systems)

double wall_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
    long long ticket = 0;
    int id = 0, nrhs = 0, mode = 0;
    const double *b = nullptr;
    double *x = nullptr;
    double t_submit = 0, t_start = 0, t_done = 0, resid = -1;
    int status = SPK_OK, iters = 0, batch_rhs = 0;
    bool done = false;
};

struct Matrix {
    int id = 0, n = 0, nparts = 0;
    char uplo = 'L';
    std::vector<double> a;
    std::vector<int> ia, ja;
    spk_system *sys = nullptr;
    long long bytes = 0;      // device footprint while resident
    long long known = 0;      // footprint last measured (kept across evictions)
    long long last_use = 0;   // LRU clock
    bool busy = false;        // in a batch (or being preprocessed)
    std::deque<Request *> pending;
};

struct Slot {
    cudaStream_t st = nullptr;
    double *dB = nullptr, *dX = nullptr, *hB = nullptr, *hX = nullptr;
    size_t cap = 0;  // doubles in each buffer
    spk::DBuf<char> ws;  // batch work columns, lent to the system being solved
    std::thread th;
};

}  // namespace

struct spk_server {
    long long budget = 0;
    long long resident = 0;     // sum of resident systems' footprints
    long long workspace = 0;    // staging buffers of the slots
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::map<int, Matrix *> mats;
    std::unordered_map<long long, Request *> reqs;
    std::vector<Slot *> slots;
    long long next_ticket = 1, clock = 0;
    long long evictions = 0, preprocs = 0, batches = 0, batched_rhs = 0, completed = 0, nomem_retries = 0;
    long long compactions = 0;
    long long rechecks = 0;
    // microseconds spent, summed over the workers: host staging in, solve (with
    // the device copies), host staging out, preprocessing
    std::atomic<long long> us_in{0}, us_solve{0}, us_out{0}, us_pre{0};
    int device = 0;
    bool stop = false;
};

namespace {

using spk::set_error;

// Host copy of a matrix registration.
int copy_csr(Matrix *M, const double *a, const int *ia, const int *ja, int n) {
    if (n <= 0 || !a || !ia || !ja) {
        set_error(SPK_ERR_ARG, "invalid matrix (n=%d)", n);
        return SPK_ERR_ARG;
    }
    const int nnz = ia[n];
    if (ia[0] != 0 || nnz <= 0) {
        set_error(SPK_ERR_INPUT, "ia must start at 0 and end at nnz > 0");
        return SPK_ERR_INPUT;
    }
    M->n = n;
    M->a.assign(a, a + nnz);
    M->ia.assign(ia, ia + n + 1);
    M->ja.assign(ja, ja + nnz);
    return SPK_OK;
}

// Device footprint for admission: the last measured one, else an estimate (the
// CSR and ELL copies and pools ~64 B per nonzero, dense spikes up to ~1 KB per
// row, one batch of work buffers 3 x 32 x 8 B per row).
long long estimate_bytes(const Matrix *M) {
    if (M->known > 0) return M->known;
    const long long nnz = (long long)M->a.size(), n = M->n;
    return 64 * nnz + 1024 * n + (long long)kBatchRhs * 8 * 3 * n;
}

// Destroy idle resident systems, least recently used first, until `need` more
// bytes fit.  Called with the lock held; returns whether they fit.
bool make_room(spk_server *S, long long need, const Matrix *keep) {
    // first the idle systems solved by chains give up the pools their solves
    // never read (spk_compact; its releases synchronize the device, so it runs
    // only when the budget asks for room)
    for (auto &kv : S->mats) {
        if (S->resident + S->workspace + need <= S->budget) break;
        Matrix *M = kv.second;
        if (M == keep || !M->sys || M->busy) continue;
        if (spk_debug_scalar(M->sys, "chain") != 1 || spk_debug_scalar(M->sys, "lean") == 1) continue;
        long long freed = 0;
        if (spk_compact(M->sys, &freed) == SPK_OK) {
            S->resident -= freed;
            M->bytes -= freed;
            S->compactions++;
        }
    }
    while (S->resident + S->workspace + need > S->budget) {
        Matrix *victim = nullptr;
        for (auto &kv : S->mats) {
            Matrix *M = kv.second;
            if (M == keep || !M->sys || M->busy) continue;
            if (!victim || M->last_use < victim->last_use) victim = M;
        }
        if (!victim) return false;
        spk_destroy(victim->sys);
        victim->sys = nullptr;
        S->resident -= victim->bytes;
        victim->bytes = 0;
        S->evictions++;
    }
    return true;
}

int ensure_slot_capacity(spk_server *S, Slot *sl, size_t doubles) {
    if (sl->cap >= doubles) return SPK_OK;
    if (sl->dB) cudaFree(sl->dB);
    if (sl->dX) cudaFree(sl->dX);
    if (sl->hB) cudaFreeHost(sl->hB);
    if (sl->hX) cudaFreeHost(sl->hX);
    sl->dB = sl->dX = sl->hB = sl->hX = nullptr;
    {
        std::lock_guard<std::mutex> g(S->mu);
        S->workspace -= (long long)(2 * sizeof(double) * sl->cap);
    }
    sl->cap = 0;
    SPK_CUDA(cudaMalloc((void **)&sl->dB, doubles * sizeof(double)));
    SPK_CUDA(cudaMalloc((void **)&sl->dX, doubles * sizeof(double)));
    SPK_CUDA(cudaHostAlloc((void **)&sl->hB, doubles * sizeof(double), cudaHostAllocDefault));
    SPK_CUDA(cudaHostAlloc((void **)&sl->hX, doubles * sizeof(double), cudaHostAllocDefault));
    sl->cap = doubles;
    std::lock_guard<std::mutex> g(S->mu);
    S->workspace += (long long)(2 * sizeof(double) * doubles);
    return SPK_OK;
}

// Host copy split across threads when large (the staging of a batch's right-hand
// sides and solutions runs at host memory bandwidth, not one core's).
void par_memcpy(void *dst, const void *src, size_t bytes) {
    constexpr size_t kSplit = 8u << 20;
    constexpr int kThreads = 4;
    if (bytes < kSplit) {
        memcpy(dst, src, bytes);
        return;
    }
    const size_t part = (bytes / kThreads + 63) & ~size_t(63);
    std::thread th[kThreads - 1];
    for (int t = 1; t < kThreads; t++) {
        const size_t off = part * t;
        if (off >= bytes) break;
        th[t - 1] = std::thread([=] { memcpy((char *)dst + off, (const char *)src + off, std::min(part, bytes - off)); });
    }
    memcpy(dst, src, std::min(part, bytes));
    for (auto &t : th)
        if (t.joinable()) t.join();
}

// The slot's workspace, grown to what a batch on this system needs.
int ensure_slot_workspace(spk_server *S, Slot *sl, spk_system *sys) {
    const long long need = spk_workspace_bytes(sys, SPK_MODE_FP32_IR, 1);
    if ((long long)sl->ws.n >= need) return SPK_OK;
    const long long old = (long long)sl->ws.n;
    SPK_TRY(sl->ws.alloc((size_t)need));
    std::lock_guard<std::mutex> g(S->mu);
    S->workspace += need - old;
    return SPK_OK;
}

// Copy-in, batched solve and copy-out of one batch on the slot's stream; the
// system borrows the slot's workspace for the batch (resident systems keep no
// batch buffers).
int run_batch(spk_server *S, Slot *sl, Matrix *M, std::vector<Request *> &batch, int mode, int *iters,
              double *resid) {
    const long long n = M->n;
    int k = 0;
    for (Request *r : batch) k += r->nrhs;
    SPK_TRY(ensure_slot_capacity(S, sl, (size_t)k * n));
    SPK_TRY(ensure_slot_workspace(S, sl, M->sys));
    SPK_TRY(spk_set_workspace(M->sys, sl->ws.p, (long long)sl->ws.n));
    const double t0 = wall_s();
    int c = 0;
    for (Request *r : batch) {
        par_memcpy(sl->hB + (size_t)c * n, r->b, sizeof(double) * r->nrhs * n);
        c += r->nrhs;
    }
    const double t1 = wall_s();
    SPK_CUDA(cudaMemcpyAsync(sl->dB, sl->hB, sizeof(double) * k * n, cudaMemcpyHostToDevice, sl->st));
    // FP32 + refinement takes kIrSteps correction steps without host
    // synchronisation and reports the final scaled residual once; every batch's
    // residual is checked by the caller (a batch above 1e-12 is solved again in FP64)
    const int rc = spk_solve_batch(M->sys, k, sl->dB, n, sl->dX, n, mode, -1.0,
                                   mode == SPK_MODE_FP32_IR ? kIrSteps : 0, (void *)sl->st, iters, resid);
    if (rc == SPK_OK) SPK_CUDA(cudaMemcpyAsync(sl->hX, sl->dX, sizeof(double) * k * n, cudaMemcpyDeviceToHost, sl->st));
    const cudaError_t e = cudaStreamSynchronize(sl->st);
    spk_set_workspace(M->sys, nullptr, 0);
    if (rc != SPK_OK) return rc;
    SPK_CUDA(e);
    SPK_TRY(spk_check(M->sys));
    const double t2 = wall_s();
    c = 0;
    for (Request *r : batch) {
        par_memcpy(r->x, sl->hX + (size_t)c * n, sizeof(double) * r->nrhs * n);
        c += r->nrhs;
    }
    const double t3 = wall_s();
    S->us_in += (long long)((t1 - t0) * 1e6);
    S->us_solve += (long long)((t2 - t1) * 1e6);
    S->us_out += (long long)((t3 - t2) * 1e6);
    return SPK_OK;
}

// The matrix whose oldest queued request is the oldest among idle matrices.
Matrix *pick(spk_server *S) {
    Matrix *best = nullptr;
    for (auto &kv : S->mats) {
        Matrix *M = kv.second;
        if (M->busy || M->pending.empty()) continue;
        if (!best || M->pending.front()->t_submit < best->pending.front()->t_submit) best = M;
    }
    return best;
}

void worker(spk_server *S, Slot *sl) {
    cudaSetDevice(S->device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        Matrix *M = nullptr;
        S->cv_work.wait(lk, [&] { return S->stop || (M = pick(S)) != nullptr; });
        if (S->stop) return;
        // batch: queued requests of one mode, up to kBatchRhs right-hand sides (at least one request)
        std::vector<Request *> batch;
        const int mode = M->pending.front()->mode;
        int k = 0;
        for (auto it = M->pending.begin(); it != M->pending.end();) {
            Request *r = *it;
            if (r->mode != mode || (!batch.empty() && k + r->nrhs > kBatchRhs)) {
                ++it;
                continue;
            }
            batch.push_back(r);
            k += r->nrhs;
            it = M->pending.erase(it);
            if (k >= kBatchRhs) break;
        }
        M->busy = true;
        int status = SPK_OK;
        if (!M->sys) {
            // admission by footprint, LRU eviction of idle systems
            const long long need = estimate_bytes(M);
            while (!make_room(S, need, M)) {
                bool others_busy = false;
                for (auto &kv : S->mats)
                    if (kv.second != M && kv.second->busy) others_busy = true;
                if (!others_busy) break;  // nothing will be released: run over budget
                S->cv_done.wait(lk);
            }
            lk.unlock();
            const double tp = wall_s();
            spk_system *sys = nullptr;
            status = spk_create(&sys);
            if (status == SPK_OK)
                status = spk_preproc(sys, M->a.data(), M->ia.data(), M->ja.data(), M->n, M->nparts, M->uplo, 1,
                                     nullptr, nullptr);
            S->us_pre += (long long)((wall_s() - tp) * 1e6);
            lk.lock();
            if (status == SPK_OK) {
                M->sys = sys;
                M->bytes = spk_debug_scalar(sys, "device_bytes");
                S->resident += M->bytes;
                S->preprocs++;
            } else if (sys) {
                spk_destroy(sys);
            }
        }
        int iters = 0;
        double resid = -1;
        const double t0 = wall_s();
        for (Request *r : batch) r->t_start = t0;
        for (int attempt = 0; status == SPK_OK && attempt < 2; attempt++) {
            lk.unlock();
            status = run_batch(S, sl, M, batch, mode, &iters, &resid);
            lk.lock();
            // the batched solves may have grown the system's work buffers
            const long long now = spk_debug_scalar(M->sys, "device_bytes");
            S->resident += now - M->bytes;
            M->bytes = now;
            M->known = std::max(M->known, now);
            if (status == SPK_OK && !(resid >= 0 && resid <= kTol)) {
                // not at the tolerance (FP32 refinement that stalls, or a bad
                // batch): solve it again in FP64 and check; fail it if still above
                const double first_resid = resid;
                lk.unlock();
                status = run_batch(S, sl, M, batch, SPK_MODE_FP64, &iters, &resid);
                lk.lock();
                S->rechecks++;
                if (status == SPK_OK && !(resid >= 0 && resid <= kTol)) {
                    set_error(SPK_ERR_INPUT, "batch scaled residual %.3e above %.0e", resid, kTol);
                    // the requests fail; the log keeps what the caller's status cannot
                    fprintf(stderr,
                            "spk server: matrix %d (n=%d, %zu requests): scaled residual %.3e after mode %d, "
                            "%.3e after FP64; the requests fail\n",
                            M->id, M->n, batch.size(), first_resid, mode, resid);
                    status = SPK_ERR_INPUT;
                }
            }
            if (status != SPK_ERR_NOMEM || attempt == 1) break;
            // device memory ran out (other workers' preprocessing or staging):
            // release every idle system and retry once
            make_room(S, S->budget, M);
            S->nomem_retries++;
            status = SPK_OK;
        }
        const double t1 = wall_s();
        for (Request *r : batch) {
            r->t_done = t1;
            r->status = status;
            r->resid = resid;
            r->iters = iters;
            r->batch_rhs = k;
            r->done = true;
        }
        M->busy = false;
        M->last_use = ++S->clock;
        S->batches++;
        S->batched_rhs += k;
        S->completed += (long long)batch.size();
        make_room(S, 0, nullptr);  // back under budget where growth pushed it over
        S->cv_done.notify_all();
        S->cv_work.notify_all();
    }
}

}  // namespace

extern "C" {

int spk_server_create(spk_server **out, long long hbm_budget_bytes, int nslots) {
    if (!out || hbm_budget_bytes <= 0 || nslots <= 0 || nslots > 64) {
        set_error(SPK_ERR_ARG, "invalid server arguments (budget=%lld, slots=%d)", hbm_budget_bytes, nslots);
        return SPK_ERR_ARG;
    }
    spk_server *S = new spk_server();
    S->budget = hbm_budget_bytes;
    cudaGetDevice(&S->device);
    for (int i = 0; i < nslots; i++) {
        Slot *sl = new Slot();
        const cudaError_t ce = cudaStreamCreateWithFlags(&sl->st, cudaStreamNonBlocking);
        if (ce != cudaSuccess) {
            delete sl;
            set_error(SPK_ERR_CUDA, "cudaStreamCreate failed: %s", cudaGetErrorString(ce));
            spk_server_destroy(S);
            return SPK_ERR_CUDA;
        }
        S->slots.push_back(sl);
    }
    for (Slot *sl : S->slots) sl->th = std::thread(worker, S, sl);
    *out = S;
    return SPK_OK;
}

int spk_server_destroy(spk_server *S) {
    if (!S) return SPK_OK;
    {
        std::lock_guard<std::mutex> g(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    for (Slot *sl : S->slots)
        if (sl->th.joinable()) sl->th.join();
    for (Slot *sl : S->slots) {
        sl->ws.release();
        if (sl->dB) cudaFree(sl->dB);
        if (sl->dX) cudaFree(sl->dX);
        if (sl->hB) cudaFreeHost(sl->hB);
        if (sl->hX) cudaFreeHost(sl->hX);
        if (sl->st) cudaStreamDestroy(sl->st);
        delete sl;
    }
    for (auto &kv : S->mats) {
        if (kv.second->sys) spk_destroy(kv.second->sys);
        delete kv.second;
    }
    for (auto &kv : S->reqs) delete kv.second;
    delete S;
    return SPK_OK;
}

int spk_server_put_matrix(spk_server *S, int id, const double *a, const int *ia, const int *ja, int n, int nparts,
                          char uplo) {
    if (!S || nparts <= 0 || nparts > n || (uplo != 'L' && uplo != 'U' && uplo != 'l' && uplo != 'u')) {
        set_error(SPK_ERR_ARG, "invalid matrix registration (n=%d, nparts=%d, uplo=%c)", n, nparts, uplo);
        return SPK_ERR_ARG;
    }
    Matrix *M = new Matrix();
    M->id = id;
    M->nparts = nparts;
    M->uplo = (uplo == 'l' || uplo == 'L') ? 'L' : 'U';
    const int rc = copy_csr(M, a, ia, ja, n);
    if (rc != SPK_OK) {
        delete M;
        return rc;
    }
    std::lock_guard<std::mutex> g(S->mu);
    auto it = S->mats.find(id);
    if (it != S->mats.end()) {
        Matrix *old = it->second;
        if (old->busy || !old->pending.empty()) {
            delete M;
            set_error(SPK_ERR_STATE, "matrix %d has requests in flight", id);
            return SPK_ERR_STATE;
        }
        if (old->sys) {
            spk_destroy(old->sys);
            S->resident -= old->bytes;
        }
        delete old;
    }
    S->mats[id] = M;
    return SPK_OK;
}

int spk_server_submit(spk_server *S, int id, int nrhs, const double *b, double *x, int mode, long long *ticket) {
    if (!S || !b || !x || !ticket || nrhs <= 0 || (mode != SPK_MODE_FP64 && mode != SPK_MODE_FP32_IR)) {
        set_error(SPK_ERR_ARG, "invalid request (nrhs=%d, mode=%d)", nrhs, mode);
        return SPK_ERR_ARG;
    }
    Request *r = new Request();
    r->id = id;
    r->nrhs = nrhs;
    r->mode = mode;
    r->b = b;
    r->x = x;
    r->t_submit = wall_s();
    {
        std::lock_guard<std::mutex> g(S->mu);
        auto it = S->mats.find(id);
        if (it == S->mats.end()) {
            delete r;
            set_error(SPK_ERR_ARG, "unknown matrix %d", id);
            return SPK_ERR_ARG;
        }
        r->ticket = S->next_ticket++;
        S->reqs[r->ticket] = r;
        it->second->pending.push_back(r);
        *ticket = r->ticket;
    }
    S->cv_work.notify_one();
    return SPK_OK;
}

int spk_server_wait(spk_server *S, long long ticket, double *latency_s, double *resid, int *iters,
                    int *batch_rhs) {
    if (!S) {
        set_error(SPK_ERR_ARG, "null server");
        return SPK_ERR_ARG;
    }
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) {
        set_error(SPK_ERR_ARG, "unknown ticket %lld", ticket);
        return SPK_ERR_ARG;
    }
    Request *r = it->second;
    S->cv_done.wait(lk, [&] { return r->done; });
    if (latency_s) *latency_s = r->t_done - r->t_submit;
    if (resid) *resid = r->resid;
    if (iters) *iters = r->iters;
    if (batch_rhs) *batch_rhs = r->batch_rhs;
    const int status = r->status;
    S->reqs.erase(it);
    delete r;
    if (status != SPK_OK) set_error(status, "request %lld failed (status %d)", ticket, status);
    return status;
}

int spk_server_stats(spk_server *S, long long *out, int count) {
    if (!S || !out) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    std::lock_guard<std::mutex> g(S->mu);
    long long nres = 0;
    for (auto &kv : S->mats) nres += kv.second->sys != nullptr;
    const long long v[16] = {S->resident,      S->workspace,    nres,           S->evictions,     S->preprocs,
                             S->batches,       S->batched_rhs,  S->completed,   S->budget,        S->nomem_retries,
                             S->rechecks,      S->us_in.load(), S->us_solve.load(), S->us_out.load(), S->us_pre.load(),
                             S->compactions};
    for (int i = 0; i < count && i < 16; i++) out[i] = v[i];
    return SPK_OK;
}

}  // extern "C"
