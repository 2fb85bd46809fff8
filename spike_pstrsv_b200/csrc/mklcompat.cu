// libspike_pstrsv_mklcompat.so: the MKL entry points the reference's drivers
// call (include/compat/mkl.h), so that its profiler (test/runtime_analysis.c)
// and example (example_usage.c) build and run against this library without
// MKL.  The profiler's two triangular-solve comparators - the sequential
// mkl_cspblas_dcsrtrsv (runtime_analysis.c:67-77) and the inspector-executor
// mkl_sparse_d_trsv (:79-87, :345-381) - become cuSPARSE SpSV on the GPU; the
// other entry points are host code with MKL's documented meaning.
//
// Kept apart from libspike_pstrsv_b200.so so that a process linking the real
// MKL never sees two definitions of these names.
#include <cuda_runtime.h>
#include <cusparse.h>
#include <omp.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <tuple>

#include "../../include/compat/mkl.h"

namespace {

int g_threads = 0;  // 0: OpenMP's default

bool cuda_ok(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return true;
    fprintf(stderr, "mkl compat: %s: %s\n", what, cudaGetErrorString(e));
    return false;
}

bool sparse_ok(cusparseStatus_t e, const char *what) {
    if (e == CUSPARSE_STATUS_SUCCESS) return true;
    fprintf(stderr, "mkl compat: %s: %s\n", what, cusparseGetErrorString(e));
    return false;
}

// One triangular CSR resident on the GPU with its SpSV analysis.
struct SvPlan {
    int m = 0, nnz = 0;
    cusparseOperation_t op = CUSPARSE_OPERATION_NON_TRANSPOSE;
    cusparseHandle_t h = nullptr;
    cudaStream_t st = nullptr;
    int *ip = nullptr, *jp = nullptr;
    double *vp = nullptr, *xp = nullptr, *yp = nullptr;
    void *buf = nullptr;
    cusparseSpMatDescr_t A = nullptr;
    cusparseDnVecDescr_t vx = nullptr, vy = nullptr;
    cusparseSpSVDescr_t sv = nullptr;
    bool ready = false;

    ~SvPlan() {
        if (sv) cusparseSpSV_destroyDescr(sv);
        if (vx) cusparseDestroyDnVec(vx);
        if (vy) cusparseDestroyDnVec(vy);
        if (A) cusparseDestroySpMat(A);
        if (h) cusparseDestroy(h);
        cudaFree(ip);
        cudaFree(jp);
        cudaFree(vp);
        cudaFree(xp);
        cudaFree(yp);
        cudaFree(buf);
        if (st) cudaStreamDestroy(st);
    }

    // rows_start[r] .. rows_end[r] - base: row r (MKL's four-array CSR).
    bool build(int rows, const int *rows_start, const int *rows_end, const int *cols, const double *vals, int base,
               bool upper, bool unit, bool trans) {
        m = rows;
        const int first = rows_start[0];
        nnz = rows_end[rows - 1] - first;
        int *hp = (int *)malloc(sizeof(int) * (rows + 1));
        int *hj = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
        double *hv = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
        if (!hp || !hj || !hv) {
            free(hp);
            free(hj);
            free(hv);
            return false;
        }
        // compact (rows_start, rows_end) into one zero-based row-pointer array
        int q = 0;
        for (int r = 0; r < rows; ++r) {
            hp[r] = q;
            for (int k = rows_start[r] - first; k < rows_end[r] - first; ++k, ++q) {
                hj[q] = cols[k] - base;
                hv[q] = vals[k];
            }
        }
        hp[rows] = q;
        nnz = q;
        bool ok = cuda_ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream") &&
                  cuda_ok(cudaMalloc(&ip, sizeof(int) * (rows + 1)), "cudaMalloc") &&
                  cuda_ok(cudaMalloc(&jp, sizeof(int) * (nnz > 0 ? nnz : 1)), "cudaMalloc") &&
                  cuda_ok(cudaMalloc(&vp, sizeof(double) * (nnz > 0 ? nnz : 1)), "cudaMalloc") &&
                  cuda_ok(cudaMalloc(&xp, sizeof(double) * rows), "cudaMalloc") &&
                  cuda_ok(cudaMalloc(&yp, sizeof(double) * rows), "cudaMalloc") &&
                  cuda_ok(cudaMemcpy(ip, hp, sizeof(int) * (rows + 1), cudaMemcpyHostToDevice), "upload") &&
                  cuda_ok(cudaMemcpy(jp, hj, sizeof(int) * nnz, cudaMemcpyHostToDevice), "upload") &&
                  cuda_ok(cudaMemcpy(vp, hv, sizeof(double) * nnz, cudaMemcpyHostToDevice), "upload");
        free(hp);
        free(hj);
        free(hv);
        if (!ok) return false;
        op = trans ? CUSPARSE_OPERATION_TRANSPOSE : CUSPARSE_OPERATION_NON_TRANSPOSE;
        cusparseFillMode_t fill = upper ? CUSPARSE_FILL_MODE_UPPER : CUSPARSE_FILL_MODE_LOWER;
        cusparseDiagType_t diag = unit ? CUSPARSE_DIAG_TYPE_UNIT : CUSPARSE_DIAG_TYPE_NON_UNIT;
        const double one = 1.0;
        size_t bytes = 0;
        ok = sparse_ok(cusparseCreate(&h), "cusparseCreate") && sparse_ok(cusparseSetStream(h, st), "stream") &&
             sparse_ok(cusparseCreateCsr(&A, rows, rows, nnz, ip, jp, vp, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                                         CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F),
                       "cusparseCreateCsr") &&
             sparse_ok(cusparseSpMatSetAttribute(A, CUSPARSE_SPMAT_FILL_MODE, &fill, sizeof(fill)), "fill mode") &&
             sparse_ok(cusparseSpMatSetAttribute(A, CUSPARSE_SPMAT_DIAG_TYPE, &diag, sizeof(diag)), "diag type") &&
             sparse_ok(cusparseCreateDnVec(&vx, rows, xp, CUDA_R_64F), "vector") &&
             sparse_ok(cusparseCreateDnVec(&vy, rows, yp, CUDA_R_64F), "vector") &&
             sparse_ok(cusparseSpSV_createDescr(&sv), "SpSV descriptor") &&
             sparse_ok(cusparseSpSV_bufferSize(h, op, &one, A, vx, vy, CUDA_R_64F, CUSPARSE_SPSV_ALG_DEFAULT, sv,
                                               &bytes),
                       "SpSV buffer size") &&
             cuda_ok(cudaMalloc(&buf, bytes ? bytes : 1), "cudaMalloc") &&
             sparse_ok(cusparseSpSV_analysis(h, op, &one, A, vx, vy, CUDA_R_64F, CUSPARSE_SPSV_ALG_DEFAULT, sv, buf),
                       "SpSV analysis") &&
             cuda_ok(cudaStreamSynchronize(st), "analysis");
        ready = ok;
        return ok;
    }

    bool solve(double alpha, const double *x, double *y) {
        return cuda_ok(cudaMemcpyAsync(xp, x, sizeof(double) * m, cudaMemcpyHostToDevice, st), "copy x") &&
               sparse_ok(cusparseSpSV_solve(h, op, &alpha, A, vx, vy, CUDA_R_64F, CUSPARSE_SPSV_ALG_DEFAULT, sv),
                         "SpSV solve") &&
               cuda_ok(cudaMemcpyAsync(y, yp, sizeof(double) * m, cudaMemcpyDeviceToHost, st), "copy y") &&
               cuda_ok(cudaStreamSynchronize(st), "solve");
    }
};

using CacheKey = std::tuple<const void *, const void *, const void *, int, int, char, char, char>;
std::mutex g_mu;
std::map<CacheKey, SvPlan *> g_cache;

}  // namespace

// The handle of mkl_sparse_d_create_csr.
struct spk_mkl_sparse_matrix {
    int rows = 0, base = 0;
    const int *rs = nullptr, *re = nullptr, *cols = nullptr;
    const double *vals = nullptr;
    bool hinted = false;
    sparse_operation_t hint_op = SPARSE_OPERATION_NON_TRANSPOSE;
    matrix_descr hint{};
    SvPlan *plan = nullptr;
    sparse_operation_t plan_op = SPARSE_OPERATION_NON_TRANSPOSE;
    matrix_descr plan_descr{};
};

extern "C" {

void *mkl_malloc(size_t size, int alignment) {
    void *p = nullptr;
    size_t al = alignment < (int)sizeof(void *) ? sizeof(void *) : (size_t)alignment;
    while (al & (al - 1)) ++al;  // posix_memalign wants a power of two
    if (posix_memalign(&p, al, size ? size : 1) != 0) return nullptr;
    return p;
}

void mkl_free(void *p) { free(p); }

void mkl_set_num_threads(int n) { g_threads = n > 0 ? n : 0; }

int mkl_get_max_threads(void) { return g_threads > 0 ? g_threads : omp_get_max_threads(); }

void cblas_dcopy(const MKL_INT n, const double *x, const MKL_INT incx, double *y, const MKL_INT incy) {
    for (MKL_INT i = 0; i < n; ++i) y[(long long)i * incy] = x[(long long)i * incx];
}

void mkl_dcsrmv(const char *transa, const MKL_INT *m, const MKL_INT *k, const double *alpha, const char *matdescra,
                const double *val, const MKL_INT *indx, const MKL_INT *pntrb, const MKL_INT *pntre, const double *x,
                const double *beta, double *y) {
    const int base = (matdescra[3] == 'F' || matdescra[3] == 'f') ? 1 : 0;
    const int first = pntrb[0];
    const bool trans = transa[0] == 'T' || transa[0] == 't' || transa[0] == 'C' || transa[0] == 'c';
    const int rows = *m;
    const int nthr = mkl_get_max_threads();
    if (!trans) {
#pragma omp parallel for num_threads(nthr) schedule(static)
        for (int r = 0; r < rows; ++r) {
            double s = 0.0;
            for (int q = pntrb[r] - first; q < pntre[r] - first; ++q) s += val[q] * x[indx[q] - base];
            y[r] = *beta * y[r] + *alpha * s;
        }
    } else {  // y (length k) := alpha A^T x + beta y
        for (int c = 0; c < *k; ++c) y[c] *= *beta;
        for (int r = 0; r < rows; ++r)
            for (int q = pntrb[r] - first; q < pntre[r] - first; ++q) y[indx[q] - base] += *alpha * val[q] * x[r];
    }
}

void mkl_cspblas_dcsrtrsv(const char *uplo, const char *transa, const char *diag, const MKL_INT *m, const double *a,
                          const MKL_INT *ia, const MKL_INT *ja, const double *x, double *y) {
    const char u = (char)(uplo[0] & ~0x20), t = (char)(transa[0] & ~0x20), d = (char)(diag[0] & ~0x20);
    const CacheKey key{a, ia, ja, *m, ia[*m], u, t, d};
    SvPlan *p = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_cache.find(key);
        if (it != g_cache.end()) {
            p = it->second;
        } else {
            p = new SvPlan();
            if (!p->build(*m, ia, ia + 1, ja, a, 0, u == 'U', d == 'U', t != 'N')) {
                delete p;
                fprintf(stderr, "mkl compat: mkl_cspblas_dcsrtrsv could not set up the GPU solve\n");
                return;
            }
            g_cache[key] = p;
        }
    }
    if (!p->solve(1.0, x, y)) fprintf(stderr, "mkl compat: mkl_cspblas_dcsrtrsv failed\n");
}

void spk_mkl_release_cache(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto &kv : g_cache) delete kv.second;
    g_cache.clear();
}

sparse_status_t mkl_sparse_d_create_csr(sparse_matrix_t *A, const sparse_index_base_t indexing, const MKL_INT rows,
                                        const MKL_INT cols, MKL_INT *rows_start, MKL_INT *rows_end,
                                        MKL_INT *col_indx, double *values) {
    if (!A || rows <= 0 || rows != cols || !rows_start || !rows_end || !col_indx || !values)
        return SPARSE_STATUS_INVALID_VALUE;
    auto *h = new (std::nothrow) spk_mkl_sparse_matrix();
    if (!h) return SPARSE_STATUS_ALLOC_FAILED;
    h->rows = rows;
    h->base = indexing == SPARSE_INDEX_BASE_ONE ? 1 : 0;
    h->rs = rows_start;
    h->re = rows_end;
    h->cols = col_indx;
    h->vals = values;
    *A = h;
    return SPARSE_STATUS_SUCCESS;
}

sparse_status_t mkl_sparse_set_sv_hint(const sparse_matrix_t A, const sparse_operation_t operation,
                                       const struct matrix_descr descr, const MKL_INT expected_calls) {
    (void)expected_calls;
    if (!A) return SPARSE_STATUS_NOT_INITIALIZED;
    A->hinted = true;
    A->hint_op = operation;
    A->hint = descr;
    return SPARSE_STATUS_SUCCESS;
}

static sparse_status_t prepare(sparse_matrix_t A, sparse_operation_t op, const matrix_descr &d) {
    if (A->plan && A->plan_op == op && A->plan_descr.mode == d.mode && A->plan_descr.diag == d.diag)
        return SPARSE_STATUS_SUCCESS;
    if (d.type != SPARSE_MATRIX_TYPE_TRIANGULAR) return SPARSE_STATUS_NOT_SUPPORTED;
    delete A->plan;
    A->plan = new (std::nothrow) SvPlan();
    if (!A->plan) return SPARSE_STATUS_ALLOC_FAILED;
    // row pointers relative to the base: rows_start/rows_end are base-indexed
    if (!A->plan->build(A->rows, A->rs, A->re, A->cols, A->vals, A->base, d.mode == SPARSE_FILL_MODE_UPPER,
                        d.diag == SPARSE_DIAG_UNIT, op == SPARSE_OPERATION_TRANSPOSE)) {
        delete A->plan;
        A->plan = nullptr;
        return SPARSE_STATUS_EXECUTION_FAILED;
    }
    A->plan_op = op;
    A->plan_descr = d;
    return SPARSE_STATUS_SUCCESS;
}

sparse_status_t mkl_sparse_optimize(sparse_matrix_t A) {
    if (!A) return SPARSE_STATUS_NOT_INITIALIZED;
    if (!A->hinted) return SPARSE_STATUS_SUCCESS;
    return prepare(A, A->hint_op, A->hint);
}

sparse_status_t mkl_sparse_d_trsv(const sparse_operation_t operation, const double alpha, const sparse_matrix_t A,
                                  const struct matrix_descr descr, const double *x, double *y) {
    if (!A) return SPARSE_STATUS_NOT_INITIALIZED;
    const sparse_status_t s = prepare(A, operation, descr);
    if (s != SPARSE_STATUS_SUCCESS) return s;
    return A->plan->solve(alpha, x, y) ? SPARSE_STATUS_SUCCESS : SPARSE_STATUS_EXECUTION_FAILED;
}

sparse_status_t mkl_sparse_destroy(sparse_matrix_t A) {
    if (!A) return SPARSE_STATUS_NOT_INITIALIZED;
    delete A->plan;
    delete A;
    return SPARSE_STATUS_SUCCESS;
}

}  // extern "C"
