// refform.cu -- the reference's GPU step as written, for comparison only.
//
// The plain FP64 GPU form of the projector step, structured as the reference
// runs it on a CuVector state (src/pdfp_kernels.jl:4-86, src/pdfp.jl:158-163):
// per PDHG step five launches --
//   cuSPARSE SpMV  Atz = A' z          (mul!(s.Atz, s.A_t, s.current_z))
//   primal kernel  (_pdfp_primal_kernel!, 256 threads per block)
//   dual_y kernel  (_pdfp_dual_y_kernel!)
//   cuSPARSE SpMV  Ax  = A x_reflected (mul!(s.Ax, s.A, s.reflected_x))
//   dual_z kernel  (_pdfp_dual_z_kernel!)
// -- on FP64 CSR copies of A and A' with int32 indices (src/pdlp.jl:79-80).
// Descriptors and the SpMV work buffer are made once (CUDA.jl makes them per
// call), and no evaluation runs between steps, so the form timed here is, if
// anything, faster than the reference's.  Built as its own library,
// libpdfp_refform.so; the projector library does not use it.
#include <cuda_runtime.h>
#include <cusparse.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pdfp_refform.h"

namespace {

thread_local std::string g_err;

struct Fail {
    std::string msg;
};

#define RF_CUDA(x)                                                                          \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess) throw Fail{std::string(#x) + ": " + cudaGetErrorString(e_)}; \
    } while (0)
#define RF_SP(x)                                                            \
    do {                                                                    \
        cusparseStatus_t e_ = (x);                                          \
        if (e_ != CUSPARSE_STATUS_SUCCESS)                                  \
            throw Fail{std::string(#x) + ": " + cusparseGetErrorString(e_)}; \
    } while (0)

__global__ void primal_kernel(double* pdhg_x, double* dual_slack, double* reflected_x,
                              double* current_x, const double* initial_x, const double* current_y,
                              const double* Atz, const double* var_lb, const double* var_ub,
                              double tau, double weight, double omega, double omw, double omwt,
                              int32_t n) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double cx = current_x[i];
    const double temp = cx - tau * (Atz[i] - current_y[i]);
    const double pdhg = fmin(fmax(temp, var_lb[i]), var_ub[i]);
    pdhg_x[i] = pdhg;
    dual_slack[i] = (pdhg - temp) / tau;
    const double refl = 2.0 * pdhg - cx;
    reflected_x[i] = refl;
    current_x[i] = weight * (omega * refl + omw * cx) + omwt * initial_x[i];
}

__global__ void dual_y_kernel(double* pdhg_y, double* current_y, double* reflected_y,
                              const double* initial_y, const double* x_tilde,
                              const double* reflected_x, const uint8_t* is_int, const double* w,
                              double sigma, double weight, double omega, double omw, double omwt,
                              int32_t n) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double cy = current_y[i];
    const double wi = w[i];
    const double y =
        is_int[i] ? fmin(fmax(cy + sigma * (x_tilde[i] - reflected_x[i]), -wi), wi) : 0.0;
    pdhg_y[i] = y;
    const double refl = 2.0 * y - cy;
    reflected_y[i] = refl;
    current_y[i] = weight * (omega * refl + omw * cy) + omwt * initial_y[i];
}

__global__ void dual_z_kernel(double* pdhg_z, double* current_z, double* reflected_z,
                              const double* initial_z, const double* Ax, const double* b,
                              const uint8_t* is_eq, double sigma, double weight, double omega,
                              double omw, double omwt, int32_t m) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const double cz = current_z[i];
    const double raw = cz + sigma * (Ax[i] - b[i]);
    const double z = is_eq[i] ? raw : fmax(raw, 0.0);
    pdhg_z[i] = z;
    const double refl = 2.0 * z - cz;
    reflected_z[i] = refl;
    current_z[i] = weight * (omega * refl + omw * cz) + omwt * initial_z[i];
}

// Vectors of the state, named as in src/pdfp.jl:15-52.
enum Vec {
    X_TILDE, W, VAR_LB, VAR_UB, INITIAL_X, CURRENT_X, PDHG_X, REFLECTED_X, INITIAL_Y, CURRENT_Y,
    PDHG_Y, REFLECTED_Y, ATZ, DUAL_SLACK, N_VECS_N
};
enum VecM { B, INITIAL_Z, CURRENT_Z, PDHG_Z, REFLECTED_Z, AX, N_VECS_M };

struct RefForm {
    int32_t m = 0, n = 0;
    int64_t nnz = 0;
    cudaStream_t stream = nullptr;
    cusparseHandle_t sp = nullptr;
    int32_t *rp = nullptr, *ci = nullptr, *rp_t = nullptr, *ci_t = nullptr;
    double *v = nullptr, *v_t = nullptr;
    double* vn[N_VECS_N] = {};
    double* vm[N_VECS_M] = {};
    uint8_t *is_int = nullptr, *is_eq = nullptr;
    cusparseSpMatDescr_t A = nullptr, At = nullptr;
    cusparseDnVecDescr_t d_z = nullptr, d_atz = nullptr, d_rx = nullptr, d_ax = nullptr;
    void* buf = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;

    ~RefForm() {
        if (A) cusparseDestroySpMat(A);
        if (At) cusparseDestroySpMat(At);
        for (auto d : {d_z, d_atz, d_rx, d_ax})
            if (d) cusparseDestroyDnVec(d);
        if (sp) cusparseDestroy(sp);
        for (void* p : {(void*)rp, (void*)ci, (void*)rp_t, (void*)ci_t, (void*)v, (void*)v_t,
                        (void*)is_int, (void*)is_eq, buf})
            if (p) cudaFree(p);
        for (auto p : vn)
            if (p) cudaFree(p);
        for (auto p : vm)
            if (p) cudaFree(p);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (stream) cudaStreamDestroy(stream);
    }
};

template <class T>
T* upload(const T* h, size_t count) {
    T* d = nullptr;
    RF_CUDA(cudaMalloc(&d, sizeof(T) * (count ? count : 1)));
    if (count) RF_CUDA(cudaMemcpy(d, h, sizeof(T) * count, cudaMemcpyHostToDevice));
    return d;
}

// CSR of A' from the CSR of A (counting sort by column: rows stay ascending).
void transpose_csr(const pdfp_csr& A, std::vector<int32_t>& rp, std::vector<int32_t>& ci,
                   std::vector<double>& v) {
    const int64_t nnz = A.row_ptr[A.m];
    rp.assign((size_t)A.n + 1, 0);
    ci.resize((size_t)nnz);
    v.resize((size_t)nnz);
    for (int64_t k = 0; k < nnz; ++k) ++rp[(size_t)A.col_idx[k] + 1];
    for (int32_t j = 0; j < A.n; ++j) rp[j + 1] += rp[j];
    std::vector<int32_t> next(rp.begin(), rp.end() - 1);
    for (int32_t i = 0; i < A.m; ++i)
        for (int32_t k = A.row_ptr[i]; k < A.row_ptr[i + 1]; ++k) {
            const int32_t p = next[A.col_idx[k]]++;
            ci[p] = i;
            v[p] = A.val[k];
        }
}

int guard(const char* what, void (*fn)(void*), void* arg) {
    try {
        fn(arg);
        return PDFP_OK;
    } catch (const Fail& f) {
        g_err = std::string(what) + ": " + f.msg;
        return PDFP_E_CUDA;
    } catch (const std::bad_alloc&) {
        g_err = std::string(what) + ": out of host memory";
        return PDFP_E_NOMEM;
    }
}

}  // namespace

extern "C" {

PDFP_API const char* pdfp_refform_last_error(void) { return g_err.c_str(); }

PDFP_API int pdfp_refform_create(const pdfp_csr* A, const double* b, const uint8_t* is_eq,
                                 const uint8_t* is_int, const double* var_lb,
                                 const double* var_ub, const double* w, void** out) {
    if (!A || !b || !is_eq || !is_int || !var_lb || !var_ub || !w || !out || A->m < 1 ||
        A->n < 1 || !A->row_ptr || !A->col_idx || !A->val) {
        g_err = "pdfp_refform_create: null argument or empty matrix";
        return PDFP_E_INVALID;
    }
    const pdfp_csr& M = *A;
    if (M.row_ptr[0] != 0) {
        g_err = "pdfp_refform_create: row_ptr[0] must be 0";
        return PDFP_E_INVALID;
    }
    for (int32_t i = 0; i < M.m; ++i)
        if (M.row_ptr[i + 1] < M.row_ptr[i]) {
            g_err = "pdfp_refform_create: row_ptr must not decrease";
            return PDFP_E_INVALID;
        }
    for (int32_t k = 0; k < M.row_ptr[M.m]; ++k)
        if (M.col_idx[k] < 0 || M.col_idx[k] >= M.n) {
            g_err = "pdfp_refform_create: column index out of range";
            return PDFP_E_INVALID;
        }
    struct Args {
        const pdfp_csr* A;
        const double *b, *lb, *ub, *w;
        const uint8_t *is_eq, *is_int;
        RefForm* r;
    } a{A, b, var_lb, var_ub, w, is_eq, is_int, new RefForm()};
    const int rc = guard("pdfp_refform_create", [](void* p) {
        Args& a = *static_cast<Args*>(p);
        RefForm& r = *a.r;
        const pdfp_csr& M = *a.A;
        r.m = M.m;
        r.n = M.n;
        r.nnz = M.row_ptr[M.m];
        std::vector<int32_t> rpt, cit;
        std::vector<double> vt;
        transpose_csr(M, rpt, cit, vt);
        RF_CUDA(cudaStreamCreateWithFlags(&r.stream, cudaStreamNonBlocking));
        RF_SP(cusparseCreate(&r.sp));
        RF_SP(cusparseSetStream(r.sp, r.stream));
        r.rp = upload(M.row_ptr, (size_t)M.m + 1);
        r.ci = upload(M.col_idx, (size_t)r.nnz);
        r.v = upload(M.val, (size_t)r.nnz);
        r.rp_t = upload(rpt.data(), rpt.size());
        r.ci_t = upload(cit.data(), cit.size());
        r.v_t = upload(vt.data(), vt.size());
        std::vector<double> zn((size_t)r.n, 0.0), zm((size_t)r.m, 0.0);
        for (int k = 0; k < N_VECS_N; ++k) r.vn[k] = upload(zn.data(), zn.size());
        for (int k = 0; k < N_VECS_M; ++k) r.vm[k] = upload(zm.data(), zm.size());
        RF_CUDA(cudaMemcpy(r.vn[W], a.w, sizeof(double) * r.n, cudaMemcpyHostToDevice));
        RF_CUDA(cudaMemcpy(r.vn[VAR_LB], a.lb, sizeof(double) * r.n, cudaMemcpyHostToDevice));
        RF_CUDA(cudaMemcpy(r.vn[VAR_UB], a.ub, sizeof(double) * r.n, cudaMemcpyHostToDevice));
        RF_CUDA(cudaMemcpy(r.vm[B], a.b, sizeof(double) * r.m, cudaMemcpyHostToDevice));
        r.is_int = upload(a.is_int, (size_t)r.n);
        r.is_eq = upload(a.is_eq, (size_t)r.m);
        RF_SP(cusparseCreateCsr(&r.A, r.m, r.n, r.nnz, r.rp, r.ci, r.v, CUSPARSE_INDEX_32I,
                                CUSPARSE_INDEX_32I, CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F));
        RF_SP(cusparseCreateCsr(&r.At, r.n, r.m, r.nnz, r.rp_t, r.ci_t, r.v_t, CUSPARSE_INDEX_32I,
                                CUSPARSE_INDEX_32I, CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F));
        RF_SP(cusparseCreateDnVec(&r.d_z, r.m, r.vm[CURRENT_Z], CUDA_R_64F));
        RF_SP(cusparseCreateDnVec(&r.d_atz, r.n, r.vn[ATZ], CUDA_R_64F));
        RF_SP(cusparseCreateDnVec(&r.d_rx, r.n, r.vn[REFLECTED_X], CUDA_R_64F));
        RF_SP(cusparseCreateDnVec(&r.d_ax, r.m, r.vm[AX], CUDA_R_64F));
        const double one = 1.0, zero = 0.0;
        size_t b1 = 0, b2 = 0;
        RF_SP(cusparseSpMV_bufferSize(r.sp, CUSPARSE_OPERATION_NON_TRANSPOSE, &one, r.At, r.d_z,
                                      &zero, r.d_atz, CUDA_R_64F, CUSPARSE_SPMV_ALG_DEFAULT, &b1));
        RF_SP(cusparseSpMV_bufferSize(r.sp, CUSPARSE_OPERATION_NON_TRANSPOSE, &one, r.A, r.d_rx,
                                      &zero, r.d_ax, CUDA_R_64F, CUSPARSE_SPMV_ALG_DEFAULT, &b2));
        RF_CUDA(cudaMalloc(&r.buf, (b1 > b2 ? b1 : b2) + 256));
        RF_CUDA(cudaEventCreate(&r.e0));
        RF_CUDA(cudaEventCreate(&r.e1));
    }, &a);
    if (rc != PDFP_OK) {
        delete a.r;
        return rc;
    }
    *out = a.r;
    return PDFP_OK;
}

PDFP_API int pdfp_refform_reset(void* h, const double* x_tilde, const double* x0) {
    if (!h || !x_tilde || !x0) {
        g_err = "pdfp_refform_reset: null argument";
        return PDFP_E_INVALID;
    }
    struct Args {
        RefForm* r;
        const double *xt, *x0;
    } a{static_cast<RefForm*>(h), x_tilde, x0};
    return guard("pdfp_refform_reset", [](void* p) {
        Args& a = *static_cast<Args*>(p);
        RefForm& r = *a.r;
        const size_t bn = sizeof(double) * r.n, bm = sizeof(double) * r.m;
        RF_CUDA(cudaMemcpyAsync(r.vn[X_TILDE], a.xt, bn, cudaMemcpyHostToDevice, r.stream));
        RF_CUDA(cudaMemcpyAsync(r.vn[CURRENT_X], a.x0, bn, cudaMemcpyHostToDevice, r.stream));
        RF_CUDA(cudaMemcpyAsync(r.vn[INITIAL_X], a.x0, bn, cudaMemcpyHostToDevice, r.stream));
        for (int k : {INITIAL_Y, CURRENT_Y, PDHG_Y, REFLECTED_Y})
            RF_CUDA(cudaMemsetAsync(r.vn[k], 0, bn, r.stream));
        for (int k : {INITIAL_Z, CURRENT_Z, PDHG_Z, REFLECTED_Z})
            RF_CUDA(cudaMemsetAsync(r.vm[k], 0, bm, r.stream));
        RF_CUDA(cudaStreamSynchronize(r.stream));
    }, &a);
}

PDFP_API int pdfp_refform_steps(void* h, double step_size, double primal_weight, int32_t k0,
                                int32_t count, float* ms) {
    if (!h || count < 0 || !(step_size > 0.0) || !(primal_weight > 0.0)) {
        g_err = "pdfp_refform_steps: invalid argument";
        return PDFP_E_INVALID;
    }
    struct Args {
        RefForm* r;
        double eta, pw;
        int32_t k0, count;
        float* ms;
    } a{static_cast<RefForm*>(h), step_size, primal_weight, k0, count, ms};
    return guard("pdfp_refform_steps", [](void* p) {
        Args& a = *static_cast<Args*>(p);
        RefForm& r = *a.r;
        const double tau = a.eta / a.pw, sigma = a.eta * a.pw, omega = 1.0, omw = 0.0;
        const double one = 1.0, zero = 0.0;
        const int gn = (r.n + 255) / 256, gm = (r.m + 255) / 256;
        RF_CUDA(cudaEventRecord(r.e0, r.stream));
        for (int32_t t = 0; t < a.count; ++t) {
            const double k = (double)(a.k0 + t);
            const double weight = k / (k + 1.0), omwt = 1.0 - weight;
            RF_SP(cusparseSpMV(r.sp, CUSPARSE_OPERATION_NON_TRANSPOSE, &one, r.At, r.d_z, &zero,
                               r.d_atz, CUDA_R_64F, CUSPARSE_SPMV_ALG_DEFAULT, r.buf));
            primal_kernel<<<gn, 256, 0, r.stream>>>(
                r.vn[PDHG_X], r.vn[DUAL_SLACK], r.vn[REFLECTED_X], r.vn[CURRENT_X], r.vn[INITIAL_X],
                r.vn[CURRENT_Y], r.vn[ATZ], r.vn[VAR_LB], r.vn[VAR_UB], tau, weight, omega, omw,
                omwt, r.n);
            dual_y_kernel<<<gn, 256, 0, r.stream>>>(
                r.vn[PDHG_Y], r.vn[CURRENT_Y], r.vn[REFLECTED_Y], r.vn[INITIAL_Y], r.vn[X_TILDE],
                r.vn[REFLECTED_X], r.is_int, r.vn[W], sigma, weight, omega, omw, omwt, r.n);
            RF_SP(cusparseSpMV(r.sp, CUSPARSE_OPERATION_NON_TRANSPOSE, &one, r.A, r.d_rx, &zero,
                               r.d_ax, CUDA_R_64F, CUSPARSE_SPMV_ALG_DEFAULT, r.buf));
            dual_z_kernel<<<gm, 256, 0, r.stream>>>(
                r.vm[PDHG_Z], r.vm[CURRENT_Z], r.vm[REFLECTED_Z], r.vm[INITIAL_Z], r.vm[AX], r.vm[B],
                r.is_eq, sigma, weight, omega, omw, omwt, r.m);
            RF_CUDA(cudaGetLastError());
        }
        RF_CUDA(cudaEventRecord(r.e1, r.stream));
        RF_CUDA(cudaEventSynchronize(r.e1));
        float t = 0.f;
        RF_CUDA(cudaEventElapsedTime(&t, r.e0, r.e1));
        if (a.ms) *a.ms = t;
    }, &a);
}

PDFP_API int pdfp_refform_get(void* h, int32_t which, double* out) {
    if (!h || !out || which < 0 || which > 3) {
        g_err = "pdfp_refform_get: invalid argument";
        return PDFP_E_INVALID;
    }
    struct Args {
        RefForm* r;
        int32_t which;
        double* out;
    } a{static_cast<RefForm*>(h), which, out};
    return guard("pdfp_refform_get", [](void* p) {
        Args& a = *static_cast<Args*>(p);
        RefForm& r = *a.r;
        const double* src = a.which == 0   ? r.vn[PDHG_X]
                            : a.which == 1 ? r.vn[CURRENT_X]
                            : a.which == 2 ? r.vm[PDHG_Z]
                                           : r.vm[CURRENT_Z];
        const size_t len = a.which < 2 ? (size_t)r.n : (size_t)r.m;
        RF_CUDA(cudaMemcpyAsync(a.out, src, sizeof(double) * len, cudaMemcpyDeviceToHost, r.stream));
        RF_CUDA(cudaStreamSynchronize(r.stream));
    }, &a);
}

PDFP_API int pdfp_refform_destroy(void* h) {
    delete static_cast<RefForm*>(h);
    return PDFP_OK;
}

}  // extern "C"
