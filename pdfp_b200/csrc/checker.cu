// checker.cu -- the pump's constraint check on the device.
//
// max_violation(milp, x) (src/milp.jl:102-114) runs once or twice per pump
// iteration on the full constraint matrix; on the host that is a sparse
// product over every nonzero.  A checker keeps the ORIGINAL (unscaled,
// unpermuted) constraints on the device and evaluates the same quantity:
// each row's activity summed sequentially over its nonzeros in ascending
// column order with separately rounded products and sums -- the order of
// Julia's CSC `A * x` and of a CSR matvec -- so the result is bit-identical to
// the host's; the maximum over rows is order-free.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>

#include "../../include/pdfp_b200.h"
#include "device.hpp"

namespace pdfp {
namespace {

__device__ __forceinline__ unsigned long long max_bits(double v) {
    return static_cast<unsigned long long>(__double_as_longlong(v));
}

// One thread per row (grid-stride); v starts at 0 and takes d (<= rows) or |d|
// (= rows) when larger, as the reference's loop does (a NaN never compares larger).
__global__ void __launch_bounds__(256) max_violation_kernel(int32_t m, const int32_t* __restrict__ rp,
                                                           const int32_t* __restrict__ ci,
                                                           const double* __restrict__ val,
                                                           const double* __restrict__ b,
                                                           const uint8_t* __restrict__ is_eq,
                                                           const double* __restrict__ x,
                                                           unsigned long long* out) {
    __shared__ double red[8];
    double v = 0.0;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) s = __dadd_rn(s, __dmul_rn(val[k], x[ci[k]]));
        const double d = __dsub_rn(s, b[i]);
        const double e = is_eq[i] ? fabs(d) : d;
        if (e > v) v = e;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_xor_sync(0xffffffffu, v, o);
        if (w > v) v = w;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
            if (red[w] > t) t = red[w];
        // non-negative doubles order like their bit patterns
        atomicMax(out, max_bits(t));
    }
}

}  // namespace

struct Checker {
    int32_t m = 0, n = 0;
    int64_t nnz = 0;
    int sms = 0;
    DeviceArena ar;
    int32_t *rp = nullptr, *ci = nullptr;
    double *val = nullptr, *b = nullptr, *x = nullptr;
    uint8_t* is_eq = nullptr;
    unsigned long long* out = nullptr;
    unsigned long long* out_h = nullptr;
    cudaStream_t stream = nullptr;
    ~Checker() {
        if (out_h) cudaFreeHost(out_h);
        if (stream) cudaStreamDestroy(stream);
    }
};

Checker* checker_create(const pdfp_csr& A, const double* b, const uint8_t* is_eq) {
    if (A.m < 0 || A.n < 0) throw Error(E_INVALID, "negative dimension");
    if (A.m > 0 && (!A.row_ptr || !b || !is_eq)) throw Error(E_INVALID, "null constraint data");
    const int64_t nnz = A.m > 0 ? A.row_ptr[A.m] : 0;
    if (nnz > 0 && (!A.col_idx || !A.val)) throw Error(E_INVALID, "null col_idx or val");
    if (A.m > 0 && A.row_ptr[0] != 0) throw Error(E_INVALID, "row_ptr[0] must be 0");
    for (int32_t i = 0; i < A.m; ++i)
        if (A.row_ptr[i + 1] < A.row_ptr[i]) throw Error(E_INVALID, "row_ptr must not decrease");
    for (int64_t k = 0; k < nnz; ++k)
        if (A.col_idx[k] < 0 || A.col_idx[k] >= A.n) throw Error(E_INVALID, "column index out of range");
    std::unique_ptr<Checker> c(new Checker());
    c->m = A.m;
    c->n = A.n;
    c->nnz = nnz;
    int dev = 0;
    PDFP_CK(cudaGetDevice(&dev));
    PDFP_CK(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, dev));
    PDFP_CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->rp = c->ar.alloc<int32_t>((size_t)A.m + 1);
    c->ci = c->ar.alloc<int32_t>((size_t)(nnz > 0 ? nnz : 1));
    c->val = c->ar.alloc<double>((size_t)(nnz > 0 ? nnz : 1));
    c->b = c->ar.alloc<double>((size_t)(A.m > 0 ? A.m : 1));
    c->is_eq = c->ar.alloc<uint8_t>((size_t)(A.m > 0 ? A.m : 1));
    c->x = c->ar.alloc<double>((size_t)(A.n > 0 ? A.n : 1));
    c->out = c->ar.alloc<unsigned long long>(1);
    if (A.m > 0) {
        PDFP_CK(cudaMemcpy(c->rp, A.row_ptr, sizeof(int32_t) * (A.m + 1), cudaMemcpyHostToDevice));
        PDFP_CK(cudaMemcpy(c->b, b, sizeof(double) * A.m, cudaMemcpyHostToDevice));
        PDFP_CK(cudaMemcpy(c->is_eq, is_eq, A.m, cudaMemcpyHostToDevice));
    }
    if (nnz > 0) {
        PDFP_CK(cudaMemcpy(c->ci, A.col_idx, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice));
        PDFP_CK(cudaMemcpy(c->val, A.val, sizeof(double) * nnz, cudaMemcpyHostToDevice));
    }
    PDFP_CK(cudaMallocHost(&c->out_h, sizeof(unsigned long long)));
    return c.release();
}

double checker_max_violation(Checker& c, const double* x) {
    if (c.m == 0) return 0.0;
    if (c.n > 0 && !x) throw Error(E_INVALID, "null x");
    if (c.n > 0)
        PDFP_CK(cudaMemcpyAsync(c.x, x, sizeof(double) * c.n, cudaMemcpyHostToDevice, c.stream));
    PDFP_CK(cudaMemsetAsync(c.out, 0, sizeof(unsigned long long), c.stream));
    int blocks = (c.m + 255) / 256;
    if (blocks > 8 * c.sms) blocks = 8 * c.sms;
    max_violation_kernel<<<blocks, 256, 0, c.stream>>>(c.m, c.rp, c.ci, c.val, c.b, c.is_eq, c.x, c.out);
    PDFP_CK(cudaGetLastError());
    PDFP_CK(cudaMemcpyAsync(c.out_h, c.out, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c.stream));
    PDFP_CK(cudaStreamSynchronize(c.stream));
    double v = 0.0;
    std::memcpy(&v, c.out_h, sizeof(double));
    return v;
}

void checker_destroy(Checker* c) { delete c; }

}  // namespace pdfp
