// gatherprobe.cu -- the random-gather ceiling of the GPU, measured
// (libpdfp_bench.so: benchmark and test support, not part of the solver library).
//
// The step kernels of a matrix with scattered column indices are bound by the
// rate at which the SMs can serve independent 4-byte loads from an L2-resident
// vector (each costs a 32-byte sector and an uncoalesced L1 request), not by
// HBM bandwidth.  pdfp_measure_gather_rate measures that ceiling with the
// simplest kernel that reaches it: streamed, coalesced 128-bit loads of
// indices and values, four independent gathers per load, a sum per thread --
// no row structure, no shared memory.  The benchmark reports the step kernel's
// gathers per second against this number beside the HBM roofline.
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "../../include/pdfp_bench.h"

namespace pdfp {
namespace {

__global__ void probe_init_kernel(int32_t* idx, float* val, int64_t nnz, int32_t m, float* vec) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += stride) {
        uint64_t h = (uint64_t)k * 0x9E3779B97F4A7C15ull;  // SplitMix64 finaliser
        h ^= h >> 31;
        h *= 0xBF58476D1CE4E5B9ull;
        h ^= h >> 27;
        idx[k] = (int32_t)(h % (uint64_t)m);
        val[k] = (float)((h >> 40) & 1023u) * (1.0f / 1024.0f) - 0.5f;
        if (k < m) vec[k] = (float)(k % 97) * 0.01f;
    }
}

template <int U>
__global__ void probe_gather_kernel(const int4* __restrict__ idx, const float4* __restrict__ val,
                                    const float* __restrict__ vec, int64_t quads, float* out) {
    float acc = 0.f;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q0 < quads; q0 += U * stride) {
        int4 c[U];
        float4 a[U];
        float g[U][4];
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (q0 + u * stride < quads) {
                c[u] = __ldcs(idx + q0 + u * stride);
                a[u] = __ldcs(val + q0 + u * stride);
            }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (q0 + u * stride < quads) {
                g[u][0] = vec[c[u].x];
                g[u][1] = vec[c[u].y];
                g[u][2] = vec[c[u].z];
                g[u][3] = vec[c[u].w];
            }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (q0 + u * stride < quads)
                acc += a[u].x * g[u][0] + a[u].y * g[u][1] + a[u].z * g[u][2] + a[u].w * g[u][3];
    }
    out[blockIdx.x * (int64_t)blockDim.x + threadIdx.x] = acc;
}

}  // namespace

thread_local std::string g_bench_err;

struct BenchError : std::runtime_error {
    int code;
    BenchError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define PB_CK(expr)                                                                          \
    do {                                                                                     \
        cudaError_t e_ = (expr);                                                             \
        if (e_ != cudaSuccess)                                                               \
            throw BenchError(e_ == cudaErrorMemoryAllocation ? PDFP_E_NOMEM : PDFP_E_CUDA,   \
                             std::string(#expr) + ": " + cudaGetErrorString(e_));            \
    } while (0)

// Device buffers of one measurement, freed on every exit path.
struct Buffers {
    void* p[4] = {nullptr, nullptr, nullptr, nullptr};
    ~Buffers() {
        for (void* q : p)
            if (q) cudaFree(q);
    }
};

// Gathers per second (best over a few launch shapes) of `nnz` random 4-byte
// gathers from an m-entry FP32 vector.
double measure_gather_rate(int64_t nnz, int32_t m, int32_t repeats) {
    if (nnz < 4 || nnz % 4 != 0 || nnz > (int64_t(1) << 31) - 4 || m < 1 || repeats < 1)
        throw BenchError(PDFP_E_INVALID, "pdfp_measure_gather_rate: need nnz a positive multiple of 4 "
                                         "below 2^31, m >= 1, repeats >= 1");
    int dev = 0, sms = 0;
    PB_CK(cudaGetDevice(&dev));
    PB_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    Buffers b;
    PB_CK(cudaMalloc(&b.p[0], sizeof(int32_t) * (size_t)nnz));
    PB_CK(cudaMalloc(&b.p[1], sizeof(float) * (size_t)nnz));
    PB_CK(cudaMalloc(&b.p[2], sizeof(float) * (size_t)m));
    PB_CK(cudaMalloc(&b.p[3], sizeof(float) * (size_t)sms * 2048));
    int32_t* idx = static_cast<int32_t*>(b.p[0]);
    float* val = static_cast<float*>(b.p[1]);
    float* vec = static_cast<float*>(b.p[2]);
    float* out = static_cast<float*>(b.p[3]);
    // one pass fills the indices, the values and the first min(nnz, m) vector entries
    PB_CK(cudaMemset(vec, 0, sizeof(float) * (size_t)m));
    probe_init_kernel<<<sms * 8, 256>>>(idx, val, nnz, m, vec);
    PB_CK(cudaGetLastError());
    PB_CK(cudaDeviceSynchronize());
    cudaEvent_t e0, e1;
    PB_CK(cudaEventCreate(&e0));
    PB_CK(cudaEventCreate(&e1));
    const int64_t quads = nnz / 4;
    double best = 0.0;
    const int shapes[][2] = {{256, 2}, {256, 4}, {512, 2}};  // threads, blocks per SM (<= 2048 per SM)
    try {
        for (const auto& sh : shapes) {
            const int threads = sh[0], blocks = sh[1] * sms;
            auto run = [&] {
                probe_gather_kernel<2><<<blocks, threads>>>(reinterpret_cast<const int4*>(idx),
                                                            reinterpret_cast<const float4*>(val), vec,
                                                            quads, out);
            };
            run();
            run();
            PB_CK(cudaGetLastError());
            PB_CK(cudaEventRecord(e0));
            for (int r = 0; r < repeats; ++r) run();
            PB_CK(cudaEventRecord(e1));
            PB_CK(cudaEventSynchronize(e1));
            PB_CK(cudaGetLastError());
            float ms = 0.f;
            PB_CK(cudaEventElapsedTime(&ms, e0, e1));
            const double rate = (double)nnz * repeats / (ms * 1e-3);
            if (rate > best) best = rate;
        }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

}  // namespace pdfp

extern "C" {

PDFP_API const char* pdfp_bench_last_error(void) { return pdfp::g_bench_err.c_str(); }

PDFP_API int pdfp_measure_gather_rate(int64_t nnz, int32_t m, int32_t repeats, double* gathers_per_s) {
    try {
        pdfp::g_bench_err.clear();
        if (!gathers_per_s) throw pdfp::BenchError(PDFP_E_INVALID, "pdfp_measure_gather_rate: null output");
        int n = 0;
        if (nnz >= 4 && nnz % 4 == 0 && m >= 1 && repeats >= 1 &&
            (cudaGetDeviceCount(&n) != cudaSuccess || n == 0))
            throw pdfp::BenchError(PDFP_E_NODEVICE, "no CUDA device available");
        *gathers_per_s = pdfp::measure_gather_rate(nnz, m, repeats);
        return PDFP_OK;
    } catch (const pdfp::BenchError& e) {
        pdfp::g_bench_err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        pdfp::g_bench_err = e.what();
        return PDFP_E_INVALID;
    }
}

}  // extern "C"
