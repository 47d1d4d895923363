// gatherprobe.cu -- the random-gather ceiling of the GPU, measured.
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
#include <string>

#include "../../include/pdfp_b200.h"
#include "device.hpp"

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

// Gathers per second (best over a few launch shapes) of `nnz` random 4-byte
// gathers from an m-entry FP32 vector.
double measure_gather_rate(int64_t nnz, int32_t m, int32_t repeats) {
    if (nnz < 4 || nnz % 4 != 0 || nnz > (int64_t(1) << 31) - 4 || m < 1 || repeats < 1)
        throw Error(E_INVALID, "pdfp_measure_gather_rate: need nnz a positive multiple of 4 "
                               "below 2^31, m >= 1, repeats >= 1");
    int dev = 0, sms = 0;
    PDFP_CK(cudaGetDevice(&dev));
    PDFP_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    DeviceArena ar;
    int32_t* idx = ar.alloc<int32_t>((size_t)nnz);
    float* val = ar.alloc<float>((size_t)nnz);
    float* vec = ar.alloc<float>((size_t)m);
    float* out = ar.alloc<float>((size_t)sms * 2048);
    // one pass fills the indices, the values and the first min(nnz, m) vector entries
    probe_init_kernel<<<sms * 8, 256>>>(idx, val, nnz, m, vec);
    PDFP_CK(cudaGetLastError());
    PDFP_CK(cudaDeviceSynchronize());
    cudaEvent_t e0, e1;
    PDFP_CK(cudaEventCreate(&e0));
    PDFP_CK(cudaEventCreate(&e1));
    const int64_t quads = nnz / 4;
    double best = 0.0;
    const int shapes[][2] = {{256, 2}, {256, 4}, {512, 2}};  // threads, blocks per SM (<= 2048 per SM)
    for (const auto& sh : shapes) {
        const int threads = sh[0], blocks = sh[1] * sms;
        auto run = [&] {
            probe_gather_kernel<2><<<blocks, threads>>>(reinterpret_cast<const int4*>(idx),
                                                        reinterpret_cast<const float4*>(val), vec,
                                                        quads, out);
        };
        run();
        run();
        PDFP_CK(cudaGetLastError());
        PDFP_CK(cudaEventRecord(e0));
        for (int r = 0; r < repeats; ++r) run();
        PDFP_CK(cudaEventRecord(e1));
        PDFP_CK(cudaEventSynchronize(e1));
        PDFP_CK(cudaGetLastError());
        float ms = 0.f;
        PDFP_CK(cudaEventElapsedTime(&ms, e0, e1));
        const double rate = (double)nnz * repeats / (ms * 1e-3);
        if (rate > best) best = rate;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

}  // namespace pdfp
