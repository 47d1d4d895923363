// common.cuh -- device helpers shared by every kernel of libpdfp_b200.
//
// * Julia scalar semantics (Base.clamp/max/min on Float64) so that the FP64
//   form evaluates the reference's expressions (src/pdfp.jl:119-156) exactly.
// * Inline-PTX wrappers for the sm_100a bulk-copy pipeline: mbarrier
//   init/expect_tx/try_wait and cp.async.bulk (global -> shared, no multicast).
// * Bounded waits: every spin in this library gives up after a fixed number of
//   tries, records PDFP_DEV_ERR_TIMEOUT in the device error word and returns.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#ifndef PDFP_WAIT_LIMIT
#define PDFP_WAIT_LIMIT (1u << 24)  // try_wait polls before a wait is declared hung
#endif

namespace pdfp {

enum : int32_t { DEV_ERR_NONE = 0, DEV_ERR_TIMEOUT = 1 };

// ---- Julia scalar semantics --------------------------------------------------
template <typename T>
__device__ __forceinline__ T jl_clamp(T x, T lo, T hi) {  // Base.clamp
    return x > hi ? hi : (x < lo ? lo : x);
}
template <typename T>
__device__ __forceinline__ T jl_max(T x, T y) {  // Base.max: NaN wins, -0.0 < 0.0
    bool take_y = (y > x) || (signbit(y) < signbit(x));
    return take_y ? (isnan(x) ? x : y) : (isnan(y) ? y : x);
}
template <typename T>
__device__ __forceinline__ T jl_min(T x, T y) {  // Base.min
    bool take_y = (y < x) || (signbit(y) > signbit(x));
    return take_y ? (isnan(x) ? x : y) : (isnan(y) ? y : x);
}

// Round-to-nearest arithmetic without FMA contraction, so that the FP64 form
// rounds every product and sum as Julia does.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }

// ---- shared-memory async copies (sm_90+ bulk copy engine) ------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
// 1-D bulk copy global -> shared (no multicast); dst, src 16-byte aligned,
// bytes a positive multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes,
                                              uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait on an mbarrier phase.  Returns false (and records the timeout
// in *err) if the phase did not complete within PDFP_WAIT_LIMIT polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int32_t* err) {
    for (uint32_t i = 0; i < PDFP_WAIT_LIMIT; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicExch(err, DEV_ERR_TIMEOUT);
    return false;
}

// Streaming loads that should not displace the gathered vectors from L2.
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const double* p) { return __ldcs(p); }

// ---- block reductions (fixed order: deterministic for a fixed block size) ----
template <int NT, int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* scratch /* K*NT/32 */) {
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int NW = NT / 32;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) scratch[k * NW + warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double t = lane < NW ? scratch[k * NW + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            v[k] = t;
        }
    }
    __syncthreads();
}

}  // namespace pdfp
