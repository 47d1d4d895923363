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

#ifndef PDFP_WAIT_LIMIT_NS
#define PDFP_WAIT_LIMIT_NS 4000000000ull  // a device wait longer than 4 s is declared hung
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
// The same with an L2 cache-eviction policy (createpolicy) for the source lines.
__device__ __forceinline__ void bulk_copy_g2s_hint(void* dst, const void* src, uint32_t bytes,
                                                   uint64_t* bar, uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1], %2, [%3], %4;" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
        : "memory");
}
// L2 policy: lines fetched under it are the first to be evicted (data read once).
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
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
// try_wait with a suspend-time hint: a waiting thread sleeps (up to `ns`)
// instead of spinning.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, uint32_t parity, uint32_t ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(ns)
        : "memory");
    return ok != 0;
}
// Non-blocking test of a phase (acquire on success).
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
// ---- per-thread async copies (cp.async, global -> shared, no registers held) ----
// One 4-byte copy, cached in L1 on the way.
__device__ __forceinline__ void cp_async_4(uint32_t dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}
// Arrive on `bar` once every cp.async this thread issued before has landed; the
// arrival counts toward the barrier's expected count (.noinc).
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t* bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}
// Block until every cp.async this thread issued has landed (before the thread exits).
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// ---- programmatic dependent launch ------------------------------------------
// Wait until the grids this one depends on have completed and their writes are
// visible (returns at once for a grid launched without the programmatic attribute).
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// Let the dependent grid be scheduled once every block of this grid has done so
// (or exited).
__device__ __forceinline__ void griddep_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
// Named barrier among the first `nthreads` threads of the block (id 1..15).
__device__ __forceinline__ void named_sync(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait on an mbarrier phase.  Returns false (and records the timeout
// in *err) if the phase did not complete within limit_ns (PDFP_WAIT_LIMIT_NS;
// the self-test passes a shorter one).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int32_t* err,
                                                  uint64_t limit_ns = PDFP_WAIT_LIMIT_NS) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    while (!mbar_try_wait_sleep(bar, parity, 20000u)) {
        if (globaltimer_ns() - t0 > limit_ns) {
            if (err) atomicExch(err, DEV_ERR_TIMEOUT);
            return false;
        }
    }
    return true;
}

// A group of `nthreads` threads (named barrier `id`) waits for a phase: one
// elected thread sleeps on the barrier, the group meets at the named barrier,
// then every thread takes its own acquire with a non-blocking test (already
// complete, so it passes at once).  Returns false if the wait gave up.
__device__ __forceinline__ bool group_wait(uint64_t* bar, uint32_t parity, int32_t* err,
                                           bool elected, int id, int nthreads, int32_t* flag,
                                           uint64_t limit_ns = PDFP_WAIT_LIMIT_NS) {
    if (elected && !mbar_wait_bounded(bar, parity, err, limit_ns)) *flag = 1;
    named_sync(id, nthreads);
    if (*flag) return false;
    if (!mbar_test_wait(bar, parity)) return mbar_wait_bounded(bar, parity, err, limit_ns);
    return true;
}

// Streaming loads that should not displace the gathered vectors from L2.
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const double* p) { return __ldcs(p); }

// ---- block reductions (fixed order: deterministic for a fixed block size) ----
// Sum over the first NT threads; BAR = 0 uses __syncthreads, otherwise the
// named barrier BAR among those NT threads.
template <int NT, int K, int BAR = 0>
__device__ __forceinline__ void block_sum(double (&v)[K], double* scratch /* K*NT/32 */,
                                          int tid /* index within the NT threads */) {
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    const int warp = tid >> 5, lane = tid & 31;
    constexpr int NW = NT / 32;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) scratch[k * NW + warp] = v[k];
    if (BAR) named_sync(BAR, NT); else __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double t = lane < NW ? scratch[k * NW + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            v[k] = t;
        }
    }
    if (BAR) named_sync(BAR, NT); else __syncthreads();
}

}  // namespace pdfp
