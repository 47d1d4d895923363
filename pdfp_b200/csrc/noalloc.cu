// noalloc.cu -- ||A||_2 by power iteration with no device allocation.
//
// pdfp_estimate_max_singular_value (precond.cu) uploads the matrix and
// allocates its vectors on every call.  This variant works on matrices the
// caller already holds on the device and keeps its three work vectors in a
// fixed-size array of this library's own device memory, so it never calls
// cudaMalloc or cudaFree.  That matters to callers whose device memory is
// already owned by a framework allocator (a process that reserved most of
// HBM up front, where a fresh cudaMalloc fails or fragments the pool), and to
// callers sharing the GPU with latency-sensitive streams, where the device-wide
// synchronisation of cudaFree would stall them.
//
// The scratch array (kNoAllocDoubles FP64 values, 8 MiB) is a file-scope
// __device__ variable.  Under CUDA's lazy module loading (the default) the
// driver commits it on a device when this file's module is first used there --
// the first call of the entry point on that device -- or when the library is
// loaded if CUDA_MODULE_LOADING=EAGER; from then on the device holds it until
// the process exits.  A caller whose allocator reserves device memory up front
// should therefore make one call per device before that reservation, and
// before any stream capture.  Host code cannot use the array's name as a
// device address: the entry point resolves the address with
// cudaGetSymbolAddress, with the caller's device current, once per CUDA
// context (keyed by the context's unique id, so a context created after
// cudaDeviceReset, or a non-primary context, resolves its own address).  All
// calls share the array and it keeps the last call's contents: every call
// overwrites what it reads before reading it, and calls that overlap on the
// GPU race on it.
//
// Cost: the whole iteration runs in one 1024-thread block (one SM), reading A
// and A' once per iteration; at the scratch limit (2m + n + 2 = 2^20 values,
// e.g. 349k rows x 349k columns) with a few million nonzeros an iteration
// takes on the order of a millisecond, so the 5000-iteration cap of the
// reference's default costs seconds there.  It is meant for small and
// mid-sized matrices.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <map>
#include <mutex>
#include <string>

#include "../../include/pdfp_b200.h"
#include "common.cuh"
#include "device.hpp"

namespace pdfp {

constexpr int64_t kNoAllocDoubles = int64_t(1) << 20;  // 8 MiB per device: 2m + n + 2 values
constexpr int kNoAllocThreads = 1024;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// The driver's current-context query, reached through the runtime so that the
// library links no driver library of its own.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

static std::mutex g_noalloc_mu;
static std::map<unsigned long long, double*> g_noalloc_addr;  // context id -> scratch address

// Unique id of the calling thread's current CUDA context (0 when none is current).
static unsigned long long current_context_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!get_current || !get_id) {
        void* f1 = nullptr;
        void* f2 = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1) !=
                cudaSuccess || q1 != cudaDriverEntryPointSuccess || !f1 ||
            cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2) !=
                cudaSuccess || q2 != cudaDriverEntryPointSuccess || !f2)
            throw Error(E_CUDA, "the driver's context queries are unavailable");
        get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
        get_id = reinterpret_cast<CtxGetIdFn>(f2);
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    unsigned long long id = 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) throw Error(E_CUDA, "cuCtxGetId failed");
    return id;
}

// Device address of the scratch array in the current context: resolved with
// cudaGetSymbolAddress (with the caller's device current) the first time a
// context calls, then taken from the cache.
static double* noalloc_scratch_address() {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    unsigned long long id = current_context_id();
    if (id != 0) {
        auto it = g_noalloc_addr.find(id);
        if (it != g_noalloc_addr.end()) return it->second;
    }
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // binds a context if none is current
    if (e != cudaSuccess || !p)
        throw Error(E_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    id = current_context_id();
    if (id != 0) g_noalloc_addr[id] = static_cast<double*>(p);
    return static_cast<double*>(p);
}

__device__ __forceinline__ uint64_t splitmix64_at(uint64_t seed, uint64_t k) {
    // the k-th output (k >= 1) of the SplitMix64 stream started at `seed`
    uint64_t z = seed + k * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Sum over the whole (kNoAllocThreads) block; every thread gets the total.
__device__ __forceinline__ double block_total(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = lane < kNoAllocThreads / 32 ? red[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    return t;
}

// estimate_max_singular_value (src/preconditioner.jl:108-125) in one block:
// the same start vector, products summed per row in ascending storage order.
// out = scratch + 2m + n: {sigma^2, iterations}.
__global__ void __launch_bounds__(kNoAllocThreads)
    power_noalloc_kernel(int32_t m, int32_t n, const int32_t* __restrict__ rp,
                         const int32_t* __restrict__ ci, const double* __restrict__ v,
                         const int32_t* __restrict__ rpt, const int32_t* __restrict__ cit,
                         const double* __restrict__ vt, int32_t max_it, double tol,
                         double* __restrict__ scratch) {
    __shared__ double red[kNoAllocThreads / 32];
    double* eig = scratch;
    double* nxt = scratch + m;
    double* dual = scratch + 2 * (int64_t)m;
    double* out = scratch + 2 * (int64_t)m + n;
    const double two_pi = 6.283185307179586;
    for (int32_t i = threadIdx.x; i < m; i += kNoAllocThreads) {
        const double u1 = (static_cast<double>(splitmix64_at(20240517ull, 2 * (uint64_t)i + 1) >> 11) + 0.5) * 0x1.0p-53;
        const double u2 = (static_cast<double>(splitmix64_at(20240517ull, 2 * (uint64_t)i + 2) >> 11) + 0.5) * 0x1.0p-53;
        eig[i] = sqrt(-2.0 * log(u1)) * cos(two_pi * u2);
    }
    __syncthreads();
    double sigma_sq = 1.0;
    int32_t it = 0;
    while (it < max_it) {
        ++it;
        double s = 0.0;
        for (int32_t i = threadIdx.x; i < m; i += kNoAllocThreads) s += eig[i] * eig[i];
        const double nrm = sqrt(block_total(s, red));
        if (nrm == 0.0) break;
        for (int32_t i = threadIdx.x; i < m; i += kNoAllocThreads) nxt[i] = eig[i] / nrm;
        __syncthreads();
        for (int32_t j = threadIdx.x; j < n; j += kNoAllocThreads) {
            double acc = 0.0;
            for (int32_t q = rpt[j]; q < rpt[j + 1]; ++q) acc = __dadd_rn(acc, __dmul_rn(vt[q], nxt[cit[q]]));
            dual[j] = acc;
        }
        __syncthreads();
        double d = 0.0;
        for (int32_t i = threadIdx.x; i < m; i += kNoAllocThreads) {
            double acc = 0.0;
            for (int32_t q = rp[i]; q < rp[i + 1]; ++q) acc = __dadd_rn(acc, __dmul_rn(v[q], dual[ci[q]]));
            eig[i] = acc;
            d += nxt[i] * acc;
        }
        sigma_sq = block_total(d, red);
        double r = 0.0;
        for (int32_t i = threadIdx.x; i < m; i += kNoAllocThreads) {
            const double e = __dsub_rn(eig[i], __dmul_rn(sigma_sq, nxt[i]));
            nxt[i] = e;
            r += e * e;
        }
        if (sqrt(block_total(r, red)) < tol) break;
    }
    if (threadIdx.x == 0) {
        out[0] = sigma_sq;
        out[1] = static_cast<double>(it);
    }
}

}  // namespace pdfp

extern "C" int pdfp_estimate_max_singular_value_noalloc(
    int32_t m, int32_t n, const int32_t* row_ptr, const int32_t* col_idx, const double* val,
    const int32_t* row_ptr_t, const int32_t* col_idx_t, const double* val_t,
    int32_t max_iterations, double tolerance, void* stream, double* sigma, int32_t* iterations) {
    try {
        pdfp::set_last_error("");
        if (m < 0 || n < 0) throw pdfp::Error(PDFP_E_INVALID, "negative dimension");
        const int64_t need = 2 * static_cast<int64_t>(m) + n + 2;
        if (need > pdfp::kNoAllocDoubles)
            throw pdfp::Error(PDFP_E_UNSUPPORTED,
                              "no-allocation power iteration needs 2m + n + 2 = " + std::to_string(need) +
                                  " FP64 scratch values; its fixed scratch holds " +
                                  std::to_string(pdfp::kNoAllocDoubles) + " (8 MiB)");
        if (!sigma) throw pdfp::Error(PDFP_E_INVALID, "null output");
        // the nonzero count lives on the device: any row (column) may hold some
        if ((m > 0 && (!row_ptr || !col_idx || !val)) || (n > 0 && (!row_ptr_t || !col_idx_t || !val_t)))
            throw pdfp::Error(PDFP_E_INVALID, "null matrix array (row pointers, column indices or values)");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
            throw pdfp::Error(PDFP_E_NODEVICE, "no CUDA device available");
        double* scratch = pdfp::noalloc_scratch_address();
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        pdfp::power_noalloc_kernel<<<1, pdfp::kNoAllocThreads, 0, s>>>(
            m, n, row_ptr, col_idx, val, row_ptr_t, col_idx_t, val_t, max_iterations, tolerance, scratch);
        PDFP_CK(cudaGetLastError());
        double out[2] = {0.0, 0.0};
        PDFP_CK(cudaMemcpyAsync(out, scratch + 2 * static_cast<int64_t>(m) + n, sizeof(out),
                                cudaMemcpyDeviceToHost, s));
        PDFP_CK(cudaStreamSynchronize(s));
        const double s2 = out[0];
        *sigma = std::isnan(s2) ? s2 : std::sqrt(s2 > 0.0 ? s2 : 0.0);
        if (iterations) *iterations = static_cast<int32_t>(out[1]);
        return PDFP_OK;
    } catch (const pdfp::Error& e) {
        pdfp::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        pdfp::set_last_error(e.what());
        return PDFP_E_INVALID;
    }
}
