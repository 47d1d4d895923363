// selftest.cu -- the library's bounded device waits, made to run out on purpose.
//
// Every spin of this library's kernels is bounded: the tile engine's mbarrier
// waits (mbar_wait_bounded / group_wait, common.cuh) and the cooperative
// window's grid barrier (grid_barrier, medium_steps.cuh) give up after their
// limit, record the timeout in a device error word and return, and the host
// turns that word into PDFP_E_TIMEOUT with the context still usable.  Nothing
// in a correct solve reaches those limits, so pdfp_selftest_bounded_wait runs
// the same wait functions in a small kernel whose wait cannot complete -- an
// mbarrier that expects one more arrival than it gets, or a grid barrier that
// expects one more block than were launched -- with a short limit.  No copy is
// in flight when a wait gives up, and nothing faults or traps.
#include <cuda_runtime.h>

#include <string>

#include "../../include/pdfp_b200.h"
#include "common.cuh"
#include "device.hpp"
#include "medium_steps.cuh"

namespace pdfp {
namespace {

constexpr int kSelfTestThreads = 64;

// The reducers' wait of the tile engine: thread 0 sleeps on a phase that never
// completes (two arrivals expected, one made), the group meets on a named barrier.
__global__ void __launch_bounds__(kSelfTestThreads) selftest_mbar_kernel(int32_t* err, uint64_t limit_ns) {
    __shared__ uint64_t bar;
    __shared__ int32_t flag;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 2);
        flag = 0;
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_arrive(&bar);
    group_wait(&bar, 0u, err, threadIdx.x == 0, 1, kSelfTestThreads, &flag, limit_ns);
}

// The cooperative window's grid barrier, expecting one block more than launched.
__global__ void __launch_bounds__(kSelfTestThreads) selftest_grid_kernel(GridBar g, int32_t* err,
                                                                           uint64_t limit_ns) {
    grid_barrier(g, err, gridDim.x + 1, limit_ns);
}

}  // namespace

// Runs one self-test; throws E_TIMEOUT when the wait gave up as designed.
void selftest_bounded_wait(int which, double limit_seconds) {
    if (which != 0 && which != 1) throw Error(E_INVALID, "self-test: which must be 0 or 1");
    if (!(limit_seconds > 0.0) || limit_seconds > 4.0)
        throw Error(E_INVALID, "self-test: limit_seconds must lie in (0, 4]");
    const uint64_t limit_ns = static_cast<uint64_t>(limit_seconds * 1e9);
    DeviceArena ar;
    int32_t* err = ar.alloc<int32_t>(1);
    unsigned* words = ar.alloc<unsigned>(4);  // count, generation, abort
    cudaStream_t s = nullptr;
    PDFP_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaError_t launched;
    if (which == 0) {
        selftest_mbar_kernel<<<1, kSelfTestThreads, 0, s>>>(err, limit_ns);
    } else {
        // two blocks of 64 threads are resident together on any GPU
        selftest_grid_kernel<<<2, kSelfTestThreads, 0, s>>>(GridBar{words, words + 1, words + 2}, err, limit_ns);
    }
    launched = cudaGetLastError();
    int32_t h_err = 0;
    cudaError_t done = launched == cudaSuccess ? cudaMemcpyAsync(&h_err, err, sizeof(h_err), cudaMemcpyDeviceToHost, s)
                                               : launched;
    if (done == cudaSuccess) done = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    PDFP_CK(done);
    if (h_err == DEV_ERR_NONE)
        throw Error(E_INVALID, "self-test: the wait completed although nothing could complete it");
    throw Error(E_TIMEOUT, std::string("a bounded device wait gave up (self-test: ") +
                               (which == 0 ? "mbarrier" : "grid barrier") + ")");
}

}  // namespace pdfp

extern "C" int pdfp_selftest_bounded_wait(int32_t which, double limit_seconds) {
    try {
        pdfp::set_last_error("");
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
            throw pdfp::Error(PDFP_E_NODEVICE, "no CUDA device available");
        pdfp::selftest_bounded_wait(which, limit_seconds);
        return PDFP_OK;
    } catch (const pdfp::Error& e) {
        pdfp::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        pdfp::set_last_error(e.what());
        return PDFP_E_INVALID;
    }
}
