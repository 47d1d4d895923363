// medium_steps.cuh -- a window's minor steps in one cooperative launch, for
// instances too large for one block and too small to fill the GPU per launch.
//
// Between a few thousand and about a million nonzeros a PDHG step launch costs
// more in launch latency and drain than in work.  Here one 256-thread block per
// SM runs steps i0 .. i1-1 of an evaluation window: each block owns a fixed, nonzero-
// balanced range of A' rows (columns) and of A rows, runs the Ops' passes over
// its ranges (G lanes per row, the Op's own per-row epilogue, as the one-block
// path does) and meets the other blocks at a grid barrier after each pass.  The
// vectors a pass gathers were written by other blocks, so the gathers read L2
// (the Ops' L2-only gather policy); everything a block reads otherwise it wrote
// itself.  The barrier is a counter and a generation word in global memory with
// a bounded wait: after kMediumWaitNs a block records the error, raises the abort
// word and returns, and every block that sees the abort word returns too.  The
// launch is cooperative, so all blocks are resident together.
#pragma once
#include "common.cuh"
#include "tiny_steps.cuh"
#include "vec_spmv.cuh"

namespace pdfp {

constexpr int kMediumThreads = 256;  // one block per SM (1024 threads measured slower)
constexpr uint64_t kMediumWaitNs = 2000000000ull;  // 2 s

struct GridBar {
    unsigned* count;  // arrivals in the current generation
    unsigned* gen;    // generation
    unsigned* abort;  // raised when a wait gave up
};

// All blocks of the grid meet; false when the barrier was abandoned.  `expected`
// arrivals complete a generation (0: the grid's blocks); the self-test asks for
// more than it launches, with a short limit, to make the wait run out.
__device__ __forceinline__ bool grid_barrier(const GridBar& g, int32_t* err, unsigned expected = 0,
                                             uint64_t limit_ns = kMediumWaitNs) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        const unsigned my_gen = *reinterpret_cast<volatile unsigned*>(g.gen);
        __threadfence();  // this block's writes before its arrival
        if (atomicAdd(g.count, 1u) == (expected ? expected : gridDim.x) - 1) {
            *g.count = 0;
            __threadfence();
            atomicAdd(g.gen, 1u);
        } else {
            const uint64_t t0 = globaltimer_ns();
            while (*reinterpret_cast<volatile unsigned*>(g.gen) == my_gen) {
                if (*reinterpret_cast<volatile unsigned*>(g.abort)) {
                    ok = 0;
                    break;
                }
                if (globaltimer_ns() - t0 > limit_ns) {
                    atomicExch(g.abort, 1u);
                    if (err) atomicExch(err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();  // the other blocks' writes before this block's reads
    }
    __syncthreads();
    return ok != 0;
}

// The pass of one side over this block's row range [ra, rb): the rows of every
// active instance inside it, instance by instance.
template <class Op>
__device__ __forceinline__ void medium_pass(const Op& op, const int32_t* __restrict__ rp,
                                            const int32_t* __restrict__ ci,
                                            const int32_t* __restrict__ off, int K, int32_t ra,
                                            int32_t rb) {
    if (ra >= rb) return;
    int lo = 0, hi = K;  // first instance whose range ends after ra
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (off[mid + 1] <= ra) lo = mid + 1; else hi = mid;
    }
    for (int p = lo; p < K && off[p] < rb; ++p) {
        if (!op.active(p)) continue;  // block-uniform
        const int32_t a = off[p] > ra ? off[p] : ra;
        const int32_t b = off[p + 1] < rb ? off[p + 1] : rb;
        if (a < b) tiny_pass<Op, kMediumThreads, 4>(op, rp, ci, a, b, p);  // 4: its register budget
    }
}

// Steps i0 .. i1-1 (minor) of every instance: POp on the rows of A' (columns),
// DOp on the rows of A; part_t / part_a hold each block's row range (gridDim.x + 1).
template <class POp, class DOp>
__global__ void __launch_bounds__(kMediumThreads)
    medium_steps_kernel(POp pop, DOp dop, const int32_t* __restrict__ rp_t,
                        const int32_t* __restrict__ ci_t, const int32_t* __restrict__ rp_a,
                        const int32_t* __restrict__ ci_a, const int32_t* __restrict__ col_off,
                        const int32_t* __restrict__ row_off, int K,
                        const int32_t* __restrict__ part_t, const int32_t* __restrict__ part_a,
                        GridBar bar, int32_t i0, int32_t i1) {
    const int32_t ta = part_t[blockIdx.x], tb = part_t[blockIdx.x + 1];
    const int32_t aa = part_a[blockIdx.x], ab = part_a[blockIdx.x + 1];
    for (int32_t i = i0; i < i1; ++i) {
        pop.k_offset = i;
        dop.k_offset = i;
        medium_pass(pop, rp_t, ci_t, col_off, K, ta, tb);  // the A'-side pass (primal update)
        if (!grid_barrier(bar, pop.err())) return;
        medium_pass(dop, rp_a, ci_a, row_off, K, aa, ab);  // the A-side pass (dual update)
        if (!grid_barrier(bar, pop.err())) return;
    }
}

// The vec engine's window: steps i0 .. i1-1 (minor) of every instance in one
// cooperative launch of every resident block, the A'-side items (POp), a grid
// barrier, the A-side items (DOp), a grid barrier, step after step.  Each warp
// takes the same items in every step (warp w: items w, w + W, ...), so every row's
// epilogue reads per-row vectors that only its own warp writes; the gathered
// vectors, written by other blocks, are read from L2 (the Ops' L2-only policy).
// The host uses it only for sides without long-row pieces, whose epilogues would
// move between warps from step to step.
template <class POp, class DOp>
__global__ void __launch_bounds__(kVecThreads, 4)
    vec_window_kernel(const VecDev ps, const VecDev ds, POp pop, DOp dop, GridBar bar,
                      int32_t i0, int32_t i1) {
    for (int32_t i = i0; i < i1; ++i) {
        pop.k_offset = i;
        dop.k_offset = i;
        vec_pass<POp>(ps, pop);  // the A'-side pass (primal update)
        if (!grid_barrier(bar, pop.err())) return;
        vec_pass<DOp>(ds, dop);  // the A-side pass (dual update)
        if (!grid_barrier(bar, pop.err())) return;
    }
}

}  // namespace pdfp
