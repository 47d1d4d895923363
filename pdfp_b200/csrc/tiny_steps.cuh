// tiny_steps.cuh -- the minor steps of a window in one launch, for small instances.
//
// For instances of a few thousand rows and columns every step launch is
// latency-bound: two launches per PDHG step cost more than the step itself.
// Here one block per batch member runs steps i0 .. i1-1 of an evaluation window
// back to back, with a block barrier between the A'-side and the A-side pass
// and after each step; vectors stay in global memory (L1/L2-resident at these
// sizes).  Each pass sums a row with G lanes, lane-strided partial sums reduced
// by an xor tree -- G = 1, a sequential sum in storage order (the reference's
// order), whenever the side has more than half as many rows as the block has
// threads -- and applies the Op's own per-row epilogue.  The first and last
// (major) steps of a window, the evaluations and the controller run as before.
#pragma once
#include "common.cuh"

namespace pdfp {

constexpr int kTinyThreads = 256;

// A lane's share of one row's sum: its nonzeros k0, k0 + G, ... below `end`, U at a
// time, added to s in storage order.  All U index, value and gather loads of a group
// are issued before its first product is added.
template <int U, class Op>
__device__ __forceinline__ void tiny_row_sum(const Op& op, const int32_t* __restrict__ ci,
                                             const typename Op::MT* vals, int32_t k0, int32_t end,
                                             int G, typename Op::AT& s) {
    using AT = typename Op::AT;
    using GT = typename Op::GT;
    for (; k0 < end; k0 += U * G) {
        int32_t c[U];
        AT a[U];
        GT g[U][1];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int32_t kk = k0 + u * G;
            c[u] = kk < end ? ci[kk] : 0;
            a[u] = kk < end ? static_cast<AT>(vals[kk]) : AT(0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (k0 + u * G < end) op.gather(c[u], g[u]);
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (k0 + u * G < end) s = add_rn(s, mul_rn(a[u], static_cast<AT>(g[u][0])));
    }
}

template <class Op, int NTH = kTinyThreads, int UONE = 8>
__device__ __forceinline__ void tiny_pass(const Op& op, const int32_t* __restrict__ rp,
                                          const int32_t* __restrict__ ci, int32_t r0, int32_t r1,
                                          int inst) {
    using AT = typename Op::AT;
    using VT = typename Op::VT;
    constexpr int NVEC = Op::NVEC;
    const VT* sv[NVEC];
#pragma unroll
    for (int k = 0; k < NVEC; ++k) sv[k] = op.staged(k);
    const typename Op::TileP tp = op.tile_params(inst);
    const auto* vals = op.values();
    double none[1] = {0.0};
    const int32_t R = r1 - r0;
    int G = 1;
    while (G < 32 && G * 2 * R <= NTH) G *= 2;
    const int groups = NTH / G;
    const int gid = threadIdx.x / G, lane = threadIdx.x & (G - 1);
    for (int32_t b = 0; b < R; b += groups) {
        const int32_t rr = b + gid;
        AT s = AT(0);
        if (rr < R) {
            const int32_t row = r0 + rr;
            // a row summed by one thread is a chain of dependent adds: UONE (eight)
            // loads in flight per group let it wait for memory once per eight
            // nonzeros (rows of 50-70 nonzeros on the reference's examples); rows
            // shared by G > 1 lanes are short per lane and take four
            if (G == 1)
                tiny_row_sum<UONE>(op, ci, vals, rp[row], rp[row + 1], 1, s);
            else
                tiny_row_sum<4>(op, ci, vals, rp[row] + lane, rp[row + 1], G, s);
        }
        for (int o = G >> 1; o > 0; o >>= 1) s = add_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
        if (rr < R && lane == 0) {
            const AT sums[1] = {s};
            op.row(r0 + rr, r0 + rr, inst, tp, sv, sums, none);
        }
    }
}

// One evaluation pass of instance `inst` over rows [r0, r1), in one block: each row's
// NV sums of products (G lanes per row, as tiny_pass) go to shared memory
// (rowsum[q * R + rr]), then the Op's per-row terms accumulate into acc with row rr on
// thread rr % NTH -- the tile engine epilogue's assignment -- so that the block sum
// that follows adds them in the same order as a one-tile evaluation launch.
// The NV sums of an evaluation Op over a lane's share of one row (as tiny_row_sum).
template <int U, class Op>
__device__ __forceinline__ void tiny_row_sums(const Op& op, const int32_t* __restrict__ ci,
                                              const typename Op::MT* vals, int32_t k0, int32_t end,
                                              int G, typename Op::AT (&s)[Op::NV]) {
    using AT = typename Op::AT;
    using GT = typename Op::GT;
    constexpr int NV = Op::NV;
    for (; k0 < end; k0 += U * G) {
        int32_t c[U];
        AT a[U];
        GT g[U][NV];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int32_t kk = k0 + u * G;
            c[u] = kk < end ? ci[kk] : 0;
            a[u] = kk < end ? static_cast<AT>(vals[kk]) : AT(0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (k0 + u * G < end) op.gather(c[u], g[u]);
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (k0 + u * G < end)
#pragma unroll
                for (int q = 0; q < NV; ++q) s[q] = add_rn(s[q], mul_rn(a[u], static_cast<AT>(g[u][q])));
    }
}

template <class Op, int NTH = kTinyThreads>
__device__ __forceinline__ void tiny_eval_pass(const Op& op, const int32_t* __restrict__ rp,
                                               const int32_t* __restrict__ ci, int32_t r0,
                                               int32_t r1, int inst, typename Op::AT* rowsum,
                                               double* acc) {
    using AT = typename Op::AT;
    using GT = typename Op::GT;
    constexpr int NV = Op::NV;
    const auto* vals = op.values();
    const int32_t R = r1 - r0;
    int G = 1;
    while (G < 32 && G * 2 * R <= NTH) G *= 2;
    const int groups = NTH / G;
    const int gid = threadIdx.x / G, lane = threadIdx.x & (G - 1);
    for (int32_t b = 0; b < R; b += groups) {
        const int32_t rr = b + gid;
        AT s[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) s[q] = AT(0);
        if (rr < R) {
            const int32_t row = r0 + rr;
            // one lane per row: four of its nonzeros in flight at a time; several lanes
            // per row: one at a time (added in storage order either way)
            if (G == 1)
                tiny_row_sums<4>(op, ci, vals, rp[row], rp[row + 1], 1, s);
            else
                tiny_row_sums<1>(op, ci, vals, rp[row] + lane, rp[row + 1], G, s);
        }
        for (int o = G >> 1; o > 0; o >>= 1)
#pragma unroll
            for (int q = 0; q < NV; ++q) s[q] = add_rn(s[q], __shfl_xor_sync(0xffffffffu, s[q], o));
        if (rr < R && lane == 0)
#pragma unroll
            for (int q = 0; q < NV; ++q) rowsum[q * R + rr] = s[q];
    }
    __syncthreads();
    const typename Op::TileP tp = op.tile_params(inst);
    const typename Op::VT* none[1] = {nullptr};
    for (int32_t rr = threadIdx.x; rr < R; rr += NTH) {
        AT sums[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) sums[q] = rowsum[q * R + rr];
        op.row(r0 + rr, rr, inst, tp, none, sums, acc);
    }
    __syncthreads();  // rowsum is reused by the next pass
}

// Steps i0 .. i1-1 (minor: no pdhg_* / reflected_* outputs) of instance blockIdx.x:
// POp runs on the rows of A' (columns), DOp on the rows of A; both carry the step
// index in k_offset.
template <class POp, class DOp>
__global__ void __launch_bounds__(kTinyThreads)
    tiny_steps_kernel(POp pop, DOp dop,
                      const int32_t* __restrict__ rp_t, const int32_t* __restrict__ ci_t,
                      const int32_t* __restrict__ rp_a, const int32_t* __restrict__ ci_a,
                      const int32_t* __restrict__ col_off, const int32_t* __restrict__ row_off,
                      int32_t i0, int32_t i1) {
    const int p = blockIdx.x;
    if (!pop.active(p)) return;  // block-uniform; status changes only in the controller
    const int32_t c0 = col_off[p], c1 = col_off[p + 1], r0 = row_off[p], r1 = row_off[p + 1];
    for (int32_t i = i0; i < i1; ++i) {
        pop.k_offset = i;
        dop.k_offset = i;
        tiny_pass(pop, rp_t, ci_t, c0, c1, p);  // the A'-side pass (primal update)
        __syncthreads();
        tiny_pass(dop, rp_a, ci_a, r0, r1, p);  // the A-side pass (dual update)
        __syncthreads();
    }
}

}  // namespace pdfp
