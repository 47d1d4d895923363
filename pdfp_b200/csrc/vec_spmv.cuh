// vec_spmv.cuh -- the third step engine: rows read straight from the CSR arrays.
//
// The step passes (PrimalOp, DualOp) with no tiles, no shared memory and no
// block barriers.  The work is a host-built list of items (VecItem, layout.hpp),
// each taken by one warp:
//
//   * a run of rows of one instance with G = 2^lg lanes per row: the warp holds
//     32 / G rows at a time; the G lanes of a row load its column indices and
//     values with coalesced streaming loads (consecutive rows are adjacent in
//     memory, so a warp's loads cover one contiguous stretch), gather four
//     vector entries per lane at a time, sum their products in the Op's
//     arithmetic type and reduce across the G lanes with shuffles; the row's
//     first lane runs the Op's per-row epilogue on the per-row vectors in
//     global memory.  The host picks G from the row length so that each lane
//     holds about `lane_nnz` nonzeros.
//   * one piece (at most kVecPiece nonzeros) of a long row: the whole warp sums
//     the piece in FP64 and stores it in the piece's slot; the warp that
//     completes the row's last piece (a counter per row, reset by that warp for
//     the next launch) adds the row's slots in piece order and runs the
//     epilogue, so the result does not depend on which warp finishes last.
//
// Items are ordered by decreasing work (long-row pieces first), and warp w takes
// items w, w + W, w + 2W, ... of the list (W warps in the grid): a static
// longest-first schedule.  Against the tile engine it trades the staged,
// pipelined tiles for more gathers in flight per SM and no hand-offs; which is
// faster depends on the matrix, so the autotuner times it with the others.  The
// FP32 steps only: its lane sums change the order in which a row's terms are
// added, which the FP64 form (that takes the oracle's steps) does not allow.
#pragma once
#include "common.cuh"
#include "layout.hpp"

namespace pdfp {

constexpr int kVecThreads = 256;  // 8 warps per block
#ifndef PDFP_VEC_MIN_BLOCKS
#define PDFP_VEC_MIN_BLOCKS 5
#endif
// resident blocks per SM the step kernels are compiled for (48 registers a thread: at 6
// blocks and 40 registers the A'-side kernel spills and runs slower)
constexpr int kVecMinBlocks = PDFP_VEC_MIN_BLOCKS;

template <class Op>
__device__ __forceinline__ void vec_rows(const VecDev& s, const Op& op, const VecItem& m,
                                         const typename Op::TileP& tp, int lane) {
    using AT = typename Op::AT;
    using MT = typename Op::MT;
    using GT = typename Op::GT;
    using VT = typename Op::VT;
    const MT* vals = op.values();
    const int lg = m.lg, G = 1 << lg;
    const int grp = lane >> lg, gl = lane & (G - 1);
    const int per = 32 >> lg;
    for (int32_t b = m.r0; b < m.r1; b += per) {
        const int32_t r = b + grp;
        const bool valid = r < m.r1;
        // the row's first lane loads the epilogue's per-row inputs now, so that their
        // latency passes under the gathers instead of after them
        VT pv[Op::NVEC];
        if (valid && gl == 0) op.load_row(r, pv);
        AT acc = AT(0);
        if (valid) {
            const int32_t e = s.rp[r + 1];
            for (int32_t k = s.rp[r] + gl; k < e; k += 4 * G) {
                int32_t c[4];
                MT a[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int32_t kk = k + u * G;
                    c[u] = kk < e ? __ldcs(s.ci + kk) : -1;
                    a[u] = kk < e ? __ldcs(vals + kk) : MT(0);
                }
                GT g[4][1] = {};
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (c[u] >= 0) op.gather(c[u], g[u]);
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (c[u] >= 0) acc = add_rn(acc, mul_rn(static_cast<AT>(a[u]), static_cast<AT>(g[u][0])));
            }
        }
        for (int o = G >> 1; o > 0; o >>= 1) acc = add_rn(acc, __shfl_xor_sync(0xffffffffu, acc, o));
        if (valid && gl == 0) {
            const AT sums[1] = {acc};
            op.row_vals(r, tp, pv, sums);
        }
    }
}

template <class Op>
__device__ __forceinline__ void vec_piece(const VecDev& s, const Op& op, const VecItem& m,
                                          const typename Op::TileP& tp, int lane) {
    using AT = typename Op::AT;
    using MT = typename Op::MT;
    using GT = typename Op::GT;
    using VT = typename Op::VT;
    const MT* vals = op.values();
    double part = 0.0;
    for (int32_t k = m.k0 + lane; k < m.k1; k += 128) {
        int32_t c[4];
        MT a[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int32_t kk = k + 32 * u;
            c[u] = kk < m.k1 ? __ldcs(s.ci + kk) : -1;
            a[u] = kk < m.k1 ? __ldcs(vals + kk) : MT(0);
        }
        GT g[4][1] = {};
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (c[u] >= 0) op.gather(c[u], g[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (c[u] >= 0) part += static_cast<double>(mul_rn(static_cast<AT>(a[u]), static_cast<AT>(g[u][0])));
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if (lane == 0) {
        s.piece_sum[m.slot] = part;
        __threadfence();
        const int32_t first = m.r1;  // the row's first slot, which also holds its counter
        if (atomicAdd(s.piece_cnt + first, 1) == m.np - 1) {
            __threadfence();
            double tot = 0.0;
            for (int32_t q = 0; q < m.np; ++q) tot += __ldcg(s.piece_sum + first + q);
            s.piece_cnt[first] = 0;
            const AT sums[1] = {static_cast<AT>(tot)};
            VT pv[Op::NVEC];
            op.load_row(m.r0, pv);
            op.row_vals(m.r0, tp, pv, sums);
        }
    }
}

// One pass over a side's items: warp w of the grid takes items w, w + W, ...  Lane
// l < 8 holds field l of the warp's next item, loaded while the current one runs;
// the step parameters are recomputed only when the instance changes.
template <class Op>
__device__ __forceinline__ void vec_pass(const VecDev& s, const Op& op) {
    static_assert(Op::NV == 1 && Op::NP == 0, "the vec engine runs the step passes");
    static_assert(sizeof(VecItem) == 8 * sizeof(int32_t), "VecItem is eight int32 fields");
    const int lane = threadIdx.x & 31;
    const int32_t w0 = static_cast<int32_t>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int32_t nw = static_cast<int32_t>((gridDim.x * blockDim.x) >> 5);
    const int32_t* fields = reinterpret_cast<const int32_t*>(s.items);
    int32_t it = w0;
    int32_t nxt = it < s.n_items && lane < 8 ? __ldg(fields + 8 * static_cast<int64_t>(it) + lane) : 0;
    int32_t cur_inst = -1;
    bool act = false;
    // the step parameters of the warp's current instance sit in a per-warp shared
    // slot: they are read only by the epilogue, and in registers they would be live
    // across every gather
    __shared__ typename Op::TileP tp_slot[kVecThreads / 32];
    typename Op::TileP& tp = tp_slot[threadIdx.x >> 5];
    while (it < s.n_items) {
        VecItem m;
        m.r0 = __shfl_sync(0xffffffffu, nxt, 0);
        m.r1 = __shfl_sync(0xffffffffu, nxt, 1);
        m.inst = __shfl_sync(0xffffffffu, nxt, 2);
        m.lg = __shfl_sync(0xffffffffu, nxt, 3);
        m.k0 = __shfl_sync(0xffffffffu, nxt, 4);
        m.k1 = __shfl_sync(0xffffffffu, nxt, 5);
        m.slot = __shfl_sync(0xffffffffu, nxt, 6);
        m.np = __shfl_sync(0xffffffffu, nxt, 7);
        it += nw;
        nxt = it < s.n_items && lane < 8 ? __ldg(fields + 8 * static_cast<int64_t>(it) + lane) : 0;
        if (m.inst != cur_inst) {
            cur_inst = m.inst;
            act = op.active(m.inst);
            __syncwarp();
            if (act && lane == 0) tp = op.tile_params(m.inst);
            __syncwarp();
        }
        if (!act) continue;
        if (m.lg < 0)
            vec_piece<Op>(s, op, m, tp, lane);
        else
            vec_rows<Op>(s, op, m, tp, lane);
    }
}

template <class Op>
__global__ void __launch_bounds__(kVecThreads, kVecMinBlocks) vec_spmv_kernel(const VecDev s, const Op op) {
    vec_pass<Op>(s, op);
}

}  // namespace pdfp
