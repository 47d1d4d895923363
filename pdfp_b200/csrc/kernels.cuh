// kernels.cuh -- launch helpers and the small kernels around the tile engine.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "common.cuh"
#include "layout.hpp"
#include "state.hpp"
#include "flat_spmv.cuh"
#include "tile_spmv.cuh"
#include "vec_spmv.cuh"
#include "seg_spmv.cuh"

namespace pdfp {

// ---- launching the tile engine ----------------------------------------------------

template <class Op>
size_t tile_dyn_smem(const SideDev& s) {
    size_t nv = Op::NV > 0 ? Op::NV : 1;
    return static_cast<size_t>(s.stages) * static_cast<size_t>(s.stage_bytes) +
           ((nv * s.max_tile_rows * sizeof(typename Op::AT) + 127) & ~size_t(127));
}

// Persistent grid size for an Op on a side (blocks resident on all SMs).
template <class Op, bool ASYNC, int NR>
int tile_grid_of(const SideDev& s, int num_sms) {
    const size_t smem = tile_dyn_smem<Op>(s);
    // The attribute belongs to the kernel, shared by every tiling launched with
    // it: only ever raise it.
    static size_t attr = 0;
    if (smem > attr) {
        cudaFuncSetAttribute(tile_spmv_kernel<Op, ASYNC, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
        attr = smem;
    }
    int blocks = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, tile_spmv_kernel<Op, ASYNC, NR>,
                                                  Op::NT + NR + 32, smem);
    const int per_sm = blocks > 0 ? blocks : 1;
    int g = per_sm * num_sms;
    return g < s.n_tiles ? g : s.n_tiles;
}

// Ops with a half-size reducer role (Op::NT / 2 reducer threads): the FP32 steps
template <class Op>
constexpr bool kHalfReducers = HasGatherSrc<Op>::value && sizeof(typename Op::MT) == 4;

// async: the Op's gathers by per-thread async copies (gather policy 2); half_red:
// Op::NT / 2 reducer threads; both ignored for Ops that have no such variant
template <class Op>
int tile_grid(const SideDev& s, int num_sms, bool async = false, bool half_red = false) {
    if constexpr (kAsyncEligible<Op>)
        if (async) return tile_grid_of<Op, true, Op::NT>(s, num_sms);
    if constexpr (kHalfReducers<Op>)
        if (half_red) return tile_grid_of<Op, false, Op::NT / 2>(s, num_sms);
    return tile_grid_of<Op, false, Op::NT>(s, num_sms);
}

template <class Op, bool ASYNC, int NR>
void launch_tile_k(const SideDev& s, const Op& op, int grid, cudaStream_t stream, bool overlap,
                   int carveout) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(grid));
    cfg.blockDim = dim3(Op::NT + NR + 32);
    cfg.dynamicSmemBytes = tile_dyn_smem<Op>(s);
    if constexpr (HasPrologue<Op>::value) cfg.dynamicSmemBytes += op.extra_smem();
    cfg.stream = stream;
    cudaLaunchAttribute at[2];
    int na = 0;
    if (overlap) {
        at[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[na].val.programmaticStreamSerializationAllowed = 1;
        ++na;
    }
    if (carveout >= 0) {
        at[na].id = cudaLaunchAttributePreferredSharedMemoryCarveout;
        at[na].val.sharedMemCarveout = static_cast<unsigned>(carveout);
        ++na;
    }
    cfg.attrs = at;
    cfg.numAttrs = na;
    cudaLaunchKernelEx(&cfg, tile_spmv_kernel<Op, ASYNC, NR>, s, op);  // errors: cudaGetLastError
}

// Share of the SM's unified L1 / shared memory (percent) that `blocks` resident
// blocks of this Op need as shared memory on side s: the rest stays L1.
template <class Op>
int tile_carveout(const SideDev& s, int blocks, int max_smem_per_sm) {
    const size_t per_block = tile_dyn_smem<Op>(s) + sizeof(TileKernelSmem<Op>) + 1024;  // + reserved
    const size_t need = per_block * static_cast<size_t>(blocks);
    const int pct = static_cast<int>((100 * need + max_smem_per_sm - 1) / max_smem_per_sm);
    return pct > 100 ? 100 : pct;
}

// overlap: the launch may start while the previous grid on the stream drains
// (programmatic dependent launch; only directly after another tile-engine launch
// of a step -- see tile_spmv.cuh).  carveout >= 0: the preferred shared-memory
// share of the unified L1 (percent) for this launch.  half_red: Op::NT / 2 reducers.
template <class Op>
void launch_tile(const SideDev& s, const Op& op, int grid, cudaStream_t stream, bool overlap = false,
                 int carveout = -1, bool half_red = false) {
    if (s.n_tiles <= 0 || grid <= 0) return;
    if constexpr (kAsyncEligible<Op>)
        if (op.gather_l2 == 2) {
            launch_tile_k<Op, true, Op::NT>(s, op, grid, stream, overlap, carveout);
            return;
        }
    if constexpr (kHalfReducers<Op>)
        if (half_red) {
            launch_tile_k<Op, false, Op::NT / 2>(s, op, grid, stream, overlap, carveout);
            return;
        }
    launch_tile_k<Op, false, Op::NT>(s, op, grid, stream, overlap, carveout);
}

// ---- launching the flat engine ---------------------------------------------------

template <class Op, int QPT>
int flat_grid(const SideDev& s, int num_sms) {
    int blocks = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, flat_spmv_kernel<Op, QPT>, kFlatThreads, 0);
    const int g = (blocks > 0 ? blocks : 1) * num_sms;
    return g < s.n_tiles ? g : s.n_tiles;
}

template <class Op>
int flat_grid(const SideDev& s, int qpt, int num_sms) {
    return qpt == 1 ? flat_grid<Op, 1>(s, num_sms) : flat_grid<Op, 2>(s, num_sms);
}

template <class Op>
void launch_flat(const SideDev& s, const Op& op, int qpt, int grid, cudaStream_t stream) {
    if (s.n_tiles <= 0 || grid <= 0) return;
    if (qpt == 1)
        flat_spmv_kernel<Op, 1><<<grid, kFlatThreads, 0, stream>>>(s, op);
    else
        flat_spmv_kernel<Op, 2><<<grid, kFlatThreads, 0, stream>>>(s, op);
}

// ---- launching the vec engine -----------------------------------------------------

// Blocks resident on all SMs, no more than the items need (8 warps per block).
template <class Op>
int vec_grid(const VecDev& s, int num_sms) {
    int blocks = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, vec_spmv_kernel<Op>, kVecThreads, 0);
    const int g = (blocks > 0 ? blocks : 1) * num_sms;
    const int need = (s.n_items + kVecThreads / 32 - 1) / (kVecThreads / 32);
    return g < need ? g : need;
}

template <class Op>
void launch_vec(const VecDev& s, const Op& op, int grid, cudaStream_t stream) {
    if (s.n_items <= 0 || grid <= 0) return;
    vec_spmv_kernel<Op><<<grid, kVecThreads, 0, stream>>>(s, op);
}

// ---- launching the segmented long rows ------------------------------------------

template <int NT, class DOp>
SegPartialOp<NT> seg_partial_op(const SideDev& pairs, const SegDev& g, const DOp& dop) {
    SegPartialOp<NT> op{};
    op.x = dop.v.rx;  // x_bar, which the A-side step gathers
    op.vals = g.val;
    op.partial = g.partial;
    op.nseg = g.nseg;
    op.seg_len = g.seg_len;
    op.n_cols = g.n_cols;
    op.n_long = g.n_long;
    op.xs_off = static_cast<uint32_t>(tile_dyn_smem<SegPartialOp<NT>>(pairs));
    op.errp = dop.errp;
    return op;
}

// Raises the partials kernel's shared-memory limit for this tiling; false when a
// block cannot have that much.
template <int NT, class DOp>
bool seg_attr(const SideDev& pairs, const SegDev& g, const DOp& dop, int max_smem_optin) {
    using SOp = SegPartialOp<NT>;
    const SOp op = seg_partial_op<NT>(pairs, g, dop);
    const size_t smem = tile_dyn_smem<SOp>(pairs) + op.extra_smem();
    if (smem > static_cast<size_t>(max_smem_optin)) return false;
    static size_t attr = 0;  // per kernel: only ever raised
    if (smem > attr) {
        if (cudaFuncSetAttribute(tile_spmv_kernel<SOp, false, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)) != cudaSuccess)
            return false;
        attr = smem;
    }
    return true;
}

// The long rows' partials (bps blocks per segment) and their finish.
template <class DOp>
void launch_seg(const SideDev& pairs, const SegDev& g, int nt, int bps, const DOp& dop,
                cudaStream_t stream) {
    if (g.n_long <= 0 || g.nseg <= 0) return;
    const int grid = g.nseg * bps;
    if (nt == 256)
        launch_tile_k<SegPartialOp<256>, false, 256>(pairs, seg_partial_op<256>(pairs, g, dop), grid,
                                                     stream, false, -1);
    else
        launch_tile_k<SegPartialOp<128>, false, 128>(pairs, seg_partial_op<128>(pairs, g, dop), grid,
                                                     stream, false, -1);
    const unsigned blocks = static_cast<unsigned>((g.n_long + 31) / 32);
    seg_finish_kernel<DOp><<<blocks, 32 * kSegFinWarps, 0, stream>>>(g, dop);
}

// ---- per-tile elementwise reductions and per-instance finalisation ---------------
// A RowsOp walks the rows of each tile of a tiling (one block per tile, one
// thread per row), accumulating NP FP64 partial sums per tile.

template <class RowsOp>
__global__ void __launch_bounds__(256) tile_rows_kernel(const SideDev s, const RowsOp op) {
    constexpr int NP = RowsOp::NP;
    __shared__ double red[(NP > 0 ? NP : 1) * 8];
    const int32_t t = blockIdx.x;
    const int32_t inst = s.tile_inst[t];
    if (!op.active(inst)) return;
    const int32_t r0 = s.tile_row[t], r1 = s.tile_row[t + 1];
    double acc[NP > 0 ? NP : 1];
#pragma unroll
    for (int k = 0; k < (NP > 0 ? NP : 1); ++k) acc[k] = 0.0;
    for (int32_t r = r0 + threadIdx.x; r < r1; r += 256) op.row(r, inst, acc);
    if (NP > 0) {
        block_sum<256, (NP > 0 ? NP : 1)>(acc, red, threadIdx.x);
        if (threadIdx.x == 0) op.write_partials(t, acc);
    }
}

template <class RowsOp>
void launch_rows(const SideDev& s, const RowsOp& op, cudaStream_t stream) {
    if (s.n_tiles <= 0) return;
    tile_rows_kernel<RowsOp><<<s.n_tiles, 256, 0, stream>>>(s, op);
}

// One block per instance: reduce NA partials from tiling A (tiles
// [ta0[p], ta0[p+1])) and NB from tiling B, then op.finalize(p, sums).
template <class FinOp>
__global__ void __launch_bounds__(256) finalize_kernel(const FinOp op) {
    constexpr int NA = FinOp::NA, NB = FinOp::NB, N = NA + NB;
    __shared__ double red[N * 8];
    const int p = blockIdx.x;
    if (!op.active(p)) return;
    double a[N];
#pragma unroll
    for (int k = 0; k < N; ++k) a[k] = 0.0;
    if (NA > 0)
        for (int32_t t = op.ta0[p] + threadIdx.x; t < op.ta0[p + 1]; t += 256)
#pragma unroll
            for (int k = 0; k < (NA > 0 ? NA : 1); ++k) a[k] += op.pa[t * (NA > 0 ? NA : 1) + k];
    if (NB > 0)
        for (int32_t t = op.tb0[p] + threadIdx.x; t < op.tb0[p + 1]; t += 256)
#pragma unroll
            for (int k = 0; k < (NB > 0 ? NB : 1); ++k) a[NA + k] += op.pb[t * (NB > 0 ? NB : 1) + k];
    block_sum<256, N>(a, red, threadIdx.x);
    if (threadIdx.x == 0) op.finalize(p, a);
}

template <class FinOp>
void launch_finalize(int K, const FinOp& op, cudaStream_t stream) {
    if (K <= 0) return;
    finalize_kernel<FinOp><<<K, 256, 0, stream>>>(op);
}

// Per-instance elementwise kernel: blockIdx.y = instance, x strides its range.
template <class ElemOp>
__global__ void __launch_bounds__(256) inst_elem_kernel(const ElemOp op) {
    const int p = blockIdx.y;
    if (!op.active(p)) return;
    const int32_t b = op.begin(p), e = op.end(p);
    for (int32_t i = b + blockIdx.x * 256 + threadIdx.x; i < e; i += gridDim.x * 256) op.elem(p, i);
}

template <class ElemOp>
void launch_elem(int K, int64_t max_len, const ElemOp& op, cudaStream_t stream) {
    if (K <= 0 || max_len <= 0) return;
    int64_t gx = (max_len + 255) / 256;
    if (gx > 2048) gx = 2048;
    dim3 grid(static_cast<unsigned>(gx), static_cast<unsigned>(K));
    inst_elem_kernel<ElemOp><<<grid, 256, 0, stream>>>(op);
}

}  // namespace pdfp
