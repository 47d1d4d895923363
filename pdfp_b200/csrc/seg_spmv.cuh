// seg_spmv.cuh -- A x_bar for the long rows of A, gathered from shared memory.
//
// On a matrix whose long rows hold most of the nonzeros (zipf-lp: 12k of 1M rows,
// 512 to 2,048 nonzeros each, hold 69% of them), the A-side step kernel spends its
// time on random 4-byte gathers of x_bar from L2.  Here those rows are regrouped by
// column segment (SegDev, layout.hpp) and the A side runs in three launches:
//
//   partials   the tile engine over the regrouped entries, whose "rows" are the
//       (segment, long row) pairs, with SegPartialOp: block b runs only tiles of
//       segment b mod nseg (the tiling interleaves the segments' tiles and the grid
//       has bps blocks per segment, which share out the segment's tiles), its
//       gatherers first copy that segment of x_bar into
//       shared memory and then gather from there; the epilogue stores each pair's
//       sum as the long row's partial for the segment (empty pairs as zero).  The
//       matrix entries stream through the engine's bulk-copy stages as usual.
//   finish     seg_finish_kernel: the partials of each long row added in a fixed
//       order (FP64), then the Op's per-row epilogue.
//   the rest   the tile engine with the step's own Op over a tiling that leaves the
//       long rows out.
//
// FP32 steps only: the regrouping changes the order in which a long row's terms
// are added.
#pragma once
#include "common.cuh"
#include "layout.hpp"

namespace pdfp {

// The partial sums of the (segment, long row) pairs; bps blocks per segment.
template <int NTHREADS>
struct SegPartialOp {
    using MT = float;
    using VT = float;
    using AT = float;
    using GT = float;
    struct TileP {
        int32_t seg;
    };
    static constexpr int NT = NTHREADS, NV = 1, NVEC = 0, NP = 0;
    const float* x;      // the gathered vector (x_bar), packed columns
    const float* vals;   // the regrouped entries' values
    float* partial;      // nseg x n_long: segment-major, so each block writes its own range
    int32_t nseg, seg_len, n_cols, n_long;
    uint32_t xs_off;     // byte offset of the segment copy in dynamic shared memory
    int32_t* errp;
    int32_t gather_l2 = 0;

    __device__ const float* values() const { return vals; }
    __device__ const float* staged(int) const { return nullptr; }
    __device__ int32_t* err() const { return errp; }
    __device__ bool active(int inst) const { return inst >= 0; }  // padding tiles: -1
    __device__ TileP tile_params(int inst) const { return TileP{inst}; }
    size_t extra_smem() const { return (static_cast<size_t>(seg_len) * 4 + 127) & ~size_t(127); }
    // The block's segment of x_bar into shared memory: 16-byte loads, eight in flight
    // per thread (seg_len is a multiple of 4, so every segment starts 16-byte aligned;
    // the last one may read up to 3 entries past the vector, inside its padding).
    __device__ void prologue(int tid, int nthreads) const {
        extern __shared__ __align__(128) unsigned char dyn_smem[];
        float4* xs = reinterpret_cast<float4*>(dyn_smem + xs_off);
        const int32_t c0 = static_cast<int32_t>(blockIdx.x % static_cast<unsigned>(nseg)) * seg_len;
        const int32_t len = min(seg_len, n_cols - c0);
        const int32_t n4 = (len + 3) >> 2;
        const float4* src = reinterpret_cast<const float4*>(x + c0);
        for (int32_t j = tid; j < n4; j += 8 * nthreads) {
            float4 v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (j + u * nthreads < n4) v[u] = __ldcg(src + j + u * nthreads);
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (j + u * nthreads < n4) xs[j + u * nthreads] = v[u];
        }
    }
    __device__ void gather(int32_t col, float (&g)[1]) const {
        extern __shared__ __align__(128) unsigned char dyn_smem[];
        g[0] = reinterpret_cast<const float*>(dyn_smem + xs_off)[col];
    }
    __device__ void row(int32_t i, int32_t, int, const TileP& t, const float* const*,
                        const float (&s)[1], double*) const {
        partial[i] = s[0];  // pair i = seg * n_long + q
    }
};

// One block of kSegFinWarps warps per 32 long rows (lane = row): warp w adds the
// partials of segments w, w + kSegFinWarps, ... (coalesced across the 32 rows), the
// block combines the warps' sums in warp order (FP64), and the rows' epilogues run
// on the first warp.
constexpr int kSegFinWarps = 8;

template <class Op>
__global__ void __launch_bounds__(32 * kSegFinWarps) seg_finish_kernel(const SegDev g, const Op op) {
    using AT = typename Op::AT;
    using VT = typename Op::VT;
    constexpr int NVEC = Op::NVEC;
    __shared__ double part[kSegFinWarps][32];
    const int lane = static_cast<int>(threadIdx.x & 31), w = static_cast<int>(threadIdx.x >> 5);
    const int32_t q = static_cast<int32_t>(blockIdx.x) * 32 + lane;
    const bool valid = q < g.n_long;
    const int32_t inst = valid ? g.long_inst[q] : -1;
    const bool act = valid && op.active(inst);
    double acc = 0.0;
    if (act) {
        for (int32_t s0 = w; s0 < g.nseg; s0 += 4 * kSegFinWarps) {  // four loads in flight
            float v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int32_t s = s0 + u * kSegFinWarps;
                v[u] = s < g.nseg ? __ldcg(g.partial + static_cast<size_t>(s) * g.n_long + q) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) acc += static_cast<double>(v[u]);
        }
    }
    part[w][lane] = acc;
    __syncthreads();
    if (w == 0 && act) {
        double tot = 0.0;
#pragma unroll
        for (int k = 0; k < kSegFinWarps; ++k) tot += part[k][lane];
        const VT* sv[NVEC > 0 ? NVEC : 1];
#pragma unroll
        for (int k = 0; k < NVEC; ++k) sv[k] = op.staged(k);
        const typename Op::TileP tp = op.tile_params(inst);
        const AT sums[1] = {static_cast<AT>(tot)};
        double none[1] = {0.0};
        const int32_t i = g.long_row[q];
        op.row(i, i, inst, tp, sv, sums, none);
    }
}

}  // namespace pdfp
