// flat_spmv.cuh -- the step engine without shared-memory staging.
//
// The second engine the autotuner can pick for the two PDHG step passes
// (PrimalOp, DualOp).  It walks the same tiles of whole rows as the tile engine
// (layout.hpp) with no producer and no role split.  For each tile every thread
// of the block
//
//   1. holds QPT quads of four consecutive column indices and values, loaded
//      straight from global memory (128-bit, streaming: read once per step),
//      and the QPT x 4 vector entries they gather;
//   2. writes the products to shared memory, where rows are summed (G lanes
//      per row; G = 1 adds a row's terms sequentially in storage order, the
//      reference's order);
//   3. runs the Op's per-row epilogue on consecutive threads, reading and
//      writing the per-row vectors in global memory directly.
//
// The block works on two tiles at once: the indices and values of the next
// tile are loaded before the products of the current one are formed, and its
// gathers are issued before the current tile's row sums and epilogue, so the
// gather latency of one tile overlaps the reductions and vector traffic of the
// other.  A row longer than a tile is its own tile of several chunks and is
// summed by the whole block (FP64 partial sums), outside the pipeline.
//
// Against the tile engine it trades the bulk copies of indices and values into
// shared memory (and the mbarrier hand-offs between roles) for plain coalesced
// loads; which is faster depends on the matrix, so the autotuner times both.
#pragma once
#include "common.cuh"
#include "layout.hpp"

namespace pdfp {

constexpr int kFlatThreads = 256;  // threads per block; tile caps in layout.hpp

template <class Op>
struct FlatSmem {
    typename Op::AT prod[kFlatCapMax];
    typename Op::AT rowsum[kFlatMaxRows];
    int32_t rp[kFlatMaxRows + 1];
    double red[kFlatThreads / 32];
};

// One multi-row tile's streams and gathers in registers.
template <class Op, int QPT>
struct FlatRegs {
    int4 cc[QPT];
    typename Op::MT aa[QPT][4];
    typename Op::GT gv[QPT][4][1];
};

struct FlatTile {
    int32_t t, inst, r0, r1, k0, k1, base, quads;
    bool is_long;
};

__device__ __forceinline__ FlatTile flat_tile(const SideDev& s, int32_t t) {
    FlatTile f;
    f.t = t;
    f.inst = s.tile_inst[t];
    f.r0 = s.tile_row[t];
    f.r1 = s.tile_row[t + 1];
    const int32_t c0 = s.tile_chunk[t];
    const ChunkDesc d0 = s.chunks[c0];
    f.is_long = (d0.flags & CHUNK_LONG) != 0;
    f.k0 = d0.k0;
    f.k1 = f.is_long ? s.chunks[s.tile_chunk[t + 1] - 1].k1 : d0.k1;
    f.base = f.k0 & ~3;
    f.quads = (f.k1 - f.base + 3) >> 2;
    return f;
}

// First tile at or after t (stepping by the grid) whose instance is active.
template <class Op>
__device__ __forceinline__ int32_t flat_next(const SideDev& s, const Op& op, int32_t t) {
    while (t < s.n_tiles && !op.active(s.tile_inst[t])) t += gridDim.x;
    return t;
}

template <class Op, int QPT>
__device__ __forceinline__ void flat_load(const SideDev& s, const Op& op, const FlatTile& f,
                                          FlatRegs<Op, QPT>& r) {
    using MT = typename Op::MT;
    const MT* vals = op.values();
#pragma unroll
    for (int h = 0; h < QPT; ++h) {
        const int32_t q = threadIdx.x + h * kFlatThreads;
        if (q < f.quads) {
            r.cc[h] = __ldcs(reinterpret_cast<const int4*>(s.ci + f.base) + q);
            if constexpr (sizeof(MT) == 4) {
                const float4 a = __ldcs(reinterpret_cast<const float4*>(vals + f.base) + q);
                r.aa[h][0] = a.x; r.aa[h][1] = a.y; r.aa[h][2] = a.z; r.aa[h][3] = a.w;
            } else {
                const double2 a = __ldcs(reinterpret_cast<const double2*>(vals + f.base) + 2 * q);
                const double2 b = __ldcs(reinterpret_cast<const double2*>(vals + f.base) + 2 * q + 1);
                r.aa[h][0] = a.x; r.aa[h][1] = a.y; r.aa[h][2] = b.x; r.aa[h][3] = b.y;
            }
        }
    }
}

template <class Op, int QPT>
__device__ __forceinline__ void flat_gather(const Op& op, const FlatTile& f, FlatRegs<Op, QPT>& r) {
#pragma unroll
    for (int h = 0; h < QPT; ++h) {
        const int32_t q = threadIdx.x + h * kFlatThreads;
        if (q < f.quads) {
            const int32_t e = f.base + 4 * q;
            const int cols[4] = {r.cc[h].x, r.cc[h].y, r.cc[h].z, r.cc[h].w};
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (e + j >= f.k0 && e + j < f.k1) op.gather(cols[j], r.gv[h][j]);
        }
    }
}

// One tile of the pipeline.  On entry `cur` holds tile t's streams and
// gathers when `have` is set; on return `nxt` holds those of the tile
// returned (when *have is set).  Returns the next tile to process.
template <class Op, int QPT>
__device__ __forceinline__ int32_t flat_step(const SideDev& s, const Op& op, FlatSmem<Op>& sh,
                                             const typename Op::VT* const* sv, int32_t t,
                                             FlatRegs<Op, QPT>& cur, FlatRegs<Op, QPT>& nxt,
                                             bool* have) {
    using AT = typename Op::AT;
    using GT = typename Op::GT;
    constexpr int NT = kFlatThreads;
    const int tid = threadIdx.x;
    double none[1] = {0.0};
    const FlatTile f = flat_tile(s, t);
    const typename Op::TileP tp = op.tile_params(f.inst);
    if (f.is_long) {
        // one long row: block-strided products, FP64 sum
        const typename Op::MT* vals = op.values();
        double part[1] = {0.0};
        for (int32_t k = f.k0 + tid; k < f.k1; k += NT) {
            GT g[1];
            op.gather(s.ci[k], g);
            part[0] += static_cast<double>(mul_rn(static_cast<AT>(vals[k]), static_cast<AT>(g[0])));
        }
        block_sum<NT, 1, 0>(part, sh.red, tid);
        if (tid == 0) {
            const AT sums[1] = {static_cast<AT>(part[0])};
            op.row(f.r0, f.r0, f.inst, tp, sv, sums, none);
        }
        __syncthreads();
        *have = false;
        return flat_next(s, op, t + (int32_t)gridDim.x);
    }
    if (!*have) {
        flat_load<Op, QPT>(s, op, f, cur);
        flat_gather<Op, QPT>(op, f, cur);
    }
    // the next tile's streams are in flight while this tile's gathers land
    const int32_t tn = flat_next(s, op, t + (int32_t)gridDim.x);
    FlatTile fn{};
    bool pre = false;
    if (tn < s.n_tiles) {
        fn = flat_tile(s, tn);
        pre = !fn.is_long;
        if (pre) flat_load<Op, QPT>(s, op, fn, nxt);
    }
    const int32_t R = f.r1 - f.r0;
    for (int32_t i = tid; i <= R; i += NT) sh.rp[i] = s.rp[f.r0 + i] - f.base;
#pragma unroll
    for (int h = 0; h < QPT; ++h) {
        const int32_t q = tid + h * NT;
        if (q < f.quads) {
            const int32_t e = f.base + 4 * q;
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (e + j >= f.k0 && e + j < f.k1)
                    sh.prod[4 * q + j] = mul_rn(static_cast<AT>(cur.aa[h][j]), static_cast<AT>(cur.gv[h][j][0]));
        }
    }
    __syncthreads();
    // the next tile's gathers are in flight during this tile's sums and epilogue
    if (pre) flat_gather<Op, QPT>(op, fn, nxt);
    *have = pre;

    int G = 1;
    while (G < 32 && G * 2 * R <= NT) G *= 2;
    const int groups = NT / G;
    const int gid = tid / G, lane = tid & (G - 1);
    for (int32_t b = 0; b < R; b += groups) {
        const int32_t rr = b + gid;
        AT acc = AT(0);
        if (rr < R)
            for (int32_t k = sh.rp[rr] + lane; k < sh.rp[rr + 1]; k += G) acc = add_rn(acc, sh.prod[k]);
        for (int o = G >> 1; o > 0; o >>= 1) acc = add_rn(acc, __shfl_xor_sync(0xffffffffu, acc, o));
        if (rr < R && lane == 0) sh.rowsum[rr] = acc;
    }
    __syncthreads();
    for (int32_t rr = tid; rr < R; rr += NT) {
        const AT sums[1] = {sh.rowsum[rr]};
        op.row(f.r0 + rr, f.r0 + rr, f.inst, tp, sv, sums, none);
    }
    __syncthreads();  // prod, rowsum and rp are reused by the next tile
    return tn;
}

template <class Op, int QPT>
__global__ void __launch_bounds__(kFlatThreads, (sizeof(typename Op::MT) == 4 ? 3 : 2) + (QPT == 1 ? 1 : 0))
    flat_spmv_kernel(const SideDev s, const Op op) {
    using VT = typename Op::VT;
    static_assert(Op::NV == 1 && Op::NP == 0, "the flat engine runs the step passes");
    static_assert(QPT * 4 * kFlatThreads <= kFlatCapMax, "tile cap");
    constexpr int NVEC = Op::NVEC;
    __shared__ __align__(16) FlatSmem<Op> sh;
    const VT* sv[NVEC > 0 ? NVEC : 1];
#pragma unroll
    for (int k = 0; k < NVEC; ++k) sv[k] = op.staged(k);

    // two register sets trade roles tile by tile (no copies of in-flight loads)
    FlatRegs<Op, QPT> a, b;
    bool have = false;
    int32_t t = flat_next(s, op, (int32_t)blockIdx.x);
    while (t < s.n_tiles) {
        t = flat_step<Op, QPT>(s, op, sh, sv, t, a, b, &have);
        if (t >= s.n_tiles) break;
        t = flat_step<Op, QPT>(s, op, sh, sv, t, b, a, &have);
    }
}

}  // namespace pdfp
