// tile_spmv.cuh -- the sparse-product engine behind every pass of the solvers.
//
// One side of a matrix (A, or its explicit transpose A') is stored as CSR in
// the packed, permuted numbering of the handle (see layout.hpp).  Its rows are
// cut into TILES of whole rows whose data fit one shared-memory stage; a row
// too long for a stage gets a tile of its own, split into several CHUNKS.
//
// A persistent kernel walks the tiles assigned to its block (round robin),
// double buffered: while chunk u is being processed, one thread has already
// issued the cp.async.bulk copies of chunk u+1 (row pointers, column indices,
// values and -- on a tile's last chunk -- the slices of the per-row vectors the
// epilogue reads) into the other stage, completing on an mbarrier.  Per chunk:
//
//   1. products   p_k = a_k * g[col_k]   for every nonzero, thread-strided, so
//                 all gathers of the chunk are in flight at once (the gathered
//                 vector is L2-resident);
//   2. row sums   in shared memory: G lanes per row (G = 1 sums a row
//                 sequentially in ascending storage order, which is the
//                 reference's order); long rows use a block reduction;
//   3. epilogue   one thread per row, consecutive rows on consecutive threads:
//                 the fused PDHG update (or an evaluation term) of the Op.
//
// The Op supplies the types, the gathered vectors, the staged vectors and the
// per-row epilogue; see pdfp_ops.cuh.  Evaluation Ops also reduce per-tile
// partial sums (FP64, fixed order) into a partials array.
#pragma once
#include "common.cuh"
#include "layout.hpp"

namespace pdfp {

// Where each region of a chunk lives inside a stage buffer.
template <int NVEC>
struct ChunkView {
    int32_t k0, k1, r0, r1, tile;
    bool last, single;  // single: tile is one (possibly multi-chunk) long row
    StageLayout lay;
    uint32_t sh_rp, sh_ci, sh_v, sh_vec;
};

template <int NVEC, int NV>
__device__ __forceinline__ ChunkView<NVEC> chunk_view(const SideDev& s, int32_t c, int esize_v,
                                                      int esize_vec, int esize_acc) {
    ChunkView<NVEC> cv;
    cv.k0 = s.chunk_k0[c];
    cv.k1 = s.chunk_k1[c];
    cv.tile = s.chunk_tile[c];
    const int32_t f = s.chunk_flags[c];
    cv.last = (f & CHUNK_LAST) != 0;
    cv.single = (f & CHUNK_LONG) != 0;
    cv.r0 = s.tile_row[cv.tile];
    cv.r1 = s.tile_row[cv.tile + 1];
    cv.lay = stage_layout(esize_v, esize_vec, esize_acc, NVEC, NV, cv.k0, cv.k1, cv.r0, cv.r1,
                          cv.last, cv.single);
    cv.sh_rp = window16_shift(cv.r0, 4);
    cv.sh_ci = window16_shift(cv.k0, 4);
    cv.sh_v = window16_shift(cv.k0, esize_v);
    cv.sh_vec = window16_shift(cv.r0, esize_vec);
    return cv;
}

template <class Op>
struct TileKernelSmem {
    static constexpr int NP = Op::NP > 0 ? Op::NP : 1;
    uint64_t bar[2];
    int32_t stage_chunk[2];
    int32_t flag;
    typename Op::AT long_acc[Op::NV];
    double red[(NP > 2 ? NP : 2) * (Op::NT / 32)];
};

// Issue the bulk copies of chunk c into stage buffer `buf` (one thread).
template <class Op>
__device__ __forceinline__ void issue_chunk(const SideDev& s, const Op& op, int32_t c,
                                            unsigned char* buf, uint64_t* bar) {
    using MT = typename Op::MT;
    using VT = typename Op::VT;
    using AT = typename Op::AT;
    const ChunkView<Op::NVEC> cv =
        chunk_view<Op::NVEC, Op::NV>(s, c, sizeof(MT), sizeof(VT), sizeof(AT));
    const uint32_t b_rp = (cv.last && !cv.single) ? window16_bytes(cv.r0, cv.r1 + 1, 4) : 0u;
    const uint32_t b_ci = window16_bytes(cv.k0, cv.k1, 4);
    const uint32_t b_v = window16_bytes(cv.k0, cv.k1, sizeof(MT));
    const uint32_t b_vec = (cv.last && Op::NVEC > 0) ? window16_bytes(cv.r0, cv.r1, sizeof(VT)) : 0u;
    const uint32_t bytes = b_rp + b_ci + b_v + b_vec * Op::NVEC;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(bar, bytes);
    if (b_rp)
        bulk_copy_g2s(buf + cv.lay.off_rp, s.rp + (cv.r0 - (int32_t)cv.sh_rp), b_rp, bar);
    if (b_ci)
        bulk_copy_g2s(buf + cv.lay.off_ci, s.ci + (cv.k0 - (int32_t)cv.sh_ci), b_ci, bar);
    if (b_v)
        bulk_copy_g2s(buf + cv.lay.off_v, op.values() + (cv.k0 - (int32_t)cv.sh_v), b_v, bar);
    if (b_vec) {
#pragma unroll
        for (int k = 0; k < Op::NVEC; ++k)
            bulk_copy_g2s(buf + cv.lay.off_vec0 + k * cv.lay.vec_stride,
                          op.staged(k) + (cv.r0 - (int32_t)cv.sh_vec), b_vec, bar);
    }
}

// Next chunk of this block's work list, skipping tiles of inactive instances.
// State (tile, chunk) lives in registers of thread 0.
struct WorkIter {
    int32_t tile, chunk, chunk_end;
};
template <class Op>
__device__ __forceinline__ int32_t next_chunk(const SideDev& s, const Op& op, WorkIter& it) {
    if (it.chunk < it.chunk_end) return it.chunk++;
    while (true) {
        it.tile += (it.tile < 0) ? (int32_t)blockIdx.x + 1 : (int32_t)gridDim.x;
        if (it.tile >= s.n_tiles) return -1;
        if (!op.active(s.tile_inst[it.tile])) continue;
        it.chunk = s.tile_chunk[it.tile];
        it.chunk_end = s.tile_chunk[it.tile + 1];
        if (it.chunk < it.chunk_end) return it.chunk++;
    }
}

template <class Op>
__global__ void __launch_bounds__(Op::NT) tile_spmv_kernel(const SideDev s, const Op op) {
    using MT = typename Op::MT;
    using VT = typename Op::VT;
    using AT = typename Op::AT;
    using GT = typename Op::GT;
    constexpr int NT = Op::NT, NV = Op::NV, NVEC = Op::NVEC, NP = Op::NP;
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    __shared__ TileKernelSmem<Op> sh;
    unsigned char* stage[2] = {dyn_smem, dyn_smem + s.stage_bytes};
    AT* rowsum = reinterpret_cast<AT*>(dyn_smem + 2 * (size_t)s.stage_bytes);  // [NV][max_rows]

    WorkIter it{-1, 0, 0};
    if (threadIdx.x == 0) {
        mbar_init(&sh.bar[0], 1);
        mbar_init(&sh.bar[1], 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int st = 0; st < 2; ++st) {
            int32_t c = next_chunk(s, op, it);
            sh.stage_chunk[st] = c;
            if (c >= 0) issue_chunk(s, op, c, stage[st], &sh.bar[st]);
        }
    }
    __syncthreads();

    uint32_t phase[2] = {0u, 0u};
    double acc[NP > 0 ? NP : 1];
#pragma unroll
    for (int j = 0; j < (NP > 0 ? NP : 1); ++j) acc[j] = 0.0;
    typename Op::TileP tp{};
    int32_t cur_tile = -1;

    for (uint32_t u = 0;; ++u) {
        const int st = u & 1;
        const int32_t c = sh.stage_chunk[st];
        if (c < 0) break;
        const bool ok = mbar_wait_bounded(&sh.bar[st], phase[st], op.err());
        phase[st] ^= 1u;
        if (__syncthreads_or(!ok)) break;  // a bulk copy never completed: give up (error recorded)

        unsigned char* buf = stage[st];
        const ChunkView<NVEC> cv = chunk_view<NVEC, NV>(s, c, sizeof(MT), sizeof(VT), sizeof(AT));
        const int32_t K = cv.k1 - cv.k0;
        const int32_t* ci_s = reinterpret_cast<const int32_t*>(buf + cv.lay.off_ci) + cv.sh_ci;
        MT* v_s = reinterpret_cast<MT*>(buf + cv.lay.off_v) + cv.sh_v;
        AT* p1 = reinterpret_cast<AT*>(v_s);  // products overwrite the values in place
        AT* p2 = reinterpret_cast<AT*>(buf + cv.lay.off_p2);
        const int32_t inst = s.tile_inst[cv.tile];
        if (cv.tile != cur_tile) {
            cur_tile = cv.tile;
            tp = op.tile_params(inst);
        }

        // 1. products
        if (NV > 0) {
            for (int32_t k = threadIdx.x; k < K; k += 4 * NT) {
                int32_t col[4];
                MT a[4];
                GT g[4][NV > 0 ? NV : 1];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int32_t kk = k + q * NT;
                    col[q] = kk < K ? ci_s[kk] : 0;
                    a[q] = kk < K ? v_s[kk] : MT(0);
                }
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (k + q * NT < K) op.gather(col[q], g[q]);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int32_t kk = k + q * NT;
                    if (kk < K) {
                        p1[kk] = mul_rn(static_cast<AT>(a[q]), static_cast<AT>(g[q][0]));
                        if (NV > 1) p2[kk] = mul_rn(static_cast<AT>(a[q]), static_cast<AT>(g[q][NV - 1]));
                    }
                }
            }
        }
        __syncthreads();

        // 2. row sums
        const int32_t R = cv.r1 - cv.r0;
        if (cv.single) {
            // one long row: block reduction over this chunk, accumulated over chunks
            double part[2] = {0.0, 0.0};
            for (int32_t k = threadIdx.x; k < K; k += NT) {
                part[0] += static_cast<double>(p1[k]);
                if (NV > 1) part[1] += static_cast<double>(p2[k]);
            }
            block_sum<NT, 2>(part, sh.red);
            if (threadIdx.x == 0) {
                const bool first = (c == s.tile_chunk[cv.tile]);
                sh.long_acc[0] = (first ? AT(0) : sh.long_acc[0]) + static_cast<AT>(part[0]);
                if (NV > 1) sh.long_acc[NV - 1] = (first ? AT(0) : sh.long_acc[NV - 1]) + static_cast<AT>(part[1]);
            }
        } else if (NV > 0) {
            const int32_t* rp_s = reinterpret_cast<const int32_t*>(buf + cv.lay.off_rp) + cv.sh_rp;
            int G = 1;
            while (G < 32 && G * 2 * R <= NT) G *= 2;
            const int groups = NT / G;
            const int gid = threadIdx.x / G, lane = threadIdx.x & (G - 1);
            for (int32_t base = 0; base < R; base += groups) {
                const int32_t rr = base + gid;
                AT s1 = AT(0), s2 = AT(0);
                if (rr < R) {
                    const int32_t e0 = rp_s[rr] - cv.k0, e1 = rp_s[rr + 1] - cv.k0;
                    for (int32_t k = e0 + lane; k < e1; k += G) {
                        s1 = add_rn(s1, p1[k]);
                        if (NV > 1) s2 = add_rn(s2, p2[k]);
                    }
                }
                for (int o = G >> 1; o > 0; o >>= 1) {
                    s1 = add_rn(s1, __shfl_xor_sync(0xffffffffu, s1, o));
                    if (NV > 1) s2 = add_rn(s2, __shfl_xor_sync(0xffffffffu, s2, o));
                }
                if (rr < R && lane == 0) {
                    rowsum[rr] = s1;
                    if (NV > 1) rowsum[s.max_tile_rows + rr] = s2;
                }
            }
        }

        // 3. epilogue on the tile's last chunk
        if (cv.last) {
            __syncthreads();
            const VT* sv[NVEC > 0 ? NVEC : 1];
#pragma unroll
            for (int k = 0; k < NVEC; ++k)
                sv[k] = reinterpret_cast<const VT*>(buf + cv.lay.off_vec0 + k * cv.lay.vec_stride) + cv.sh_vec;
            for (int32_t rr = threadIdx.x; rr < R; rr += NT) {
                AT sums[NV > 0 ? NV : 1];
                if (cv.single) {
#pragma unroll
                    for (int q = 0; q < NV; ++q) sums[q] = sh.long_acc[q];
                } else {
#pragma unroll
                    for (int q = 0; q < NV; ++q) sums[q] = rowsum[q * s.max_tile_rows + rr];
                }
                op.row(cv.r0 + rr, rr, inst, tp, sv, sums, acc);
            }
            if constexpr (NP > 0) {
                block_sum<NT, NP>(acc, sh.red);
                if (threadIdx.x == 0) op.write_partials(cv.tile, acc);
#pragma unroll
                for (int j = 0; j < (NP > 0 ? NP : 1); ++j) acc[j] = 0.0;
            }
        }
        __syncthreads();  // stage `st` fully consumed
        if (threadIdx.x == 0) {
            int32_t nc = next_chunk(s, op, it);
            sh.stage_chunk[st] = nc;
            if (nc >= 0) issue_chunk(s, op, nc, stage[st], &sh.bar[st]);
        }
        __syncthreads();
    }
}

}  // namespace pdfp
