// tile_spmv.cuh -- the sparse-product engine behind every pass of the solvers.
//
// One side of a matrix (A, or its explicit transpose A') is stored as CSR in
// the packed, permuted numbering of the handle (see layout.hpp).  Its rows are
// cut into TILES of whole rows whose data fit one shared-memory stage; a row
// too long for a stage gets a tile of its own, split into several CHUNKS.
//
// A persistent, warp-specialised kernel walks the tiles assigned to its block
// (round robin) with three roles and kStages shared-memory stages:
//
//   PRODUCER  (one lane of the last warp) issues, for each chunk, the
//             cp.async.bulk copies of the row pointers, column indices, values
//             and -- on a tile's last chunk -- the slices of the per-row vectors
//             the epilogue reads, completing on the stage's FULL mbarrier; it
//             waits on the stage's EMPTY mbarrier before reusing it.
//   GATHERERS (NT threads) each wait on FULL and compute their share of the
//             products p_k = a_k * g[col_k], thread-strided with up to sixteen
//             gathers in flight per thread (the gathered vector is L2-resident),
//             in place over the staged values; then each arrives on PROD (which
//             completes when all NT have).  No barrier joins them, so threads
//             drift up to kStages stages apart and gathers of several stages
//             overlap.
//   REDUCERS  (NRED threads: NT, or NT / 2 for FP32 steps) wait on PROD, sum
//             each row in shared memory (G lanes per row; G = 1 sums a row
//             sequentially in ascending storage order, which is the
//             reference's order; a long row uses a block
//             reduction accumulated over its chunks) and, on a tile's last
//             chunk, run the epilogue -- one thread per row, consecutive rows on
//             consecutive threads: the fused PDHG update (or an evaluation
//             term) of the Op; then arrive on EMPTY.
//
// So the gathers of one chunk are in flight while the rows of the previous one
// are reduced and updated.  The reducers synchronise among themselves with a
// named barrier; every wait is bounded.
//
// Back-to-back step launches may overlap (programmatic dependent launch): the
// producer reads only data no grid of the chain still writes -- the matrix, the
// per-row vectors last written two launches back, the instance states -- so it
// starts staging while the previous grid drains; gatherers and reducers first
// wait for the previous grid (griddepcontrol.wait).  The next grid is let in when
// every block's producer has staged its last chunk, after a wait of its own, so a
// launch never starts before the one two back is done.
//
// The Op supplies the types, the gathered vectors, the staged vectors and the
// per-row epilogue; see pdfp_ops.cuh.  Evaluation Ops also reduce per-tile
// partial sums (FP64, fixed order) into a partials array.
#pragma once
#include <type_traits>
#include <utility>

#include "common.cuh"
#include "layout.hpp"

namespace pdfp {

constexpr int kStages = 4;     // most shared-memory stages per block (SideDev::stages: 2..4)
constexpr int kReduceBar = 2;  // named barrier id of the reducer threads

// Where each region of a chunk lives inside a stage buffer.
struct ChunkView {
    ChunkDesc d;
    bool last, single;  // single: tile is one (possibly multi-chunk) long row
    StageLayout lay;
    uint32_t sh_rp, sh_ci, sh_v, sh_vec;
};

template <int NVEC, int NV>
__device__ __forceinline__ ChunkView chunk_view(const SideDev& s, int32_t c, int esize_v,
                                                int esize_vec, int esize_acc) {
    ChunkView cv;
    cv.d = s.chunks[c];
    cv.last = (cv.d.flags & CHUNK_LAST) != 0;
    cv.single = (cv.d.flags & CHUNK_LONG) != 0;
    cv.lay = stage_layout(esize_v, esize_vec, esize_acc, NVEC, NV, cv.d.k0, cv.d.k1, cv.d.r0,
                          cv.d.r1, cv.last, cv.single);
    cv.sh_rp = window16_shift(cv.d.r0, 4);
    cv.sh_ci = window16_shift(cv.d.k0, 4);
    cv.sh_v = window16_shift(cv.d.k0, esize_v);
    cv.sh_vec = window16_shift(cv.d.r0, esize_vec);
    return cv;
}

// Ops whose gathered vector can be fetched by per-thread async copies expose it as
// gather_src() and select that policy with gather_l2 == 2 (see the gatherers).
template <class Op, class = void>
struct HasGatherSrc : std::false_type {};
template <class Op>
struct HasGatherSrc<Op, std::void_t<decltype(std::declval<const Op&>().gather_src())>>
    : std::true_type {};

template <class Op>
constexpr bool kAsyncEligible = HasGatherSrc<Op>::value && sizeof(typename Op::MT) == 4 &&
                                sizeof(typename Op::AT) == 4 && Op::NV == 1;

// Ops that gather from a block-private copy in shared memory (after the stages and
// row sums; extra_smem() bytes) fill it in prologue(), run by the gatherers, which
// then meet at a named barrier before their first gather.
template <class Op, class = void>
struct HasPrologue : std::false_type {};
template <class Op>
struct HasPrologue<Op, std::void_t<decltype(std::declval<const Op&>().prologue(0, 0))>>
    : std::true_type {};
constexpr int kGatherBar = 3;  // named barrier id of the gatherer threads

template <class Op>
struct TileKernelSmem {
    static constexpr int NP = Op::NP > 0 ? Op::NP : 1;
    uint64_t full[kStages];
    uint64_t prod[kStages];
    uint64_t empty[kStages];
    int32_t stage_chunk[kStages];
    int32_t flag;
    typename Op::AT long_acc[Op::NV > 0 ? Op::NV : 1];
    double red[(NP > 2 ? NP : 2) * (Op::NT / 32)];  // sized for up to Op::NT reducers
};

// Issue the bulk copies of chunk c into stage buffer `buf` (producer lane).
template <class Op>
__device__ __forceinline__ void issue_chunk(const SideDev& s, const Op& op, int32_t c,
                                            unsigned char* buf, uint64_t* bar, uint64_t policy) {
    using MT = typename Op::MT;
    using VT = typename Op::VT;
    using AT = typename Op::AT;
    const ChunkView cv = chunk_view<Op::NVEC, Op::NV>(s, c, sizeof(MT), sizeof(VT), sizeof(AT));
    const int32_t k0 = cv.d.k0, k1 = cv.d.k1, r0 = cv.d.r0, r1 = cv.d.r1;
    const uint32_t b_rp = (cv.last && !cv.single) ? window16_bytes(r0, r1 + 1, 4) : 0u;
    const uint32_t b_ci = window16_bytes(k0, k1, 4);
    const uint32_t b_v = window16_bytes(k0, k1, sizeof(MT));
    const uint32_t b_vec = (cv.last && Op::NVEC > 0) ? window16_bytes(r0, r1, sizeof(VT)) : 0u;
    const uint32_t bytes = b_rp + b_ci + b_v + b_vec * Op::NVEC;
    mbar_arrive_expect_tx(bar, bytes);
    // the matrix streams through once per launch; with s.evict_first its lines leave
    // L2 first, so the gathered vector and the iterates stay resident
    if (s.evict_first) {
        if (b_rp) bulk_copy_g2s_hint(buf + cv.lay.off_rp, s.rp + (r0 - (int32_t)cv.sh_rp), b_rp, bar, policy);
        if (b_ci) bulk_copy_g2s_hint(buf + cv.lay.off_ci, s.ci + (k0 - (int32_t)cv.sh_ci), b_ci, bar, policy);
        if (b_v) bulk_copy_g2s_hint(buf + cv.lay.off_v, op.values() + (k0 - (int32_t)cv.sh_v), b_v, bar, policy);
    } else {
        if (b_rp) bulk_copy_g2s(buf + cv.lay.off_rp, s.rp + (r0 - (int32_t)cv.sh_rp), b_rp, bar);
        if (b_ci) bulk_copy_g2s(buf + cv.lay.off_ci, s.ci + (k0 - (int32_t)cv.sh_ci), b_ci, bar);
        if (b_v) bulk_copy_g2s(buf + cv.lay.off_v, op.values() + (k0 - (int32_t)cv.sh_v), b_v, bar);
    }
    if (b_vec) {
#pragma unroll
        for (int k = 0; k < Op::NVEC; ++k)
            bulk_copy_g2s(buf + cv.lay.off_vec0 + k * cv.lay.vec_stride,
                          op.staged(k) + (r0 - (int32_t)cv.sh_vec), b_vec, bar);
    }
}

// Next chunk of this block's work list, skipping tiles of inactive instances.
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

// ASYNC (a separate instantiation, so the register-gather path keeps its own register
// budget): the gatherers fetch by per-thread async copies; eligible Ops only.
// NRED: reducer threads (a multiple of 32, at most Op::NT); the gatherers are Op::NT.
template <class Op, bool ASYNC = false, int NRED = Op::NT>
__global__ void __launch_bounds__(Op::NT + NRED + 32) tile_spmv_kernel(const SideDev s, const Op op) {
    using MT = typename Op::MT;
    using VT = typename Op::VT;
    using AT = typename Op::AT;
    using GT = typename Op::GT;
    constexpr int NT = Op::NT, NV = Op::NV, NVEC = Op::NVEC, NP = Op::NP;
    constexpr int NR = NRED;
    static_assert(NR % 32 == 0 && NR <= NT, "reducers: a multiple of 32, at most the gatherers");
    constexpr int UNROLL = sizeof(MT) == 4 ? 16 : 8;  // scalar path: gathers in flight per thread
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    __shared__ TileKernelSmem<Op> sh;
    const int NS = s.stages;  // stages in use
    AT* rowsum = reinterpret_cast<AT*>(dyn_smem + NS * (size_t)s.stage_bytes);  // [NV][max_rows]

    if (threadIdx.x == 0) {
        for (int i = 0; i < kStages; ++i) {
            mbar_init(&sh.full[i], 1);
            mbar_init(&sh.prod[i], Op::NT);  // every gatherer arrives
            mbar_init(&sh.empty[i], 1);
        }
        sh.flag = 0;
        fence_barrier_init();
    }
    __syncthreads();

    if (threadIdx.x >= NT + NR) {
        // ---- producer: one lane walks the work list and issues the copies ----
        if (threadIdx.x == NT + NR) {
            const uint64_t policy = l2_policy_evict_first();
            WorkIter it{-1, 0, 0};
            for (uint32_t u = 0;; ++u) {
                const int st = u % NS;
                if (u >= (uint32_t)NS &&
                    !mbar_wait_bounded(&sh.empty[st], ((u / NS) - 1) & 1u, op.err())) {
                    sh.flag = 1;  // the stage was never released: stop feeding
                    sh.stage_chunk[st] = -1;
                    mbar_arrive(&sh.full[st]);
                    break;
                }
                const int32_t c = next_chunk(s, op, it);
                sh.stage_chunk[st] = c;
                if (c < 0) {
                    mbar_arrive(&sh.full[st]);  // completes the phase: the end of the work
                    // this block has staged all its work: the next grid may be
                    // scheduled once every block got here (after this grid's own wait)
                    griddep_wait();
                    griddep_launch_dependents();
                    break;
                }
                issue_chunk(s, op, c, dyn_smem + st * (size_t)s.stage_bytes, &sh.full[st], policy);
            }
        }
        return;
    }

    constexpr bool async = ASYNC && kAsyncEligible<Op>;
    if (threadIdx.x < NT) {
        // ---- gatherers: products of each chunk, in place over its values ----
        const int g = threadIdx.x;
        griddep_wait();  // the gathered vector comes from the previous grid
        if constexpr (HasPrologue<Op>::value) {
            op.prologue(g, NT);
            named_sync(kGatherBar, NT);
        }
        for (uint32_t u = 0;; ++u) {
            const int st = u % NS;
            // Each gatherer waits and arrives on its own: with no barrier among them a
            // thread whose gathers have landed runs ahead into the next stages while
            // slower gathers of the previous one are still in flight.
            const bool ok = mbar_wait_bounded(&sh.full[st], (u / NS) & 1u, op.err());
            if (!ok) sh.flag = 1;
            const int32_t c = ok ? sh.stage_chunk[st] : -1;
            if (c >= 0 && NV > 0) {
                unsigned char* buf = dyn_smem + st * (size_t)s.stage_bytes;
                const ChunkView cv = chunk_view<NVEC, NV>(s, c, sizeof(MT), sizeof(VT), sizeof(AT));
                const int32_t K = cv.d.k1 - cv.d.k0;
                if constexpr (sizeof(MT) == 4 && sizeof(AT) == 4 && NV == 1) {
                    // 32-bit values: the index and value windows start 16-byte
                    // aligned with the same shift, so each thread takes four
                    // consecutive nonzeros with 128-bit shared loads and stores
                    const int32_t sh0 = static_cast<int32_t>(cv.sh_ci);
                    const int4* ci4 = reinterpret_cast<const int4*>(buf + cv.lay.off_ci);
                    float4* v4 = reinterpret_cast<float4*>(buf + cv.lay.off_v);
                    const int32_t quads = (sh0 + K + 3) >> 2;
                    constexpr int QH = 4;  // quads per thread per pass: 16 gathers in flight
                    if constexpr (async) {
                        // async policy: each gathered entry is copied (cp.async, 4 bytes)
                        // over its own column index in the stage, and the products are
                        // left to the reducers; no register waits on the gathers, whose
                        // completion arrives on PROD by itself
                        {
                            const GT* src = op.gather_src();
                            const uint32_t ci_base = smem_addr(buf + cv.lay.off_ci);
                            for (int32_t q0 = g; q0 < quads; q0 += QH * NT) {
                                int4 cc[QH];
#pragma unroll
                                for (int h = 0; h < QH; ++h)
                                    if (q0 + h * NT < quads) cc[h] = ci4[q0 + h * NT];
#pragma unroll
                                for (int h = 0; h < QH; ++h) {
                                    const int32_t q = q0 + h * NT;
                                    if (q < quads) {
                                        const int32_t e = 4 * q - sh0;
                                        const int cols[4] = {cc[h].x, cc[h].y, cc[h].z, cc[h].w};
#pragma unroll
                                        for (int j = 0; j < 4; ++j)
                                            if (e + j >= 0 && e + j < K)
                                                cp_async_4(ci_base + 16u * q + 4u * j, src + cols[j]);
                                    }
                                }
                            }
                        }
                    } else
                    for (int32_t q0 = g; q0 < quads; q0 += QH * NT) {
                        int4 cc[QH];
                        GT gv[QH][4][1];
#pragma unroll
                        for (int h = 0; h < QH; ++h) {
                            const int32_t q = q0 + h * NT;
                            if (q < quads) cc[h] = ci4[q];
                        }
#pragma unroll
                        for (int h = 0; h < QH; ++h) {
                            const int32_t q = q0 + h * NT;
                            if (q < quads) {
                                const int32_t e = 4 * q - sh0;  // nonzero index of the quad's first lane
                                const int cols[4] = {cc[h].x, cc[h].y, cc[h].z, cc[h].w};
#pragma unroll
                                for (int j = 0; j < 4; ++j)
                                    if (e + j >= 0 && e + j < K) op.gather(cols[j], gv[h][j]);
                            }
                        }
#pragma unroll
                        for (int h = 0; h < QH; ++h) {
                            const int32_t q = q0 + h * NT;
                            if (q < quads) {
                                // the values are read only now, after the gathers were
                                // issued: fewer registers live across their latency
                                const int32_t e = 4 * q - sh0;
                                const float4 a = v4[q];
                                float4 p = a;
                                if (e + 0 >= 0 && e + 0 < K) p.x = mul_rn(static_cast<float>(a.x), static_cast<float>(gv[h][0][0]));
                                if (e + 1 >= 0 && e + 1 < K) p.y = mul_rn(static_cast<float>(a.y), static_cast<float>(gv[h][1][0]));
                                if (e + 2 >= 0 && e + 2 < K) p.z = mul_rn(static_cast<float>(a.z), static_cast<float>(gv[h][2][0]));
                                if (e + 3 >= 0 && e + 3 < K) p.w = mul_rn(static_cast<float>(a.w), static_cast<float>(gv[h][3][0]));
                                v4[q] = p;
                            }
                        }
                    }
                } else {
                    const int32_t* ci_s = reinterpret_cast<const int32_t*>(buf + cv.lay.off_ci) + cv.sh_ci;
                    MT* v_s = reinterpret_cast<MT*>(buf + cv.lay.off_v) + cv.sh_v;
                    AT* p1 = reinterpret_cast<AT*>(v_s);
                    AT* p2 = reinterpret_cast<AT*>(buf + cv.lay.off_p2);
                    // one gathered vector: the values are read only after the gathers
                    // are issued (fewer registers live across their latency); two: the
                    // values first (the other order spills in the evaluation kernels)
                    constexpr bool kLate = NV == 1;
                    for (int32_t k = g; k < K; k += UNROLL * NT) {
                        int32_t col[UNROLL];
                        MT a[kLate ? 1 : UNROLL];
                        GT gv[UNROLL][NV > 0 ? NV : 1];
#pragma unroll
                        for (int q = 0; q < UNROLL; ++q) {
                            const int32_t kk = k + q * NT;
                            col[q] = kk < K ? ci_s[kk] : 0;
                            if constexpr (!kLate) a[q] = kk < K ? v_s[kk] : MT(0);
                        }
#pragma unroll
                        for (int q = 0; q < UNROLL; ++q)
                            if (k + q * NT < K) op.gather(col[q], gv[q]);
#pragma unroll
                        for (int q = 0; q < UNROLL; ++q) {
                            const int32_t kk = k + q * NT;
                            if (kk < K) {
                                const MT av = kLate ? v_s[kk] : a[kLate ? 0 : q];
                                p1[kk] = mul_rn(static_cast<AT>(av), static_cast<AT>(gv[q][0]));
                                if (NV > 1)
                                    p2[kk] = mul_rn(static_cast<AT>(av), static_cast<AT>(gv[q][NV > 1 ? NV - 1 : 0]));
                            }
                        }
                    }
                }
            }
            if (async && c >= 0)
                cp_async_arrive_noinc(&sh.prod[st]);  // arrives once this thread's copies land
            else
                mbar_arrive(&sh.prod[st]);  // this thread's products of the stage are in place
            if (c < 0) break;
        }
        if constexpr (async) cp_async_wait_all();
        return;
    }

    // ---- reducers: row sums and the epilogue ----
    const int r = threadIdx.x - NT;
    griddep_wait();  // the epilogue writes what the previous grid may still read
    double acc[NP > 0 ? NP : 1];
#pragma unroll
    for (int j = 0; j < (NP > 0 ? NP : 1); ++j) acc[j] = 0.0;
    typename Op::TileP tp{};
    int32_t cur_tile = -1;

    for (uint32_t u = 0;; ++u) {
        const int st = u % NS;
        if (!group_wait(&sh.prod[st], (u / NS) & 1u, op.err(), r == 0, kReduceBar, NR, &sh.flag))
            break;  // a wait gave up (error recorded)
        const int32_t c = sh.stage_chunk[st];
        if (c < 0) break;

        unsigned char* buf = dyn_smem + st * (size_t)s.stage_bytes;
        const ChunkView cv = chunk_view<NVEC, NV>(s, c, sizeof(MT), sizeof(VT), sizeof(AT));
        const int32_t K = cv.d.k1 - cv.d.k0;
        const AT* p1 = reinterpret_cast<const AT*>(reinterpret_cast<MT*>(buf + cv.lay.off_v) + cv.sh_v);
        const AT* p2 = reinterpret_cast<const AT*>(buf + cv.lay.off_p2);
        // product k of the first gathered vector: in place over the values, or -- async
        // policy -- the value times the gathered entry that replaced its column index
        const AT* g1 = reinterpret_cast<const AT*>(reinterpret_cast<const int32_t*>(buf + cv.lay.off_ci) + cv.sh_ci);
        auto prod1 = [&](int32_t k) -> AT {
            if constexpr (async) return mul_rn(p1[k], g1[k]);
            else return p1[k];
        };
        const int32_t inst = cv.d.inst;
        if (cv.d.tile != cur_tile) {
            cur_tile = cv.d.tile;
            tp = op.tile_params(inst);
        }

        // row sums
        const int32_t R = cv.d.r1 - cv.d.r0;
        if (cv.single) {
            // one long row: block reduction over this chunk, accumulated over chunks
            double part[2] = {0.0, 0.0};
            for (int32_t k = r; k < K; k += NR) {
                part[0] += static_cast<double>(prod1(k));
                if (NV > 1) part[1] += static_cast<double>(p2[k]);
            }
            block_sum<NR, 2, kReduceBar>(part, sh.red, r);
            if (r == 0) {
                const bool first = cv.d.first != 0;
                sh.long_acc[0] = (first ? AT(0) : sh.long_acc[0]) + static_cast<AT>(part[0]);
                if (NV > 1) sh.long_acc[NV - 1] = (first ? AT(0) : sh.long_acc[NV - 1]) + static_cast<AT>(part[1]);
            }
        } else if (NV > 0) {
            const int32_t* rp_s = reinterpret_cast<const int32_t*>(buf + cv.lay.off_rp) + cv.sh_rp;
            int G = 1;
            while (G < 32 && G * 2 * R <= NR) G *= 2;
            const int groups = NR / G;
            const int gid = r / G, lane = r & (G - 1);
            for (int32_t base = 0; base < R; base += groups) {
                const int32_t rr = base + gid;
                AT s1 = AT(0), s2 = AT(0);
                if (rr < R) {
                    const int32_t e0 = rp_s[rr] - cv.d.k0, e1 = rp_s[rr + 1] - cv.d.k0;
                    for (int32_t k = e0 + lane; k < e1; k += G) {
                        s1 = add_rn(s1, prod1(k));
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

        // epilogue on the tile's last chunk
        if (cv.last) {
            named_sync(kReduceBar, NR);
            const VT* sv[NVEC > 0 ? NVEC : 1];
#pragma unroll
            for (int k = 0; k < NVEC; ++k)
                sv[k] = reinterpret_cast<const VT*>(buf + cv.lay.off_vec0 + k * cv.lay.vec_stride) + cv.sh_vec;
            for (int32_t rr = r; rr < R; rr += NR) {
                AT sums[NV > 0 ? NV : 1];
                if (cv.single) {
#pragma unroll
                    for (int q = 0; q < NV; ++q) sums[q] = sh.long_acc[q];
                } else {
#pragma unroll
                    for (int q = 0; q < NV; ++q) sums[q] = rowsum[q * s.max_tile_rows + rr];
                }
                op.row(cv.d.r0 + rr, rr, inst, tp, sv, sums, acc);
            }
            if constexpr (NP > 0) {
                block_sum<NR, NP, kReduceBar>(acc, sh.red, r);
                if (r == 0) op.write_partials(cv.d.tile, acc);
#pragma unroll
                for (int j = 0; j < NP; ++j) acc[j] = 0.0;
            }
        }
        named_sync(kReduceBar, NR);  // stage `st` fully consumed
        if (r == 0) {
            fence_proxy_async_smem();  // generic-proxy writes (products) before the next bulk copy
            mbar_arrive(&sh.empty[st]);
        }
    }
}

}  // namespace pdfp
