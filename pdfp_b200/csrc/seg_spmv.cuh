// seg_spmv.cuh -- the FP32 step passes with the gathered vector in cluster shared memory.
//
// A step pass multiplies one side of the matrix (A, or A') by a vector it gathers
// at random (x_bar, or z).  On a matrix with scattered column indices the tile
// engine's gathers go to L2 one 32-byte sector each, and their rate, not HBM,
// bounds the pass.  This engine keeps the gathered vector in the shared memory of
// a thread-block cluster instead and reads it with ld.shared::cluster:
//
//   * the columns are cut into SEGMENTS of kSegQ * SL entries; a cluster of kSegQ
//     CTAs holds one segment at a time, SL entries per CTA, double-buffered: while
//     the CTAs work on segment s, each one's slice of segment s + 1 arrives by a
//     bulk copy (cp.async.bulk, global -> its own shared memory, no multicast);
//   * every CTA owns a contiguous range of rows (balanced by nonzeros) and, per
//     segment, streams the nonzeros of its rows that fall in the segment -- a
//     32-bit key (row in the CTA << 17 | column in the segment) and an FP32 value,
//     stored segment-major per CTA and sorted by (row, column) within a segment --
//     gathering each product's vector entry from the cluster's shared memory;
//   * row sums accumulate in the CTA's shared memory across the segments: a warp
//     takes 32 consecutive nonzeros, sums each row's run by a segmented shuffle
//     scan, and the one window where a row starts adds its run directly while the
//     windows that continue it leave partials that a second pass adds in window
//     order -- so the result does not depend on timing (no atomics);
//   * after the last segment each CTA runs the Op's per-row epilogue (the fused
//     PDHG update) on its rows, reading the per-row vectors from global memory.
//
// One cluster barrier per segment orders everything: when it completes, every
// CTA's slice of segment s is in place and every CTA is done with segment s - 1,
// whose buffer then receives segment s + 1.  Waits on the bulk copies are bounded
// (an error word, as in the tile engine); the cluster barrier is the hardware's.
// No load reads another GPU's memory, and none uses multicast.
#pragma once
#include <type_traits>

#include "common.cuh"

namespace pdfp {

constexpr int kSegQ = 8;          // CTAs per cluster (the portable cluster size)
constexpr int kSegColBits = 17;   // column-in-segment bits of a key
constexpr int kSegThreads = 512;  // threads per CTA

// One side of the matrix in the segmented layout (device view).
struct SegDev {
    int32_t G;       // CTAs (a multiple of kSegQ)
    int32_t S;       // segments
    int32_t sl_log;  // log2 of each CTA's slice of a segment (vector entries)
    int32_t rmax;    // most rows of one CTA
    int32_t wmax;    // most 32-nonzero windows of one (CTA, segment) chunk
    int32_t ncols;   // length of the gathered vector
    const int32_t* row_start;  // G + 1: the CTAs' row ranges (packed numbering)
    const int32_t* chunk_off;  // G * S + 1: nonzeros of CTA g in segment s
    const uint32_t* key;       // row in the CTA << kSegColBits | column in the segment
    const float* val;
};

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ uint32_t cluster_cta_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// The shared-memory address `a` (this CTA's) as seen in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t map_shared_rank(uint32_t a, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}
__device__ __forceinline__ float ld_shared_cluster(uint32_t a) {
    float v;
    asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(a) : "memory");
    return v;
}

// Dynamic shared memory of a launch: two slices, the row sums, the window partials.
inline size_t seg_smem_bytes(int sl_log, int rmax, int wmax) {
    return sizeof(float) * (2 * (size_t(1) << sl_log) + static_cast<size_t>(rmax) + static_cast<size_t>(wmax));
}

template <class Op, int SL_LOG>
__global__ void __launch_bounds__(kSegThreads) seg_spmv_kernel(const SegDev s, const Op op) {
    static_assert(std::is_same<typename Op::AT, float>::value && std::is_same<typename Op::MT, float>::value &&
                      Op::NV == 1,
                  "the segmented engine runs FP32 steps with one gathered vector");
    constexpr int SL = 1 << SL_LOG;
    constexpr int SEG = kSegQ * SL;
    static_assert(SEG <= (1 << kSegColBits), "a segment's columns must fit the key");
    constexpr int NT = kSegThreads, NW = NT / 32;
    extern __shared__ __align__(128) float seg_sm[];
    float* xb[2] = {seg_sm, seg_sm + SL};
    float* acc = seg_sm + 2 * SL;
    float* side = acc + s.rmax;
    __shared__ uint64_t bar[2];
    if (!op.active(0)) return;  // one instance: the same on every CTA of the grid

    const int g = blockIdx.x;
    const uint32_t rank = cluster_cta_rank();
    const int32_t ra = s.row_start[g], rows = s.row_start[g + 1] - ra;
    const float* vec = op.gather_src();
    for (int32_t i = threadIdx.x; i < rows; i += NT) acc[i] = 0.f;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_barrier_init();
    }
    __syncthreads();
    // this CTA's slice of segment `seg` into buffer seg & 1 (rounded up to 16 bytes;
    // every vector is padded by 64 bytes)
    auto issue = [&](int seg) {
        const int64_t lo = static_cast<int64_t>(seg) * SEG + static_cast<int64_t>(rank) * SL;
        int64_t cnt = static_cast<int64_t>(s.ncols) - lo;
        cnt = cnt < 0 ? 0 : (cnt > SL ? SL : cnt);
        const uint32_t bytes = static_cast<uint32_t>((cnt * 4 + 15) & ~int64_t(15));
        if (bytes) {
            mbar_arrive_expect_tx(&bar[seg & 1], bytes);
            bulk_copy_g2s(xb[seg & 1], vec + lo, bytes, &bar[seg & 1]);
        } else {
            mbar_arrive(&bar[seg & 1]);
        }
    };
    if (threadIdx.x == 0) issue(0);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int seg = 0; seg < s.S; ++seg) {
        if (threadIdx.x == 0) mbar_wait_bounded(&bar[seg & 1], (seg >> 1) & 1, op.err());
        __syncthreads();
        cluster_sync_all();  // every CTA's slice of `seg` is in place; all are done with seg - 1
        if (threadIdx.x == 0 && seg + 1 < s.S) {
            fence_proxy_async_smem();  // this CTA's reads of the old buffer before the copy over it
            issue(seg + 1);
        }
        const uint32_t base = smem_addr(xb[seg & 1]);
        const int32_t k0 = s.chunk_off[g * s.S + seg], k1 = s.chunk_off[g * s.S + seg + 1];
        for (int32_t w = k0 + warp * 32; w < k1; w += NW * 32) {
            const int32_t k = w + lane;
            const bool valid = k < k1;
            const uint32_t kk = valid ? __ldcs(s.key + k) : 0xFFFFFFFFu;
            float p = 0.f;
            if (valid) {
                const float a = __ldcs(s.val + k);
                const uint32_t col = kk & ((1u << kSegColBits) - 1u);
                p = mul_rn(a, ld_shared_cluster(map_shared_rank(base + 4u * (col & (SL - 1)), col >> SL_LOG)));
            }
            // segmented inclusive scan over the lanes of each row's run (rows ascend)
            const uint32_t row = kk >> kSegColBits;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const float t = __shfl_up_sync(0xffffffffu, p, d);
                const uint32_t tr = __shfl_up_sync(0xffffffffu, row, d);
                if (lane >= d && tr == row) p = add_rn(t, p);
            }
            const uint32_t next = __shfl_down_sync(0xffffffffu, row, 1);
            const uint32_t row0 = __shfl_sync(0xffffffffu, row, 0);
            if (valid && (lane == 31 || next != row)) {
                // the run of lane 0 continues a row of the previous window: a partial
                const bool cont = row == row0 && w > k0 && (__ldg(s.key + w - 1) >> kSegColBits) == row0;
                if (cont) side[(w - k0) >> 5] = p;
                else acc[row] = add_rn(acc[row], p);
            }
        }
        __syncthreads();
        // the continuing windows' partials, added in window order, one thread per row run
        const int32_t nwin = (k1 - k0 + 31) >> 5;
        for (int32_t wi = 1 + threadIdx.x; wi < nwin; wi += NT) {
            const int32_t ws = k0 + wi * 32;
            const uint32_t r0 = __ldg(s.key + ws) >> kSegColBits;
            if ((__ldg(s.key + ws - 1) >> kSegColBits) != r0) continue;  // the window starts a row
            if (wi >= 2 && (__ldg(s.key + ws - 32) >> kSegColBits) == r0 &&
                (__ldg(s.key + ws - 33) >> kSegColBits) == r0)
                continue;  // an earlier window of the same run adds this one
            float t = side[wi];
            for (int32_t wj = wi + 1; wj < nwin; ++wj) {
                const int32_t vs = k0 + wj * 32;
                if ((__ldg(s.key + vs) >> kSegColBits) != r0 || (__ldg(s.key + vs - 1) >> kSegColBits) != r0)
                    break;
                t = add_rn(t, side[wj]);
            }
            acc[r0] = add_rn(acc[r0], t);
        }
        // the next segment's cluster barrier orders these adds before its direct ones
    }
    __syncthreads();
    // the Op's per-row epilogue on this CTA's rows (consecutive rows, consecutive threads)
    using VT = typename Op::VT;
    constexpr int NVEC = Op::NVEC;
    const VT* sv[NVEC > 0 ? NVEC : 1];
#pragma unroll
    for (int k = 0; k < NVEC; ++k) sv[k] = op.staged(k) + ra;
    const typename Op::TileP tp = op.tile_params(0);
    double none[1] = {0.0};
    for (int32_t rr = threadIdx.x; rr < rows; rr += NT) {
        const float sums[1] = {acc[rr]};
        op.row(ra + rr, rr, 0, tp, sv, sums, none);
    }
    cluster_sync_all();  // no CTA leaves while its peers may still read its slices
}

}  // namespace pdfp
