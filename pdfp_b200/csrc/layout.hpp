// layout.hpp -- how a batch of problems is laid out in HBM.
//
// K instances are packed block-diagonally: instance p owns packed rows
// [row_off[p], row_off[p+1]) and packed columns [col_off[p], col_off[p+1]).
// Within an instance, rows are permuted so that equality rows come first (the
// row kernel tests `local_row < n_eq` instead of reading a flag vector) and
// each group is ordered by decreasing length; columns are ordered by decreasing
// length.  Inside every CSR row the nonzeros keep the caller's ascending
// ORIGINAL index order, so sequential row sums add terms in the reference's
// order (Julia's CSC mul!).
//
// Both A (rows i) and an explicit A' (rows = columns j) are stored: int32
// row pointers and column indices, FP64 values, and FP32 values for the mixed
// precision iterations.  Each side is cut into tiles (see tile_spmv.cuh) once
// per stage geometry.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#ifdef __CUDACC__
#define PDFP_HD __host__ __device__
#else
#define PDFP_HD
#endif

namespace pdfp {

enum : int32_t { CHUNK_LAST = 1, CHUNK_LONG = 2 };

// Byte size of the 16-byte-aligned window covering elements [e0, e1) of an
// array with `esize`-byte elements (0 for an empty range), and the number of
// elements between the window start and e0.
PDFP_HD inline uint32_t window16_bytes(int64_t e0, int64_t e1, int esize) {
    if (e1 <= e0) return 0;
    const int64_t b0 = (e0 * esize) & ~int64_t(15);
    const int64_t b1 = (e1 * esize + 15) & ~int64_t(15);
    return static_cast<uint32_t>(b1 - b0);
}
PDFP_HD inline uint32_t window16_shift(int64_t e0, int esize) {
    return static_cast<uint32_t>(((e0 * esize) & int64_t(15)) / esize);
}
PDFP_HD inline uint32_t align128(uint32_t b) { return (b + 127u) & ~127u; }

// Offsets of the regions of one chunk inside a shared-memory stage: row
// pointers (last chunk of a multi-row tile), column indices, values, the
// second product array (nv > 1), and nvec staged per-row vector slices (last
// chunk only).  This one function sizes tiles on the host and lays out the
// stage in the kernel.
struct StageLayout {
    uint32_t off_rp, off_ci, off_v, off_p2, off_vec0, vec_stride, total;
};
PDFP_HD inline StageLayout stage_layout(int esize_v, int esize_vec, int esize_acc, int nvec, int nv,
                                        int64_t k0, int64_t k1, int64_t r0, int64_t r1, bool last,
                                        bool single) {
    StageLayout s;
    uint32_t off = 0;
    s.off_rp = 0;
    if (last && !single) off += align128(window16_bytes(r0, r1 + 1, 4));
    s.off_ci = off;
    off += align128(window16_bytes(k0, k1, 4));
    s.off_v = off;
    off += align128(window16_bytes(k0, k1, esize_v));
    s.off_p2 = off;
    if (nv > 1) off += align128(static_cast<uint32_t>((k1 - k0) * esize_acc));
    s.off_vec0 = off;
    s.vec_stride = (last && nvec > 0) ? align128(window16_bytes(r0, r1, esize_vec)) : 0u;
    off += s.vec_stride * static_cast<uint32_t>(nvec > 0 ? nvec : 0);
    s.total = off;
    return s;
}

// Everything a kernel needs to know about one chunk, in one 32-byte load.
struct alignas(32) ChunkDesc {
    int32_t k0, k1;  // nonzero range of the chunk
    int32_t r0, r1;  // rows of its tile
    int32_t tile, inst, flags, first;  // first: this is the tile's first chunk
};

// Device view of one side of the matrix plus one tiling of it.
struct SideDev {
    int32_t rows;
    int32_t n_tiles, n_chunks, max_tile_rows, stage_bytes;
    int32_t stages = 4;  // shared-memory stages per block of the tile engine (2..4)
    int32_t evict_first = 0;  // tile engine: stream the matrix under an L2 evict-first policy
    const int32_t* rp;
    const int32_t* ci;
    const int32_t* tile_row;     // n_tiles + 1
    const int32_t* tile_chunk;   // n_tiles + 1: first chunk of each tile
    const int32_t* tile_inst;    // n_tiles
    const ChunkDesc* chunks;     // n_chunks
};

// Sizes of what one chunk stages (must match chunk_view in tile_spmv.cuh).
struct StageGeom {
    int esize_v;    // matrix value bytes
    int esize_vec;  // staged per-row vector element bytes
    int esize_acc;  // accumulator bytes
    int nvec;       // staged per-row vectors
    int nv;         // simultaneous products (gathered vectors)
    int32_t stage_bytes;
    int32_t max_rows;  // cap on rows per tile
};

inline uint32_t chunk_stage_bytes(const StageGeom& g, int64_t k0, int64_t k1, int64_t r0,
                                  int64_t r1, bool last, bool single) {
    return stage_layout(g.esize_v, g.esize_vec, g.esize_acc, g.nvec, g.nv, k0, k1, r0, r1, last,
                        single)
        .total;
}

struct HostCsr {
    int32_t rows = 0, cols = 0;
    std::vector<int32_t> rp, ci;
    std::vector<double> v;
};

struct HostTiling {
    std::vector<int32_t> tile_row, tile_chunk, tile_inst, chunk_k0, chunk_k1, chunk_tile,
        chunk_flags;
    std::vector<int32_t> tile_row_end;  // n_tiles: one past each tile's last row
    std::vector<int32_t> inst_tile0;  // K + 1: tiles of instance p are [inst_tile0[p], inst_tile0[p+1])
    int32_t max_tile_rows = 1;
    StageGeom geom{};
};

// Tiles of whole rows in row order; rows with (*skip)[r] != 0 are left out (their
// neighbours then fall in different tiles, so only the tile engine, which reads
// each chunk's row range, may run a tiling with skipped rows).
void build_tiling(const HostCsr& csr, const std::vector<int32_t>& inst_row_off,
                  const StageGeom& g, HostTiling& t, const std::vector<uint8_t>* skip = nullptr);

// Caps of the flat step engine (flat_spmv.cuh): a multi-row tile holds at most
// kFlatMaxRows rows and its nonzeros, counted from the 4-aligned element below
// the first, at most `cap` (1024 or kFlatCapMax, the engine's two variants).
constexpr int kFlatCapMax = 2048;
constexpr int kFlatMaxRows = 256;

// Stage size handed to the tiler for the flat engine: with at least one
// 128-byte block for the row pointers, the 16-byte window of the column
// indices can take at most 4 * cap bytes, the values' window correspondingly
// (checked on every tiling by flat_tiling_fits).
inline int32_t flat_stage_bytes(int esize_v, int cap) {
    return static_cast<int32_t>(128u + 4u * cap + align128(static_cast<uint32_t>(esize_v) * cap));
}

inline bool flat_tiling_fits(const HostTiling& t, int cap) {
    const size_t nt = t.tile_inst.size();
    for (size_t i = 0; i < nt; ++i) {
        const int32_t c = t.tile_chunk[i];
        if (t.chunk_flags[c] & CHUNK_LONG) continue;
        if (t.tile_chunk[i + 1] != c + 1 || t.tile_row[i + 1] - t.tile_row[i] > kFlatMaxRows ||
            t.chunk_k1[c] - (t.chunk_k0[c] & ~3) > cap)
            return false;
    }
    return true;
}

// Work items of the vec step engine (vec_spmv.cuh), one warp each.  lg >= 0:
// rows [r0, r1) of instance `inst` with 2^lg lanes per row.  lg = -1: the
// nonzeros [k0, k1) of long row r0, piece `slot - r1` of its `np` pieces, whose
// FP64 partial sums occupy slots [r1, r1 + np) (slot r1 also indexes the row's
// completion counter).
struct alignas(32) VecItem {
    int32_t r0, r1, inst, lg, k0, k1, slot, np;
};

// Nonzeros per piece of a long row.  A row of up to this many nonzeros is summed by one
// warp; longer rows are cut into pieces summed by several warps.  On the zipf-lp
// matrix (8,710 rows of 1,025-1,305 nonzeros, 56% of the nonzeros) 2,048 took the
// A-side step from 104.0 to 96.5 us against 1,024: the pieces' FP64 partial sums,
// completion counters and finishing warps cost more than a longer warp loop.
constexpr int kVecPiece = 2048;

// Device view of one side of the matrix as vec-engine items.
struct VecDev {
    int32_t n_items = 0;
    int32_t n_slots = 0;  // long-row piece slots (0: no row longer than kVecPiece)
    const int32_t* rp = nullptr;
    const int32_t* ci = nullptr;
    const VecItem* items = nullptr;
    double* piece_sum = nullptr;  // n_slots
    int32_t* piece_cnt = nullptr;  // n_slots, all zero between launches
};

// Items of one side: rows longer than kVecPiece are cut into pieces; the other
// rows get the lanes per row that give each lane about `lane_nnz` nonzeros (a
// power of two up to 32), and runs of rows with equal lanes are cut into items
// of (32 / lanes) x `groups` rows (groups <= 0: max(1, 8 / lane_nnz)), fewer where
// the item would hold more than 2048 nonzeros.  Items are ordered longest-first:
// pieces, then by decreasing lanes per row, each group in row order.  Returns the
// slot count.
int32_t build_vec_items(const HostCsr& csr, const std::vector<int32_t>& inst_row_off,
                        int lane_nnz, std::vector<VecItem>& items, int groups = 0);

// The long rows of A by column segment (seg_spmv.cuh).  The packed columns are cut
// into nseg segments of seg_len (a multiple of 4; the last segments may be short
// or empty); each long row's nonzeros are regrouped segment by
// segment into a CSR whose rows are the (segment, long row) pairs, segment-major
// (row s * n_long + q holds long row q's entries in segment s, in the row's
// storage order), with column indices relative to the segment start.  One block
// per segment, holding that segment of the gathered vector in shared memory,
// forms every pair's sum: the long row's partial for the segment.
struct SegDev {
    int32_t nseg = 0, seg_len = 0, n_cols = 0, n_long = 0;
    const int32_t* long_row = nullptr;   // n_long: packed row index of each long row
    const int32_t* long_inst = nullptr;  // n_long: its instance
    const float* val = nullptr;          // the regrouped entries' values (FP32)
    float* partial = nullptr;            // nseg x n_long partial sums (pair order)
};

struct HostSeg {
    int32_t nseg = 0, seg_len = 0, n_cols = 0;
    std::vector<int32_t> long_row, long_inst;
    HostCsr pairs;                 // rows: the pairs; ci: column - segment start; v: values
    std::vector<uint8_t> is_long;  // per row of A: 1 for the long rows
};

// Long rows: at least `long_min` nonzeros.  Returns false (and leaves `out` empty)
// when no row qualifies or a segment would span more than 65,536 columns.
bool build_seg(const HostCsr& csr, const std::vector<int32_t>& inst_row_off, int nseg,
               int long_min, HostSeg& out);

// The tiles of a tiling whose instances are the segments (tiles of segment s are
// [inst_tile0[s], inst_tile0[s+1])), reordered so that tile j * nseg + s is the
// j-th tile of segment s: a grid of nseg blocks walking tiles b, b + nseg, ...
// then gives block s exactly the tiles of segment s.  Segments with fewer tiles
// are padded with empty tiles of instance -1.
void interleave_tiles(const HostTiling& in, int nseg, HostTiling& out);

// One problem as handed to the library (CSR, caller's numbering).
struct ProblemIn {
    int32_t m, n;
    const int32_t* rp;
    const int32_t* ci;
    const double* v;
    const uint8_t* is_eq;  // nullable: all inequality
};

struct HostLayout {
    int32_t K = 0;
    int64_t M = 0, N = 0, NNZ = 0;
    std::vector<int32_t> row_off, col_off, n_eq;  // K+1, K+1, K
    std::vector<int32_t> row_orig, col_orig;      // packed -> caller index within the instance
    HostCsr A, At;                                // packed numbering
};

// Validates every CSR (monotone row pointers, column indices in range,
// ascending within rows); returns an error message or "" and fills `out`.
std::string build_layout(const std::vector<ProblemIn>& probs, bool permute, HostLayout& out);

}  // namespace pdfp
