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
    std::vector<int32_t> inst_tile0;  // K + 1: tiles of instance p are [inst_tile0[p], inst_tile0[p+1])
    int32_t max_tile_rows = 1;
    StageGeom geom{};
};

void build_tiling(const HostCsr& csr, const std::vector<int32_t>& inst_row_off,
                  const StageGeom& g, HostTiling& t);

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
