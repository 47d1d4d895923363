// layout_check.cpp -- CPU checks of the host layout and tiling builder
// (pdfp_b200/csrc/layout.cpp): permutations, A/A' consistency, storage order,
// tile coverage and the shared-memory stage bound of every chunk.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "../../pdfp_b200/csrc/layout.hpp"

using namespace pdfp;

static int check_tiling(const HostCsr& csr, const std::vector<int32_t>& off, const StageGeom& g,
                        int64_t* n_tiles, int64_t* n_long, int flat_cap = 0) {
    HostTiling t;
    build_tiling(csr, off, g, t);
    if (flat_cap && !flat_tiling_fits(t, flat_cap)) return 26;
    const int K = static_cast<int>(off.size()) - 1;
    if (t.tile_row.size() != t.tile_inst.size() + 1) return 10;
    if ((int)t.inst_tile0.size() != K + 1) return 11;
    int32_t r = 0;
    for (int p = 0; p < K; ++p) {
        for (int32_t tt = t.inst_tile0[p]; tt < t.inst_tile0[p + 1]; ++tt) {
            if (t.tile_inst[tt] != p) return 12;
            if (t.tile_row[tt] != r) return 13;
            if (t.tile_row_end[tt] != t.tile_row[tt + 1]) return 27;  // no row left out
            const int32_t r0 = t.tile_row[tt], r1 = t.tile_row[tt + 1];
            if (r1 <= r0) return 14;
            if (r0 < off[p] || r1 > off[p + 1]) return 15;  // a tile never crosses an instance
            if (r1 - r0 > t.max_tile_rows) return 16;
            int64_t k = csr.rp[r0];
            const int32_t c0 = t.tile_chunk[tt], c1 = t.tile_chunk[tt + 1];
            if (c1 <= c0) return 17;
            for (int32_t c = c0; c < c1; ++c) {
                if (t.chunk_tile[c] != tt) return 18;
                if (t.chunk_k0[c] != k) return 19;
                const bool last = (t.chunk_flags[c] & CHUNK_LAST) != 0;
                const bool single = (t.chunk_flags[c] & CHUNK_LONG) != 0;
                if (last != (c == c1 - 1)) return 20;
                if (single && r1 - r0 != 1) return 21;
                if (c1 - c0 > 1 && !single) return 22;
                if (chunk_stage_bytes(g, t.chunk_k0[c], t.chunk_k1[c], r0, r1, last, single) >
                    static_cast<uint32_t>(g.stage_bytes))
                    return 23;
                k = t.chunk_k1[c];
                if (single) ++*n_long;
            }
            if (k != csr.rp[r1]) return 24;
            r = r1;
        }
        if (r != off[p + 1] && off[p + 1] != off[p]) return 25;
        r = off[p + 1];
    }
    *n_tiles += static_cast<int64_t>(t.tile_inst.size());
    return 0;
}

// Vec-engine items (build_vec_items): every row once, in a multi-row item of its
// instance or as pieces that cover its nonzeros in order; lanes and sizes in range.
static int check_vec(const HostCsr& csr, const std::vector<int32_t>& off, int lane_nnz,
                     int groups = 0) {
    std::vector<VecItem> items;
    const int32_t slots = build_vec_items(csr, off, lane_nnz, items, groups);
    const int K = static_cast<int>(off.size()) - 1;
    std::vector<int> seen(csr.rows, 0);
    std::vector<int32_t> next_k(csr.rows, -1);
    std::vector<int> slot_used(slots > 0 ? slots : 1, 0);
    bool pieces_done = false;
    int last_lg = 6;
    for (const VecItem& it : items) {
        if (it.inst < 0 || it.inst >= K) return 1;
        if (it.lg < 0) {
            if (pieces_done) return 2;  // pieces come first
            const int32_t r = it.r0;
            if (r < off[it.inst] || r >= off[it.inst + 1]) return 3;
            const int32_t len = csr.rp[r + 1] - csr.rp[r];
            if (len <= kVecPiece || it.np != (len + kVecPiece - 1) / kVecPiece) return 4;
            if (next_k[r] < 0) next_k[r] = csr.rp[r];
            if (it.k0 != next_k[r] || it.k1 <= it.k0 || it.k1 - it.k0 > kVecPiece) return 5;
            if (it.slot != it.r1 + (it.k0 - csr.rp[r]) / kVecPiece || it.slot >= slots) return 6;
            slot_used[it.slot]++;
            next_k[r] = it.k1;
            if (it.k1 == csr.rp[r + 1]) seen[r]++;
            continue;
        }
        pieces_done = true;
        if (it.lg > 5 || it.lg > last_lg) return 7;  // by decreasing lanes per row
        last_lg = it.lg;
        if (it.r1 <= it.r0 || it.r0 < off[it.inst] || it.r1 > off[it.inst + 1]) return 8;
        for (int32_t r = it.r0; r < it.r1; ++r) {
            if (csr.rp[r + 1] - csr.rp[r] > kVecPiece) return 9;
            seen[r]++;
        }
    }
    for (int32_t r = 0; r < csr.rows; ++r)
        if (seen[r] != 1) return 10;
    for (int32_t q = 0; q < slots; ++q)
        if (slot_used[q] != 1) return 11;
    return 0;
}

// Segmented long rows (build_seg), the interleaved tiling of their pairs and the
// tiling of the other rows: the long rows are exactly those of at least long_min
// nonzeros, each pair holds the row's entries of its segment in storage order, block
// s of an nseg grid walks exactly segment s's tiles, and the tiling with the long
// rows left out covers every other row once.
static int check_seg(const HostCsr& A, const std::vector<int32_t>& off, int nseg, int long_min,
                     int stage_bytes, int64_t* n_long_out) {
    HostSeg h;
    const bool ok = build_seg(A, off, nseg, long_min, h);
    const int K = static_cast<int>(off.size()) - 1;
    const int64_t seg_len = A.cols > 0 ? (((A.cols + nseg - 1) / nseg + 3) & ~int64_t(3)) : 0;
    int64_t n_want = 0;
    for (int32_t r = 0; r < A.rows; ++r) n_want += A.rp[r + 1] - A.rp[r] >= long_min;
    if (!ok) return (n_want == 0 || seg_len > 65536 || A.cols == 0) && h.long_row.empty() ? 0 : 1;
    const int64_t nl = static_cast<int64_t>(h.long_row.size());
    if (nl != n_want || h.seg_len != seg_len || (int64_t)h.is_long.size() != A.rows) return 2;
    for (int32_t r = 0; r < A.rows; ++r)
        if (h.is_long[r] != (A.rp[r + 1] - A.rp[r] >= long_min)) return 3;
    for (int64_t q = 0; q < nl; ++q) {
        const int32_t r = h.long_row[q];
        if (!h.is_long[r] || (q > 0 && r <= h.long_row[q - 1])) return 4;
        const int p = h.long_inst[q];
        if (p < 0 || p >= K || r < off[p] || r >= off[p + 1]) return 5;
    }
    const HostCsr& P = h.pairs;
    if (P.rows != nseg * nl || (int64_t)P.rp.size() != P.rows + 1 || P.rp[0] != 0) return 6;
    for (size_t i = 1; i < P.rp.size(); ++i)
        if (P.rp[i] < P.rp[i - 1]) return 6;
    if (P.rp.back() != (int32_t)P.ci.size() || P.ci.size() != P.v.size()) return 7;
    // each pair: the long row's entries of its segment, in storage order
    int64_t total = 0;
    for (int64_t q = 0; q < nl; ++q) {
        const int32_t r = h.long_row[q];
        for (int s = 0; s < nseg; ++s) {
            int32_t e = P.rp[s * nl + q];
            const int32_t e1 = P.rp[s * nl + q + 1];
            total += e1 - e;
            for (int32_t k = A.rp[r]; k < A.rp[r + 1]; ++k) {
                if (A.ci[k] / seg_len != s) continue;
                if (e >= e1) return 9;
                if (P.ci[e] + s * seg_len != A.ci[k] || P.ci[e] < 0 || P.ci[e] >= seg_len ||
                    P.v[e] != A.v[k])
                    return 10;
                ++e;
            }
            if (e != e1) return 11;
        }
    }
    if (total != P.rp.back()) return 11;
    // tiles by segment, interleaved
    std::vector<int32_t> soff(nseg + 1);
    for (int s = 0; s <= nseg; ++s) soff[s] = static_cast<int32_t>(s * nl);
    const StageGeom gs{4, 4, 4, 0, 1, stage_bytes, 2048};
    HostTiling by, t;
    build_tiling(P, soff, gs, by);
    interleave_tiles(by, nseg, t);
    if (t.tile_chunk.size() != t.tile_inst.size() + 1 || t.tile_row_end.size() != t.tile_inst.size() ||
        t.tile_inst.size() % nseg != 0)
        return 12;
    std::vector<int> pair_cover(P.rows, 0);
    for (int b = 0; b < nseg; ++b)
        for (size_t tt = b; tt < t.tile_inst.size(); tt += nseg) {
            const int32_t p = t.tile_inst[tt];
            if (p == -1) {
                if (t.tile_chunk[tt + 1] != t.tile_chunk[tt]) return 13;
                continue;
            }
            if (p != b) return 14;  // block b sees only its own segment
            const int32_t r0 = t.tile_row[tt], r1 = t.tile_row_end[tt];
            if (r1 <= r0 || r0 < soff[b] || r1 > soff[b + 1]) return 15;
            int64_t k = P.rp[r0];
            for (int32_t c = t.tile_chunk[tt]; c < t.tile_chunk[tt + 1]; ++c) {
                if (t.chunk_tile[c] != (int32_t)tt || t.chunk_k0[c] != k) return 16;
                k = t.chunk_k1[c];
            }
            if (k != P.rp[r1]) return 17;
            for (int32_t r = r0; r < r1; ++r) pair_cover[r]++;
        }
    for (int32_t r = 0; r < P.rows; ++r)
        if (pair_cover[r] != 1) return 18;
    // the tiling of the other rows
    const StageGeom g{4, 4, 4, 3, 1, 16 * 1024, 2048};
    HostTiling o;
    build_tiling(A, off, g, o, &h.is_long);
    std::vector<int> cover(A.rows, 0);
    for (size_t tt = 0; tt < o.tile_inst.size(); ++tt) {
        const int32_t r0 = o.tile_row[tt], r1 = o.tile_row_end[tt];
        const int p = o.tile_inst[tt];
        if (r1 <= r0 || r0 < off[p] || r1 > off[p + 1]) return 19;
        int64_t k = A.rp[r0];
        for (int32_t c = o.tile_chunk[tt]; c < o.tile_chunk[tt + 1]; ++c) {
            if (o.chunk_k0[c] != k) return 20;
            k = o.chunk_k1[c];
        }
        if (k != A.rp[r1]) return 21;
        for (int32_t r = r0; r < r1; ++r) cover[r]++;
    }
    for (int32_t r = 0; r < A.rows; ++r)
        if (cover[r] != (h.is_long[r] ? 0 : 1)) return 22;
    *n_long_out += nl;
    return 0;
}

extern "C" int layout_check(int K, const int32_t* ms, const int32_t* ns, const int32_t* const* rps,
                            const int32_t* const* cis, const double* const* vs,
                            const uint8_t* const* is_eqs, int stage_bytes, int64_t* stats) {
    std::vector<ProblemIn> probs;
    for (int p = 0; p < K; ++p) probs.push_back(ProblemIn{ms[p], ns[p], rps[p], cis[p], vs[p], is_eqs[p]});
    HostLayout L;
    if (!build_layout(probs, true, L).empty()) return 1;
    // permutations are bijections per instance; equality rows first
    for (int p = 0; p < K; ++p) {
        std::vector<int> seen_r(ms[p], 0), seen_c(ns[p], 0);
        for (int32_t i = 0; i < ms[p]; ++i) seen_r[L.row_orig[L.row_off[p] + i]]++;
        for (int32_t j = 0; j < ns[p]; ++j) seen_c[L.col_orig[L.col_off[p] + j]]++;
        for (int v : seen_r) if (v != 1) return 2;
        for (int v : seen_c) if (v != 1) return 3;
        for (int32_t i = 0; i < ms[p]; ++i) {
            const bool eq = is_eqs[p] && is_eqs[p][L.row_orig[L.row_off[p] + i]];
            if (eq != (i < L.n_eq[p])) return 4;
        }
    }
    // A rows: same entries as the caller's row, ascending caller column index
    std::vector<int32_t> cpos(L.N);
    for (int p = 0; p < K; ++p)
        for (int32_t j = 0; j < ns[p]; ++j) cpos[L.col_off[p] + j] = L.col_orig[L.col_off[p] + j];
    for (int p = 0; p < K; ++p) {
        for (int32_t i = 0; i < ms[p]; ++i) {
            const int32_t pr = L.row_off[p] + i, orow = L.row_orig[pr];
            const int32_t a0 = L.A.rp[pr], a1 = L.A.rp[pr + 1];
            if (a1 - a0 != rps[p][orow + 1] - rps[p][orow]) return 5;
            for (int32_t q = a0; q < a1; ++q) {
                const int32_t oq = rps[p][orow] + (q - a0);
                if (cpos[L.A.ci[q]] != cis[p][oq] || L.A.v[q] != vs[p][oq]) return 6;
                if (L.A.ci[q] < L.col_off[p] || L.A.ci[q] >= L.col_off[p + 1]) return 7;
            }
        }
    }
    // A' is the transpose of A, each row in ascending caller row index
    std::vector<int64_t> cnt(L.N, 0);
    for (int64_t q = 0; q < L.NNZ; ++q) cnt[L.A.ci[q]]++;
    for (int64_t j = 0; j < L.N; ++j)
        if (L.At.rp[j + 1] - L.At.rp[j] != cnt[j]) return 8;
    for (int64_t j = 0; j < L.N; ++j)
        for (int32_t q = L.At.rp[j] + 1; q < L.At.rp[j + 1]; ++q)
            if (L.row_orig[L.At.ci[q]] <= L.row_orig[L.At.ci[q - 1]]) return 9;
    // tilings of the iteration and evaluation geometries
    const StageGeom geoms[] = {
        {4, 4, 4, 8, 1, stage_bytes, 2048}, {4, 4, 4, 3, 1, stage_bytes, 2048},
        {8, 8, 8, 8, 1, stage_bytes, 2048}, {8, 8, 8, 3, 1, stage_bytes, 2048},
        {8, 8, 8, 0, 2, stage_bytes, 2048}};
    stats[0] = stats[1] = 0;
    for (const StageGeom& g : geoms) {
        int rc = check_tiling(L.At, L.col_off, g, &stats[0], &stats[1]);
        if (rc) return rc;
        rc = check_tiling(L.A, L.row_off, g, &stats[0], &stats[1]);
        if (rc) return 100 + rc;
    }
    // the flat engine's geometries (FP32 and FP64 values, no staged vectors)
    for (int e : {4, 8})
        for (int cap : {1024, kFlatCapMax}) {
            const StageGeom g{e, e, e, 0, 1, flat_stage_bytes(e, cap), kFlatMaxRows};
            int rc = check_tiling(L.At, L.col_off, g, &stats[0], &stats[1], cap);
            if (rc) return 200 + rc;
            rc = check_tiling(L.A, L.row_off, g, &stats[0], &stats[1], cap);
            if (rc) return 300 + rc;
        }
    // the vec engine's items
    for (int lane : {1, 2, 4, 8})
        for (int groups : {0, 32 / lane}) {  // the default rows per item and four times them
            int rc = check_vec(L.At, L.col_off, lane, groups);
            if (rc) return 400 + rc;
            rc = check_vec(L.A, L.row_off, lane, groups);
            if (rc) return 500 + rc;
        }
    // segmented long rows: small stages, so that pairs span several tiles and long
    // pairs several chunks
    stats[2] = 0;
    const int segs[][3] = {{1, 1, 8192}, {3, 2, 8192}, {16, 4, 8192}, {64, 64, 16384}, {7, 16, 8192}};
    for (const auto& c : segs) {
        int rc = check_seg(L.A, L.row_off, c[0], c[1], c[2], &stats[2]);
        if (rc) return 600 + rc;
    }
    return 0;
}
