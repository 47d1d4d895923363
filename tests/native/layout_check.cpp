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
    return 0;
}
