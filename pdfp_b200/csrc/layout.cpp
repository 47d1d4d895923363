// layout.cpp -- host construction of the packed, permuted device layout.
#include "layout.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <string>

namespace pdfp {

void build_tiling(const HostCsr& csr, const std::vector<int32_t>& inst_row_off,
                  const StageGeom& g, HostTiling& t) {
    t = HostTiling();
    t.geom = g;
    const int K = static_cast<int>(inst_row_off.size()) - 1;
    const std::vector<int32_t>& rp = csr.rp;
    t.tile_row.push_back(0);
    t.tile_chunk.push_back(0);
    t.inst_tile0.push_back(0);
    int32_t max_rows = 1;
    for (int p = 0; p < K; ++p) {
        int32_t r = inst_row_off[p];
        const int32_t rend = inst_row_off[p + 1];
        while (r < rend) {
            const int32_t tile = static_cast<int32_t>(t.tile_inst.size());
            if (chunk_stage_bytes(g, rp[r], rp[r + 1], r, r + 1, true, false) >
                static_cast<uint32_t>(g.stage_bytes)) {
                // a long row: one tile, several chunks
                int64_t fixed = chunk_stage_bytes(g, 0, 0, r, r + 1, true, true);
                int64_t per = 4 + g.esize_v + (g.nv > 1 ? g.esize_acc : 0);
                int64_t kc = (static_cast<int64_t>(g.stage_bytes) - fixed - 3 * 160) / per;
                kc = std::max<int64_t>(kc & ~int64_t(31), 32);
                while (kc > 32 && chunk_stage_bytes(g, 0, kc, r, r + 1, true, true) >
                                      static_cast<uint32_t>(g.stage_bytes))
                    kc -= 32;
                for (int64_t k = rp[r]; k < rp[r + 1]; k += kc) {
                    int64_t ke = std::min<int64_t>(k + kc, rp[r + 1]);
                    t.chunk_k0.push_back(static_cast<int32_t>(k));
                    t.chunk_k1.push_back(static_cast<int32_t>(ke));
                    t.chunk_tile.push_back(tile);
                    t.chunk_flags.push_back(CHUNK_LONG | (ke == rp[r + 1] ? CHUNK_LAST : 0));
                }
                r += 1;
            } else {
                int32_t r1 = r + 1;
                while (r1 < rend && (r1 + 1 - r) <= g.max_rows &&
                       chunk_stage_bytes(g, rp[r], rp[r1 + 1], r, r1 + 1, true, false) <=
                           static_cast<uint32_t>(g.stage_bytes))
                    ++r1;
                t.chunk_k0.push_back(rp[r]);
                t.chunk_k1.push_back(rp[r1]);
                t.chunk_tile.push_back(tile);
                t.chunk_flags.push_back(CHUNK_LAST);
                max_rows = std::max(max_rows, r1 - r);
                r = r1;
            }
            t.tile_inst.push_back(p);
            t.tile_row.push_back(r);
            t.tile_chunk.push_back(static_cast<int32_t>(t.chunk_k0.size()));
        }
        t.inst_tile0.push_back(static_cast<int32_t>(t.tile_inst.size()));
    }
    t.max_tile_rows = max_rows;
}

std::string build_layout(const std::vector<ProblemIn>& probs, bool permute, HostLayout& L) {
    L = HostLayout();
    const int K = static_cast<int>(probs.size());
    L.K = K;
    L.row_off.assign(K + 1, 0);
    L.col_off.assign(K + 1, 0);
    L.n_eq.assign(K, 0);
    int64_t nnz_total = 0;
    for (int p = 0; p < K; ++p) {
        const ProblemIn& P = probs[p];
        if (P.m < 0 || P.n < 0) return "negative dimension";
        if (P.m > 0 && (!P.rp)) return "null row_ptr";
        const int64_t nnz = P.m > 0 ? P.rp[P.m] : 0;
        if (P.m > 0 && P.rp[0] != 0) return "row_ptr[0] must be 0";
        for (int32_t i = 0; i < P.m; ++i) {
            if (P.rp[i + 1] < P.rp[i]) return "row_ptr is not monotone";
            for (int32_t q = P.rp[i]; q < P.rp[i + 1]; ++q) {
                if (P.ci[q] < 0 || P.ci[q] >= P.n) return "column index out of range";
                if (q > P.rp[i] && P.ci[q] <= P.ci[q - 1])
                    return "column indices must be strictly ascending within a row";
                if (!std::isfinite(P.v[q])) return "non-finite matrix value";
            }
        }
        L.row_off[p + 1] = L.row_off[p] + P.m;
        L.col_off[p + 1] = L.col_off[p] + P.n;
        nnz_total += nnz;
        if (L.row_off[p + 1] < 0 || L.col_off[p + 1] < 0 || nnz_total > 0x7fffff00LL)
            return "problem too large for int32 indexing";
    }
    L.M = L.row_off[K];
    L.N = L.col_off[K];
    L.NNZ = nnz_total;
    L.row_orig.resize(L.M);
    L.col_orig.resize(L.N);
    HostCsr& A = L.A;
    HostCsr& At = L.At;
    A.rows = static_cast<int32_t>(L.M);
    A.cols = static_cast<int32_t>(L.N);
    At.rows = static_cast<int32_t>(L.N);
    At.cols = static_cast<int32_t>(L.M);
    A.rp.assign(L.M + 1, 0);
    A.ci.resize(nnz_total);
    A.v.resize(nnz_total);
    At.rp.assign(L.N + 1, 0);
    At.ci.resize(nnz_total);
    At.v.resize(nnz_total);

    int64_t a_pos = 0;
    for (int p = 0; p < K; ++p) {
        const ProblemIn& P = probs[p];
        const int32_t m = P.m, n = P.n, r0 = L.row_off[p], c0 = L.col_off[p];
        std::vector<int32_t> rlen(m), clen(n, 0);
        for (int32_t i = 0; i < m; ++i) {
            rlen[i] = P.rp[i + 1] - P.rp[i];
            for (int32_t q = P.rp[i]; q < P.rp[i + 1]; ++q) clen[P.ci[q]]++;
        }
        // row order: equality rows first, then by decreasing length (stable)
        std::vector<int32_t> rord(m), cord(n);
        std::iota(rord.begin(), rord.end(), 0);
        std::iota(cord.begin(), cord.end(), 0);
        int32_t neq = 0;
        for (int32_t i = 0; i < m; ++i) neq += (P.is_eq && P.is_eq[i]) ? 1 : 0;
        std::stable_sort(rord.begin(), rord.end(), [&](int32_t a, int32_t b) {
            bool ea = P.is_eq && P.is_eq[a], eb = P.is_eq && P.is_eq[b];
            if (ea != eb) return ea;
            return permute ? rlen[a] > rlen[b] : false;
        });
        if (permute)
            std::stable_sort(cord.begin(), cord.end(),
                             [&](int32_t a, int32_t b) { return clen[a] > clen[b]; });
        L.n_eq[p] = neq;
        std::vector<int32_t> cnew(n);
        for (int32_t j = 0; j < n; ++j) {
            cnew[cord[j]] = j;
            L.col_orig[c0 + j] = cord[j];
        }
        std::vector<int32_t> rnew(m);
        for (int32_t i = 0; i < m; ++i) {
            rnew[rord[i]] = i;
            L.row_orig[r0 + i] = rord[i];
        }
        // A: packed rows in the new order, entries in the caller's column order
        const int64_t base = a_pos;  // this instance's nonzeros start here in A and in A'
        for (int32_t i = 0; i < m; ++i) {
            const int32_t orow = rord[i];
            A.rp[r0 + i] = static_cast<int32_t>(a_pos);
            for (int32_t q = P.rp[orow]; q < P.rp[orow + 1]; ++q) {
                A.ci[a_pos] = c0 + cnew[P.ci[q]];
                A.v[a_pos] = P.v[q];
                ++a_pos;
            }
        }
        // A': packed columns in the new order, entries in ascending caller row index
        std::vector<int64_t> cstart(n + 1, 0);
        for (int32_t j = 0; j < n; ++j) cstart[j + 1] = cstart[j] + clen[cord[j]];
        std::vector<int64_t> fill(n);
        for (int32_t j = 0; j < n; ++j) {
            fill[j] = base + cstart[j];
            At.rp[c0 + j] = static_cast<int32_t>(base + cstart[j]);
        }
        for (int32_t orow = 0; orow < m; ++orow)
            for (int32_t q = P.rp[orow]; q < P.rp[orow + 1]; ++q) {
                const int32_t j = cnew[P.ci[q]];
                At.ci[fill[j]] = r0 + rnew[orow];
                At.v[fill[j]] = P.v[q];
                ++fill[j];
            }
    }
    A.rp[L.M] = static_cast<int32_t>(a_pos);
    At.rp[L.N] = static_cast<int32_t>(a_pos);
    return "";
}

}  // namespace pdfp
