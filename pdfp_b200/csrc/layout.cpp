// layout.cpp -- host construction of the packed, permuted device layout.
#include "layout.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <string>

namespace pdfp {

void build_tiling(const HostCsr& csr, const std::vector<int32_t>& inst_row_off,
                  const StageGeom& g, HostTiling& t, const std::vector<uint8_t>* skip) {
    t = HostTiling();
    t.geom = g;
    const int K = static_cast<int>(inst_row_off.size()) - 1;
    const std::vector<int32_t>& rp = csr.rp;
    auto skipped = [&](int32_t r) { return skip && (*skip)[r] != 0; };
    std::vector<int32_t> starts;
    t.tile_chunk.push_back(0);
    t.inst_tile0.push_back(0);
    int32_t max_rows = 1;
    for (int p = 0; p < K; ++p) {
        int32_t r = inst_row_off[p];
        const int32_t rend = inst_row_off[p + 1];
        while (r < rend) {
            if (skipped(r)) {
                ++r;
                continue;
            }
            const int32_t tile = static_cast<int32_t>(t.tile_inst.size());
            starts.push_back(r);
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
                while (r1 < rend && !skipped(r1) && (r1 + 1 - r) <= g.max_rows &&
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
            t.tile_row_end.push_back(r);
            t.tile_chunk.push_back(static_cast<int32_t>(t.chunk_k0.size()));
        }
        t.inst_tile0.push_back(static_cast<int32_t>(t.tile_inst.size()));
    }
    // tile t covers rows [tile_row[t], tile_row_end[t]); without skipped rows the
    // tiles are contiguous and tile_row[t + 1] == tile_row_end[t]
    t.tile_row = starts;
    t.tile_row.push_back(t.tile_row_end.empty() ? (K > 0 ? inst_row_off[K] : 0) : t.tile_row_end.back());
    t.max_tile_rows = max_rows;
}

int32_t build_vec_items(const HostCsr& csr, const std::vector<int32_t>& inst_row_off,
                        int lane_nnz, std::vector<VecItem>& items, int groups) {
    items.clear();
    const int K = static_cast<int>(inst_row_off.size()) - 1;
    const std::vector<int32_t>& rp = csr.rp;
    const int rpg = groups > 0 ? groups : std::max(1, 8 / std::max(1, lane_nnz));
    auto lanes_log2 = [&](int64_t len) {
        int lg = 0;
        while (lg < 5 && (int64_t(1) << lg) * lane_nnz < len) ++lg;
        return lg;
    };
    std::vector<VecItem> pieces;
    int32_t slots = 0;
    for (int p = 0; p < K; ++p) {
        int32_t r = inst_row_off[p];
        const int32_t rend = inst_row_off[p + 1];
        while (r < rend) {
            const int64_t len = rp[r + 1] - rp[r];
            if (len > kVecPiece) {
                const int32_t np = static_cast<int32_t>((len + kVecPiece - 1) / kVecPiece);
                for (int32_t q = 0; q < np; ++q) {
                    const int32_t k0 = rp[r] + q * kVecPiece;
                    const int32_t k1 = std::min<int32_t>(k0 + kVecPiece, rp[r + 1]);
                    pieces.push_back(VecItem{r, slots, p, -1, k0, k1, slots + q, np});
                }
                slots += np;
                ++r;
                continue;
            }
            const int lg = lanes_log2(len);
            int32_t cap = (32 >> lg) * rpg;
            while (cap > (32 >> lg) && static_cast<int64_t>(cap) * len > 2048) cap -= 32 >> lg;
            int32_t r1 = r + 1;
            while (r1 < rend && r1 - r < cap) {
                const int64_t l1 = rp[r1 + 1] - rp[r1];
                if (l1 > kVecPiece || lanes_log2(l1) != lg) break;
                ++r1;
            }
            items.push_back(VecItem{r, r1, p, lg, 0, 0, 0, 0});
            r = r1;
        }
    }
    std::stable_sort(items.begin(), items.end(),
                     [](const VecItem& a, const VecItem& b) { return a.lg > b.lg; });
    items.insert(items.begin(), pieces.begin(), pieces.end());
    return slots;
}

bool build_seg(const HostCsr& csr, const std::vector<int32_t>& inst_row_off, int nseg,
               int long_min, HostSeg& o) {
    o = HostSeg();
    const int K = static_cast<int>(inst_row_off.size()) - 1;
    const int64_t ncols = csr.cols;
    if (nseg <= 0 || ncols <= 0 || K <= 0 || long_min <= 0) return false;
    // a multiple of 4, so that each segment of an FP32 vector starts 16-byte aligned
    const int64_t seg_len = ((ncols + nseg - 1) / nseg + 3) & ~int64_t(3);
    if (seg_len > 65536) return false;
    const std::vector<int32_t>& rp = csr.rp;
    const std::vector<int32_t>& ci = csr.ci;
    o.is_long.assign(csr.rows, 0);
    for (int p = 0; p < K; ++p)
        for (int32_t r = inst_row_off[p]; r < inst_row_off[p + 1]; ++r) {
            if (rp[r + 1] - rp[r] < long_min) continue;
            o.is_long[r] = 1;
            o.long_row.push_back(r);
            o.long_inst.push_back(p);
        }
    const int64_t nl = static_cast<int64_t>(o.long_row.size());
    if (nl == 0 || static_cast<int64_t>(nseg) * nl > 0x7ffffff0LL) {
        o = HostSeg();
        return false;
    }
    o.nseg = nseg;
    o.seg_len = static_cast<int32_t>(seg_len);
    o.n_cols = static_cast<int32_t>(ncols);
    HostCsr& P = o.pairs;
    P.rows = static_cast<int32_t>(nseg * nl);
    P.cols = static_cast<int32_t>(seg_len);
    P.rp.assign(static_cast<size_t>(P.rows) + 1, 0);
    for (int64_t q = 0; q < nl; ++q) {
        const int32_t r = o.long_row[q];
        for (int32_t k = rp[r]; k < rp[r + 1]; ++k) ++P.rp[static_cast<size_t>(ci[k] / seg_len) * nl + q + 1];
    }
    for (size_t i = 1; i < P.rp.size(); ++i) P.rp[i] += P.rp[i - 1];
    P.ci.resize(P.rp.back());
    P.v.resize(P.rp.back());
    std::vector<int32_t> cur(nseg);
    for (int64_t q = 0; q < nl; ++q) {
        const int32_t r = o.long_row[q];
        for (int s = 0; s < nseg; ++s) cur[s] = P.rp[s * nl + q];
        for (int32_t k = rp[r]; k < rp[r + 1]; ++k) {
            const int32_t s = static_cast<int32_t>(ci[k] / seg_len);
            const int32_t e = cur[s]++;
            P.ci[e] = static_cast<int32_t>(ci[k] - s * seg_len);
            P.v[e] = csr.v[k];
        }
    }
    return true;
}

void interleave_tiles(const HostTiling& in, int nseg, HostTiling& t) {
    t = HostTiling();
    t.geom = in.geom;
    t.max_tile_rows = in.max_tile_rows;
    int32_t most = 0;
    for (int s = 0; s < nseg; ++s) most = std::max(most, in.inst_tile0[s + 1] - in.inst_tile0[s]);
    t.tile_chunk.push_back(0);
    for (int32_t j = 0; j < most; ++j)
        for (int s = 0; s < nseg; ++s) {
            const int32_t tile = static_cast<int32_t>(t.tile_inst.size());
            const int32_t src = in.inst_tile0[s] + j;
            if (src < in.inst_tile0[s + 1]) {
                t.tile_row.push_back(in.tile_row[src]);
                t.tile_row_end.push_back(in.tile_row_end[src]);
                t.tile_inst.push_back(s);
                for (int32_t c = in.tile_chunk[src]; c < in.tile_chunk[src + 1]; ++c) {
                    t.chunk_k0.push_back(in.chunk_k0[c]);
                    t.chunk_k1.push_back(in.chunk_k1[c]);
                    t.chunk_tile.push_back(tile);
                    t.chunk_flags.push_back(in.chunk_flags[c]);
                }
            } else {  // padding: no rows, no chunks
                t.tile_row.push_back(0);
                t.tile_row_end.push_back(0);
                t.tile_inst.push_back(-1);
            }
            t.tile_chunk.push_back(static_cast<int32_t>(t.chunk_k0.size()));
        }
    t.tile_row.push_back(in.tile_row.empty() ? 0 : in.tile_row.back());
    t.inst_tile0.assign(1, 0);
    t.inst_tile0.push_back(static_cast<int32_t>(t.tile_inst.size()));
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
