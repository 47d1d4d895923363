// seg_layout_check.cpp -- CPU checks of the segmented engine's layout
// (build_seg_layout, pdfp_b200/csrc/layout.cpp) and of its row-sum bookkeeping
// (seg_spmv.cuh), replayed on the host: every key decodes to a nonzero of the CSR,
// each exactly once, sorted by (row, column) within its chunk, inside the CTA's rows
// and the segment's columns; and the warp-window sums -- each row's run summed per
// 32-nonzero window, added directly by the window where the row starts and through
// the continuation partials otherwise, in window order -- give every row's sum.
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../pdfp_b200/csrc/layout.hpp"

using namespace pdfp;

extern "C" int seg_layout_check(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                                const double* v, int G, int q, int sl_log, int64_t* stats) {
    HostCsr C;
    C.rows = m;
    C.cols = n;
    C.rp.assign(rp, rp + m + 1);
    C.ci.assign(ci, ci + rp[m]);
    C.v.assign(v, v + rp[m]);
    SegHost h;
    if (!build_seg_layout(C, G, q, sl_log, h).empty()) return 1;
    const int64_t seg = static_cast<int64_t>(q) << sl_log;
    const int64_t nnz = rp[m];
    if (h.G != G || h.S != (n + seg - 1) / seg || h.ncols != n) return 2;
    if ((int64_t)h.row_start.size() != G + 1 || h.row_start[0] != 0 || h.row_start[G] != m) return 3;
    int32_t rmax = 0;
    for (int g = 0; g < G; ++g) {
        if (h.row_start[g + 1] < h.row_start[g]) return 4;
        rmax = std::max(rmax, h.row_start[g + 1] - h.row_start[g]);
    }
    if (rmax != h.rmax || rmax >= (1 << 15)) return 5;
    if ((int64_t)h.chunk_off.size() != (int64_t)G * h.S + 1 || h.chunk_off[0] != 0 ||
        h.chunk_off.back() != nnz)
        return 6;
    std::vector<int> seen(nnz, 0);
    std::vector<double> x(n), ref(m, 0.0), got(m, 0.0);
    for (int32_t j = 0; j < n; ++j) x[j] = 1.0 + 0.001 * (j % 997);
    for (int32_t i = 0; i < m; ++i)
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) ref[i] += static_cast<double>(static_cast<float>(v[k])) * x[ci[k]];
    int64_t wmax = 0, cont_windows = 0;
    for (int g = 0; g < G; ++g)
        for (int s = 0; s < h.S; ++s) {
            const int64_t c = static_cast<int64_t>(g) * h.S + s;
            const int32_t k0 = h.chunk_off[c], k1 = h.chunk_off[c + 1];
            if (k1 < k0) return 7;
            wmax = std::max<int64_t>(wmax, (k1 - k0 + 31) / 32);
            int64_t prev = -1;
            for (int32_t k = k0; k < k1; ++k) {
                const int32_t row = h.row_start[g] + static_cast<int32_t>(h.key[k] >> 17);
                const int64_t col = s * seg + (h.key[k] & ((1u << 17) - 1u));
                if (row >= h.row_start[g + 1] || col >= n) return 8;
                const int64_t order = static_cast<int64_t>(row) * n + col;
                if (order <= prev) return 9;  // sorted by (row, column), no duplicates
                prev = order;
                const int32_t* b = ci + rp[row];
                const int32_t* e = ci + rp[row + 1];
                const int32_t* it = std::lower_bound(b, e, static_cast<int32_t>(col));
                if (it == e || *it != col) return 10;
                const int64_t kk = it - ci;
                if (seen[kk]++) return 11;
                if (h.val[k] != static_cast<float>(v[kk])) return 12;
            }
            // the kernel's window bookkeeping for this chunk
            const int32_t nwin = (k1 - k0 + 31) / 32;
            std::vector<double> side(nwin, 0.0);
            auto rowof = [&](int32_t k) { return static_cast<int32_t>(h.key[k] >> 17); };
            for (int32_t w = 0; w < nwin; ++w) {
                const int32_t ws = k0 + 32 * w, we = std::min(ws + 32, k1);
                const int32_t row0 = rowof(ws);
                for (int32_t a = ws; a < we;) {
                    int32_t b = a;
                    double sum = 0.0;
                    while (b < we && rowof(b) == rowof(a)) {
                        const int64_t col = s * seg + (h.key[b] & ((1u << 17) - 1u));
                        sum += static_cast<double>(h.val[b]) * x[col];
                        ++b;
                    }
                    const bool cont = rowof(a) == row0 && ws > k0 && rowof(ws - 1) == row0;
                    if (cont) {
                        side[w] = sum;
                        ++cont_windows;
                    } else {
                        got[h.row_start[g] + rowof(a)] += sum;
                    }
                    a = b;
                }
            }
            for (int32_t wi = 1; wi < nwin; ++wi) {
                const int32_t ws = k0 + 32 * wi;
                const int32_t r0 = rowof(ws);
                if (rowof(ws - 1) != r0) continue;
                if (wi >= 2 && rowof(ws - 32) == r0 && rowof(ws - 33) == r0) continue;
                double t = side[wi];
                for (int32_t wj = wi + 1; wj < nwin; ++wj) {
                    const int32_t vs = k0 + 32 * wj;
                    if (rowof(vs) != r0 || rowof(vs - 1) != r0) break;
                    t += side[wj];
                }
                got[h.row_start[g] + r0] += t;
            }
        }
    for (int64_t k = 0; k < nnz; ++k)
        if (seen[k] != 1) return 13;
    if (wmax != h.wmax && !(wmax == 0 && h.wmax == 1)) return 14;
    for (int32_t i = 0; i < m; ++i)
        if (std::fabs(got[i] - ref[i]) > 1e-9 * (1.0 + std::fabs(ref[i]))) return 15;
    stats[0] = h.S;
    stats[1] = cont_windows;
    return 0;
}
