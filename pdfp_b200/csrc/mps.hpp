// mps.hpp -- the canonical MILP an MPS file reads into (mps.cpp).
#pragma once
#include <cstdint>
#include <vector>

namespace pdfp {

// min c'x + c0  s.t.  A x <= b / A x = b (is_eq), l <= x <= u, x_j integer on int_idx.
struct MpsModel {
    int32_t m = 0, n = 0;
    std::vector<double> c, b, l, u;
    double c0 = 0.0;
    std::vector<int32_t> rp, ci, int_idx;  // CSR of A, rows listing columns ascending
    std::vector<double> v;
    std::vector<uint8_t> is_eq;
};

MpsModel* read_mps_file(const char* path);
void mps_destroy(MpsModel* m);

}  // namespace pdfp
