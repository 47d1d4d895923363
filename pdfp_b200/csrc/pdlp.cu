// pdlp.cu -- the root-LP solver (placeholder until the PDLP engine lands).
#include "device.hpp"
#include "solvers.hpp"

namespace pdfp {

void solve_lp_relaxation_device(const pdfp_csr&, const double*, const double*, const double*,
                                const double*, const uint8_t*, double, double, bool, int, double*,
                                double*, pdfp_result*) {
    throw Error(E_UNSUPPORTED, "pdlp_solve_relaxation is not built yet");
}

}  // namespace pdfp
