// controller.cuh -- the restart rules shared by the projector and the root LP.
//
// should_restart and update_primal_weight! (src/pdlp.jl:167-205) evaluated on
// the device from one instance's state, by the controller kernels.
#pragma once
#include "common.cuh"
#include "state.hpp"

namespace pdfp {

// should_restart, src/pdlp.jl:167-181
__device__ __forceinline__ bool should_restart(InstState& s) {
    bool restart = false;
    const int64_t freq = s.freq;
    if (s.total == freq) {
        restart = true;
    } else if (s.total > freq) {
        if (s.fpe <= s.suff * s.initial_fpe) restart = true;
        if (s.fpe <= s.nec * s.initial_fpe && s.fpe > s.last_trial_fpe) restart = true;
        if (static_cast<double>(s.inner) >= s.art * static_cast<double>(s.total)) restart = true;
    }
    s.last_trial_fpe = s.fpe;
    return restart;
}

// update_primal_weight!, src/pdlp.jl:185-205
__device__ __forceinline__ void update_primal_weight(InstState& s, double primal_dist,
                                                     double dual_dist) {
    const double eps = 2.220446049250313e-16;
    const double ratio = s.rel_d / jl_max(s.rel_p, eps);
    if (1e-16 < primal_dist && primal_dist < 1e12 && 1e-16 < dual_dist && dual_dist < 1e12 &&
        1e-8 < ratio && ratio < 1e8) {
        const double err = log(dual_dist) - log(primal_dist) - log(s.primal_weight);
        s.err_sum *= s.ismooth;
        s.err_sum += err;
        const double delta_err = err - s.last_err;
        s.primal_weight *= exp(s.kp * err + s.ki * s.err_sum + s.kd * delta_err);
        s.last_err = err;
    } else {
        s.primal_weight = s.best_primal_weight;
        s.err_sum = 0.0;
        s.last_err = 0.0;
    }
    const double gap = fabs(log10(s.rel_d / jl_max(s.rel_p, eps)));
    if (gap < s.best_gap) {
        s.best_gap = gap;
        s.best_primal_weight = s.primal_weight;
    }
}

}  // namespace pdfp
