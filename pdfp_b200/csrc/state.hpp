// state.hpp -- per-instance solver state kept on the device.
//
// Every scalar the reference's pdfp_solve! / pdlp_solve! keeps in the state
// struct (src/pdfp.jl:15-52, src/pdlp.jl:33-76) lives here, one entry per
// batch member, in FP64.  Kernels read step sizes, the Halpern counter and the
// status from it; the controller kernel updates it after every evaluation, so
// a whole evaluation window runs without the host.
#pragma once
#include <cstdint>

namespace pdfp {

enum : int32_t { ST_RUNNING = 0, ST_OPTIMAL = 1, ST_ITERATION_LIMIT = 2, ST_TIME_LIMIT = 3,
                 ST_PRIMAL_INFEASIBLE = 4, ST_DUAL_INFEASIBLE = 5 };
enum : int32_t { MODE_FP64 = 0, MODE_FP32 = 1 };

struct InstState {
    // step sizes and primal weight (src/pdfp.jl:34-40)
    double step_size, primal_weight, best_primal_weight, best_gap, err_sum, last_err;
    double tau, sigma;  // step_size / primal_weight, step_size * primal_weight
    // restart bookkeeping (src/pdfp.jl:41-45)
    double fpe, initial_fpe, last_trial_fpe;
    // termination (src/pdfp.jl:46-50)
    double rel_p, rel_d, rel_gap, l1;
    double dual_den, gap_den, b_norm;
    double max_sv;  // ||A||_2 of the instance, NaN until estimated
    // PDLP (src/pdlp.jl:46-74)
    double bound_scale, objective_scale, cbn, ovn, objective_value;
    double max_primal_ray_inf, primal_ray_lin_obj, max_dual_ray_inf, dual_ray_obj;
    // parameters of the current solve
    double eps_opt, eps_feas, time_limit, omega;
    double art, suff, nec, kp, ki, kd, ismooth;
    double best_score;  // mixed precision: best KKT score seen (stall test)
    double fp32_floor;  // mixed precision: relative residual the FP32 phase aims for
    int64_t inner, total, iter_limit;
    int64_t fp64_iters;  // PDHG iterations of this solve run in FP64
    uint64_t t_start_ns;
    int32_t status, do_restart, restart_now, restarts;
    int32_t freq, mode, stall, stall_limit;  // stall_limit: evaluations without progress before the polish (0: never)
    int32_t nnz_zero, pad0, pad1, pad2;
};

// One solve's parameters for one instance (SolverParameters, src/pdlp.jl:21-31).
struct SolveParams {
    double eps_opt, eps_feas, time_limit, omega;
    double art, suff, nec, kp, ki, kd, ismooth;
    double primal_weight;
    double fp32_floor;
    int64_t iter_limit;
    int32_t freq, mode;
    int32_t stall_limit;
    int32_t resume;  // 1: the instance is running from an earlier call; keep its state
};

// What the host polls after every window.
struct InstFlags {
    int32_t status, mode, polish_request, pad;
};

// Power iteration state (src/preconditioner.jl:108-125).
struct PowerState {
    double nrm, sigma_sq, dot, res_sq, eig_sq, tol;
    int32_t it, max_it, done, pad;
};

}  // namespace pdfp
