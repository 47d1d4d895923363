// solvers.hpp -- the handle-free solver entry points behind the C ABI.
#pragma once
#include "../../include/pdfp_b200.h"

namespace pdfp {

// scale_problem (src/preconditioner.jl:26-99) on the device.
void scale_problem_device(const pdfp_csr& A, const double* c, const double* var_lb,
                          const double* var_ub, const double* con_lb, const double* con_ub,
                          int32_t ruiz_iterations, double alpha, bool rescale, double* val_out,
                          double* c_out, double* var_lb_out, double* var_ub_out, double* con_lb_out,
                          double* con_ub_out, double* D_r, double* D_c, double* bound_scale,
                          double* objective_scale);

// estimate_max_singular_value (src/preconditioner.jl:108-125) on the device.
double estimate_sv_device(const pdfp_csr& A, int32_t max_iterations, double tolerance,
                          int32_t* iterations);

// solve_lp_relaxation (src/pdlp.jl:381-393) on the device.
void solve_lp_relaxation_device(const pdfp_csr& A, const double* c, const double* l,
                                const double* u, const double* b, const uint8_t* is_le,
                                double tolerance, double time_limit, bool cupdlpx, int precision,
                                double* x_out, double* dual_slack_out, pdfp_result* r);


// The pump's constraint check on the device (checker.cu).
struct Checker;
Checker* checker_create(const pdfp_csr& A, const double* b, const uint8_t* is_eq);
double checker_max_violation(Checker& c, const double* x);
void checker_destroy(Checker* c);

// The pump's constraint-propagation rounding on the host (rounding.cpp).
struct Rounder;
Rounder* rounder_create(const pdfp_csr* A, const double* b, const uint8_t* is_le, const double* l,
                        const double* u, const uint8_t* is_int);
void rounder_destroy(Rounder* r);
void rounder_round(const Rounder& r, const double* x_star, const int32_t* first, int32_t n_first,
                   int32_t batch_phase, const int32_t* batch, int32_t n_batch, const int32_t* after,
                   int32_t n_after, const int32_t* int_idx, int32_t n_int, const uint8_t* direction,
                   int64_t max_pops, double* xt, int32_t* infeasible);

}  // namespace pdfp
