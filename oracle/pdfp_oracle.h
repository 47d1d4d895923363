/*
 * pdfp_oracle.h -- CPU FP64 restatement of the PDFP reference's hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * B200 library (pdfp_b200/).  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline legs of bench.py may load it.  The product never links it.
 *
 * It restates, operation for operation and in FP64, the reference's CPU code
 * path (`use_gpu = false`) of MIT-Lu-Lab/PDFP v0.1.0:
 *   src/preconditioner.jl:26-125  (Ruiz + Pock-Chambolle scaling, power iteration)
 *   src/pdfp.jl:98-288            (restarted Halpern PDHG with reflection, l1 projection)
 *   src/pdlp.jl:10-393            (restarted Halpern PDHG for the root LP, cuPDLPx rules)
 *
 * Numerics: sparse products accumulate each output in ascending index order
 * (what Julia's SparseMatrixCSC mul! does), elementwise expressions are
 * evaluated in the reference's order, and the library is compiled with
 * -ffp-contract=off.  Norms, dots and sums are plain sequential sums (Julia
 * uses BLAS nrm2/dot and pairwise sums), so scalars agree with the reference
 * to rounding, not bitwise.  The power iteration starts from the SplitMix64 /
 * Box-Muller vector of or_normal_vector, not Julia's MersenneTwister stream;
 * the estimate of ||A||_2 therefore agrees with the reference only to the
 * iteration's tolerance.
 */
#ifndef PDFP_ORACLE_H
#define PDFP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_UNSPECIFIED = 0, OR_OPTIMAL = 1, OR_ITERATION_LIMIT = 2, OR_TIME_LIMIT = 3,
       OR_PRIMAL_INFEASIBLE = 4, OR_DUAL_INFEASIBLE = 5 };

/* SolverParameters + RestartParameters, src/pdlp.jl:10-31. */
typedef struct {
    double eps_optimal_relative;
    double eps_feasible_relative;
    int64_t iteration_limit;
    double time_limit;
    int32_t termination_evaluation_frequency;
    int32_t sv_max_iterations;
    double reflection_coefficient;
    double sv_tolerance;
    double artificial_restart_threshold;
    double sufficient_reduction_for_restart;
    double necessary_reduction_for_restart;
    double k_p, k_i, k_d, i_smooth;
} or_params;

typedef struct {
    int32_t status;
    int32_t restarts;
    int64_t total_count;
    double rel_primal, rel_dual, rel_gap;
    double primal_weight, step_size, max_singular_value, fixed_point_error;
    double objective_value;   /* PDLP only */
} or_result;

/* Fill or_params with the reference defaults (src/pdlp.jl:10-31). */
void or_default_params(or_params* p);

/* Deterministic N(0,1) vector: SplitMix64 stream from `seed`, two uniforms per
 * entry u1,u2 in (0,1) as ((z>>11)+0.5)*2^-53, value sqrt(-2 log u1) cos(2 pi u2).
 * Stands in for randn(MersenneTwister(20240517), m) at src/preconditioner.jl:111. */
void or_normal_vector(uint64_t seed, int64_t m, double* out);

/* scale_problem, src/preconditioner.jl:26-99, on a CSR matrix (0-based,
 * ascending column indices within each row).  Outputs may alias nothing. */
int or_scale_problem(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                     const double* c, const double* var_lb, const double* var_ub,
                     const double* con_lb, const double* con_ub,
                     int32_t ruiz_iterations, double pock_chambolle_alpha,
                     int32_t bound_objective_rescaling,
                     double* v_out, double* c_out, double* var_lb_out, double* var_ub_out,
                     double* con_lb_out, double* con_ub_out, double* D_r, double* D_c,
                     double* bound_scale, double* objective_scale);

/* estimate_max_singular_value, src/preconditioner.jl:108-125, started from
 * or_normal_vector(20240517, m). */
double or_estimate_max_singular_value(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                                      const double* v, int32_t max_iterations, double tolerance,
                                      int32_t* iterations_out);

/* ---- PDFP projector (src/pdfp.jl) ---- */
typedef struct or_pdfp or_pdfp;

/* PDFPState(A, b, is_eq, is_int, var_lb, var_ub, w), src/pdfp.jl:60-76. */
or_pdfp* or_pdfp_create(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                        const double* b, const uint8_t* is_eq, const uint8_t* is_int,
                        const double* var_lb, const double* var_ub, const double* w);
void or_pdfp_destroy(or_pdfp* s);
/* original_primal_residual!, src/pdfp.jl:85-90. */
void or_pdfp_original_primal_residual(or_pdfp* s, const double* D_r);
/* copyto!(s.current_x / s.initial_x, x), src/pump.jl:305-306. */
void or_pdfp_set_x(or_pdfp* s, const double* x);
/* set_target!, src/pdfp.jl:98-101 (copies the target, then warm_start!). */
void or_pdfp_set_target(or_pdfp* s, const double* x_tilde);
/* warm_start!, src/pdfp.jl:104-114. */
void or_pdfp_warm_start(or_pdfp* s);
/* pdfp_solve!, src/pdfp.jl:252-288. */
int32_t or_pdfp_solve(or_pdfp* s, const or_params* p, double primal_weight, or_result* r);
/* Read a state vector: which = 0 pdhg_x, 1 pdhg_y, 2 pdhg_z, 3 current_x,
 * 4 current_y, 5 current_z, 6 dual_slack, 7 reflected_x. */
void or_pdfp_get(const or_pdfp* s, int32_t which, double* out);
/* Run `count` PDHG steps with Halpern offsets k0..k0+count-1 (test hook). */
void or_pdfp_steps(or_pdfp* s, double step_size, double primal_weight, int32_t k0, int32_t count);
/* Seed the per-run cache of ||A||_2 that pdfp_solve! fills on its first call
 * (src/pdfp.jl:225-229), as a pump run that already estimated it has it
 * (benchmark hook: the CPU baseline times solves, not the estimate). */
void or_pdfp_set_max_singular_value(or_pdfp* s, double sigma);

/* ---- root LP (src/pdlp.jl) ---- */
/* solve_lp_relaxation, src/pdlp.jl:381-393, for the canonical MILP rows
 * (is_le[i] = 1: A_i x <= b_i, else A_i x = b_i).  x_out: original units;
 * dual_slack_out: scaled units. */
int32_t or_solve_lp_relaxation(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                               const double* v, const double* c, const double* l, const double* u,
                               const double* b, const uint8_t* is_le, double tolerance,
                               double time_limit, int32_t cupdlpx_termination,
                               double* x_out, double* dual_slack_out, or_result* r);

/* The PDLP state itself (for finer tests): pdlp_solve! on a scaled problem. */
int32_t or_pdlp_solve_scaled(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                             const double* v, const double* c, const double* var_lb,
                             const double* var_ub, const double* con_lb, const double* con_ub,
                             double bound_scale, double objective_scale,
                             const double* D_r /* nullable: cuPDLPx termination if set */,
                             const double* D_c, const or_params* p,
                             double* pdhg_primal, double* pdhg_dual, double* dual_slack,
                             or_result* r);

/* Number of OpenMP threads used by the sparse products and vector loops
 * (1 unless the library was built with -fopenmp). */
void or_set_threads(int32_t threads);
int32_t or_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
