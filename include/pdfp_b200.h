/*
 * pdfp_b200.h -- C ABI of libpdfp_b200.so, the B200 projector and root-LP
 * solver of the PDFP feasibility pump.
 *
 * The library owns every device buffer of a handle for the handle's lifetime
 * (the whole pump run); host pointers passed in are borrowed for the duration
 * of the call and copied.  Every entry point returns 0 on success or a
 * negative PDFP_E* code; pdfp_last_error() gives the message of the last
 * failure on the calling thread.  Nothing aborts the process.
 *
 * Each entry point cites the reference interface (MIT-Lu-Lab/PDFP v0.1.0,
 * paths relative to its source tree) that it replaces.
 *
 * Indices are 0-based int32 CSR with ascending column indices per row; the
 * reference's Julia shim converts its 1-based Int64 CSC (a transpose-free
 * conversion: CSC of A' is the CSR of A).
 *
 * Threading: a handle is not re-entrant; separate handles may be used from
 * separate threads.  All work of a handle runs on one CUDA stream owned by it.
 */
#ifndef PDFP_B200_H
#define PDFP_B200_H
#include <stdint.h>

#if defined(__GNUC__)
#define PDFP_API __attribute__((visibility("default")))
#else
#define PDFP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------- */
#define PDFP_OK 0
#define PDFP_E_INVALID (-1)      /* bad argument (shape, CSR structure, NaN input) */
#define PDFP_E_CUDA (-2)         /* CUDA runtime error */
#define PDFP_E_NOMEM (-3)        /* device allocation failed */
#define PDFP_E_TIMEOUT (-4)      /* a bounded device wait gave up */
#define PDFP_E_UNSUPPORTED (-5)  /* size beyond the library's limits */
#define PDFP_E_NODEVICE (-6)     /* no CUDA device */

/* Termination reasons, the reference's Symbols (src/pdfp.jl:276-286,
 * src/pdlp.jl:352-370). */
#define PDFP_UNSPECIFIED 0
#define PDFP_OPTIMAL 1
#define PDFP_ITERATION_LIMIT 2
#define PDFP_TIME_LIMIT 3
#define PDFP_PRIMAL_INFEASIBLE 4
#define PDFP_DUAL_INFEASIBLE 5

/* Arithmetic of the iterations.  FP64: plain FP64 form.  MIXED: iterates,
 * matrix values and row accumulation in FP32; KKT/gap/restart reductions,
 * Halpern weights and the reported distance in FP64 on the device; an FP64
 * polish takes over when the FP32 residual stalls above tolerance or reaches
 * the FP32 floor under a tighter tolerance (pdfp_set_polish). */
#define PDFP_FP64 0
#define PDFP_MIXED 1

/* Which state vector pdfp_get_vector reads (all in scaled units). */
#define PDFP_VEC_PDHG_X 0
#define PDFP_VEC_PDHG_Y 1
#define PDFP_VEC_PDHG_Z 2
#define PDFP_VEC_CURRENT_X 3
#define PDFP_VEC_CURRENT_Y 4
#define PDFP_VEC_CURRENT_Z 5
#define PDFP_VEC_DUAL_SLACK 6
#define PDFP_VEC_REFLECTED_X 7

typedef struct pdfp_handle pdfp_handle;

/* A sparse matrix: m rows, n columns, row_ptr[m+1], col_idx/val[row_ptr[m]]. */
typedef struct {
    int32_t m, n;
    const int32_t* row_ptr;
    const int32_t* col_idx;
    const double* val;
} pdfp_csr;

/* SolverParameters + RestartParameters, src/pdlp.jl:10-31 (same meaning and
 * defaults; see pdfp_default_params). */
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
} pdfp_params;

/* Outcome of one solve (per instance for batches). */
typedef struct {
    int32_t status;              /* PDFP_OPTIMAL, ... (termination_reason) */
    int32_t restarts;
    int64_t total_count;         /* PDHG iterations of this solve (multiple of the evaluation frequency) */
    double rel_primal, rel_dual, rel_gap;
    double primal_weight, step_size, max_singular_value, fixed_point_error;
    double objective_value;      /* PDLP: c'x in original units; PDFP: l1 distance sum_I w|x - x~| (scaled data) */
    int32_t polished;            /* MIXED: 1 if the FP64 polish finished this solve */
    int32_t precision;           /* arithmetic at termination (PDFP_FP64 / PDFP_MIXED) */
    double device_ms;            /* device time of the solve: CUDA events on the handle's stream */
    double kernel_ms_primal;     /* timing mode: mean device time of the A'-side step kernel */
    double kernel_ms_dual;       /* timing mode: mean device time of the A-side step kernel */
    int64_t kernel_samples;      /* timing mode: minor steps in the timed runs */
    int64_t fp64_iterations;     /* PDHG iterations of this solve run in FP64 (MIXED: the polish) */
} pdfp_result;

/* One projection problem (the data of PDFPState, src/pdfp.jl:15-52), already
 * scaled.  is_eq[m], is_int[n] are 0/1 bytes; w[n] the y-box half widths
 * (used on is_int columns); row_unscale[m] (nullable) = 1 ./ D_r switches the
 * primal residual to original units (original_primal_residual!). */
typedef struct {
    pdfp_csr A;
    const double* b;
    const uint8_t* is_eq;
    const uint8_t* is_int;
    const double* var_lb;
    const double* var_ub;
    const double* w;
    const double* row_unscale;
} pdfp_problem;

/* ---- library ---------------------------------------------------------------- */

/* Fill the reference defaults (src/pdlp.jl:10-31). */
PDFP_API void pdfp_default_params(pdfp_params* p);
/* Message of the last failure on the calling thread ("" if none). */
PDFP_API const char* pdfp_last_error(void);
/* Name of the CUDA device the library uses (the pump log's "device" line,
 * src/pump.jl:442). */
PDFP_API int pdfp_device_name(char* buf, int32_t len);
/* Make `device` the calling thread's CUDA device for this library's later calls
 * (one process per GPU: each rank selects its own; the library otherwise uses the
 * thread's current device). */
PDFP_API int pdfp_set_device(int32_t device);
/* Version string of this library. */
PDFP_API const char* pdfp_version(void);

/* ---- projector: PDFPState and its methods (src/pdfp.jl) ---------------------- */

/* PDFPState(A, b, is_eq, is_int, var_lb, var_ub, w; use_gpu = true),
 * src/pdfp.jl:60-76, plus original_primal_residual!(s, D_r), src/pdfp.jl:85-90
 * when row_unscale (= 1 ./ D_r) is not NULL. */
PDFP_API int pdfp_create(const pdfp_csr* A, const double* b, const uint8_t* is_eq, const uint8_t* is_int,
                const double* var_lb, const double* var_ub, const double* w,
                const double* row_unscale, int32_t precision, pdfp_handle** out);

/* k independent projections packed block-diagonally into one handle: one
 * launch sequence advances all of them, each with its own restart and
 * termination state on the device.  Replaces the reference's concurrent
 * trajectory processes (scripts/solve.jl:121-148) with batch members. */
PDFP_API int pdfp_create_batch(int32_t k, const pdfp_problem* problems, int32_t precision,
                      pdfp_handle** out);

/* copyto!(s.current_x, x); copyto!(s.initial_x, x), src/pump.jl:305-306. */
PDFP_API int pdfp_set_x(pdfp_handle* h, int32_t instance, const double* x);
/* set_target!(s, x_tilde_scaled), src/pdfp.jl:98-101 (then warm_start!). */
PDFP_API int pdfp_set_target(pdfp_handle* h, int32_t instance, const double* x_tilde);
/* warm_start!(s), src/pdfp.jl:104-114. */
PDFP_API int pdfp_warm_start(pdfp_handle* h, int32_t instance);
/* pdfp_solve!(s, p, primal_weight), src/pdfp.jl:252-288: instance 0 of the
 * handle (single-problem handles). */
PDFP_API int pdfp_solve(pdfp_handle* h, const pdfp_params* p, double primal_weight, pdfp_result* r);
/* pdfp_solve! for every member of a batch handle at once; params,
 * primal_weights and results hold one entry per instance. */
PDFP_API int pdfp_solve_batch(pdfp_handle* h, const pdfp_params* params, const double* primal_weights,
                     pdfp_result* results);
/* pdfp_solve! for the members of a batch handle, returning as soon as at least one
 * member that was running has stopped (checked at evaluation-window boundaries);
 * the others stop at their next window boundary and report status 0 (still
 * running).  A later call with resume[p] != 0 continues member p exactly where it
 * stopped (its tolerances, limits, restart state and counters stand; params[p] is
 * not read for it); members with resume[p] == 0 (or resume == NULL) start a new
 * solve as in pdfp_solve_batch.  Resuming a member that is not running from the
 * previous call, or after pdfp_set_target / pdfp_warm_start on it, is an error.
 * This lets concurrent pump trajectories each advance at their own pace, as the
 * reference's separate pump processes do (scripts/solve.jl:121-148), instead of
 * every pump iteration waiting for the slowest member's projection. */
PDFP_API int pdfp_solve_batch_any(pdfp_handle* h, const pdfp_params* params,
                                  const double* primal_weights, const uint8_t* resume,
                                  pdfp_result* results);
/* Read a state vector of an instance (s.pdhg_x etc., scaled units, the
 * caller's variable/row order). */
PDFP_API int pdfp_get_vector(pdfp_handle* h, int32_t instance, int32_t which, double* out);
/* s.pdhg_x of an instance: the projection in scaled units (src/pump.jl:338). */
PDFP_API int pdfp_get_x(pdfp_handle* h, int32_t instance, double* x_scaled);

/* ---- the pump's column scaling on the device (src/pump.jl:300-354) ----------
 * The pump feeds the projector x ./ D_c and x_tilde ./ D_c and reads back
 * D_c .* s.pdhg_x (src/pump.jl:305-306, 331, 338, 354).  After
 * pdfp_set_col_scale, the *_unscaled calls take and return vectors in the
 * model's own units and do the division and product on the device, correctly
 * rounded in FP64: bit-identical to the host arithmetic they replace.
 * D_c: n entries, positive and finite (E_INVALID otherwise); the unscaled
 * calls return E_INVALID until it is set for the instance. */
PDFP_API int pdfp_set_col_scale(pdfp_handle* h, int32_t instance, const double* D_c);
/* pdfp_set_x(h, instance, x ./ D_c), src/pump.jl:305-306. */
PDFP_API int pdfp_set_x_unscaled(pdfp_handle* h, int32_t instance, const double* x);
/* pdfp_set_target(h, instance, x_tilde ./ D_c), src/pump.jl:331. */
PDFP_API int pdfp_set_target_unscaled(pdfp_handle* h, int32_t instance, const double* x_tilde);
/* D_c .* (a primal column vector: PDFP_VEC_PDHG_X, _CURRENT_X or _REFLECTED_X). */
PDFP_API int pdfp_get_vector_unscaled(pdfp_handle* h, int32_t instance, int32_t which, double* out);
/* D_c .* s.pdhg_x, src/pump.jl:338. */
PDFP_API int pdfp_get_x_unscaled(pdfp_handle* h, int32_t instance, double* x);

/* Page-locked host memory for the vectors passed to the setters and getters:
 * host <-> device copies from it run at DMA speed instead of through the
 * driver's pageable staging.  Any host pointer is accepted by every call;
 * this is only faster.  Free with pdfp_host_free. */
PDFP_API int pdfp_host_alloc(int64_t bytes, void** out);
PDFP_API int pdfp_host_free(void* p);
/* Instance count, rows and columns of an instance. */
PDFP_API int pdfp_shape(const pdfp_handle* h, int32_t instance, int32_t* k, int32_t* m, int32_t* n);
/* Release every device buffer of the handle (the Julia finalizer). */
PDFP_API int pdfp_destroy(pdfp_handle* h);

/* Timing mode: when on, every evaluation window of later solves also records
 * CUDA events around a run of its minor steps (the middle half of them, with no
 * other event inside, so that they run as in any window) and around each kernel
 * of up to eight single minor steps outside the run; pdfp_result reports the
 * run's mean step time split between the two step kernels in the proportion of
 * the single steps (benchmark support; off by default). */
PDFP_API int pdfp_set_kernel_timing(pdfp_handle* h, int32_t on);

/* Mixed precision (PDFP_MIXED handles): an instance starts each solve in FP32;
 * the FP64 polish -- the iterates converted to FP64 on the device, the solve
 * continued in FP64 to its tolerance -- takes over after `stall_evaluations`
 * evaluations without a 10% improvement of the KKT score (the largest
 * residual-to-tolerance ratio) while above tolerance, or as soon as the
 * relative residuals reach `fp32_floor` while the requested tolerance is
 * tighter.  Defaults 10 and 1e-6.  stall_evaluations = 0 switches the polish
 * off (an instance whose tolerance is below fp32_floor then runs in FP64 from
 * the start).  The reference has no mixed form; its loop is pdfp_solve!,
 * src/pdfp.jl:252-288. */
PDFP_API int pdfp_set_polish(pdfp_handle* h, int32_t stall_evaluations, double fp32_floor);

/* The step-kernel configuration the autotuner chose at creation.  It times, on
 * the handle's own matrix, the tile engine (shared-memory stage size x threads
 * per role x gather policy) and the flat engine (both cache policies) and
 * keeps the fastest per side; below 256K nonzeros it keeps the default.
 * Gather policy: 0 = register gathers cached in L1, 1 = register gathers cached
 * in L2 only, 2 = per-thread async copies into the shared-memory stage (FP32
 * steps of the tile engine; the reducers form the products, with the same
 * roundings in the same order, so results do not depend on the policy).
 * The FP32 steps may also run on the vec engine (warps over rows read straight
 * from the CSR arrays, lanes per row by row length; threads per role 32, "stage
 * bytes" its target nonzeros per lane 1, 2, 4 or 8; gather policy 0 or 1).
 * PDFP_AUTOTUNE=0 / =1 switches it off / on regardless of size, and
 * PDFP_STEP_ENGINE=tile / =flat / =flat1 / =vec fixes the engine with its default
 * settings (flat1: the flat engine's one-quad-per-thread variant; vec: the FP32
 * steps, the FP64 steps stay on the tile engine), and
 * PDFP_TUNING="s,t,l,s,t,l[,n,n[,b,b]]" pins both sides for handles created
 * while it is set: stage bytes, threads per role and the gather policy of A',
 * then of A, with the values out[] below reports, and optionally the stage
 * counts of A' and A (pdfp_get_tuning_stages; default 4), their caps on
 * resident blocks per SM (pdfp_get_tuning_blocks; default 0) and their reducer
 * threads (pdfp_get_tuning_reducers; 0: as many as gatherers).
 * out[8] = {A' stage bytes, A' threads per role (0: flat engine, 32: vec
 * engine), A' tiles (vec engine: work items), A stage bytes, A threads per role,
 * A tiles, A' gather policy, A gather policy}. */
PDFP_API int pdfp_get_tuning(const pdfp_handle* h, int32_t* out);
/* Shared-memory stages per block of the tile engine on each side: out[2] =
 * {A', A} (2..4; 4 for the flat engine, which has none). */
PDFP_API int pdfp_get_tuning_stages(const pdfp_handle* h, int32_t* out);
/* Cap on resident blocks per SM of the tile engine on each side: out[2] = {A', A}
 * (0: as many as shared memory and registers allow).  With a cap the launch asks
 * for only those blocks' shared memory, leaving the rest of the SM's unified
 * L1 / shared memory as L1, where a gather-bound kernel keeps its misses in flight. */
PDFP_API int pdfp_get_tuning_blocks(const pdfp_handle* h, int32_t* out);
/* Reducer threads per block of the tile engine on each side: out[2] = {A', A}
 * (the gatherers are the threads per role of pdfp_get_tuning; FP32 steps may run
 * half as many reducers as gatherers; 0 for the flat engine). */
PDFP_API int pdfp_get_tuning_reducers(const pdfp_handle* h, int32_t* out);
/* The A-side step of the FP32 steps with its long rows regrouped by column
 * segment: out[2] = {segments, long-row threshold in nonzeros}, {0, 0} when the
 * handle runs it without.  The rows with at least that many nonzeros are summed
 * by one block per column segment, gathering from that segment of x_bar held in
 * shared memory, and finished one warp per row (FP64 sum of the segments'
 * partials in segment order); the other rows stay on the tile engine.  Off
 * by default.  PDFP_SEG=tune lets the autotuner try a few segmentations on
 * handles of at least 2^22 nonzeros and keep one only if it beats the tile
 * engine's A-side step; PDFP_SEG="n,l[,s,t,k[,b]]" fixes n segments and
 * threshold l (and the partials pass's stage bytes, threads per role, stages
 * and blocks per segment); PDFP_SEG=0: off. */
PDFP_API int pdfp_get_tuning_seg(const pdfp_handle* h, int32_t* out);
/* How a window's minor steps run: *out = 0, two step launches per step replayed
 * from a captured graph; 1, one cooperative launch of the per-block row passes
 * (PDFP_MEDIUM=1); 2, one cooperative launch of the vec engine's warp items
 * (PDFP_VEC_WINDOW=1, both FP32 sides on the vec engine without long-row
 * pieces); 3, whole windows of each small member in one block's launch. */
PDFP_API int pdfp_get_window_form(const pdfp_handle* h, int32_t* out);
/* Every measurement the autotuner took: up to `cap` rows, ms[i] the mean
 * launch time, cfg[7i..7i+6] = {side (0: A', 1: A), stage bytes, gatherer
 * threads (0: flat engine; 32: vec engine, whose stage bytes are its nonzeros
 * per lane), gather policy, stages, blocks per SM cap, reducer threads}; side 2:
 * the A side with segmented long rows (pdfp_get_tuning_seg), {2, segments,
 * long-row threshold, gather policy of the other rows, then the partials pass's
 * stages, stage bytes and threads per role}; *count receives the number of rows. */
PDFP_API int pdfp_get_tuning_table(const pdfp_handle* h, float* ms, int32_t* cfg, int32_t cap,
                                   int32_t* count);

/* Kernel timing of the two fused PDHG step kernels, over `iterations` steps
 * of instance state as it stands (benchmark support; state advances). ms_*
 * receive the mean device time per launch. */
PDFP_API int pdfp_profile_step(pdfp_handle* h, int32_t iterations, float* ms_primal, float* ms_dual,
                      double* bytes_primal, double* bytes_dual);

/* ---- preconditioner (src/preconditioner.jl) --------------------------------- */

/* scale_problem(A, c, var_lb, var_ub, con_lb, con_ub; ruiz_iterations,
 * pock_chambolle_alpha, bound_objective_rescaling), src/preconditioner.jl:26-99,
 * computed on the device.  val_out has A's sparsity pattern. */
PDFP_API int pdfp_scale_problem(const pdfp_csr* A, const double* c, const double* var_lb,
                       const double* var_ub, const double* con_lb, const double* con_ub,
                       int32_t ruiz_iterations, double pock_chambolle_alpha,
                       int32_t bound_objective_rescaling, double* val_out, double* c_out,
                       double* var_lb_out, double* var_ub_out, double* con_lb_out,
                       double* con_ub_out, double* D_r, double* D_c, double* bound_scale,
                       double* objective_scale);

/* read_mps (src/milp.jl:42-94) on the host, in C++: an MPS file, plain or
 * gzip-compressed (zlib), into the pump's canonical form -- min c'x + c0 s.t.
 * A x <= b (is_eq[i] == 0) / A x = b (is_eq[i] != 0), l <= x <= u, x_j integer
 * for j in int_idx -- with the reference's canonicalisation (maximisation
 * negated, binaries clipped to [0, 1], equal finite row bounds -> equality,
 * else hi row then -lo row, |v| >= 1e20 infinite).  CSR rows list their
 * columns ascending (0-based).  pdfp_mps_dims gives the sizes, pdfp_mps_get
 * copies the arrays out (c, l, u: n; b, is_eq: m; row_ptr: m + 1; col_idx,
 * val: nnz; int_idx: n_int).  Needs no GPU. */
typedef struct pdfp_mps pdfp_mps;
PDFP_API int pdfp_mps_read(const char* path, pdfp_mps** out);
PDFP_API int pdfp_mps_dims(const pdfp_mps* p, int32_t* m, int32_t* n, int64_t* nnz, int32_t* n_int);
PDFP_API int pdfp_mps_get(const pdfp_mps* p, double* c, double* c0, int32_t* row_ptr,
                          int32_t* col_idx, double* val, double* b, uint8_t* is_eq, double* l,
                          double* u, int32_t* int_idx);
PDFP_API int pdfp_mps_destroy(pdfp_mps* p);

/* ---- the pump's constraint-propagation rounding, on the host ----------------
 * FP 2.0's CPR rounding as the reference runs it on the CPU: activity-based
 * bound propagation (src/propagation.jl:1-276) behind the guarded two-phase
 * rounding (src/rounding.jl:117-256), native.  Needs no GPU.
 * pdfp_rounder_create: the model part (PropagationData, src/propagation.jl:19-84)
 * from the canonical rows A x <= b (is_le[i] = 1) or A x = b, column indices
 * strictly ascending within each row, bounds l <= x <= u (infinite allowed),
 * is_int per column. */
typedef struct pdfp_rounder pdfp_rounder;
PDFP_API int pdfp_rounder_create(const pdfp_csr* A, const double* b, const uint8_t* is_le,
                                 const double* l, const double* u, const uint8_t* is_int,
                                 pdfp_rounder** out);
/* One rounding of x_star (n values) into xt (n values) on fresh domains:
 * xt = x_star; the columns first[0..n_first) are fixed one by one in that order,
 * each rounded to nearest (ties to even) inside its current domain -- moved by
 * one toward the domain if that leaves it, or chosen by the row violations when
 * direction[j] is set (direction may be NULL) -- and propagated after each fix
 * (_round_sequentially, src/rounding.jl:152-174); with batch_phase set, the
 * columns batch[0..n_batch) are then all fixed at their rounded values and
 * propagated once (the guard: *infeasible = 2 and an incomplete xt when that
 * leaves the domains infeasible); then after[0..n_after) as `first`; finally the
 * columns int_idx[0..n_int) read their values off the domains (fixed: the bound;
 * else the rounded clamped x_star).  max_pops caps the rows popped per
 * propagation (src/propagation.jl:235-244).  Otherwise *infeasible reports the
 * final domains' state (1: infeasible, 0: not found infeasible). */
PDFP_API int pdfp_rounder_round(const pdfp_rounder* r, const double* x_star, const int32_t* first,
                                int32_t n_first, int32_t batch_phase, const int32_t* batch,
                                int32_t n_batch, const int32_t* after, int32_t n_after,
                                const int32_t* int_idx, int32_t n_int, const uint8_t* direction,
                                int64_t max_pops, double* xt, int32_t* infeasible);
PDFP_API int pdfp_rounder_destroy(pdfp_rounder* r);

/* max_violation(milp, x), src/milp.jl:102-114, on the device: the largest
 * violation of A x <= b (rows with is_eq[i] == 0) and A x = b (is_eq[i] != 0)
 * over the ORIGINAL constraints (caller's numbering, 0-based CSR, ascending
 * column indices), 0 when nothing is violated.  Rows are summed in ascending
 * column order with separately rounded operations, so the value equals the
 * host's A * x evaluation bit for bit.  A checker owns device copies of A, b
 * and is_eq; pdfp_checker_max_violation copies x (n values) to the device and
 * returns when the value is on the host.  Not re-entrant. */
typedef struct pdfp_checker pdfp_checker;
PDFP_API int pdfp_checker_create(const pdfp_csr* A, const double* b, const uint8_t* is_eq,
                                 pdfp_checker** out);
PDFP_API int pdfp_checker_max_violation(pdfp_checker* c, const double* x, double* violation);
PDFP_API int pdfp_checker_destroy(pdfp_checker* c);

/* Self-test of the library's bounded device waits (no counterpart in the
 * reference, whose loop ends only on its time and iteration limits,
 * src/pdfp.jl:279-282).  Every spin of this library's kernels gives up after a
 * limit and turns into PDFP_E_TIMEOUT with the CUDA context still usable; no
 * correct solve reaches those limits.  This call runs the same wait code in a
 * small kernel whose wait cannot complete -- which = 0: the tile engine's
 * mbarrier wait, on a phase that gets one arrival fewer than it expects;
 * which = 1: the cooperative window's grid barrier, expecting one block more
 * than launched -- with a limit of limit_seconds (0 < limit <= 4), no copy in
 * flight.  Returns PDFP_E_TIMEOUT when the wait gave up as designed. */
PDFP_API int pdfp_selftest_bounded_wait(int32_t which, double limit_seconds);

/* estimate_max_singular_value(A, A_t, m; max_iterations, tolerance),
 * src/preconditioner.jl:108-125, on the device. */
PDFP_API int pdfp_estimate_max_singular_value(const pdfp_csr* A, int32_t max_iterations, double tolerance,
                                     double* sigma, int32_t* iterations);

/* ||A||_2 by power iteration on matrices already on the device, with no
 * device allocation (no counterpart in the reference).  For callers that
 * cannot call cudaMalloc: processes whose device memory a framework allocator
 * reserved up front (a new cudaMalloc fails or fragments its pool) and callers
 * that must not trigger the device-wide synchronisation of cudaFree.  A and
 * A' are device CSR arrays (0-based, ascending indices per row; none may be
 * NULL when its side has rows); the work vectors live in a fixed 8 MiB array
 * of this library's device memory, so 2m + n + 2 must not exceed 1,048,576
 * (PDFP_E_UNSUPPORTED otherwise).  The driver commits that array on a device
 * at the first call there (CUDA's default lazy module loading; at library load
 * under CUDA_MODULE_LOADING=EAGER) and the device keeps it until the process
 * exits: make one call per device before reserving device memory up front, and
 * before any stream capture (that call also resolves the array's address for
 * the calling context).  Calls share the array and it keeps the last call's
 * contents: calls that overlap on the GPU race.  The iteration runs in one
 * thread block; near the size limit an iteration costs about a millisecond.
 * `stream` is a cudaStream_t (NULL: the default stream); the call returns when
 * the result is on the host.  Same algorithm, start vector and summation order
 * as pdfp_estimate_max_singular_value. */
PDFP_API int pdfp_estimate_max_singular_value_noalloc(
    int32_t m, int32_t n, const int32_t* row_ptr, const int32_t* col_idx, const double* val,
    const int32_t* row_ptr_t, const int32_t* col_idx_t, const double* val_t,
    int32_t max_iterations, double tolerance, void* stream, double* sigma, int32_t* iterations);

/* ---- root LP (src/pdlp.jl) --------------------------------------------------- */

/* solve_lp_relaxation(milp; tolerance, time_limit, use_gpu = true,
 * cupdlpx_termination), src/pdlp.jl:381-393, for the canonical MILP rows
 * (is_le[i] = 1: A_i x <= b_i, else A_i x = b_i).  x_out in original units,
 * dual_slack_out in scaled units, as the reference returns them. */
PDFP_API int pdlp_solve_relaxation(const pdfp_csr* A, const double* c, const double* l, const double* u,
                          const double* b, const uint8_t* is_le, double tolerance,
                          double time_limit, int32_t cupdlpx_termination, int32_t precision,
                          double* x_out, double* dual_slack_out, pdfp_result* r);

#ifdef __cplusplus
}
#endif
#endif
