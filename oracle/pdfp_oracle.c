/*
 * pdfp_oracle.c -- CPU FP64 restatement of the PDFP reference's hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the parity checker); see pdfp_oracle.h.
 * Every routine cites the reference function it restates (paths relative to
 * the MIT-Lu-Lab/PDFP source tree).  Compile with -ffp-contract=off.
 *
 * Sparse products and per-element loops may run on several OpenMP threads;
 * each output element is still computed by one thread in the reference's
 * order, and every reduction is a sequential loop, so the results do not
 * depend on the thread count.
 */
#define _POSIX_C_SOURCE 200809L
#include "pdfp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PAR_MIN 16384 /* loops shorter than this stay on one thread */

static double now_seconds(void) {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

void or_set_threads(int32_t threads) {
#ifdef _OPENMP
    omp_set_num_threads(threads > 0 ? threads : 1);
#else
    (void)threads;
#endif
}

int32_t or_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---- Julia scalar semantics ------------------------------------------------ */

/* Base.max / Base.min for Float64: NaN-propagating, -0.0 < 0.0. */
static inline double jl_max(double x, double y) {
    int take_y = (y > x) || (signbit(y) < signbit(x));
    return take_y ? (isnan(x) ? x : y) : (isnan(y) ? y : x);
}
static inline double jl_min(double x, double y) {
    int take_y = (y < x) || (signbit(y) > signbit(x));
    return take_y ? (isnan(x) ? x : y) : (isnan(y) ? y : x);
}
/* Base.clamp(x, lo, hi) = x > hi ? hi : (x < lo ? lo : x). */
static inline double jl_clamp(double x, double lo, double hi) {
    return x > hi ? hi : (x < lo ? lo : x);
}
/* Float64 * Bool: x * true = x, x * false = copysign(0, x). */
static inline double jl_mulbool(double x, int b) { return b ? x : copysign(0.0, x); }

static const double JL_EPS = 2.220446049250313e-16; /* eps(Float64) */

/* ---- CSR helpers ------------------------------------------------------------ */

typedef struct {
    int32_t m, n;      /* rows, columns */
    int64_t nnz;
    int32_t* rp;       /* m+1 */
    int32_t* ci;       /* nnz, ascending per row */
    double* v;         /* nnz */
} csr_t;

static void csr_free(csr_t* a) {
    free(a->rp); free(a->ci); free(a->v);
    memset(a, 0, sizeof(*a));
}

static void csr_copy(csr_t* dst, int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                     const double* v) {
    dst->m = m; dst->n = n; dst->nnz = rp[m];
    dst->rp = (int32_t*)malloc(sizeof(int32_t) * ((size_t)m + 1));
    dst->ci = (int32_t*)malloc(sizeof(int32_t) * ((size_t)dst->nnz + 1));
    dst->v = (double*)malloc(sizeof(double) * ((size_t)dst->nnz + 1));
    memcpy(dst->rp, rp, sizeof(int32_t) * ((size_t)m + 1));
    if (dst->nnz) {
        memcpy(dst->ci, ci, sizeof(int32_t) * (size_t)dst->nnz);
        memcpy(dst->v, v, sizeof(double) * (size_t)dst->nnz);
    }
}

/* sparse(transpose(A)): row j of the result lists the rows i of A holding
 * column j, in ascending i (a counting sort over rows in ascending order). */
static void csr_transpose(const csr_t* a, csr_t* t) {
    t->m = a->n; t->n = a->m; t->nnz = a->nnz;
    t->rp = (int32_t*)calloc((size_t)a->n + 1, sizeof(int32_t));
    t->ci = (int32_t*)malloc(sizeof(int32_t) * ((size_t)a->nnz + 1));
    t->v = (double*)malloc(sizeof(double) * ((size_t)a->nnz + 1));
    for (int64_t p = 0; p < a->nnz; ++p) t->rp[a->ci[p] + 1]++;
    for (int32_t j = 0; j < a->n; ++j) t->rp[j + 1] += t->rp[j];
    int32_t* fill = (int32_t*)malloc(sizeof(int32_t) * ((size_t)a->n + 1));
    memcpy(fill, t->rp, sizeof(int32_t) * ((size_t)a->n + 1));
    for (int32_t i = 0; i < a->m; ++i)
        for (int32_t p = a->rp[i]; p < a->rp[i + 1]; ++p) {
            int32_t q = fill[a->ci[p]]++;
            t->ci[q] = i;
            t->v[q] = a->v[p];
        }
    free(fill);
}

/* mul!(y, A, x) with Julia's CSC loop order: y_i = sum over ascending j. */
static void spmv(const csr_t* a, const double* x, double* y) {
    const int32_t m = a->m;
#pragma omp parallel for schedule(static) if (a->nnz > PAR_MIN)
    for (int32_t i = 0; i < m; ++i) {
        double s = 0.0;
        for (int32_t p = a->rp[i]; p < a->rp[i + 1]; ++p) s += a->v[p] * x[a->ci[p]];
        y[i] = s;
    }
}

static double sum_sq(const double* x, int64_t n) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += x[i] * x[i];
    return s;
}
static double nrm2(const double* x, int64_t n) { return sqrt(sum_sq(x, n)); }
static double dotp(const double* x, const double* y, int64_t n) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += x[i] * y[i];
    return s;
}
static double* dalloc(int64_t n) { return (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

/* ---- defaults and the start vector ------------------------------------------ */

void or_default_params(or_params* p) {
    /* src/pdlp.jl:10-31 */
    p->eps_optimal_relative = 1e-4;
    p->eps_feasible_relative = 1e-4;
    p->iteration_limit = 100000;
    p->time_limit = 3600.0;
    p->termination_evaluation_frequency = 200;
    p->reflection_coefficient = 1.0;
    p->sv_max_iterations = 5000;
    p->sv_tolerance = 1e-4;
    p->artificial_restart_threshold = 0.36;
    p->sufficient_reduction_for_restart = 0.2;
    p->necessary_reduction_for_restart = 0.5;
    p->k_p = 0.99;
    p->k_i = 0.01;
    p->k_d = 0.0;
    p->i_smooth = 0.3;
}

static uint64_t splitmix64(uint64_t* state) {
    uint64_t z = (*state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void or_normal_vector(uint64_t seed, int64_t m, double* out) {
    uint64_t st = seed;
    const double two_pi = 6.283185307179586;
    for (int64_t i = 0; i < m; ++i) {
        double u1 = ((double)(splitmix64(&st) >> 11) + 0.5) * 0x1.0p-53;
        double u2 = ((double)(splitmix64(&st) >> 11) + 0.5) * 0x1.0p-53;
        out[i] = sqrt(-2.0 * log(u1)) * cos(two_pi * u2);
    }
}

/* ---- scale_problem, src/preconditioner.jl:26-99 --------------------------- */

static const double SCALING_EPSILON = 1e-12; /* src/preconditioner.jl:11 */

int or_scale_problem(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                     const double* c, const double* var_lb, const double* var_ub,
                     const double* con_lb, const double* con_ub, int32_t ruiz_iterations,
                     double alpha, int32_t rescale, double* vals, double* c_s, double* var_lb_s,
                     double* var_ub_s, double* con_lb_s, double* con_ub_s, double* D_r,
                     double* D_c, double* bound_scale, double* objective_scale) {
    const int64_t nnz = rp[m];
    if (nnz) memcpy(vals, v, sizeof(double) * (size_t)nnz);
    for (int32_t i = 0; i < m; ++i) D_r[i] = 1.0;
    for (int32_t j = 0; j < n; ++j) D_c[j] = 1.0;
    double* row_max = dalloc(m);
    double* col_max = dalloc(n);
    double* rscale = dalloc(m);
    double* cscale = dalloc(n);

    /* Ruiz, :36-49 -- max |a| per row and column (order-free), then
     * vals *= rscale[i] * cscale[j]. */
    for (int32_t it = 0; it < ruiz_iterations; ++it) {
        memset(row_max, 0, sizeof(double) * (size_t)(m > 0 ? m : 1));
        memset(col_max, 0, sizeof(double) * (size_t)(n > 0 ? n : 1));
        for (int32_t i = 0; i < m; ++i)
            for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
                double a = fabs(vals[p]);
                if (a > row_max[i]) row_max[i] = a;
                if (a > col_max[ci[p]]) col_max[ci[p]] = a;
            }
        for (int32_t i = 0; i < m; ++i)
            rscale[i] = row_max[i] < SCALING_EPSILON ? 1.0 : 1.0 / sqrt(row_max[i]);
        for (int32_t j = 0; j < n; ++j)
            cscale[j] = col_max[j] < SCALING_EPSILON ? 1.0 : 1.0 / sqrt(col_max[j]);
        for (int32_t i = 0; i < m; ++i)
            for (int32_t p = rp[i]; p < rp[i + 1]; ++p) vals[p] *= rscale[i] * cscale[ci[p]];
        for (int32_t i = 0; i < m; ++i) D_r[i] *= rscale[i];
        for (int32_t j = 0; j < n; ++j) D_c[j] *= cscale[j];
    }

    /* Pock-Chambolle, :51-64.  Julia walks the CSC matrix column by column:
     * row sums receive their terms in ascending column order and column sums
     * in ascending row order -- exactly what a row-major walk gives. */
    memset(row_max, 0, sizeof(double) * (size_t)(m > 0 ? m : 1)); /* row_sum */
    memset(col_max, 0, sizeof(double) * (size_t)(n > 0 ? n : 1)); /* col_sum */
    for (int32_t i = 0; i < m; ++i)
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            double a = fabs(vals[p]);
            row_max[i] += alpha == 1.0 ? a : pow(a, alpha);
            col_max[ci[p]] += (2.0 - alpha) == 1.0 ? a : pow(a, 2.0 - alpha);
        }
    for (int32_t i = 0; i < m; ++i)
        rscale[i] = row_max[i] < SCALING_EPSILON ? 1.0 : 1.0 / sqrt(row_max[i]);
    for (int32_t j = 0; j < n; ++j)
        cscale[j] = col_max[j] < SCALING_EPSILON ? 1.0 : 1.0 / sqrt(col_max[j]);
    for (int32_t i = 0; i < m; ++i)
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) vals[p] *= rscale[i] * cscale[ci[p]];
    for (int32_t i = 0; i < m; ++i) D_r[i] *= rscale[i];
    for (int32_t j = 0; j < n; ++j) D_c[j] *= cscale[j];

    /* :66-70 */
    for (int32_t j = 0; j < n; ++j) {
        c_s[j] = c[j] * D_c[j];
        var_lb_s[j] = isfinite(var_lb[j]) ? var_lb[j] / D_c[j] : var_lb[j];
        var_ub_s[j] = isfinite(var_ub[j]) ? var_ub[j] / D_c[j] : var_ub[j];
    }
    for (int32_t i = 0; i < m; ++i) {
        con_lb_s[i] = isfinite(con_lb[i]) ? con_lb[i] * D_r[i] : con_lb[i];
        con_ub_s[i] = isfinite(con_ub[i]) ? con_ub[i] * D_r[i] : con_ub[i];
    }

    /* Bound/objective rescaling, :72-96. */
    double bs = 1.0, os = 1.0;
    if (rescale) {
        double bound_sq = 0.0;
        for (int32_t i = 0; i < m; ++i) {
            int flo = isfinite(con_lb[i]), fhi = isfinite(con_ub[i]);
            double lo = con_lb_s[i], hi = con_ub_s[i];
            if (flo && (!fhi || fabs(lo - hi) > SCALING_EPSILON)) bound_sq += lo * lo;
            if (fhi) bound_sq += hi * hi;
        }
        bs = 1.0 / (sqrt(bound_sq) + 1.0);
        os = 1.0 / (sqrt(sum_sq(c_s, n)) + 1.0);
        for (int32_t i = 0; i < m; ++i) {
            if (isfinite(con_lb[i])) con_lb_s[i] *= bs;
            if (isfinite(con_ub[i])) con_ub_s[i] *= bs;
        }
        for (int32_t j = 0; j < n; ++j) {
            if (isfinite(var_lb[j])) var_lb_s[j] *= bs;
            if (isfinite(var_ub[j])) var_ub_s[j] *= bs;
            c_s[j] *= os;
        }
    }
    *bound_scale = bs;
    *objective_scale = os;
    free(row_max); free(col_max); free(rscale); free(cscale);
    return 0;
}

/* ---- estimate_max_singular_value, src/preconditioner.jl:108-125 ----------- */

static double power_iteration(const csr_t* a, const csr_t* at, int32_t max_iterations,
                              double tolerance, int32_t* iters) {
    const int32_t m = a->m, n = a->n;
    double* eig = dalloc(m);
    double* nxt = dalloc(m);
    double* dual = dalloc(n);
    or_normal_vector(20240517ull, m, eig);
    double sigma_sq = 1.0;
    int32_t it = 0;
    for (; it < max_iterations;) {
        ++it;
        memcpy(nxt, eig, sizeof(double) * (size_t)(m > 0 ? m : 1));
        double nrm = nrm2(nxt, m);
        if (nrm == 0.0) break;
        for (int32_t i = 0; i < m; ++i) nxt[i] /= nrm;
        spmv(at, nxt, dual);
        spmv(a, dual, eig);
        sigma_sq = dotp(nxt, eig, m);
        for (int32_t i = 0; i < m; ++i) nxt[i] = eig[i] - sigma_sq * nxt[i];
        if (nrm2(nxt, m) < tolerance) break;
    }
    if (iters) *iters = it;
    free(eig); free(nxt); free(dual);
    return sqrt(jl_max(sigma_sq, 0.0));
}

double or_estimate_max_singular_value(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                                      const double* v, int32_t max_iterations, double tolerance,
                                      int32_t* iterations_out) {
    csr_t a, at;
    csr_copy(&a, m, n, rp, ci, v);
    csr_transpose(&a, &at);
    double s = power_iteration(&a, &at, max_iterations, tolerance, iterations_out);
    csr_free(&a); csr_free(&at);
    return s;
}

/* ---- shared restart rules, src/pdlp.jl:167-205 ---------------------------- */

typedef struct {
    double primal_weight, best_primal_weight, best_gap, err_sum, last_err;
    double fixed_point_error, initial_fpe, last_trial_fpe;
    int64_t inner, total;
    double rel_p, rel_d;
} restart_state_t;

/* should_restart, src/pdlp.jl:167-181 */
static int should_restart(restart_state_t* s, const or_params* p) {
    int restart = 0;
    int64_t freq = p->termination_evaluation_frequency;
    if (s->total == freq) {
        restart = 1;
    } else if (s->total > freq) {
        if (s->fixed_point_error <= p->sufficient_reduction_for_restart * s->initial_fpe) restart = 1;
        if (s->fixed_point_error <= p->necessary_reduction_for_restart * s->initial_fpe &&
            s->fixed_point_error > s->last_trial_fpe)
            restart = 1;
        if ((double)s->inner >= p->artificial_restart_threshold * (double)s->total) restart = 1;
    }
    s->last_trial_fpe = s->fixed_point_error;
    return restart;
}

/* update_primal_weight!, src/pdlp.jl:185-205 */
static void update_primal_weight(restart_state_t* s, const or_params* p, double primal_dist,
                                 double dual_dist) {
    double ratio = s->rel_d / jl_max(s->rel_p, JL_EPS);
    if (1e-16 < primal_dist && primal_dist < 1e12 && 1e-16 < dual_dist && dual_dist < 1e12 &&
        1e-8 < ratio && ratio < 1e8) {
        double err = log(dual_dist) - log(primal_dist) - log(s->primal_weight);
        s->err_sum *= p->i_smooth;
        s->err_sum += err;
        double delta_err = err - s->last_err;
        s->primal_weight *= exp(p->k_p * err + p->k_i * s->err_sum + p->k_d * delta_err);
        s->last_err = err;
    } else {
        s->primal_weight = s->best_primal_weight;
        s->err_sum = 0.0;
        s->last_err = 0.0;
    }
    double gap = fabs(log10(s->rel_d / jl_max(s->rel_p, JL_EPS)));
    if (gap < s->best_gap) {
        s->best_gap = gap;
        s->best_primal_weight = s->primal_weight;
    }
}

/* ---- PDFP projector, src/pdfp.jl ------------------------------------------- */

struct or_pdfp {
    csr_t A, At;
    int32_t m, n;
    double *b, *lb, *ub, *xt, *w;
    uint8_t *is_eq, *is_int;
    double *ix, *cx, *px, *rx, *iy, *cy, *py, *ry, *iz, *cz, *pz, *rz;
    double *Ax, *Atz, *tmp_n, *tmp_m, *ds, *dx, *dy, *dz;
    int opr;
    double* row_unscale;
    double b_norm_original;
    double max_sv, step_size;
    restart_state_t r;
    double rel_gap, dual_den, gap_den;
    int32_t status, restarts;
};

or_pdfp* or_pdfp_create(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                        const double* b, const uint8_t* is_eq, const uint8_t* is_int,
                        const double* var_lb, const double* var_ub, const double* w) {
    or_pdfp* s = (or_pdfp*)calloc(1, sizeof(or_pdfp));
    s->m = m; s->n = n;
    csr_copy(&s->A, m, n, rp, ci, v);
    csr_transpose(&s->A, &s->At);
    s->b = dalloc(m); memcpy(s->b, b, sizeof(double) * (size_t)m);
    s->lb = dalloc(n); memcpy(s->lb, var_lb, sizeof(double) * (size_t)n);
    s->ub = dalloc(n); memcpy(s->ub, var_ub, sizeof(double) * (size_t)n);
    s->w = dalloc(n); memcpy(s->w, w, sizeof(double) * (size_t)n);
    s->xt = dalloc(n);
    s->is_eq = (uint8_t*)calloc((size_t)m + 1, 1); memcpy(s->is_eq, is_eq, (size_t)m);
    s->is_int = (uint8_t*)calloc((size_t)n + 1, 1); memcpy(s->is_int, is_int, (size_t)n);
    double** nv[] = {&s->ix, &s->cx, &s->px, &s->rx, &s->iy, &s->cy, &s->py, &s->ry,
                     &s->Atz, &s->tmp_n, &s->ds, &s->dx, &s->dy};
    for (size_t k = 0; k < sizeof(nv) / sizeof(nv[0]); ++k) *nv[k] = dalloc(n);
    double** mv[] = {&s->iz, &s->cz, &s->pz, &s->rz, &s->Ax, &s->tmp_m, &s->dz};
    for (size_t k = 0; k < sizeof(mv) / sizeof(mv[0]); ++k) *mv[k] = dalloc(m);
    s->max_sv = NAN;
    s->r.primal_weight = 1.0;
    s->r.best_primal_weight = 1.0;
    s->r.best_gap = INFINITY;
    s->r.fixed_point_error = INFINITY;
    s->r.initial_fpe = INFINITY;
    s->r.last_trial_fpe = INFINITY;
    s->r.rel_p = INFINITY; s->r.rel_d = INFINITY;
    s->rel_gap = INFINITY;
    s->dual_den = 1.0; s->gap_den = 1.0;
    s->b_norm_original = NAN;
    return s;
}

void or_pdfp_destroy(or_pdfp* s) {
    if (!s) return;
    csr_free(&s->A); csr_free(&s->At);
    double* all[] = {s->b, s->lb, s->ub, s->xt, s->w, s->ix, s->cx, s->px, s->rx, s->iy,
                     s->cy, s->py, s->ry, s->iz, s->cz, s->pz, s->rz, s->Ax, s->Atz,
                     s->tmp_n, s->tmp_m, s->ds, s->dx, s->dy, s->dz, s->row_unscale};
    for (size_t k = 0; k < sizeof(all) / sizeof(all[0]); ++k) free(all[k]);
    free(s->is_eq); free(s->is_int);
    free(s);
}

void or_pdfp_original_primal_residual(or_pdfp* s, const double* D_r) {
    /* src/pdfp.jl:85-90 */
    free(s->row_unscale);
    s->row_unscale = dalloc(s->m);
    double* t = dalloc(s->m);
    for (int32_t i = 0; i < s->m; ++i) {
        s->row_unscale[i] = 1.0 / D_r[i];
        t[i] = s->b[i] / D_r[i];
    }
    s->b_norm_original = nrm2(t, s->m);
    free(t);
    s->opr = 1;
}

void or_pdfp_set_x(or_pdfp* s, const double* x) {
    memcpy(s->cx, x, sizeof(double) * (size_t)s->n);
    memcpy(s->ix, x, sizeof(double) * (size_t)s->n);
}

void or_pdfp_warm_start(or_pdfp* s) {
    /* src/pdfp.jl:104-114 */
    memcpy(s->ix, s->cx, sizeof(double) * (size_t)s->n);
    memcpy(s->iy, s->cy, sizeof(double) * (size_t)s->n);
    memcpy(s->iz, s->cz, sizeof(double) * (size_t)s->m);
    s->r.inner = 0;
    s->r.total = 0;
    s->r.fixed_point_error = INFINITY;
    s->r.last_trial_fpe = INFINITY;
    s->status = OR_UNSPECIFIED;
}

void or_pdfp_set_target(or_pdfp* s, const double* x_tilde) {
    memcpy(s->xt, x_tilde, sizeof(double) * (size_t)s->n);
    or_pdfp_warm_start(s);
}

/* primal_step! + dual_y_step! + dual_z_step!, src/pdfp.jl:119-163. */
static void pdfp_step(or_pdfp* s, int32_t k_offset, double omega) {
    const int32_t n = s->n, m = s->m;
    const double tau = s->step_size / s->r.primal_weight;
    const double sigma = s->step_size * s->r.primal_weight;
    const double k = (double)(s->r.inner + k_offset);
    const double weight = k / (k + 1.0), omw = 1.0 - omega, omwt = 1.0 - weight;
    spmv(&s->At, s->cz, s->Atz);
#pragma omp parallel for schedule(static) if (n > PAR_MIN)
    for (int32_t j = 0; j < n; ++j) {
        /* primal_step!, :119-131 */
        double cx = s->cx[j];
        double t = cx - tau * (s->Atz[j] - s->cy[j]);
        double xh = jl_clamp(t, s->lb[j], s->ub[j]);
        s->px[j] = xh;
        s->ds[j] = (xh - t) / tau;
        double rx = 2.0 * xh - cx;
        s->rx[j] = rx;
        s->cx[j] = weight * (omega * rx + omw * cx) + omwt * s->ix[j];
        /* dual_y_step!, :134-143 */
        double cy = s->cy[j];
        double yh = s->is_int[j]
                        ? jl_clamp(cy + sigma * (s->xt[j] - rx), -s->w[j], s->w[j])
                        : 0.0;
        s->py[j] = yh;
        double ry = 2.0 * yh - cy;
        s->ry[j] = ry;
        s->cy[j] = weight * (omega * ry + omw * cy) + omwt * s->iy[j];
    }
    /* dual_z_step!, :146-156 */
    spmv(&s->A, s->rx, s->Ax);
#pragma omp parallel for schedule(static) if (m > PAR_MIN)
    for (int32_t i = 0; i < m; ++i) {
        double cz = s->cz[i];
        double raw = cz + sigma * (s->Ax[i] - s->b[i]);
        double zh = s->is_eq[i] ? raw : jl_max(raw, 0.0);
        s->pz[i] = zh;
        double rz = 2.0 * zh - cz;
        s->rz[i] = rz;
        s->cz[i] = weight * (omega * rz + omw * cz) + omwt * s->iz[i];
    }
}

/* compute_fixed_point_error!, src/pdfp.jl:167-178 */
static void pdfp_fixed_point_error(or_pdfp* s) {
    const int32_t n = s->n, m = s->m;
    for (int32_t j = 0; j < n; ++j) {
        s->dx[j] = s->px[j] - s->rx[j];
        s->dy[j] = s->py[j] - s->ry[j];
    }
    for (int32_t i = 0; i < m; ++i) s->dz[i] = s->pz[i] - s->rz[i];
    double pw = s->r.primal_weight;
    double movement = sum_sq(s->dx, n) * pw + (sum_sq(s->dy, n) + sum_sq(s->dz, m)) / pw;
    spmv(&s->At, s->dz, s->Atz);
    for (int32_t j = 0; j < n; ++j) s->tmp_n[j] = s->Atz[j] - s->dy[j];
    double interaction = 2.0 * s->step_size * dotp(s->tmp_n, s->dx, n);
    s->r.fixed_point_error = sqrt(jl_max(movement + interaction, 0.0));
}

/* perform_restart!, src/pdfp.jl:180-192 */
static void pdfp_restart(or_pdfp* s, const or_params* p) {
    const int32_t n = s->n, m = s->m;
    for (int32_t j = 0; j < n; ++j) {
        s->dx[j] = s->ix[j] - s->px[j];
        s->dy[j] = s->iy[j] - s->py[j];
    }
    for (int32_t i = 0; i < m; ++i) s->dz[i] = s->iz[i] - s->pz[i];
    update_primal_weight(&s->r, p, nrm2(s->dx, n), sqrt(sum_sq(s->dy, n) + sum_sq(s->dz, m)));
    memcpy(s->ix, s->px, sizeof(double) * (size_t)n); memcpy(s->cx, s->px, sizeof(double) * (size_t)n);
    memcpy(s->iy, s->py, sizeof(double) * (size_t)n); memcpy(s->cy, s->py, sizeof(double) * (size_t)n);
    memcpy(s->iz, s->pz, sizeof(double) * (size_t)m); memcpy(s->cz, s->pz, sizeof(double) * (size_t)m);
    s->r.inner = 0;
    s->r.last_trial_fpe = INFINITY;
    s->restarts++;
}

/* compute_residual!, src/pdfp.jl:200-218 */
static void pdfp_residual(or_pdfp* s) {
    const int32_t n = s->n, m = s->m;
    spmv(&s->A, s->px, s->Ax);
    for (int32_t i = 0; i < m; ++i) {
        double d = s->Ax[i] - s->b[i];
        s->tmp_m[i] = s->is_eq[i] ? fabs(d) : jl_max(d, 0.0);
        if (s->opr) s->tmp_m[i] *= s->row_unscale[i];
    }
    double b_norm = s->opr ? s->b_norm_original : nrm2(s->b, m);
    s->r.rel_p = nrm2(s->tmp_m, m) / (1.0 + b_norm);
    spmv(&s->At, s->pz, s->Atz);
    for (int32_t j = 0; j < n; ++j) s->tmp_n[j] = s->Atz[j] - s->py[j] - s->ds[j];
    s->r.rel_d = nrm2(s->tmp_n, n) / s->dual_den;
    double l1 = 0.0, y_term = 0.0, z_term = 0.0;
    for (int32_t j = 0; j < n; ++j) l1 += s->is_int[j] ? s->w[j] * fabs(s->px[j] - s->xt[j]) : 0.0;
    for (int32_t j = 0; j < n; ++j) y_term += s->is_int[j] ? s->py[j] * (s->xt[j] - s->px[j]) : 0.0;
    for (int32_t i = 0; i < m; ++i) z_term += s->pz[i] * (s->Ax[i] - s->b[i]);
    s->rel_gap = fabs(y_term + z_term - l1) / s->gap_den;
}

/* initialize_step_size_and_primal_weight!, src/pdfp.jl:220-241 */
static void pdfp_initialize(or_pdfp* s, const or_params* p, double primal_weight) {
    if (s->A.nnz == 0) {
        s->step_size = 1.0;
    } else {
        if (isnan(s->max_sv))
            s->max_sv = power_iteration(&s->A, &s->At, p->sv_max_iterations, p->sv_tolerance, NULL);
        s->step_size = 0.998 / sqrt(1.0 + s->max_sv * s->max_sv);
    }
    s->r.primal_weight = primal_weight;
    s->r.best_primal_weight = primal_weight;
    s->r.err_sum = 0.0;
    s->r.last_err = 0.0;
    double sq = 0.0, l1 = 0.0;
    for (int32_t j = 0; j < s->n; ++j) {
        double wi = s->is_int[j] ? s->w[j] : 0.0;
        sq += wi * wi;
        l1 += s->is_int[j] ? s->w[j] * fabs(s->xt[j]) : 0.0;
    }
    s->dual_den = 1.0 + sqrt(sq);
    s->gap_den = 1.0 + l1;
}

int32_t or_pdfp_solve(or_pdfp* s, const or_params* p, double primal_weight, or_result* res) {
    /* pdfp_solve!, src/pdfp.jl:252-288 */
    double t_start = now_seconds();
    pdfp_initialize(s, p, primal_weight);
    const double omega = p->reflection_coefficient;
    const int32_t freq = p->termination_evaluation_frequency;
    int do_restart = 0;
    while (s->r.total < p->iteration_limit) {
        pdfp_step(s, 1, omega);
        if (do_restart) {
            pdfp_fixed_point_error(s);
            s->r.initial_fpe = s->r.fixed_point_error;
            do_restart = 0;
        }
        for (int32_t i = 2; i <= freq; ++i) pdfp_step(s, i, omega);
        pdfp_fixed_point_error(s);
        pdfp_residual(s);
        s->r.inner += freq;
        s->r.total += freq;
        if (s->r.rel_p <= p->eps_feasible_relative && s->r.rel_d <= p->eps_optimal_relative &&
            s->rel_gap <= p->eps_optimal_relative) {
            s->status = OR_OPTIMAL;
            break;
        }
        if (now_seconds() - t_start > p->time_limit) {
            s->status = OR_TIME_LIMIT;
            break;
        }
        do_restart = should_restart(&s->r, p);
        if (do_restart) pdfp_restart(s, p);
    }
    if (s->status == OR_UNSPECIFIED) s->status = OR_ITERATION_LIMIT;
    if (res) {
        memset(res, 0, sizeof(*res));
        res->status = s->status;
        res->restarts = s->restarts;
        res->total_count = s->r.total;
        res->rel_primal = s->r.rel_p;
        res->rel_dual = s->r.rel_d;
        res->rel_gap = s->rel_gap;
        res->primal_weight = s->r.primal_weight;
        res->step_size = s->step_size;
        res->max_singular_value = s->max_sv;
        res->fixed_point_error = s->r.fixed_point_error;
        res->objective_value = NAN;
    }
    return s->status;
}

void or_pdfp_get(const or_pdfp* s, int32_t which, double* out) {
    const double* src = NULL;
    int64_t len = s->n;
    switch (which) {
        case 0: src = s->px; break;
        case 1: src = s->py; break;
        case 2: src = s->pz; len = s->m; break;
        case 3: src = s->cx; break;
        case 4: src = s->cy; break;
        case 5: src = s->cz; len = s->m; break;
        case 6: src = s->ds; break;
        case 7: src = s->rx; break;
        default: return;
    }
    if (len) memcpy(out, src, sizeof(double) * (size_t)len);
}

void or_pdfp_set_max_singular_value(or_pdfp* s, double sigma) { s->max_sv = sigma; }

void or_pdfp_steps(or_pdfp* s, double step_size, double primal_weight, int32_t k0, int32_t count) {
    s->step_size = step_size;
    s->r.primal_weight = primal_weight;
    for (int32_t i = 0; i < count; ++i) pdfp_step(s, k0 + i, 1.0);
}

/* ---- PDLP, src/pdlp.jl ------------------------------------------------------ */

typedef struct {
    csr_t A, At;
    int32_t m, n;
    const double *c, *lb, *ub, *clb, *cub;
    double *ix, *cx, *px, *rx, *iy, *cy, *py, *ry;
    double *pp, *dp, *tmp_n, *tmp_m, *ds, *dpr, *ddu;
    double bound_scale, objective_scale;
    int cupdlpx;
    double *row_unscale, *col_unscale;
    double eps_inf, cbn, ovn, step_size;
    restart_state_t r;
    double rel_gap, objective_value;
    double max_primal_ray_inf, primal_ray_lin_obj, max_dual_ray_inf, dual_ray_obj;
    int32_t status, restarts;
} pdlp_t;

/* primal_step!, src/pdlp.jl:115-132 */
static void pdlp_primal_step(pdlp_t* s, int32_t k_offset, double omega, int major) {
    const double step = s->step_size / s->r.primal_weight;
    const double k = (double)(s->r.inner + k_offset);
    const double weight = k / (k + 1.0), omw = 1.0 - omega, omwt = 1.0 - weight;
    const int32_t n = s->n;
#pragma omp parallel for schedule(static) if (n > PAR_MIN)
    for (int32_t j = 0; j < n; ++j) {
        double cx = s->cx[j];
        double t = cx - step * (s->c[j] - s->dp[j]);
        double xh = jl_clamp(t, s->lb[j], s->ub[j]);
        if (major) s->ds[j] = (xh - t) / step;
        s->px[j] = xh;
        double rx = 2.0 * xh - cx;
        s->rx[j] = rx;
        s->cx[j] = weight * (omega * rx + omw * cx) + omwt * s->ix[j];
    }
}

/* dual_step!, src/pdlp.jl:134-145 */
static void pdlp_dual_step(pdlp_t* s, int32_t k_offset, double omega, int major) {
    const double step = s->step_size * s->r.primal_weight;
    const double k = (double)(s->r.inner + k_offset);
    const double weight = k / (k + 1.0), omw = 1.0 - omega, omwt = 1.0 - weight;
    const int32_t m = s->m;
#pragma omp parallel for schedule(static) if (m > PAR_MIN)
    for (int32_t i = 0; i < m; ++i) {
        double cy = s->cy[i];
        double t = cy / step - s->pp[i];
        double yh = (t - jl_clamp(t, -s->cub[i], -s->clb[i])) * step;
        if (major) s->py[i] = yh;
        double ry = 2.0 * yh - cy;
        s->ry[i] = ry;
        s->cy[i] = weight * (omega * ry + omw * cy) + omwt * s->iy[i];
    }
}

/* pdhg_step!, src/pdlp.jl:147-153 */
static void pdlp_step(pdlp_t* s, int32_t k_offset, double omega, int major) {
    spmv(&s->At, s->cy, s->dp);
    pdlp_primal_step(s, k_offset, omega, major);
    spmv(&s->A, s->rx, s->pp);
    pdlp_dual_step(s, k_offset, omega, major);
}

/* compute_fixed_point_error!, src/pdlp.jl:157-165 */
static void pdlp_fixed_point_error(pdlp_t* s) {
    for (int32_t j = 0; j < s->n; ++j) s->dpr[j] = s->px[j] - s->rx[j];
    for (int32_t i = 0; i < s->m; ++i) s->ddu[i] = s->py[i] - s->ry[i];
    double pw = s->r.primal_weight;
    double movement = sum_sq(s->dpr, s->n) * pw + sum_sq(s->ddu, s->m) / pw;
    spmv(&s->At, s->ddu, s->dp);
    double interaction = 2.0 * s->step_size * dotp(s->dp, s->dpr, s->n);
    s->r.fixed_point_error = sqrt(jl_max(movement + interaction, 0.0));
}

/* perform_restart!, src/pdlp.jl:207-216 */
static void pdlp_restart(pdlp_t* s, const or_params* p) {
    for (int32_t j = 0; j < s->n; ++j) s->dpr[j] = s->ix[j] - s->px[j];
    for (int32_t i = 0; i < s->m; ++i) s->ddu[i] = s->iy[i] - s->py[i];
    update_primal_weight(&s->r, p, nrm2(s->dpr, s->n), nrm2(s->ddu, s->m));
    size_t bn = sizeof(double) * (size_t)s->n, bm = sizeof(double) * (size_t)s->m;
    memcpy(s->ix, s->px, bn); memcpy(s->cx, s->px, bn);
    memcpy(s->iy, s->py, bm); memcpy(s->cy, s->py, bm);
    s->r.inner = 0;
    s->r.last_trial_fpe = INFINITY;
    s->restarts++;
}

/* compute_residual!, src/pdlp.jl:220-242 */
static void pdlp_residual(pdlp_t* s) {
    const int32_t m = s->m, n = s->n;
    spmv(&s->A, s->px, s->pp);
    for (int32_t i = 0; i < m; ++i) {
        s->tmp_m[i] = s->pp[i] - jl_clamp(s->pp[i], s->clb[i], s->cub[i]);
        if (s->cupdlpx) s->tmp_m[i] *= s->row_unscale[i];
    }
    double primal_residual = nrm2(s->tmp_m, m) / s->bound_scale;
    spmv(&s->At, s->py, s->dp);
    for (int32_t j = 0; j < n; ++j) {
        s->tmp_n[j] = s->c[j] - s->dp[j] - s->ds[j];
        if (s->cupdlpx) s->tmp_n[j] *= s->col_unscale[j];
    }
    double dual_residual = nrm2(s->tmp_n, n) / s->objective_scale;
    s->r.rel_p = primal_residual / (1.0 + s->cbn);
    s->r.rel_d = dual_residual / (1.0 + s->ovn);
    double scale = s->bound_scale * s->objective_scale;
    s->objective_value = dotp(s->c, s->px, n) / scale;
    double sum_m = 0.0;
    for (int32_t i = 0; i < m; ++i) {
        double lo = fabs(s->clb[i]) < 1e19 ? s->clb[i] : 0.0;
        double hi = fabs(s->cub[i]) < 1e19 ? s->cub[i] : 0.0;
        sum_m += jl_max(s->py[i], 0.0) * lo + jl_min(s->py[i], 0.0) * hi;
    }
    double dual_objective = (dotp(s->ds, s->px, n) + sum_m) / scale;
    s->rel_gap = fabs(s->objective_value - dual_objective) /
                 (1.0 + fabs(s->objective_value) + fabs(dual_objective));
}

/* compute_infeasibility_information!, src/pdlp.jl:247-285 */
static void pdlp_infeasibility(pdlp_t* s) {
    const int32_t m = s->m, n = s->n;
    double* d = s->dpr;
    double* y = s->ddu;
    for (int32_t j = 0; j < n; ++j) {
        d[j] = -d[j];
        if (isfinite(s->lb[j])) d[j] = jl_max(d[j], 0.0);
        if (isfinite(s->ub[j])) d[j] = jl_min(d[j], 0.0);
    }
    for (int32_t i = 0; i < m; ++i) {
        y[i] = -y[i];
        if (!isfinite(s->clb[i])) y[i] = jl_min(y[i], 0.0);
        if (!isfinite(s->cub[i])) y[i] = jl_max(y[i], 0.0);
    }
    double prn = 0.0;
    for (int32_t j = 0; j < n; ++j) prn = jl_max(prn, fabs(d[j]));
    if (prn > 0.0)
        for (int32_t j = 0; j < n; ++j) d[j] /= prn;
    double drn = 0.0;
    for (int32_t i = 0; i < m; ++i) drn = jl_max(drn, fabs(y[i]));
    spmv(&s->A, d, s->pp);
    spmv(&s->At, y, s->dp);
    double scale = s->bound_scale * s->objective_scale;
    s->primal_ray_lin_obj = dotp(s->c, d, n) / scale;
    double primal_slack = 0.0;
    for (int32_t i = 0; i < m; ++i)
        primal_slack += jl_max(y[i], 0.0) * (isfinite(s->clb[i]) ? s->clb[i] : 0.0) +
                        jl_min(y[i], 0.0) * (isfinite(s->cub[i]) ? s->cub[i] : 0.0);
    double dual_slack = 0.0;
    for (int32_t j = 0; j < n; ++j)
        dual_slack += jl_max(-s->dp[j], 0.0) * (isfinite(s->lb[j]) ? s->lb[j] : 0.0) +
                      jl_min(-s->dp[j], 0.0) * (isfinite(s->ub[j]) ? s->ub[j] : 0.0);
    s->dual_ray_obj = (primal_slack + dual_slack) / scale;
    double mpri = 0.0;
    for (int32_t i = 0; i < m; ++i) {
        double t = jl_mulbool(jl_max(0.0, -s->pp[i]), isfinite(s->clb[i])) +
                   jl_mulbool(jl_max(0.0, s->pp[i]), isfinite(s->cub[i]));
        t *= s->row_unscale[i];
        mpri = jl_max(mpri, fabs(t));
    }
    double dsn = 0.0;
    for (int32_t j = 0; j < n; ++j) {
        double t = jl_mulbool(jl_max(0.0, -s->dp[j]), !isfinite(s->lb[j])) -
                   jl_mulbool(jl_min(0.0, -s->dp[j]), !isfinite(s->ub[j]));
        t *= s->col_unscale[j];
        dsn = jl_max(dsn, fabs(t));
    }
    s->max_primal_ray_inf = mpri;
    double scaling = jl_max(drn, dsn);
    if (scaling > 0.0) {
        s->max_dual_ray_inf = dsn / scaling;
        s->dual_ray_obj /= scaling;
    } else {
        s->max_dual_ray_inf = 0.0;
        s->dual_ray_obj = 0.0;
    }
}

/* initialize_step_size_and_primal_weight!, src/pdlp.jl:292-316 */
static void pdlp_initialize(pdlp_t* s, const or_params* p) {
    if (s->A.nnz == 0) {
        s->step_size = 1.0;
    } else {
        double sv = power_iteration(&s->A, &s->At, p->sv_max_iterations, p->sv_tolerance, NULL);
        s->step_size = (isfinite(sv) && sv > 0) ? 0.998 / sv : 0.998;
    }
    double lo_sq = 0.0, hi_sq = 0.0;
    if (s->cupdlpx) {
        double sq = 0.0;
        for (int32_t j = 0; j < s->n; ++j) {
            double t = s->c[j] * s->col_unscale[j];
            sq += t * t;
        }
        s->ovn = sqrt(sq) / s->objective_scale;
        for (int32_t i = 0; i < s->m; ++i) {
            double lo = s->clb[i] * s->row_unscale[i] / s->bound_scale;
            double hi = s->cub[i] * s->row_unscale[i] / s->bound_scale;
            double a = (isfinite(lo) && s->clb[i] != s->cub[i]) ? lo : 0.0;
            double b = isfinite(hi) ? hi : 0.0;
            lo_sq += a * a;
            hi_sq += b * b;
        }
    } else {
        s->ovn = nrm2(s->c, s->n);
        for (int32_t i = 0; i < s->m; ++i) {
            double lo = s->clb[i], hi = s->cub[i];
            double a = (isfinite(lo) && s->clb[i] != s->cub[i]) ? lo : 0.0;
            double b = isfinite(hi) ? hi : 0.0;
            lo_sq += a * a;
            hi_sq += b * b;
        }
    }
    s->cbn = sqrt(lo_sq + hi_sq);
    s->r.primal_weight = 1.0;
    s->r.best_primal_weight = 1.0;
}

/* pdlp_solve!, src/pdlp.jl:325-372 */
static int32_t pdlp_solve(pdlp_t* s, const or_params* p) {
    double t_start = now_seconds();
    pdlp_initialize(s, p);
    const double omega = p->reflection_coefficient;
    const int32_t freq = p->termination_evaluation_frequency;
    int do_restart = 0;
    while (s->r.total < p->iteration_limit) {
        pdlp_step(s, 1, omega, 1);
        if (do_restart) {
            pdlp_fixed_point_error(s);
            s->r.initial_fpe = s->r.fixed_point_error;
            do_restart = 0;
        }
        for (int32_t i = 2; i <= freq - 1; ++i) pdlp_step(s, i, omega, 0);
        pdlp_step(s, freq, omega, 1);
        pdlp_fixed_point_error(s);
        pdlp_residual(s);
        if (s->cupdlpx) pdlp_infeasibility(s);
        s->r.inner += freq;
        s->r.total += freq;
        if (s->r.rel_p <= p->eps_feasible_relative && s->r.rel_d <= p->eps_feasible_relative &&
            s->rel_gap <= p->eps_optimal_relative) {
            s->status = OR_OPTIMAL;
            break;
        }
        if (s->cupdlpx && s->dual_ray_obj > 0.0 &&
            s->max_dual_ray_inf / s->dual_ray_obj <= s->eps_inf) {
            s->status = OR_PRIMAL_INFEASIBLE;
            break;
        }
        if (s->cupdlpx && s->primal_ray_lin_obj < 0.0 &&
            s->max_primal_ray_inf / (-s->primal_ray_lin_obj) <= s->eps_inf) {
            s->status = OR_DUAL_INFEASIBLE;
            break;
        }
        if (now_seconds() - t_start > p->time_limit) {
            s->status = OR_TIME_LIMIT;
            break;
        }
        do_restart = should_restart(&s->r, p);
        if (do_restart) pdlp_restart(s, p);
    }
    if (s->status == OR_UNSPECIFIED) s->status = OR_ITERATION_LIMIT;
    return s->status;
}

int32_t or_pdlp_solve_scaled(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                             const double* v, const double* c, const double* var_lb,
                             const double* var_ub, const double* con_lb, const double* con_ub,
                             double bound_scale, double objective_scale, const double* D_r,
                             const double* D_c, const or_params* p, double* pdhg_primal,
                             double* pdhg_dual, double* dual_slack, or_result* res) {
    pdlp_t s;
    memset(&s, 0, sizeof(s));
    s.m = m; s.n = n;
    csr_copy(&s.A, m, n, rp, ci, v);
    csr_transpose(&s.A, &s.At);
    s.c = c; s.lb = var_lb; s.ub = var_ub; s.clb = con_lb; s.cub = con_ub;
    double** nv[] = {&s.ix, &s.cx, &s.px, &s.rx, &s.dp, &s.tmp_n, &s.ds, &s.dpr};
    for (size_t k = 0; k < sizeof(nv) / sizeof(nv[0]); ++k) *nv[k] = dalloc(n);
    double** mv[] = {&s.iy, &s.cy, &s.py, &s.ry, &s.pp, &s.tmp_m, &s.ddu};
    for (size_t k = 0; k < sizeof(mv) / sizeof(mv[0]); ++k) *mv[k] = dalloc(m);
    s.bound_scale = bound_scale;
    s.objective_scale = objective_scale;
    s.eps_inf = 1e-14;
    if (D_r && D_c) {
        /* cupdlpx_termination!, src/pdlp.jl:105-110 */
        s.cupdlpx = 1;
        s.row_unscale = dalloc(m);
        s.col_unscale = dalloc(n);
        for (int32_t i = 0; i < m; ++i) s.row_unscale[i] = 1.0 / D_r[i];
        for (int32_t j = 0; j < n; ++j) s.col_unscale[j] = 1.0 / D_c[j];
    }
    s.r.primal_weight = 1.0;
    s.r.best_primal_weight = 1.0;
    s.r.best_gap = INFINITY;
    s.r.fixed_point_error = INFINITY;
    s.r.initial_fpe = INFINITY;
    s.r.last_trial_fpe = INFINITY;
    s.r.rel_p = INFINITY; s.r.rel_d = INFINITY;
    s.rel_gap = INFINITY;
    s.objective_value = NAN;
    int32_t st = pdlp_solve(&s, p);
    if (pdhg_primal && n) memcpy(pdhg_primal, s.px, sizeof(double) * (size_t)n);
    if (pdhg_dual && m) memcpy(pdhg_dual, s.py, sizeof(double) * (size_t)m);
    if (dual_slack && n) memcpy(dual_slack, s.ds, sizeof(double) * (size_t)n);
    if (res) {
        memset(res, 0, sizeof(*res));
        res->status = st;
        res->restarts = s.restarts;
        res->total_count = s.r.total;
        res->rel_primal = s.r.rel_p;
        res->rel_dual = s.r.rel_d;
        res->rel_gap = s.rel_gap;
        res->primal_weight = s.r.primal_weight;
        res->step_size = s.step_size;
        res->max_singular_value = NAN;
        res->fixed_point_error = s.r.fixed_point_error;
        res->objective_value = s.objective_value;
    }
    csr_free(&s.A); csr_free(&s.At);
    double* all[] = {s.ix, s.cx, s.px, s.rx, s.dp, s.tmp_n, s.ds, s.dpr, s.iy, s.cy, s.py,
                     s.ry, s.pp, s.tmp_m, s.ddu, s.row_unscale, s.col_unscale};
    for (size_t k = 0; k < sizeof(all) / sizeof(all[0]); ++k) free(all[k]);
    return st;
}

int32_t or_solve_lp_relaxation(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                               const double* v, const double* c, const double* l, const double* u,
                               const double* b, const uint8_t* is_le, double tolerance,
                               double time_limit, int32_t cupdlpx_termination, double* x_out,
                               double* dual_slack_out, or_result* res) {
    /* solve_lp_relaxation, src/pdlp.jl:381-393 */
    const int64_t nnz = rp[m];
    double* con_lb = dalloc(m);
    for (int32_t i = 0; i < m; ++i) con_lb[i] = is_le[i] ? -INFINITY : b[i];
    double* vals = dalloc(nnz);
    double *c_s = dalloc(n), *lb_s = dalloc(n), *ub_s = dalloc(n), *D_c = dalloc(n);
    double *clb_s = dalloc(m), *cub_s = dalloc(m), *D_r = dalloc(m);
    double bs, os;
    or_scale_problem(m, n, rp, ci, v, c, l, u, con_lb, b, 10, 1.0, 1, vals, c_s, lb_s, ub_s,
                     clb_s, cub_s, D_r, D_c, &bs, &os);
    or_params p;
    or_default_params(&p);
    p.iteration_limit = 5000000;
    p.eps_optimal_relative = tolerance;
    p.eps_feasible_relative = tolerance;
    p.time_limit = time_limit;
    double* px = dalloc(n);
    int32_t st = or_pdlp_solve_scaled(m, n, rp, ci, vals, c_s, lb_s, ub_s, clb_s, cub_s, bs, os,
                                      cupdlpx_termination ? D_r : NULL,
                                      cupdlpx_termination ? D_c : NULL, &p, px, NULL,
                                      dual_slack_out, res);
    for (int32_t j = 0; j < n; ++j) x_out[j] = (D_c[j] * px[j]) / bs;
    free(con_lb); free(vals); free(c_s); free(lb_s); free(ub_s); free(D_c);
    free(clb_s); free(cub_s); free(D_r); free(px);
    return st;
}
