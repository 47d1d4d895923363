// pdlp_ops.cuh -- the root-LP solver's fused passes (src/pdlp.jl, src/pdlp_kernels.jl).
//
// min c'x  s.t.  con_lb <= A x <= con_ub,  var_lb <= x <= var_ub, by restarted
// Halpern PDHG with reflection (cuPDLPx).  One PDHG step (pdhg_step!,
// src/pdlp.jl:147-153) is two tile-engine launches:
//   LpPrimalOp (rows of A' = columns j): A'y, then primal_step! (:115-132);
//              pdhg_primal is stored every step, dual_slack on major steps only;
//   LpDualOp   (rows i of A): A x_bar, then dual_step! (:134-145); pdhg_dual
//              is stored on major steps only.
// Evaluation (compute_fixed_point_error!, compute_residual!, :157-242) is
// LpEvalColOp + LpEvalRowOp producing FP64 per-tile partial sums; cuPDLPx
// infeasibility detection (compute_infeasibility_information!, :247-285) adds
// four passes whose maxima are reduced with an order-free atomic max.
#pragma once
#include "common.cuh"
#include "layout.hpp"
#include "pdfp_ops.cuh"
#include "state.hpp"

namespace pdfp {

template <typename T>
struct LpVecs {  // one precision's copy of the LP state (packed order)
    T *cx, *ix, *px, *rx, *ds;  // n
    T *cy, *iy, *py, *ry;       // m
    T *c, *lb, *ub;             // n
    T *clb, *cub;               // m
    T *val_t, *val_a;
};

struct LpData {  // FP64 data for evaluation and infeasibility detection
    const double *c, *lb, *ub, *clb, *cub;  // scaled
    const double *row_unscale, *col_unscale;  // 1 ./ D_r, 1 ./ D_c (null: scaled units)
    const double *val_t, *val_a;
    double *dray, *yray;                      // ray work vectors
    double* part_col;                         // eval A' tiles x 8
    double* part_row;                         // eval A tiles x 4
    unsigned long long* maxes;                // [4] order-free maxima (bits of non-negative doubles)
};

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* slot, double v) {
    atomicMax(slot, static_cast<unsigned long long>(__double_as_longlong(v)));
}

template <typename T, bool MAJOR, int NTHREADS>
struct LpPrimalOp {
    using MT = T;
    using VT = T;
    using AT = T;
    using GT = T;
    using TileP = StepParams<T>;
    static constexpr int NT = NTHREADS, NV = 1, NVEC = 5, NP = 0;
    LpVecs<T> v;
    const InstState* st;
    int32_t k_offset, mode;
    int32_t* errp;
    __device__ const T* values() const { return v.val_t; }
    __device__ const T* staged(int k) const {
        return k == 0 ? v.cx : (k == 1 ? v.ix : (k == 2 ? v.c : (k == 3 ? v.lb : v.ub)));
    }
    __device__ int32_t* err() const { return errp; }
    __device__ bool active(int inst) const {
        return st[inst].status == ST_RUNNING && st[inst].mode == mode;
    }
    __device__ TileP tile_params(int inst) const { return step_params<T>(st[inst], k_offset); }
    __device__ void gather(int32_t col, T (&g)[1]) const { g[0] = v.cy[col]; }
    __device__ void row(int32_t j, int32_t rr, int, const TileP& p, const T* const* sv,
                        const T (&s)[1], double*) const {
        const T cx = sv[0][rr], ix = sv[1][rr], c = sv[2][rr], lb = sv[3][rr], ub = sv[4][rr];
        // primal_step!, src/pdlp.jl:115-132 (tau is the primal step here)
        const T t = sub_rn(cx, mul_rn(p.tau, sub_rn(c, s[0])));
        const T xh = jl_clamp(t, lb, ub);
        if (MAJOR) v.ds[j] = sub_rn(xh, t) / p.tau;
        v.px[j] = xh;
        const T rx = sub_rn(mul_rn(T(2), xh), cx);
        v.rx[j] = rx;
        v.cx[j] = halpern(p.weight, p.omega, p.omw, p.omwt, rx, cx, ix);
    }
    __device__ void write_partials(int32_t, const double*) const {}
};

template <typename T, bool MAJOR, int NTHREADS>
struct LpDualOp {
    using MT = T;
    using VT = T;
    using AT = T;
    using GT = T;
    using TileP = StepParams<T>;
    static constexpr int NT = NTHREADS, NV = 1, NVEC = 4, NP = 0;
    LpVecs<T> v;
    const InstState* st;
    int32_t k_offset, mode;
    int32_t* errp;
    __device__ const T* values() const { return v.val_a; }
    __device__ const T* staged(int k) const {
        return k == 0 ? v.cy : (k == 1 ? v.iy : (k == 2 ? v.clb : v.cub));
    }
    __device__ int32_t* err() const { return errp; }
    __device__ bool active(int inst) const {
        return st[inst].status == ST_RUNNING && st[inst].mode == mode;
    }
    __device__ TileP tile_params(int inst) const { return step_params<T>(st[inst], k_offset); }
    __device__ void gather(int32_t col, T (&g)[1]) const { g[0] = v.rx[col]; }
    __device__ void row(int32_t i, int32_t rr, int, const TileP& p, const T* const* sv,
                        const T (&s)[1], double*) const {
        const T cy = sv[0][rr], iy = sv[1][rr], clb = sv[2][rr], cub = sv[3][rr];
        // dual_step!, src/pdlp.jl:134-145 (sigma is the dual step here)
        const T t = sub_rn(cy / p.sigma, s[0]);
        const T yh = mul_rn(sub_rn(t, jl_clamp(t, -cub, -clb)), p.sigma);
        if (MAJOR) v.py[i] = yh;
        const T ry = sub_rn(mul_rn(T(2), yh), cy);
        v.ry[i] = ry;
        v.cy[i] = halpern(p.weight, p.omega, p.omw, p.omwt, ry, cy, iy);
    }
    __device__ void write_partials(int32_t, const double*) const {}
};

// Column terms: A'y_hat and A'(y_hat - y_bar) in one pass over A'.
template <typename T, int NTHREADS>
struct LpEvalColOp {
    using MT = double;
    using VT = double;
    using AT = double;
    using GT = double;
    struct TileP {
        int32_t d;
    };
    static constexpr int NT = NTHREADS, NV = 2, NVEC = 0, NP = 8;
    LpVecs<T> v;
    LpData d;
    const InstState* st;
    int32_t which, mode;
    int32_t* errp;
    __device__ const double* values() const { return d.val_t; }
    __device__ const double* staged(int) const { return nullptr; }
    __device__ int32_t* err() const { return errp; }
    __device__ bool active(int inst) const {
        const InstState& s = st[inst];
        return s.status == ST_RUNNING && s.mode == mode && (which == EVAL_FULL || s.do_restart);
    }
    __device__ TileP tile_params(int) const { return TileP{0}; }
    __device__ void gather(int32_t col, double (&g)[2]) const {
        const double py = static_cast<double>(v.py[col]);
        g[0] = py;
        g[1] = sub_rn(py, static_cast<double>(v.ry[col]));  // delta_dual (src/pdlp.jl:159)
    }
    __device__ void row(int32_t j, int32_t, int, const TileP&, const double* const*,
                        const double (&s)[2], double* acc) const {
        const double px = v.px[j], rx = v.rx[j], ds = v.ds[j];
        const double dp = sub_rn(px, rx);
        acc[0] += dp * dp;                           // sum(abs2, delta_primal)
        acc[1] += mul_rn(s[1], dp);                  // <A' delta_dual, delta_primal>
        double r = sub_rn(sub_rn(d.c[j], s[0]), ds);  // c - A'y - dual_slack (src/pdlp.jl:227)
        if (d.col_unscale) r = mul_rn(r, d.col_unscale[j]);
        acc[2] += r * r;
        acc[3] += mul_rn(d.c[j], px);                // objective
        acc[4] += mul_rn(ds, px);                    // dual objective, bound part
        const double e = sub_rn(static_cast<double>(v.ix[j]), px);
        acc[5] += e * e;                             // restart distance (primal)
    }
    __device__ void write_partials(int32_t t, const double* acc) const {
#pragma unroll
        for (int k = 0; k < NP; ++k) d.part_col[t * NP + k] = acc[k];
    }
};

// Row terms: A x_hat in one pass over A.
template <typename T, int NTHREADS>
struct LpEvalRowOp {
    using MT = double;
    using VT = double;
    using AT = double;
    using GT = double;
    struct TileP {
        int32_t d;
    };
    static constexpr int NT = NTHREADS, NV = 1, NVEC = 0, NP = 4;
    LpVecs<T> v;
    LpData d;
    const InstState* st;
    int32_t which, mode;
    int32_t* errp;
    __device__ const double* values() const { return d.val_a; }
    __device__ const double* staged(int) const { return nullptr; }
    __device__ int32_t* err() const { return errp; }
    __device__ bool active(int inst) const {
        const InstState& s = st[inst];
        return s.status == ST_RUNNING && s.mode == mode && (which == EVAL_FULL || s.do_restart);
    }
    __device__ TileP tile_params(int) const { return TileP{0}; }
    __device__ void gather(int32_t col, double (&g)[1]) const { g[0] = static_cast<double>(v.px[col]); }
    __device__ void row(int32_t i, int32_t, int, const TileP&, const double* const*,
                        const double (&s)[1], double* acc) const {
        const double py = v.py[i], ry = v.ry[i];
        const double dd = sub_rn(py, ry);
        acc[0] += dd * dd;                                        // sum(abs2, delta_dual)
        double r = sub_rn(s[0], jl_clamp(s[0], d.clb[i], d.cub[i]));  // src/pdlp.jl:222
        if (d.row_unscale) r = mul_rn(r, d.row_unscale[i]);
        acc[1] += r * r;
        const double lo = fabs(d.clb[i]) < 1e19 ? d.clb[i] : 0.0;   // src/pdlp.jl:236-237
        const double hi = fabs(d.cub[i]) < 1e19 ? d.cub[i] : 0.0;
        acc[2] += add_rn(mul_rn(jl_max(py, 0.0), lo), mul_rn(jl_min(py, 0.0), hi));
        const double e = sub_rn(static_cast<double>(v.iy[i]), py);
        acc[3] += e * e;                                          // restart distance (dual)
    }
    __device__ void write_partials(int32_t t, const double* acc) const {
#pragma unroll
        for (int k = 0; k < NP; ++k) d.part_row[t * NP + k] = acc[k];
    }
};

// ---- cuPDLPx infeasibility detection (src/pdlp.jl:247-285) -----------------------
// maxes[0] = max|d| (primal ray norm), [1] = max|y| (dual ray norm),
// [2] = max primal ray infeasibility, [3] = max dual scratch (original units).

template <typename T>
struct RayRowsCol {  // d = -(pdhg - reflected) on x, clipped by the finite bounds
    static constexpr int NP = 2;
    LpVecs<T> v;
    LpData d;
    const InstState* st;
    __device__ bool active(int p) const { return st[p].status == ST_RUNNING; }
    __device__ void row(int32_t j, int, double* acc) const {
        double x = sub_rn(static_cast<double>(v.rx[j]), static_cast<double>(v.px[j]));
        if (isfinite(d.lb[j])) x = jl_max(x, 0.0);
        if (isfinite(d.ub[j])) x = jl_min(x, 0.0);
        d.dray[j] = x;
        atomic_max_nonneg(&d.maxes[0], fabs(x));
    }
    __device__ void write_partials(int32_t, const double*) const {}
};

template <typename T>
struct RayRowsRow {  // y = -(pdhg - reflected) on the duals, signs from the row bounds
    static constexpr int NP = 1;
    LpVecs<T> v;
    LpData d;
    const InstState* st;
    double* part;  // per A tile: primal slack of the dual ray
    __device__ bool active(int p) const { return st[p].status == ST_RUNNING; }
    __device__ void row(int32_t i, int, double* acc) const {
        double y = sub_rn(static_cast<double>(v.ry[i]), static_cast<double>(v.py[i]));
        const bool flo = isfinite(d.clb[i]), fhi = isfinite(d.cub[i]);
        if (!flo) y = jl_min(y, 0.0);
        if (!fhi) y = jl_max(y, 0.0);
        d.yray[i] = y;
        atomic_max_nonneg(&d.maxes[1], fabs(y));
        acc[0] += add_rn(mul_rn(jl_max(y, 0.0), flo ? d.clb[i] : 0.0),
                         mul_rn(jl_min(y, 0.0), fhi ? d.cub[i] : 0.0));
    }
    __device__ void write_partials(int32_t t, const double* acc) const { part[t] = acc[0]; }
};

// A'y_ray over A': linear objective of the normalised primal ray, the dual slack
// of the dual ray and its infeasibility in original units.
template <int NTHREADS>
struct RayColOp {
    using MT = double;
    using VT = double;
    using AT = double;
    using GT = double;
    struct TileP {
        double prn;
    };
    static constexpr int NT = NTHREADS, NV = 1, NVEC = 0, NP = 2;
    LpData d;
    const InstState* st;
    double* part;  // per A' tile x 2
    int32_t* errp;
    __device__ const double* values() const { return d.val_t; }
    __device__ const double* staged(int) const { return nullptr; }
    __device__ int32_t* err() const { return errp; }
    __device__ bool active(int inst) const { return st[inst].status == ST_RUNNING; }
    __device__ TileP tile_params(int) const {
        return TileP{__longlong_as_double(static_cast<long long>(d.maxes[0]))};
    }
    __device__ void gather(int32_t col, double (&g)[1]) const { g[0] = d.yray[col]; }
    __device__ void row(int32_t j, int32_t, int, const TileP& tp, const double* const*,
                        const double (&s)[1], double* acc) const {
        const double dn = tp.prn > 0.0 ? d.dray[j] / tp.prn : d.dray[j];
        acc[0] += mul_rn(d.c[j], dn);                        // c'd
        const double mdp = -s[0];
        const bool flo = isfinite(d.lb[j]), fhi = isfinite(d.ub[j]);
        acc[1] += add_rn(mul_rn(jl_max(mdp, 0.0), flo ? d.lb[j] : 0.0),
                         mul_rn(jl_min(mdp, 0.0), fhi ? d.ub[j] : 0.0));
        double t = sub_rn(flo ? 0.0 : jl_max(0.0, mdp), fhi ? 0.0 : jl_min(0.0, mdp));
        if (d.col_unscale) t = mul_rn(t, d.col_unscale[j]);
        atomic_max_nonneg(&d.maxes[3], fabs(t));
    }
    __device__ void write_partials(int32_t t, const double* acc) const {
        part[t * 2] = acc[0];
        part[t * 2 + 1] = acc[1];
    }
};

// A d over A (d normalised by its max): the primal ray's infeasibility.
template <int NTHREADS>
struct RayRowOp {
    using MT = double;
    using VT = double;
    using AT = double;
    using GT = double;
    struct TileP {
        int32_t d;
    };
    static constexpr int NT = NTHREADS, NV = 1, NVEC = 0, NP = 0;
    LpData d;
    const InstState* st;
    int32_t* errp;
    __device__ const double* values() const { return d.val_a; }
    __device__ const double* staged(int) const { return nullptr; }
    __device__ int32_t* err() const { return errp; }
    __device__ bool active(int inst) const { return st[inst].status == ST_RUNNING; }
    __device__ TileP tile_params(int) const { return TileP{0}; }
    __device__ void gather(int32_t col, double (&g)[1]) const {
        const double prn = __longlong_as_double(static_cast<long long>(d.maxes[0]));
        g[0] = prn > 0.0 ? d.dray[col] / prn : d.dray[col];
    }
    __device__ void row(int32_t i, int32_t, int, const TileP&, const double* const*,
                        const double (&s)[1], double*) const {
        const double pp = s[0];
        double t = add_rn(isfinite(d.clb[i]) ? jl_max(0.0, -pp) : 0.0,
                          isfinite(d.cub[i]) ? jl_max(0.0, pp) : 0.0);
        if (d.row_unscale) t = mul_rn(t, d.row_unscale[i]);
        atomic_max_nonneg(&d.maxes[2], fabs(t));
    }
    __device__ void write_partials(int32_t, const double*) const {}
};

}  // namespace pdfp
