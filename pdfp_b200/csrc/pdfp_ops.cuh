// pdfp_ops.cuh -- the PDFP projector's fused passes (src/pdfp.jl, src/pdfp_kernels.jl).
//
// One PDHG step is two tile-engine launches:
//   PrimalOp  (rows of A' = columns j):  A'z gathered and summed, then
//             primal_step! and dual_y_step! fused per column
//             (src/pdfp.jl:119-143; K1+K2 of src/pdfp_kernels.jl:4-48);
//   DualOp    (rows i of A):  A x_bar, then dual_z_step! (src/pdfp.jl:146-156; K3).
// Steps whose pdhg_* / reflected_* outputs are consumed (the first step of a
// window, read by the fixed-point error after a restart, and the last step,
// read by the evaluation) are MAJOR and store them; the other steps store only
// the iterates and x_bar.
//
// Evaluation is two more launches (EvalColOp, EvalRowOp) producing per-tile
// FP64 partial sums of every term of compute_fixed_point_error! and
// compute_residual! (src/pdfp.jl:167-218) plus the restart distances of
// perform_restart! (src/pdfp.jl:180-192); the controller (pdfp_kernels.cu)
// reduces them per instance.
//
// T is the iterate type: double for the plain FP64 form, float for the mixed
// form.  Arithmetic follows the reference's expression order with explicitly
// rounded operations (no FMA contraction).
#pragma once
#include "common.cuh"
#include "layout.hpp"
#include "state.hpp"

namespace pdfp {

template <typename T>
struct IterVecs {  // one precision's copy of the projector's vectors (packed order)
    T *cx, *ix, *px, *rx, *cy, *iy, *py, *ry, *ds;  // n
    T *cz, *iz, *pz, *rz;                           // m
    T *lb, *ub, *xt, *w;                            // n (w < 0 marks a continuous column)
    T *b;                                           // m
    T* val_t;                                       // A' values in this precision
    T* val_a;                                       // A values in this precision
};

template <typename T>
__device__ __forceinline__ T halpern(T weight, T omega, T omw, T omwt, T refl, T cur, T init) {
    // weight * (omega * refl + omw * cur) + omwt * init   (src/pdfp.jl:129)
    return add_rn(mul_rn(weight, add_rn(mul_rn(omega, refl), mul_rn(omw, cur))), mul_rn(omwt, init));
}

template <typename T>
struct StepParams {
    T tau, sigma, weight, omwt, omega, omw;
};

template <typename T>
__device__ __forceinline__ StepParams<T> step_params(const InstState& st, int32_t k_offset) {
    const double k = static_cast<double>(st.inner + k_offset);
    const double weight = k / (k + 1.0);
    StepParams<T> p;
    p.tau = static_cast<T>(st.tau);
    p.sigma = static_cast<T>(st.sigma);
    p.weight = static_cast<T>(weight);
    p.omwt = static_cast<T>(1.0 - weight);
    p.omega = static_cast<T>(st.omega);
    p.omw = static_cast<T>(1.0 - st.omega);
    return p;
}

// ---- the PDHG step ------------------------------------------------------------

template <typename T, bool MAJOR, int NTHREADS>
struct PrimalOp {
    using MT = T;
    using VT = T;
    using AT = T;
    using GT = T;
    using TileP = StepParams<T>;
    static constexpr int NT = NTHREADS, NV = 1, NVEC = 8, NP = 0;
    IterVecs<T> v;
    const InstState* st;
    int32_t k_offset, mode;
    int32_t* errp;
    int32_t gather_l2;  // 1: gathers cached in L2 only (ld.global.cg); 2: async copies (tile engine)

    __device__ const T* values() const { return v.val_t; }
    __device__ const T* staged(int k) const {
        switch (k) {
            case 0: return v.cx;
            case 1: return v.ix;
            case 2: return v.cy;
            case 3: return v.iy;
            case 4: return v.lb;
            case 5: return v.ub;
            case 6: return v.xt;
            default: return v.w;
        }
    }
    __device__ int32_t* err() const { return errp; }
    __device__ bool active(int inst) const {
        return st[inst].status == ST_RUNNING && st[inst].mode == mode;
    }
    __device__ TileP tile_params(int inst) const { return step_params<T>(st[inst], k_offset); }
    __device__ void gather(int32_t col, T (&g)[1]) const {
        g[0] = gather_l2 ? __ldcg(v.cz + col) : v.cz[col];
    }
    __device__ const T* gather_src() const { return v.cz; }
    __device__ void row(int32_t j, int32_t rr, int inst, const TileP& p, const T* const* sv,
                        const T (&s)[1], double*) const {
        T pv[NVEC];
#pragma unroll
        for (int q = 0; q < NVEC; ++q) pv[q] = sv[q][rr];
        row_vals(j, p, pv, s);
    }
    // Column j's per-column inputs from global memory, in staged() order, cached in L2
    // only: L1 stays for the gathered z entries that long rows share.
    __device__ void load_row(int32_t j, T (&pv)[NVEC]) const {
#pragma unroll
        for (int q = 0; q < NVEC; ++q) pv[q] = __ldcg(staged(q) + j);
    }
    // The epilogue on column j's inputs pv (staged() order) and its sum s = (A'z)_j.
    __device__ void row_vals(int32_t j, const TileP& p, const T (&pv)[NVEC], const T (&s)[1]) const {
        const T cx = pv[0], ix = pv[1], cy = pv[2], iy = pv[3];
        const T lb = pv[4], ub = pv[5], xt = pv[6], w = pv[7];
        // primal_step!  (src/pdfp.jl:124-129)
        const T t = sub_rn(cx, mul_rn(p.tau, sub_rn(s[0], cy)));
        const T xh = jl_clamp(t, lb, ub);
        const T rx = sub_rn(mul_rn(T(2), xh), cx);
        v.cx[j] = halpern(p.weight, p.omega, p.omw, p.omwt, rx, cx, ix);
        v.rx[j] = rx;
        // dual_y_step!  (src/pdfp.jl:138-141); w < 0 marks j outside I
        const T yh = w >= T(0) ? jl_clamp(add_rn(cy, mul_rn(p.sigma, sub_rn(xt, rx))), -w, w) : T(0);
        const T ry = sub_rn(mul_rn(T(2), yh), cy);
        v.cy[j] = halpern(p.weight, p.omega, p.omw, p.omwt, ry, cy, iy);
        if (MAJOR) {
            v.px[j] = xh;
            v.ds[j] = sub_rn(xh, t) / p.tau;
            v.py[j] = yh;
            v.ry[j] = ry;
        }
    }
};

template <typename T, bool MAJOR, int NTHREADS>
struct DualOp {
    using MT = T;
    using VT = T;
    using AT = T;
    using GT = T;
    struct TileP {
        StepParams<T> p;
        int32_t eq_end;  // packed rows below this index are equality rows
    };
    static constexpr int NT = NTHREADS, NV = 1, NVEC = 3, NP = 0;
    IterVecs<T> v;
    const InstState* st;
    const int32_t* row_off;
    const int32_t* n_eq;
    int32_t k_offset, mode;
    int32_t* errp;
    int32_t gather_l2;

    __device__ const T* values() const { return v.val_a; }
    __device__ const T* staged(int k) const { return k == 0 ? v.cz : (k == 1 ? v.iz : v.b); }
    __device__ int32_t* err() const { return errp; }
    __device__ bool active(int inst) const {
        return st[inst].status == ST_RUNNING && st[inst].mode == mode;
    }
    __device__ TileP tile_params(int inst) const {
        TileP t;
        t.p = step_params<T>(st[inst], k_offset);
        t.eq_end = row_off[inst] + n_eq[inst];
        return t;
    }
    __device__ void gather(int32_t col, T (&g)[1]) const {
        g[0] = gather_l2 ? __ldcg(v.rx + col) : v.rx[col];
    }
    __device__ const T* gather_src() const { return v.rx; }
    __device__ void row(int32_t i, int32_t rr, int inst, const TileP& t, const T* const* sv,
                        const T (&s)[1], double*) const {
        T pv[NVEC];
#pragma unroll
        for (int q = 0; q < NVEC; ++q) pv[q] = sv[q][rr];
        row_vals(i, t, pv, s);
    }
    // Row i's per-row inputs from global memory, in staged() order.
    __device__ void load_row(int32_t i, T (&pv)[NVEC]) const {
#pragma unroll
        for (int q = 0; q < NVEC; ++q) pv[q] = staged(q)[i];
    }
    // The epilogue on row i's inputs pv (staged() order) and its sum s = (A x_bar)_i.
    __device__ void row_vals(int32_t i, const TileP& t, const T (&pv)[NVEC], const T (&s)[1]) const {
        const T cz = pv[0], iz = pv[1], b = pv[2];
        // dual_z_step!  (src/pdfp.jl:150-154)
        const T raw = add_rn(cz, mul_rn(t.p.sigma, sub_rn(s[0], b)));
        const T zh = i < t.eq_end ? raw : jl_max(raw, T(0));
        const T rz = sub_rn(mul_rn(T(2), zh), cz);
        v.cz[i] = halpern(t.p.weight, t.p.omega, t.p.omw, t.p.omwt, rz, cz, iz);
        if (MAJOR) {
            v.pz[i] = zh;
            v.rz[i] = rz;
        }
    }
};

// ---- evaluation -------------------------------------------------------------------

struct EvalData {  // FP64 problem data for the evaluation (packed order)
    const double *xt, *w, *b, *row_unscale;
    const double *val_t, *val_a;
    double* part_col;  // n_tiles(eval A') x 8
    double* part_row;  // n_tiles(eval A) x 4
};

enum : int32_t { EVAL_FULL = 0, EVAL_AFTER_RESTART = 1 };

// Column terms: A'z_hat and A'(z_hat - z_bar) from one pass over A'.
template <typename T, int NTHREADS>
struct EvalColOp {
    using MT = double;
    using VT = double;
    using AT = double;
    using GT = double;
    struct TileP {
        int32_t dummy;
    };
    static constexpr int NT = NTHREADS, NV = 2, NVEC = 0, NP = 8;
    IterVecs<T> v;
    EvalData d;
    const InstState* st;
    int32_t which, mode;
    int32_t* errp;

    __device__ const double* values() const { return d.val_t; }
    __device__ const double* staged(int) const { return nullptr; }
    __device__ int32_t* err() const { return errp; }
    __device__ bool active(int inst) const {
        const InstState& s = st[inst];
        return s.status == ST_RUNNING && s.mode == mode &&
               (which == EVAL_FULL || s.do_restart);
    }
    __device__ TileP tile_params(int) const { return TileP{0}; }
    __device__ void gather(int32_t col, double (&g)[2]) const {
        const double pz = static_cast<double>(v.pz[col]);
        g[0] = pz;
        g[1] = sub_rn(pz, static_cast<double>(v.rz[col]));  // delta_z (src/pdfp.jl:170)
    }
    __device__ void row(int32_t j, int32_t, int, const TileP&, const double* const*,
                        const double (&s)[2], double* acc) const {
        const double px = v.px[j], rx = v.rx[j], py = v.py[j], ry = v.ry[j];
        const double dx = sub_rn(px, rx), dy = sub_rn(py, ry);
        acc[0] += dx * dx;                               // sum(abs2, delta_x)
        acc[1] += dy * dy;                               // sum(abs2, delta_y)
        acc[2] += mul_rn(sub_rn(s[1], dy), dx);          // <A'dz - dy, dx>
        const double r = sub_rn(sub_rn(s[0], py), static_cast<double>(v.ds[j]));
        acc[3] += r * r;                                 // ||A'z - y - dual_slack||^2
        const double w = d.w[j];
        if (w >= 0.0) {
            const double xt = d.xt[j];
            acc[4] += mul_rn(w, fabs(sub_rn(px, xt)));   // l1 distance
            acc[5] += mul_rn(py, sub_rn(xt, px));        // y term of the gap
        }
        const double ex = sub_rn(static_cast<double>(v.ix[j]), px);
        const double ey = sub_rn(static_cast<double>(v.iy[j]), py);
        acc[6] += ex * ex;                               // restart distance (x)
        acc[7] += ey * ey;                               // restart distance (y)
    }
    __device__ void write_partials(int32_t tile, const double* acc) const {
#pragma unroll
        for (int k = 0; k < NP; ++k) d.part_col[tile * NP + k] = acc[k];
    }
};

// Row terms: A x_hat from one pass over A.
template <typename T, int NTHREADS>
struct EvalRowOp {
    using MT = double;
    using VT = double;
    using AT = double;
    using GT = double;
    struct TileP {
        int32_t eq_end;
    };
    static constexpr int NT = NTHREADS, NV = 1, NVEC = 0, NP = 4;
    IterVecs<T> v;
    EvalData d;
    const InstState* st;
    const int32_t* row_off;
    const int32_t* n_eq;
    int32_t which, mode;
    int32_t* errp;

    __device__ const double* values() const { return d.val_a; }
    __device__ const double* staged(int) const { return nullptr; }
    __device__ int32_t* err() const { return errp; }
    __device__ bool active(int inst) const {
        const InstState& s = st[inst];
        return s.status == ST_RUNNING && s.mode == mode &&
               (which == EVAL_FULL || s.do_restart);
    }
    __device__ TileP tile_params(int inst) const { return TileP{row_off[inst] + n_eq[inst]}; }
    __device__ void gather(int32_t col, double (&g)[1]) const { g[0] = static_cast<double>(v.px[col]); }
    __device__ void row(int32_t i, int32_t, int, const TileP& t, const double* const*,
                        const double (&s)[1], double* acc) const {
        const double b = d.b[i];
        const double dd = sub_rn(s[0], b);
        double viol = i < t.eq_end ? fabs(dd) : jl_max(dd, 0.0);   // src/pdfp.jl:202
        if (d.row_unscale) viol = mul_rn(viol, d.row_unscale[i]);  // :203
        acc[0] += viol * viol;
        const double pz = v.pz[i];
        acc[1] += mul_rn(pz, dd);                                  // z term of the gap
        const double dz = sub_rn(pz, static_cast<double>(v.rz[i]));
        acc[2] += dz * dz;                                         // sum(abs2, delta_z)
        const double ez = sub_rn(static_cast<double>(v.iz[i]), pz);
        acc[3] += ez * ez;                                         // restart distance (z)
    }
    __device__ void write_partials(int32_t tile, const double* acc) const {
#pragma unroll
        for (int k = 0; k < NP; ++k) d.part_row[tile * NP + k] = acc[k];
    }
};

}  // namespace pdfp
