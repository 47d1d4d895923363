// pdlp.cu -- the root-LP solver on the device: solve_lp_relaxation / pdlp_solve!.
//
// src/pdlp.jl:325-393: scale (bound/objective rescaling on), estimate ||A||_2,
// then windows of `freq` PDHG steps -- step 1 and step `freq` are major --
// each followed by the fixed-point error, the residuals (original units under
// cuPDLPx termination), cuPDLPx infeasibility detection, the termination tests
// and the restart rule, all on the device.  One window is one CUDA graph.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "../../include/pdfp_b200.h"
#include "controller.cuh"
#include "device.hpp"
#include "kernels.cuh"
#include "pdlp_ops.cuh"
#include "tiny_steps.cuh"
#include "power.cuh"
#include "solvers.hpp"

namespace pdfp {

constexpr int LP_NT = 256;
constexpr double LP_EPS_INFEASIBLE = 1e-14;  // src/pdlp.jl:53


// ---- initialisation: the norms of initialize_step_size_and_primal_weight! ----------

struct LpNormRowsA {  // lo_sq, hi_sq over the rows (src/pdlp.jl:304-312)
    static constexpr int NP = 2;
    LpData d;
    double bound_scale;
    double* part;
    __device__ bool active(int) const { return true; }
    __device__ void row(int32_t i, int, double* acc) const {
        double lo = d.clb[i], hi = d.cub[i];
        if (d.row_unscale) {
            lo = lo * d.row_unscale[i] / bound_scale;
            hi = hi * d.row_unscale[i] / bound_scale;
        }
        const double a = (isfinite(lo) && d.clb[i] != d.cub[i]) ? lo : 0.0;
        const double b = isfinite(hi) ? hi : 0.0;
        acc[0] += a * a;
        acc[1] += b * b;
    }
    __device__ void write_partials(int32_t t, const double* acc) const {
        part[t * 4] = acc[0];
        part[t * 4 + 1] = acc[1];
        part[t * 4 + 2] = 0.0;
        part[t * 4 + 3] = 0.0;
    }
};

struct LpNormRowsC {  // ||c|| (in original units under cuPDLPx)
    static constexpr int NP = 1;
    LpData d;
    double* part;
    __device__ bool active(int) const { return true; }
    __device__ void row(int32_t j, int, double* acc) const {
        const double t = d.col_unscale ? d.c[j] * d.col_unscale[j] : d.c[j];
        acc[0] += t * t;
    }
    __device__ void write_partials(int32_t t, const double* acc) const {
        for (int k = 0; k < 8; ++k) part[t * 8 + k] = k == 0 ? acc[0] : 0.0;
    }
};

struct LpNormFin {
    static constexpr int NA = 8, NB = 4;
    const int32_t* ta0;
    const double* pa;
    const int32_t* tb0;
    const double* pb;
    InstState* st;
    int32_t cupdlpx;
    __device__ bool active(int) const { return true; }
    __device__ void finalize(int p, const double* a) const {
        InstState& s = st[p];
        s.ovn = cupdlpx ? sqrt(a[0]) / s.objective_scale : sqrt(a[0]);
        s.cbn = sqrt(a[8] + a[9]);
    }
};

// ---- the controller ---------------------------------------------------------------------

struct LpRayFin {  // compute_infeasibility_information!, src/pdlp.jl:259-283
    static constexpr int NA = 2, NB = 1;
    const int32_t* ta0;
    const double* pa;
    const int32_t* tb0;
    const double* pb;
    InstState* st;
    const unsigned long long* maxes;
    __device__ bool active(int p) const { return st[p].status == ST_RUNNING; }
    __device__ void finalize(int p, const double* a) const {
        InstState& s = st[p];
        const double scale = s.bound_scale * s.objective_scale;
        const double drn = __longlong_as_double(static_cast<long long>(maxes[1]));
        const double dsn = __longlong_as_double(static_cast<long long>(maxes[3]));
        s.primal_ray_lin_obj = a[0] / scale;
        double dro = (a[2] + a[1]) / scale;  // (primal_slack + dual_slack) / scale
        s.max_primal_ray_inf = __longlong_as_double(static_cast<long long>(maxes[2]));
        const double scaling = jl_max(drn, dsn);
        if (scaling > 0.0) {
            s.max_dual_ray_inf = dsn / scaling;
            dro /= scaling;
        } else {
            s.max_dual_ray_inf = 0.0;
            dro = 0.0;
        }
        s.dual_ray_obj = dro;
    }
};

struct LpController {
    static constexpr int NA = 8, NB = 4;
    const int32_t* ta0;
    const double* pa;
    const int32_t* tb0;
    const double* pb;
    InstState* st;
    InstFlags* fl;
    int32_t phase, cupdlpx;
    __device__ bool active(int p) const {
        return st[p].status == ST_RUNNING && (phase == 1 || st[p].do_restart);
    }
    __device__ void finalize(int p, const double* a) const {
        InstState& s = st[p];
        const double pw = s.primal_weight;
        // compute_fixed_point_error!, src/pdlp.jl:157-165
        const double movement = a[0] * pw + a[8] / pw;
        const double interaction = 2.0 * s.step_size * a[1];
        s.fpe = sqrt(jl_max(movement + interaction, 0.0));
        if (phase == 0) {  // src/pdlp.jl:333-337
            s.initial_fpe = s.fpe;
            s.do_restart = 0;
            return;
        }
        // compute_residual!, src/pdlp.jl:220-242
        const double pr = sqrt(a[9]) / s.bound_scale;
        const double dr = sqrt(a[2]) / s.objective_scale;
        s.rel_p = pr / (1.0 + s.cbn);
        s.rel_d = dr / (1.0 + s.ovn);
        const double scale = s.bound_scale * s.objective_scale;
        const double obj = a[3] / scale;
        const double dobj = (a[4] + a[10]) / scale;
        s.objective_value = obj;
        s.rel_gap = fabs(obj - dobj) / (1.0 + fabs(obj) + fabs(dobj));
        s.inner += s.freq;
        s.total += s.freq;
        s.restart_now = 0;
        if (s.rel_p <= s.eps_feas && s.rel_d <= s.eps_feas && s.rel_gap <= s.eps_opt) {
            s.status = ST_OPTIMAL;
        } else if (cupdlpx && s.dual_ray_obj > 0.0 &&
                   s.max_dual_ray_inf / s.dual_ray_obj <= LP_EPS_INFEASIBLE) {
            s.status = ST_PRIMAL_INFEASIBLE;
        } else if (cupdlpx && s.primal_ray_lin_obj < 0.0 &&
                   s.max_primal_ray_inf / (-s.primal_ray_lin_obj) <= LP_EPS_INFEASIBLE) {
            s.status = ST_DUAL_INFEASIBLE;
        } else if (static_cast<double>(globaltimer_ns() - s.t_start_ns) * 1e-9 > s.time_limit) {
            s.status = ST_TIME_LIMIT;
        } else {
            if (should_restart(s)) {  // perform_restart!, src/pdlp.jl:207-216
                update_primal_weight(s, sqrt(a[5]), sqrt(a[11]));
                s.inner = 0;
                s.last_trial_fpe = INFINITY;
                s.restarts += 1;
                s.restart_now = 1;
                s.do_restart = 1;
            }
            s.tau = s.step_size / s.primal_weight;
            s.sigma = s.step_size * s.primal_weight;
            if (s.total >= s.iter_limit) s.status = ST_ITERATION_LIMIT;
        }
        int32_t request = 0;
        if (s.status == ST_RUNNING && s.mode == MODE_FP32) {
            // FP32 progress test: hand over to the FP64 form when the KKT score has
            // not improved by 10% over ten evaluations
            const double score = fmax(s.rel_p / s.eps_feas, fmax(s.rel_d / s.eps_feas, s.rel_gap / s.eps_opt));
            if (score < 0.9 * s.best_score) {
                s.best_score = score;
                s.stall = 0;
            } else {
                s.stall += 1;
            }
            if (s.stall >= 10 && score > 1.0) request = 1;
        }
        fl[p] = InstFlags{s.status, s.mode, request, 0};
    }
};

template <typename S, typename D>
struct LpConvert {  // the LP iterates S -> D (the FP64 polish)
    LpVecs<S> s;
    LpVecs<D> d;
    int32_t n, m;
    __device__ bool active(int) const { return true; }
    __device__ int32_t begin(int) const { return 0; }
    __device__ int32_t end(int) const { return n + m; }
    __device__ void elem(int, int32_t i) const {
        if (i < n) {
            d.cx[i] = static_cast<D>(s.cx[i]); d.ix[i] = static_cast<D>(s.ix[i]);
            d.px[i] = static_cast<D>(s.px[i]); d.rx[i] = static_cast<D>(s.rx[i]);
            d.ds[i] = static_cast<D>(s.ds[i]);
        } else {
            const int32_t r = i - n;
            d.cy[r] = static_cast<D>(s.cy[r]); d.iy[r] = static_cast<D>(s.iy[r]);
            d.py[r] = static_cast<D>(s.py[r]); d.ry[r] = static_cast<D>(s.ry[r]);
        }
    }
};

__global__ void lp_set_mode_kernel(InstState* st, int32_t mode) { st[0].mode = mode; }

template <typename T>
struct LpRestartCopy {
    LpVecs<T> v;
    const InstState* st;
    int32_t n, m;
    __device__ bool active(int p) const { return st[p].restart_now; }
    __device__ int32_t begin(int) const { return 0; }
    __device__ int32_t end(int) const { return n + m; }
    __device__ void elem(int, int32_t i) const {
        if (i < n) {
            const T x = v.px[i];
            v.ix[i] = x;
            v.cx[i] = x;
        } else {
            const int32_t r = i - n;
            const T y = v.py[r];
            v.iy[r] = y;
            v.cy[r] = y;
        }
    }
};

// ---- a small LP's whole solve in one launch ---------------------------------------------
//
// As for the projector (tiny_solve_kernel, pdfp.cu): one block runs whole evaluation
// windows of pdlp_solve! (src/pdlp.jl:332-370) -- step 1, the evaluation after a
// restart, steps 2 .. freq-1, step freq, the full evaluation, the cuPDLPx ray passes,
// the controller and the restart copy -- until the LP stops, asks for the FP64 polish,
// or max_windows windows have run.  STAGED: the LP's iterates, data, ray work vectors
// and matrix are copied into the block's shared memory for the launch (the iterates
// back at its end): the same arithmetic, bit-identical results.
constexpr int kLpTinyWindowsPerLaunch = 64;

// Shared-memory bytes of an LP's staged copy (lp_tiny_solve_kernel<T, true>).
template <typename T>
inline size_t lp_tiny_stage_bytes(int64_t n, int64_t m, int64_t nnz, bool unscale) {
    auto r16 = [](int64_t b) { return static_cast<size_t>((b + 15) & ~int64_t(15)); };
    size_t b = 8 * r16(sizeof(T) * n) + 6 * r16(sizeof(T) * m);          // iterates and data
    b += r16(4 * (n + 1)) + r16(4 * (m + 1)) + 2 * r16(4 * nnz) + 2 * r16(sizeof(T) * nnz);
    b += r16(8 * n) + r16(8 * m);                                         // ray work vectors
    if (sizeof(T) == 4) b += 3 * r16(8 * n) + 2 * r16(8 * m) + 2 * r16(8 * nnz);  // FP64 copies
    if (unscale) b += r16(8 * n) + r16(8 * m);
    return b;
}

template <typename T, bool STAGED>
__global__ void __launch_bounds__(kTinyThreads)
    lp_tiny_solve_kernel(LpVecs<T> gv, LpData gd, InstState* st, InstFlags* fl,
                         const int32_t* __restrict__ g_rp_t, const int32_t* __restrict__ g_ci_t,
                         const int32_t* __restrict__ g_rp_a, const int32_t* __restrict__ g_ci_a,
                         int32_t n, int32_t m, int32_t* err, int32_t cupdlpx, int32_t max_windows,
                         int32_t rowsum_len) {
    constexpr int NT = kTinyThreads;
    constexpr int32_t mode = std::is_same<T, float>::value ? MODE_FP32 : MODE_FP64;
    extern __shared__ __align__(16) double lp_rowsum[];  // rowsum_len doubles, then the staged copy
    __shared__ double red[8 * (NT / 32)];
    __shared__ int32_t go;
    LpVecs<T> v = gv;
    LpData d = gd;
    const int32_t *rp_t = g_rp_t, *ci_t = g_ci_t, *rp_a = g_rp_a, *ci_a = g_ci_a;
    T* const gx[5] = {gv.cx, gv.ix, gv.px, gv.rx, gv.ds};  // n-side iterates
    T* const gy[4] = {gv.cy, gv.iy, gv.py, gv.ry};         // m-side iterates
    T* sx[5] = {};
    T* sy[4] = {};
    if constexpr (STAGED) {
        unsigned char* cur = reinterpret_cast<unsigned char*>(lp_rowsum + rowsum_len);
        auto carve = [&](size_t bytes) {
            unsigned char* q = cur;
            cur += (bytes + 15) & ~size_t(15);
            return q;
        };
        auto stage = [&](const auto* src, int64_t len) {
            using E = std::remove_cv_t<std::remove_pointer_t<decltype(src)>>;
            E* q = reinterpret_cast<E*>(carve(sizeof(E) * len));
            for (int64_t i = threadIdx.x; i < len; i += NT) q[i] = src[i];
            return q;
        };
        const int32_t nnz = g_rp_a[m];
        for (int k = 0; k < 5; ++k) sx[k] = stage(gx[k], n);
        for (int k = 0; k < 4; ++k) sy[k] = stage(gy[k], m);
        v.cx = sx[0]; v.ix = sx[1]; v.px = sx[2]; v.rx = sx[3]; v.ds = sx[4];
        v.cy = sy[0]; v.iy = sy[1]; v.py = sy[2]; v.ry = sy[3];
        v.c = stage(gv.c, n);
        v.lb = stage(gv.lb, n);
        v.ub = stage(gv.ub, n);
        v.clb = stage(gv.clb, m);
        v.cub = stage(gv.cub, m);
        rp_t = stage(g_rp_t, n + 1);
        rp_a = stage(g_rp_a, m + 1);
        ci_t = stage(g_ci_t, nnz);
        ci_a = stage(g_ci_a, nnz);
        v.val_t = stage(gv.val_t, nnz);
        v.val_a = stage(gv.val_a, nnz);
        if constexpr (std::is_same<T, double>::value) {  // the FP64 data are these very arrays
            d.c = v.c;
            d.lb = v.lb;
            d.ub = v.ub;
            d.clb = v.clb;
            d.cub = v.cub;
            d.val_t = v.val_t;
            d.val_a = v.val_a;
        } else {
            d.c = stage(gd.c, n);
            d.lb = stage(gd.lb, n);
            d.ub = stage(gd.ub, n);
            d.clb = stage(gd.clb, m);
            d.cub = stage(gd.cub, m);
            d.val_t = stage(gd.val_t, nnz);
            d.val_a = stage(gd.val_a, nnz);
        }
        if (gd.row_unscale) d.row_unscale = stage(gd.row_unscale, m);
        if (gd.col_unscale) d.col_unscale = stage(gd.col_unscale, n);
        d.dray = reinterpret_cast<double*>(carve(8 * n));  // work vectors: written before read
        d.yray = reinterpret_cast<double*>(carve(8 * m));
        __syncthreads();
    }
    auto evaluate = [&](int32_t which, int32_t phase) {
        double ac[8], ar[4];
#pragma unroll
        for (int k = 0; k < 8; ++k) ac[k] = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) ar[k] = 0.0;
        tiny_eval_pass(LpEvalColOp<T, NT>{v, d, st, which, mode, err}, rp_t, ci_t, 0, n, 0, lp_rowsum, ac);
        block_sum<NT, 8>(ac, red, threadIdx.x);
        tiny_eval_pass(LpEvalRowOp<T, NT>{v, d, st, which, mode, err}, rp_a, ci_a, 0, m, 0, lp_rowsum, ar);
        block_sum<NT, 4>(ar, red, threadIdx.x);
        if (phase == 1 && cupdlpx) {  // compute_infeasibility_information!, src/pdlp.jl:247-285
            if (threadIdx.x < 4) d.maxes[threadIdx.x] = 0ull;
            __syncthreads();
            double none[2] = {0.0, 0.0};
            const RayRowsCol<T> rc{v, d, st};
            for (int32_t j = threadIdx.x; j < n; j += NT) rc.row(j, 0, none);
            double rr[1] = {0.0};
            const RayRowsRow<T> rw{v, d, st, nullptr};
            for (int32_t i = threadIdx.x; i < m; i += NT) rw.row(i, 0, rr);
            block_sum<NT, 1>(rr, red, threadIdx.x);  // its barriers also order dray, yray and the maxima
            double a2[2] = {0.0, 0.0};
            tiny_eval_pass(RayColOp<NT>{d, st, nullptr, err}, rp_t, ci_t, 0, n, 0, lp_rowsum, a2);
            block_sum<NT, 2>(a2, red, threadIdx.x);
            double a0[1] = {0.0};
            tiny_eval_pass(RayRowOp<NT>{d, st, err}, rp_a, ci_a, 0, m, 0, lp_rowsum, a0);
            if (threadIdx.x == 0) {
                const double a[3] = {a2[0], a2[1], rr[0]};
                LpRayFin{nullptr, nullptr, nullptr, nullptr, st, d.maxes}.finalize(0, a);
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            const double a[12] = {ac[0], ac[1], ac[2], ac[3], ac[4], ac[5], ac[6], ac[7],
                                  ar[0], ar[1], ar[2], ar[3]};
            LpController{nullptr, nullptr, nullptr, nullptr, st, fl, phase, cupdlpx}.finalize(0, a);
        }
        __syncthreads();
    };
    for (int32_t w = 0; w < max_windows; ++w) {
        if (threadIdx.x == 0) go = st[0].status == ST_RUNNING && st[0].mode == mode;
        __syncthreads();
        if (!go) break;
        const int32_t freq = st[0].freq;
        for (int32_t i = 1; i <= freq; ++i) {  // pdhg_step!, src/pdlp.jl:147-153
            if (i == 1 || i == freq) {
                tiny_pass(LpPrimalOp<T, true, NT>{v, st, i, mode, err}, rp_t, ci_t, 0, n, 0);
                __syncthreads();
                tiny_pass(LpDualOp<T, true, NT>{v, st, i, mode, err}, rp_a, ci_a, 0, m, 0);
            } else {
                tiny_pass(LpPrimalOp<T, false, NT>{v, st, i, mode, err}, rp_t, ci_t, 0, n, 0);
                __syncthreads();
                tiny_pass(LpDualOp<T, false, NT>{v, st, i, mode, err}, rp_a, ci_a, 0, m, 0);
            }
            __syncthreads();
            if (i == 1 && st[0].do_restart) evaluate(EVAL_AFTER_RESTART, 0);
        }
        evaluate(EVAL_FULL, 1);
        const LpRestartCopy<T> rc{v, st, n, m};
        if (rc.active(0))
            for (int32_t i = threadIdx.x; i < n + m; i += NT) rc.elem(0, i);
        if (threadIdx.x == 0) go = st[0].status == ST_RUNNING && !fl[0].polish_request;
        __syncthreads();
        if (!go) break;
    }
    if constexpr (STAGED) {  // the iterates back to global memory
        __syncthreads();
        for (int k = 0; k < 5; ++k)
            for (int32_t i = threadIdx.x; i < n; i += NT) gx[k][i] = sx[k][i];
        for (int k = 0; k < 4; ++k)
            for (int32_t i = threadIdx.x; i < m; i += NT) gy[k][i] = sy[k][i];
    }
}

__global__ void lp_begin_kernel(InstState* st) { st[0].t_start_ns = globaltimer_ns(); }
__global__ void zero_maxes_kernel(unsigned long long* m) {
    if (threadIdx.x < 4) m[threadIdx.x] = 0ull;
}

// ---- the solver ----------------------------------------------------------------------------

class LpSolver {
  public:
    // The LP in its original units; it is scaled on the device (scale_uploaded: Ruiz
    // rounds and Pock-Chambolle alpha, with the bound/objective rescaling), as
    // solve_lp_relaxation scales it first (src/pdlp.jl:381-393).
    LpSolver(const pdfp_csr& A, const double* c, const double* lb, const double* ub,
             const double* clb, const double* cub, int32_t ruiz_iterations, double alpha,
             bool cupdlpx, int precision)
        : cupdlpx_(cupdlpx), f32_(precision == PDFP_MIXED) {
        int dev = 0;
        PDFP_CK(cudaGetDevice(&dev));
        PDFP_CK(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev));
        PDFP_CK(cudaDeviceGetAttribute(&max_smem_, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        PDFP_CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        static const int32_t zero_rp = 0;
        ProblemIn in{A.m, A.n, A.m > 0 ? A.row_ptr : &zero_rp, A.col_idx, A.val, nullptr};
        std::string msg = build_layout({in}, false, M_.L);  // caller order: no permutation
        if (!msg.empty()) throw Error(E_INVALID, msg);
        // as for the projector: below 2^18 nonzeros (PDFP_MIXED_MIN_NNZ overrides)
        // every launch is latency-bound and the mixed form computes in FP64
        if (f32_) {
            const char* mm = std::getenv("PDFP_MIXED_MIN_NNZ");
            const int64_t min_nnz = mm ? std::atoll(mm) : (int64_t(1) << 18);
            if (M_.L.NNZ < min_nnz) f32_ = false;
        }
        M_.upload(ar_, f32_);  // unscaled; the FP32 copies are refreshed after the scaling
        {
            const char* te = std::getenv("PDFP_TINY");
            tiny_ = !(te && te[0] == '0') && static_cast<int64_t>(A.m) + A.n <= 4096 &&
                    M_.L.NNZ <= (1 << 16);
        }
        m_ = A.m;
        n_ = A.n;
        const int e = f32_ ? 4 : 8;
        // the step tilings serve the captured window only (a small LP runs
        // lp_tiny_solve_kernel); the evaluation tilings also serve the power iteration
        // and the initial norms
        if (!tiny_) {
            it_t_ = M_.make_tiling(ar_, true, StageGeom{e, e, e, 5, 1, 24 * 1024, 2048});
            it_a_ = M_.make_tiling(ar_, false, StageGeom{e, e, e, 4, 1, 24 * 1024, 2048});
        }
        if (f32_ && !tiny_) {  // FP64 tilings for the polish
            it64_t_ = M_.make_tiling(ar_, true, StageGeom{8, 8, 8, 5, 1, 24 * 1024, 2048});
            it64_a_ = M_.make_tiling(ar_, false, StageGeom{8, 8, 8, 4, 1, 24 * 1024, 2048});
        }
        StageGeom gev{8, 8, 8, 0, 2, 24 * 1024, 2048};
        ev_t_ = M_.make_tiling(ar_, true, gev);
        ev_a_ = M_.make_tiling(ar_, false, gev);
        alloc_vecs(v64_);
        v64_.val_t = M_.v64_t;
        v64_.val_a = M_.v64_a;
        if (f32_) {
            alloc_vecs(v32_);
            v32_.val_t = M_.v32_t;
            v32_.val_a = M_.v32_a;
        }
        // the original vectors in one copy, scaled on the device into the iterate
        // vectors; D_c and the two scales come back in one copy
        {
            const int64_t tot = 3 * int64_t(n_) + 2 * int64_t(m_);
            std::vector<double> hin(std::max<int64_t>(tot, 1));
            const double* src[5] = {c, lb, ub, clb, cub};
            const int64_t len[5] = {n_, n_, n_, m_, m_};
            double* const din = ar_.alloc<double>(hin.size());
            const double* vin[5];
            double* const vout[5] = {v64_.c, v64_.lb, v64_.ub, v64_.clb, v64_.cub};
            int64_t off = 0;
            for (int k = 0; k < 5; ++k) {
                if (len[k]) std::copy(src[k], src[k] + len[k], hin.begin() + off);
                vin[k] = din + off;
                off += len[k];
            }
            double* dsc = ar_.alloc<double>(static_cast<size_t>(n_) + m_ + 2);  // D_c, D_r, scales
            double* D_c = dsc;
            double* D_r = dsc + n_;
            double* scales = D_r + m_;
            if (tot) PDFP_CK(cudaMemcpyAsync(din, hin.data(), sizeof(double) * tot, cudaMemcpyHostToDevice, stream_));
            scale_uploaded(M_, ar_, ruiz_iterations, alpha, true, vin, vout, D_r, D_c, scales, stream_);
            if (f32_) {
                M_.refresh_f32(stream_);
                float* const f[5] = {v32_.c, v32_.lb, v32_.ub, v32_.clb, v32_.cub};
                for (int k = 0; k < 5; ++k) cast_f64_to_f32(vout[k], f[k], len[k], stream_);
            }
            d_.row_unscale = nullptr;
            d_.col_unscale = nullptr;
            if (cupdlpx) {  // cupdlpx_termination!, src/pdlp.jl:105-110: 1 ./ D_r, 1 ./ D_c
                double* dru = ar_.alloc<double>(m_);
                double* dcu = ar_.alloc<double>(n_);
                reciprocal(D_r, dru, m_, stream_);
                reciprocal(D_c, dcu, n_, stream_);
                d_.row_unscale = dru;
                d_.col_unscale = dcu;
            }
            D_c_.resize(static_cast<size_t>(n_) + 2);
            PDFP_CK(cudaMemcpyAsync(D_c_.data(), D_c, sizeof(double) * n_, cudaMemcpyDeviceToHost, stream_));
            PDFP_CK(cudaMemcpyAsync(D_c_.data() + n_, scales, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream_));
            PDFP_CK(cudaStreamSynchronize(stream_));
            bound_scale_ = D_c_[n_];
            objective_scale_ = D_c_[n_ + 1];
            D_c_.resize(n_);
        }
        d_.c = v64_.c;
        d_.lb = v64_.lb;
        d_.ub = v64_.ub;
        d_.clb = v64_.clb;
        d_.cub = v64_.cub;
        d_.val_t = M_.v64_t;
        d_.val_a = M_.v64_a;
        d_.dray = ar_.alloc<double>(n_);
        d_.yray = ar_.alloc<double>(m_);
        d_.part_col = ar_.alloc<double>(8 * static_cast<size_t>(std::max(ev_t_.dev.n_tiles, 1)));
        d_.part_row = ar_.alloc<double>(4 * static_cast<size_t>(std::max(ev_a_.dev.n_tiles, 1)));
        d_.maxes = ar_.alloc<unsigned long long>(4);
        ray_part_col_ = ar_.alloc<double>(2 * static_cast<size_t>(std::max(ev_t_.dev.n_tiles, 1)));
        ray_part_row_ = ar_.alloc<double>(static_cast<size_t>(std::max(ev_a_.dev.n_tiles, 1)));
        st_ = ar_.alloc<InstState>(1);
        flags_ = ar_.alloc<InstFlags>(2);
        err_ = ar_.alloc<int32_t>(4);
        InstState s;
        std::memset(&s, 0, sizeof(s));
        s.primal_weight = 1.0;
        s.best_primal_weight = 1.0;
        s.best_gap = INFINITY;
        s.fpe = s.initial_fpe = s.last_trial_fpe = INFINITY;
        s.rel_p = s.rel_d = s.rel_gap = INFINITY;
        s.bound_scale = bound_scale_;
        s.objective_scale = objective_scale_;
        s.objective_value = NAN;
        s.nnz_zero = (A.m == 0 || A.row_ptr[A.m] == 0) ? 1 : 0;
        s.mode = f32_ ? MODE_FP32 : MODE_FP64;
        s.status = ST_RUNNING;
        PDFP_CK(cudaMemcpy(st_, &s, sizeof(s), cudaMemcpyHostToDevice));
        PDFP_CK(cudaDeviceSynchronize());
    }

    ~LpSolver() {
        if (graph_) cudaGraphExecDestroy(graph_);
        if (stream_) cudaStreamDestroy(stream_);
    }

    int32_t solve(double tolerance, double time_limit, int32_t sv_max_it, double sv_tol,
                  double* x_scaled, double* dual_slack, pdfp_result* r);
    const std::vector<double>& col_scale() const { return D_c_; }  // D_c, host copy
    double bound_scale() const { return bound_scale_; }

  private:
    template <typename T>
    void alloc_vecs(LpVecs<T>& v) {
        T** nv[] = {&v.cx, &v.ix, &v.px, &v.rx, &v.ds, &v.c, &v.lb, &v.ub};
        for (T** q : nv) *q = ar_.alloc<T>(n_);
        T** mv[] = {&v.cy, &v.iy, &v.py, &v.ry, &v.clb, &v.cub};
        for (T** q : mv) *q = ar_.alloc<T>(m_);
    }
    template <typename T>
    void record(int freq);
    template <typename T>
    void launch_tiny_solve();
    template <typename T>
    void prepare_grids();

    bool cupdlpx_, f32_;
    std::vector<double> D_c_;
    double bound_scale_ = 1.0, objective_scale_ = 1.0;
    bool tiny_ = false;  // small LP: whole windows in one launch (lp_tiny_solve_kernel)
    int sms_ = 148;
    int max_smem_ = 232448;  // dynamic shared memory a block may opt into
    int32_t m_ = 0, n_ = 0;
    cudaStream_t stream_ = nullptr;
    DeviceArena ar_;
    DeviceMatrix M_;
    DeviceMatrix::Tiling it_t_, it_a_, it64_t_, it64_a_, ev_t_, ev_a_;
    LpVecs<double> v64_{};
    LpVecs<float> v32_{};
    LpData d_{};
    double *ray_part_col_ = nullptr, *ray_part_row_ = nullptr;
    InstState* st_ = nullptr;
    InstFlags* flags_ = nullptr;
    int32_t* err_ = nullptr;
    int gp_ = 0, gd_ = 0, gec_ = 0, ger_ = 0, grc_ = 0, grr_ = 0;
    cudaGraphExec_t graph_ = nullptr;
    bool polished_ = false;
    template <typename T>
    const DeviceMatrix::Tiling& tiling_t() const {
        return (std::is_same<T, double>::value && f32_) ? it64_t_ : it_t_;
    }
    template <typename T>
    const DeviceMatrix::Tiling& tiling_a() const {
        return (std::is_same<T, double>::value && f32_) ? it64_a_ : it_a_;
    }
    template <typename T>
    cudaGraphExec_t build_graph(int freq);
};

template <typename T>
void LpSolver::prepare_grids() {
    gp_ = tile_grid<LpPrimalOp<T, true, LP_NT>>(tiling_t<T>().dev, sms_);
    tile_grid<LpPrimalOp<T, false, LP_NT>>(tiling_t<T>().dev, sms_);
    gd_ = tile_grid<LpDualOp<T, true, LP_NT>>(tiling_a<T>().dev, sms_);
    tile_grid<LpDualOp<T, false, LP_NT>>(tiling_a<T>().dev, sms_);
    gec_ = tile_grid<LpEvalColOp<T, LP_NT>>(ev_t_.dev, sms_);
    ger_ = tile_grid<LpEvalRowOp<T, LP_NT>>(ev_a_.dev, sms_);
    grc_ = tile_grid<RayColOp<LP_NT>>(ev_t_.dev, sms_);
    grr_ = tile_grid<RayRowOp<LP_NT>>(ev_a_.dev, sms_);
}

template <typename T>
void LpSolver::record(int freq) {
    LpVecs<T>* vp = nullptr;
    if constexpr (std::is_same<T, float>::value) vp = &v32_; else vp = &v64_;
    LpVecs<T>& v = *vp;
    const int mode = std::is_same<T, float>::value ? MODE_FP32 : MODE_FP64;
    const SideDev& tt = tiling_t<T>().dev;
    const SideDev& ta = tiling_a<T>().dev;
    auto step = [&](int k, bool major) {  // pdhg_step!, src/pdlp.jl:147-153
        if (major) {
            launch_tile(tt, LpPrimalOp<T, true, LP_NT>{v, st_, k, mode, err_}, gp_, stream_);
            launch_tile(ta, LpDualOp<T, true, LP_NT>{v, st_, k, mode, err_}, gd_, stream_);
        } else {
            launch_tile(tt, LpPrimalOp<T, false, LP_NT>{v, st_, k, mode, err_}, gp_, stream_);
            launch_tile(ta, LpDualOp<T, false, LP_NT>{v, st_, k, mode, err_}, gd_, stream_);
        }
    };
    auto evals = [&](int which) {
        launch_tile(ev_t_.dev, LpEvalColOp<T, LP_NT>{v, d_, st_, which, mode, err_}, gec_, stream_);
        launch_tile(ev_a_.dev, LpEvalRowOp<T, LP_NT>{v, d_, st_, which, mode, err_}, ger_, stream_);
    };
    // src/pdlp.jl:332-341: step 1 (major), steps 2..freq-1, step freq (major)
    step(1, true);
    evals(EVAL_AFTER_RESTART);
    launch_finalize(1, LpController{ev_t_.inst_tile0, d_.part_col, ev_a_.inst_tile0, d_.part_row,
                                    st_, flags_, 0, cupdlpx_ ? 1 : 0}, stream_);
    if (tiny_ && freq > 2) {
        // a small LP: steps 2 .. freq-1 in one launch (tiny_steps.cuh)
        tiny_steps_kernel<LpPrimalOp<T, false, kTinyThreads>, LpDualOp<T, false, kTinyThreads>>
            <<<1, kTinyThreads, 0, stream_>>>(LpPrimalOp<T, false, kTinyThreads>{v, st_, 0, mode, err_},
                                              LpDualOp<T, false, kTinyThreads>{v, st_, 0, mode, err_},
                                              M_.rp_t, M_.ci_t, M_.rp_a, M_.ci_a, M_.col_off,
                                              M_.row_off, 2, freq);
        PDFP_CK(cudaGetLastError());
    } else {
        for (int i = 2; i <= freq - 1; ++i) step(i, false);
    }
    step(freq, true);
    evals(EVAL_FULL);
    if (cupdlpx_) {
        zero_maxes_kernel<<<1, 32, 0, stream_>>>(d_.maxes);
        launch_rows(ev_t_.dev, RayRowsCol<T>{v, d_, st_}, stream_);
        launch_rows(ev_a_.dev, RayRowsRow<T>{v, d_, st_, ray_part_row_}, stream_);
        launch_tile(ev_t_.dev, RayColOp<LP_NT>{d_, st_, ray_part_col_, err_}, grc_, stream_);
        launch_tile(ev_a_.dev, RayRowOp<LP_NT>{d_, st_, err_}, grr_, stream_);
        launch_finalize(1, LpRayFin{ev_t_.inst_tile0, ray_part_col_, ev_a_.inst_tile0, ray_part_row_,
                                    st_, d_.maxes}, stream_);
    }
    launch_finalize(1, LpController{ev_t_.inst_tile0, d_.part_col, ev_a_.inst_tile0, d_.part_row,
                                    st_, flags_, 1, cupdlpx_ ? 1 : 0}, stream_);
    launch_elem(1, static_cast<int64_t>(n_) + m_, LpRestartCopy<T>{v, st_, n_, m_}, stream_);
}

// A small LP: up to kLpTinyWindowsPerLaunch windows in one launch (lp_tiny_solve_kernel).
template <typename T>
void LpSolver::launch_tiny_solve() {
    LpVecs<T>* vp = nullptr;
    if constexpr (std::is_same<T, float>::value) vp = &v32_; else vp = &v64_;
    const int32_t rowsum_len = 2 * std::max(std::max(n_, m_), 1);
    const size_t base = sizeof(double) * static_cast<size_t>(rowsum_len);
    // the staged form when the LP's copy fits next to the row sums (PDFP_TINY_STAGE=0: in place)
    const char* ts = std::getenv("PDFP_TINY_STAGE");
    const size_t staged = base + lp_tiny_stage_bytes<T>(n_, m_, M_.L.NNZ, d_.row_unscale != nullptr);
    const bool stage = !(ts && ts[0] == '0') && staged <= static_cast<size_t>(max_smem_) - 8 * 1024;
    const size_t smem = stage ? staged : base;
    auto kern = stage ? lp_tiny_solve_kernel<T, true> : lp_tiny_solve_kernel<T, false>;
    if (smem > 48 * 1024)
        PDFP_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    kern<<<1, kTinyThreads, smem, stream_>>>(*vp, d_, st_, flags_, M_.rp_t, M_.ci_t, M_.rp_a, M_.ci_a, n_,
                                             m_, err_, cupdlpx_ ? 1 : 0, kLpTinyWindowsPerLaunch, rowsum_len);
    PDFP_CK(cudaGetLastError());
}

template <typename T>
cudaGraphExec_t LpSolver::build_graph(int freq) {
    prepare_grids<T>();
    cudaGraph_t g = nullptr;
    cudaGraphExec_t exec = nullptr;
    PDFP_CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    record<T>(freq);
    cudaError_t ce = cudaStreamEndCapture(stream_, &g);
    if (ce != cudaSuccess) throw Error(E_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    PDFP_CK(cudaGraphInstantiate(&exec, g, 0));
    cudaGraphDestroy(g);
    return exec;
}

int32_t LpSolver::solve(double tolerance, double time_limit, int32_t sv_max_it, double sv_tol,
                        double* x_scaled, double* dual_slack, pdfp_result* r) {
    const auto wall0 = std::chrono::steady_clock::now();
    cudaEvent_t e0, e1;
    PDFP_CK(cudaEventCreate(&e0));
    PDFP_CK(cudaEventCreate(&e1));
    PDFP_CK(cudaEventRecord(e0, stream_));
    lp_begin_kernel<<<1, 1, 0, stream_>>>(st_);
    // initialize_step_size_and_primal_weight!, src/pdlp.jl:292-316
    std::vector<int> run(1, 1);
    double sv = NAN;
    if (n_ > 0 && m_ > 0 && M_.L.NNZ > 0)
        sv = power_iteration(M_, ar_, ev_a_, ev_t_, run, sv_max_it, sv_tol, stream_, sms_, err_, nullptr)[0];
    const double step = M_.L.NNZ == 0 ? 1.0 : ((std::isfinite(sv) && sv > 0) ? 0.998 / sv : 0.998);
    InstState s;
    PDFP_CK(cudaMemcpy(&s, st_, sizeof(s), cudaMemcpyDeviceToHost));
    s.step_size = step;
    s.max_sv = sv;
    s.primal_weight = 1.0;
    s.best_primal_weight = 1.0;
    s.tau = step;
    s.sigma = step;
    s.eps_opt = tolerance;
    s.eps_feas = tolerance;
    s.time_limit = time_limit;
    s.iter_limit = 5000000;  // src/pdlp.jl:388
    s.freq = 200;
    s.omega = 1.0;
    s.art = 0.36;
    s.suff = 0.2;
    s.nec = 0.5;
    s.kp = 0.99;
    s.ki = 0.01;
    s.kd = 0.0;
    s.ismooth = 0.3;
    s.status = ST_RUNNING;
    s.best_score = INFINITY;
    s.stall = 0;
    PDFP_CK(cudaMemcpy(st_, &s, sizeof(s), cudaMemcpyHostToDevice));
    double* part4 = ar_.alloc<double>(4 * static_cast<size_t>(std::max(ev_a_.dev.n_tiles, 1)));
    double* part8 = ar_.alloc<double>(8 * static_cast<size_t>(std::max(ev_t_.dev.n_tiles, 1)));
    launch_rows(ev_a_.dev, LpNormRowsA{d_, s.bound_scale, part4}, stream_);
    launch_rows(ev_t_.dev, LpNormRowsC{d_, part8}, stream_);
    launch_finalize(1, LpNormFin{ev_t_.inst_tile0, part8, ev_a_.inst_tile0, part4, st_, cupdlpx_ ? 1 : 0}, stream_);
    PDFP_CK(cudaGetLastError());

    // a small LP's window is a dozen launches: issue them directly, with no graph to
    // capture and instantiate per solve; a larger one replays a captured window
    bool f32_window = f32_;
    if (!tiny_) graph_ = f32_ ? build_graph<float>(200) : build_graph<double>(200);

    InstFlags fh[2] = {};  // a few bytes per poll: pageable memory, no page-locked allocation
    {
        for (;;) {
            if (tiny_) {
                if (f32_window) launch_tiny_solve<float>(); else launch_tiny_solve<double>();
            } else {
                PDFP_CK(cudaGraphLaunch(graph_, stream_));
            }
            PDFP_CK(cudaMemcpyAsync(fh, flags_, sizeof(InstFlags), cudaMemcpyDeviceToHost, stream_));
            PDFP_CK(cudaMemcpyAsync(&fh[1].status, err_, sizeof(int32_t), cudaMemcpyDeviceToHost, stream_));
            PDFP_CK(cudaStreamSynchronize(stream_));
            if (fh[1].status) throw Error(E_TIMEOUT, "a bounded device wait gave up (bulk copy did not complete)");
            if (fh[0].status != ST_RUNNING) break;
            if (fh[0].polish_request && !polished_) {  // FP64 polish: convert and switch graphs
                launch_elem(1, static_cast<int64_t>(n_) + m_, LpConvert<float, double>{v32_, v64_, n_, m_}, stream_);
                lp_set_mode_kernel<<<1, 1, 0, stream_>>>(st_, MODE_FP64);
                PDFP_CK(cudaGetLastError());
                if (graph_) cudaGraphExecDestroy(graph_);
                graph_ = nullptr;
                if (!tiny_) graph_ = build_graph<double>(200);
                f32_window = false;
                polished_ = true;
            }
            const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
            if (wall > time_limit + 120.0) throw Error(E_TIMEOUT, "root LP exceeded its time limit by 120 s");
        }
    }
    PDFP_CK(cudaEventRecord(e1, stream_));
    PDFP_CK(cudaMemcpy(&s, st_, sizeof(s), cudaMemcpyDeviceToHost));
    float ms = 0.f;
    PDFP_CK(cudaEventSynchronize(e1));
    PDFP_CK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // pdhg_primal and dual_slack back to the host (scaled units)
    if (n_ > 0) {
        std::vector<float> tmp;
        if (f32_ && !polished_) {
            tmp.resize(n_);
            PDFP_CK(cudaMemcpy(tmp.data(), v32_.px, sizeof(float) * n_, cudaMemcpyDeviceToHost));
            for (int32_t j = 0; j < n_; ++j) x_scaled[j] = tmp[j];
            PDFP_CK(cudaMemcpy(tmp.data(), v32_.ds, sizeof(float) * n_, cudaMemcpyDeviceToHost));
            for (int32_t j = 0; j < n_; ++j) dual_slack[j] = tmp[j];
        } else {
            PDFP_CK(cudaMemcpy(x_scaled, v64_.px, sizeof(double) * n_, cudaMemcpyDeviceToHost));
            PDFP_CK(cudaMemcpy(dual_slack, v64_.ds, sizeof(double) * n_, cudaMemcpyDeviceToHost));
        }
    }
    std::memset(r, 0, sizeof(*r));
    r->status = s.status;
    r->restarts = s.restarts;
    r->total_count = s.total;
    r->rel_primal = s.rel_p;
    r->rel_dual = s.rel_d;
    r->rel_gap = s.rel_gap;
    r->primal_weight = s.primal_weight;
    r->step_size = s.step_size;
    r->max_singular_value = s.max_sv;
    r->fixed_point_error = s.fpe;
    r->objective_value = s.objective_value;
    r->precision = (f32_ && !polished_) ? PDFP_MIXED : PDFP_FP64;
    r->polished = polished_ ? 1 : 0;
    r->device_ms = ms;
    return s.status;
}

void solve_lp_relaxation_device(const pdfp_csr& A, const double* c, const double* l,
                                const double* u, const double* b, const uint8_t* is_le,
                                double tolerance, double time_limit, bool cupdlpx, int precision,
                                double* x_out, double* dual_slack_out, pdfp_result* r) {
    // solve_lp_relaxation, src/pdlp.jl:381-393
    if (precision != PDFP_FP64 && precision != PDFP_MIXED) throw Error(E_INVALID, "bad precision");
    const int32_t m = A.m, n = A.n;
    std::vector<double> con_lb(m);
    for (int32_t i = 0; i < m; ++i) con_lb[i] = is_le[i] ? -INFINITY : b[i];
    LpSolver lp(A, c, l, u, con_lb.data(), b, 10, 1.0, cupdlpx, precision);
    std::vector<double> px(std::max(n, 1));
    lp.solve(tolerance, time_limit, 5000, 1e-4, px.data(), dual_slack_out, r);
    const std::vector<double>& D_c = lp.col_scale();
    const double bs = lp.bound_scale();
    for (int32_t j = 0; j < n; ++j) x_out[j] = (D_c[j] * px[j]) / bs;
}

}  // namespace pdfp
