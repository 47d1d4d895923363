// pdfp.cu -- the PDFP projector: PDFPState / pdfp_solve! on the device.
//
// Restarted Halpern PDHG with reflection on the l1-projection saddle point
// (src/pdfp.jl:1-288, src/pdfp_kernels.jl:1-86), for a batch of instances
// packed block-diagonally in one handle.  One evaluation window (the
// reference's `freq` steps followed by compute_fixed_point_error!,
// compute_residual!, should_restart and perform_restart!, src/pdfp.jl:258-285)
// is a fixed launch sequence captured once as a CUDA graph; every decision in
// it is taken on the device from the per-instance state, so the host only
// replays the graph and polls one status word per instance per window.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <map>
#include <memory>

#include "../../include/pdfp_b200.h"
#include "device.hpp"
#include "kernels.cuh"
#include "pdfp_ops.cuh"
#include "controller.cuh"
#include "power.cuh"
#include "tiny_steps.cuh"
#include "medium_steps.cuh"
#include "projector.hpp"

namespace pdfp {

constexpr int NT_EVAL = 256;
constexpr int64_t kMixedMinNnz = 1 << 18;  // smaller mixed handles compute in FP64
constexpr int64_t kTinyMaxDim = 4096;      // rows + columns of a member for the one-launch steps
constexpr int64_t kTinyMaxNnz = 1 << 16;   // nonzeros of a member for the one-launch steps
constexpr int32_t kHostNanScanMax = 1 << 16;  // vectors up to this length are checked on the host

// ---- per-instance state kernels ---------------------------------------------------

__global__ void solve_begin_kernel(InstState* st, const SolveParams* sp, int K) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < K && !sp[p].resume) st[p].t_start_ns = globaltimer_ns();
}

__global__ void set_max_sv_kernel(InstState* st, const double* sv, int K) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < K && !isnan(sv[p])) st[p].max_sv = sv[p];
}

// initialize_step_size_and_primal_weight! (src/pdfp.jl:220-241) minus the two
// denominators, plus this solve's parameters.
__global__ void solve_init_kernel(InstState* st, InstFlags* fl, const SolveParams* sp, int K) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= K) return;
    InstState& s = st[p];
    const SolveParams& q = sp[p];
    if (q.resume) {  // running from an earlier call: its parameters and counters stand
        fl[p] = InstFlags{s.status, s.mode, 0, 0};
        return;
    }
    s.eps_opt = q.eps_opt;
    s.eps_feas = q.eps_feas;
    s.time_limit = q.time_limit;
    s.iter_limit = q.iter_limit;
    s.freq = q.freq;
    s.omega = q.omega;
    s.art = q.art;
    s.suff = q.suff;
    s.nec = q.nec;
    s.kp = q.kp;
    s.ki = q.ki;
    s.kd = q.kd;
    s.ismooth = q.ismooth;
    s.step_size = s.nnz_zero ? 1.0 : 0.998 / sqrt(1.0 + s.max_sv * s.max_sv);
    s.primal_weight = q.primal_weight;
    s.best_primal_weight = q.primal_weight;
    s.err_sum = 0.0;
    s.last_err = 0.0;
    s.tau = s.step_size / s.primal_weight;
    s.sigma = s.step_size * s.primal_weight;
    s.mode = q.mode;
    s.best_score = INFINITY;
    s.stall = 0;
    s.stall_limit = q.stall_limit;
    s.fp32_floor = q.fp32_floor;
    s.fp64_iters = 0;
    s.do_restart = 0;
    s.restart_now = 0;
    s.restarts = 0;
    s.status = s.total < q.iter_limit ? ST_RUNNING : ST_ITERATION_LIMIT;
    fl[p] = InstFlags{s.status, s.mode, 0, 0};
}

// warm_start! (src/pdfp.jl:104-114): the counter part.
__global__ void warm_start_state_kernel(InstState* st, int p) {
    InstState& s = st[p];
    s.inner = 0;
    s.total = 0;
    s.fpe = INFINITY;
    s.last_trial_fpe = INFINITY;
    s.status = ST_RUNNING;
}

// ---- denominators of the relative residuals (src/pdfp.jl:236-239) -----------------

struct DenRows {
    static constexpr int NP = 2;
    const double *w, *xt;
    double* part;
    __device__ bool active(int) const { return true; }
    __device__ void row(int32_t j, int, double* acc) const {
        const double w_ = w[j];
        if (w_ >= 0.0) {
            acc[0] += w_ * w_;
            acc[1] += mul_rn(w_, fabs(xt[j]));
        }
    }
    __device__ void write_partials(int32_t t, const double* acc) const {
        part[t * 8] = acc[0];
        part[t * 8 + 1] = acc[1];
#pragma unroll
        for (int k = 2; k < 8; ++k) part[t * 8 + k] = 0.0;
    }
};

struct DenFin {
    static constexpr int NA = 8, NB = 0;
    const int32_t* ta0;
    const double* pa;
    const int32_t* tb0;
    const double* pb;
    InstState* st;
    __device__ bool active(int) const { return true; }
    __device__ void finalize(int p, const double* a) const {
        st[p].dual_den = 1.0 + sqrt(a[0]);
        st[p].gap_den = 1.0 + a[1];
    }
};

// ---- the controller: restart and termination rules on the device --------------

enum : int32_t { PHASE_AFTER_FIRST = 0, PHASE_EVAL = 1 };

struct Controller {
    static constexpr int NA = 8, NB = 4;
    const int32_t* ta0;
    const double* pa;
    const int32_t* tb0;
    const double* pb;
    InstState* st;
    InstFlags* fl;
    int32_t phase, polish;
    __device__ bool active(int p) const {
        return st[p].status == ST_RUNNING && (phase == PHASE_EVAL || st[p].do_restart);
    }
    __device__ void finalize(int p, const double* a) const {
        InstState& s = st[p];
        const double pw = s.primal_weight;
        // compute_fixed_point_error!, src/pdfp.jl:171-176
        const double movement = a[0] * pw + (a[1] + a[10]) / pw;
        const double interaction = 2.0 * s.step_size * a[2];
        const double fpe = sqrt(jl_max(movement + interaction, 0.0));
        s.fpe = fpe;
        if (phase == PHASE_AFTER_FIRST) {  // src/pdfp.jl:260-264
            s.initial_fpe = fpe;
            s.do_restart = 0;
            return;
        }
        // compute_residual!, src/pdfp.jl:200-218
        s.rel_p = sqrt(a[8]) / (1.0 + s.b_norm);
        s.rel_d = sqrt(a[3]) / s.dual_den;
        s.l1 = a[4];
        s.rel_gap = fabs(a[5] + a[9] - a[4]) / s.gap_den;
        s.inner += s.freq;
        s.total += s.freq;
        if (s.mode == MODE_FP64) s.fp64_iters += s.freq;
        s.restart_now = 0;
        int32_t request = 0;
        if (s.rel_p <= s.eps_feas && s.rel_d <= s.eps_opt && s.rel_gap <= s.eps_opt) {
            s.status = ST_OPTIMAL;
        } else if (static_cast<double>(globaltimer_ns() - s.t_start_ns) * 1e-9 > s.time_limit) {
            s.status = ST_TIME_LIMIT;
        } else {
            if (should_restart(s)) {  // perform_restart!, src/pdfp.jl:180-192
                update_primal_weight(s, sqrt(a[6]), sqrt(a[7] + a[11]));
                s.inner = 0;
                s.last_trial_fpe = INFINITY;
                s.restarts += 1;
                s.restart_now = 1;
                s.do_restart = 1;
            }
            s.tau = s.step_size / s.primal_weight;
            s.sigma = s.step_size * s.primal_weight;
            if (s.total >= s.iter_limit) s.status = ST_ITERATION_LIMIT;
            if (s.status == ST_RUNNING && s.mode == MODE_FP32 && polish && s.stall_limit > 0) {
                // End of the FP32 phase: the FP64 polish takes over from the FP32
                // iterate when the KKT score (largest residual / tolerance ratio) has
                // not improved by 10% over stall_limit evaluations, or when the
                // residuals have reached the FP32 floor while the tolerance asks for
                // more than FP32 iterates carry.
                const double score = fmax(s.rel_p / s.eps_feas, fmax(s.rel_d / s.eps_opt, s.rel_gap / s.eps_opt));
                const double ff = fmax(s.eps_feas, s.fp32_floor), fo = fmax(s.eps_opt, s.fp32_floor);
                const double score32 = fmax(s.rel_p / ff, fmax(s.rel_d / fo, s.rel_gap / fo));
                if (score < 0.9 * s.best_score) {
                    s.best_score = score;
                    s.stall = 0;
                } else {
                    s.stall += 1;
                }
                if (score > 1.0 && (s.stall >= s.stall_limit || score32 <= 1.0)) request = 1;
            }
        }
        fl[p] = InstFlags{s.status, s.mode, request, 0};
    }
};

// ---- vector kernels ------------------------------------------------------------------

template <typename T>
struct RestartCopy {  // perform_restart!: initial = current = pdhg (src/pdfp.jl:186-188)
    IterVecs<T> v;
    const InstState* st;
    const int32_t *col_off, *row_off;
    int32_t mode;
    __device__ bool active(int p) const { return st[p].restart_now && st[p].mode == mode; }
    __device__ int32_t begin(int) const { return 0; }
    __device__ int32_t end(int p) const {
        return (col_off[p + 1] - col_off[p]) + (row_off[p + 1] - row_off[p]);
    }
    __device__ void elem(int p, int32_t i) const {
        const int32_t n = col_off[p + 1] - col_off[p];
        if (i < n) {
            const int32_t j = col_off[p] + i;
            const T x = v.px[j], y = v.py[j];
            v.ix[j] = x; v.cx[j] = x;
            v.iy[j] = y; v.cy[j] = y;
        } else {
            const int32_t r = row_off[p] + (i - n);
            const T z = v.pz[r];
            v.iz[r] = z; v.cz[r] = z;
        }
    }
};

template <typename T>
struct WarmStartCopy {  // initial = current (src/pdfp.jl:105-107)
    IterVecs<T> v;
    const int32_t *col_off, *row_off;
    int32_t only;
    __device__ bool active(int p) const { return p == only; }
    __device__ int32_t begin(int) const { return 0; }
    __device__ int32_t end(int p) const {
        return (col_off[p + 1] - col_off[p]) + (row_off[p + 1] - row_off[p]);
    }
    __device__ void elem(int p, int32_t i) const {
        const int32_t n = col_off[p + 1] - col_off[p];
        if (i < n) {
            const int32_t j = col_off[p] + i;
            v.ix[j] = v.cx[j];
            v.iy[j] = v.cy[j];
        } else {
            const int32_t r = row_off[p] + (i - n);
            v.iz[r] = v.cz[r];
        }
    }
};

// ---- a small member's whole solve in one launch -------------------------------------
//
// For members of a few thousand rows and columns every launch and every host poll
// costs more than the work of a window.  tiny_solve_kernel runs whole evaluation
// windows of pdfp_solve! (src/pdfp.jl:258-285) for member blockIdx.x in one block:
// step 1, the evaluation after a restart, steps 2 .. freq-1, step freq, the full
// evaluation, the controller (termination, should_restart, PID) and the restart copy,
// window after window, until the member stops, asks for the FP64 polish, or
// max_windows windows have run.  The passes are tiny_pass (the one-block steps) and
// tiny_eval_pass; the controller is the window's own (Controller::finalize), on the
// block-summed terms.
//
// STAGED: the member's iterates, data and both sides of its matrix are copied into
// the block's shared memory for the launch (and the iterates back at its end), so that
// no pass waits on a global-memory round trip for what the previous pass wrote; the
// arithmetic is the same, so the results are bit-identical to the unstaged kernel.
constexpr int kTinyWindowsPerLaunch = 64;

// Shared-memory bytes of a member's staged copy (tiny_solve_kernel<T, true>).
template <typename T>
__host__ __device__ inline size_t tiny_stage_bytes(int64_t nc, int64_t nr, int64_t nzt, int64_t nza,
                                                   bool unscale) {
    auto r16 = [](int64_t b) { return static_cast<size_t>((b + 15) & ~int64_t(15)); };
    size_t b = 13 * r16(sizeof(T) * nc) + 5 * r16(sizeof(T) * nr);  // iterates and data
    b += r16(4 * (nc + 1)) + r16(4 * (nr + 1)) + r16(4 * nzt) + r16(4 * nza);  // pointers, indices
    b += r16(sizeof(T) * nzt) + r16(sizeof(T) * nza);                       // values
    if (sizeof(T) == 4) b += 2 * r16(8 * nc) + r16(8 * nr) + r16(8 * nzt) + r16(8 * nza);  // FP64 copies
    if (unscale) b += r16(8 * nr);
    return b;
}

template <typename T, bool STAGED>
__global__ void __launch_bounds__(kTinyThreads)
    tiny_solve_kernel(IterVecs<T> gv, EvalData ged, InstState* st, InstFlags* fl,
                      const int32_t* __restrict__ g_rp_t, const int32_t* __restrict__ g_ci_t,
                      const int32_t* __restrict__ g_rp_a, const int32_t* __restrict__ g_ci_a,
                      const int32_t* __restrict__ col_off, const int32_t* __restrict__ row_off,
                      const int32_t* __restrict__ n_eq, int32_t* err, int32_t max_windows,
                      int32_t polish, int32_t rowsum_len, int32_t* any_stop) {
    constexpr int NT = kTinyThreads;
    constexpr int32_t mode = std::is_same<T, float>::value ? MODE_FP32 : MODE_FP64;
    extern __shared__ __align__(16) double tiny_rowsum[];  // rowsum_len doubles, then the staged copy
    __shared__ double red[8 * (NT / 32)];
    __shared__ int32_t go;
    const int p = blockIdx.x;
    const int32_t c0 = col_off[p], c1 = col_off[p + 1], r0 = row_off[p], r1 = row_off[p + 1];
    IterVecs<T> v = gv;
    EvalData ed = ged;
    const int32_t *rp_t = g_rp_t, *ci_t = g_ci_t, *rp_a = g_rp_a, *ci_a = g_ci_a;
    const int32_t nc = c1 - c0, nr = r1 - r0;
    T* const stv[9] = {gv.cx, gv.ix, gv.px, gv.rx, gv.cy, gv.iy, gv.py, gv.ry, gv.ds};  // n-side iterates
    T* const stz[4] = {gv.cz, gv.iz, gv.pz, gv.rz};                                      // m-side iterates
    T* loc_v[9] = {};
    T* loc_z[4] = {};
    if constexpr (STAGED) {
        // carve the copy out of the shared memory after the row sums; every region
        // starts 16-byte aligned; pointers are rebased so that the packed indices the
        // Ops use land in the copy
        unsigned char* cur = reinterpret_cast<unsigned char*>(tiny_rowsum + rowsum_len);
        auto carve = [&](size_t bytes) {
            unsigned char* q = cur;
            cur += (bytes + 15) & ~size_t(15);
            return q;
        };
        const int32_t k0t = g_rp_t[c0], k1t = g_rp_t[c1], k0a = g_rp_a[r0], k1a = g_rp_a[r1];
        auto stage_n = [&](const T* src) {
            T* d = reinterpret_cast<T*>(carve(sizeof(T) * nc));
            for (int32_t i = threadIdx.x; i < nc; i += NT) d[i] = src[c0 + i];
            return d;
        };
        auto stage_m = [&](const T* src) {
            T* d = reinterpret_cast<T*>(carve(sizeof(T) * nr));
            for (int32_t i = threadIdx.x; i < nr; i += NT) d[i] = src[r0 + i];
            return d;
        };
        for (int k = 0; k < 9; ++k) loc_v[k] = stage_n(stv[k]);
        for (int k = 0; k < 4; ++k) loc_z[k] = stage_m(stz[k]);
        T* lb = stage_n(gv.lb);
        T* ub = stage_n(gv.ub);
        T* xt = stage_n(gv.xt);
        T* w = stage_n(gv.w);
        T* b = stage_m(gv.b);
        int32_t* rpt = reinterpret_cast<int32_t*>(carve(4 * (nc + 1)));
        int32_t* rpa = reinterpret_cast<int32_t*>(carve(4 * (nr + 1)));
        int32_t* cit = reinterpret_cast<int32_t*>(carve(4 * (k1t - k0t)));
        int32_t* cia = reinterpret_cast<int32_t*>(carve(4 * (k1a - k0a)));
        T* vt = reinterpret_cast<T*>(carve(sizeof(T) * (k1t - k0t)));
        T* va = reinterpret_cast<T*>(carve(sizeof(T) * (k1a - k0a)));
        for (int32_t i = threadIdx.x; i <= nc; i += NT) rpt[i] = g_rp_t[c0 + i];
        for (int32_t i = threadIdx.x; i <= nr; i += NT) rpa[i] = g_rp_a[r0 + i];
        for (int32_t k = threadIdx.x; k < k1t - k0t; k += NT) {
            cit[k] = g_ci_t[k0t + k];
            vt[k] = gv.val_t[k0t + k];
        }
        for (int32_t k = threadIdx.x; k < k1a - k0a; k += NT) {
            cia[k] = g_ci_a[k0a + k];
            va[k] = gv.val_a[k0a + k];
        }
        T** vp[9] = {&v.cx, &v.ix, &v.px, &v.rx, &v.cy, &v.iy, &v.py, &v.ry, &v.ds};
        for (int k = 0; k < 9; ++k) *vp[k] = loc_v[k] - c0;
        T** zp[4] = {&v.cz, &v.iz, &v.pz, &v.rz};
        for (int k = 0; k < 4; ++k) *zp[k] = loc_z[k] - r0;
        v.lb = lb - c0;
        v.ub = ub - c0;
        v.xt = xt - c0;
        v.w = w - c0;
        v.b = b - r0;
        v.val_t = vt - k0t;
        v.val_a = va - k0a;
        rp_t = rpt - c0;
        rp_a = rpa - r0;
        ci_t = cit - k0t;
        ci_a = cia - k0a;
        if constexpr (std::is_same<T, double>::value) {  // the FP64 data are these very arrays
            ed.xt = v.xt;
            ed.w = v.w;
            ed.b = v.b;
            ed.val_t = v.val_t;
            ed.val_a = v.val_a;
        } else {
            auto stage64 = [&](const double* src, int64_t off, int64_t len) {
                double* d = reinterpret_cast<double*>(carve(8 * len));
                for (int64_t i = threadIdx.x; i < len; i += NT) d[i] = src[off + i];
                return d - off;
            };
            ed.xt = stage64(ged.xt, c0, nc);
            ed.w = stage64(ged.w, c0, nc);
            ed.b = stage64(ged.b, r0, nr);
            ed.val_t = stage64(ged.val_t, k0t, k1t - k0t);
            ed.val_a = stage64(ged.val_a, k0a, k1a - k0a);
        }
        if (ged.row_unscale) {
            double* d = reinterpret_cast<double*>(carve(8 * nr));
            for (int32_t i = threadIdx.x; i < nr; i += NT) d[i] = ged.row_unscale[r0 + i];
            ed.row_unscale = d - r0;
        }
        __syncthreads();
    }
    // the evaluation terms of one phase, block-summed, then the controller (thread 0)
    auto evaluate = [&](int32_t which, int32_t phase) {
        double ac[8], ar[4];
#pragma unroll
        for (int k = 0; k < 8; ++k) ac[k] = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) ar[k] = 0.0;
        tiny_eval_pass(EvalColOp<T, NT>{v, ed, st, which, mode, err}, rp_t, ci_t, c0, c1, p, tiny_rowsum, ac);
        block_sum<NT, 8>(ac, red, threadIdx.x);
        tiny_eval_pass(EvalRowOp<T, NT>{v, ed, st, row_off, n_eq, which, mode, err}, rp_a, ci_a, r0, r1, p,
                       tiny_rowsum, ar);
        block_sum<NT, 4>(ar, red, threadIdx.x);
        if (threadIdx.x == 0) {
            const double a[12] = {ac[0], ac[1], ac[2], ac[3], ac[4], ac[5], ac[6], ac[7],
                                  ar[0], ar[1], ar[2], ar[3]};
            Controller{nullptr, nullptr, nullptr, nullptr, st, fl, phase, polish}.finalize(p, a);
        }
        __syncthreads();
    };
    for (int32_t w = 0; w < max_windows; ++w) {
        // any_stop (a solve that returns once any member stops): after another
        // member's block has stopped, leave at this window boundary, still running
        if (threadIdx.x == 0)
            go = st[p].status == ST_RUNNING && st[p].mode == mode &&
                 !(any_stop && *reinterpret_cast<volatile int32_t*>(any_stop));
        __syncthreads();
        if (!go) break;
        const int32_t freq = st[p].freq;
        for (int32_t i = 1; i <= freq; ++i) {
            if (i == 1 || i == freq) {  // major steps: pdhg_* and reflected_* are read after them
                tiny_pass(PrimalOp<T, true, NT>{v, st, i, mode, err, 0}, rp_t, ci_t, c0, c1, p);
                __syncthreads();
                tiny_pass(DualOp<T, true, NT>{v, st, row_off, n_eq, i, mode, err, 0}, rp_a, ci_a, r0, r1, p);
            } else {
                tiny_pass(PrimalOp<T, false, NT>{v, st, i, mode, err, 0}, rp_t, ci_t, c0, c1, p);
                __syncthreads();
                tiny_pass(DualOp<T, false, NT>{v, st, row_off, n_eq, i, mode, err, 0}, rp_a, ci_a, r0, r1, p);
            }
            __syncthreads();
            if (i == 1 && st[p].do_restart) evaluate(EVAL_AFTER_RESTART, PHASE_AFTER_FIRST);
        }
        evaluate(EVAL_FULL, PHASE_EVAL);
        const RestartCopy<T> rc{v, st, col_off, row_off, mode};
        if (rc.active(p))
            for (int32_t i = threadIdx.x; i < (c1 - c0) + (r1 - r0); i += NT) rc.elem(p, i);
        if (threadIdx.x == 0) {
            go = st[p].status == ST_RUNNING && !fl[p].polish_request;
            if (any_stop && st[p].status != ST_RUNNING) atomicExch(any_stop, 1);
        }
        __syncthreads();
        if (!go) break;
    }
    if constexpr (STAGED) {  // the iterates back to global memory
        __syncthreads();
        for (int k = 0; k < 9; ++k)
            for (int32_t i = threadIdx.x; i < nc; i += NT) stv[k][c0 + i] = loc_v[k][i];
        for (int k = 0; k < 4; ++k)
            for (int32_t i = threadIdx.x; i < nr; i += NT) stz[k][r0 + i] = loc_z[k][i];
    }
}

// dst[packed j] = src[caller index of j] for instance `only` (columns or rows)
template <typename T>
struct PermuteIn {
    T* dst;
    T* dst2;  // optional second destination
    const double* src;
    const int32_t *off, *orig;
    int32_t only;
    __device__ bool active(int p) const { return p == only; }
    __device__ int32_t begin(int p) const { return off[p]; }
    __device__ int32_t end(int p) const { return off[p + 1]; }
    __device__ void elem(int, int32_t j) const {
        const T x = static_cast<T>(src[orig[j]]);
        dst[j] = x;
        if (dst2) dst2[j] = x;
    }
};

template <typename T>
struct PermuteOut {
    double* dst;
    const T* src;
    const int32_t *off, *orig;
    int32_t only;
    __device__ bool active(int p) const { return p == only; }
    __device__ int32_t begin(int p) const { return off[p]; }
    __device__ int32_t end(int p) const { return off[p + 1]; }
    __device__ void elem(int, int32_t j) const { dst[orig[j]] = static_cast<double>(src[j]); }
};

// Unscaled caller vector -> scaled packed vector: dst[j] = src[caller index of j] / D_c[j],
// the pump's x_tilde ./ D_c (src/pump.jl:331; x ./ D_c at 305-306) done on the
// device.  Both operands are FP64 and the quotient is correctly rounded, so the
// result equals the host's division bit for bit.
template <typename T>
struct ScaleIn {
    T* dst;
    T* dst2;  // optional second destination
    const double* src;
    const double* dc;  // D_c in packed order
    const int32_t *off, *orig;
    int32_t only;
    __device__ bool active(int p) const { return p == only; }
    __device__ int32_t begin(int p) const { return off[p]; }
    __device__ int32_t end(int p) const { return off[p + 1]; }
    __device__ void elem(int, int32_t j) const {
        const T x = static_cast<T>(__ddiv_rn(src[orig[j]], dc[j]));
        dst[j] = x;
        if (dst2) dst2[j] = x;
    }
};

// Scaled packed vector -> unscaled caller vector: dst[caller index of j] = D_c[j] * src[j],
// the pump's D_c .* s.pdhg_x (src/pump.jl:338) done on the device (one correctly
// rounded FP64 product, as on the host).
template <typename T>
struct ScaleOut {
    double* dst;
    const T* src;
    const double* dc;
    const int32_t *off, *orig;
    int32_t only;
    __device__ bool active(int p) const { return p == only; }
    __device__ int32_t begin(int p) const { return off[p]; }
    __device__ int32_t end(int p) const { return off[p + 1]; }
    __device__ void elem(int, int32_t j) const {
        dst[orig[j]] = __dmul_rn(dc[j], static_cast<double>(src[j]));
    }
};

// *nan_seen = 1 when the staged caller vector of instance `only` holds a NaN
struct NanScan {
    const double* src;
    const int32_t* off;
    int32_t only;
    int32_t* nan_seen;
    __device__ bool active(int p) const { return p == only; }
    __device__ int32_t begin(int) const { return 0; }
    __device__ int32_t end(int p) const { return off[p + 1] - off[p]; }
    __device__ void elem(int, int32_t i) const {
        if (isnan(src[i])) *nan_seen = 1;
    }
};

template <typename S, typename D>
struct ConvertVecs {  // the live iterate set of instance `only`: S -> D
    IterVecs<S> s;
    IterVecs<D> d;
    const int32_t *col_off, *row_off;
    int32_t only;
    __device__ bool active(int p) const { return p == only; }
    __device__ int32_t begin(int) const { return 0; }
    __device__ int32_t end(int p) const {
        return (col_off[p + 1] - col_off[p]) + (row_off[p + 1] - row_off[p]);
    }
    __device__ void elem(int p, int32_t i) const {
        const int32_t n = col_off[p + 1] - col_off[p];
        if (i < n) {
            const int32_t j = col_off[p] + i;
            d.cx[j] = static_cast<D>(s.cx[j]); d.ix[j] = static_cast<D>(s.ix[j]);
            d.px[j] = static_cast<D>(s.px[j]); d.rx[j] = static_cast<D>(s.rx[j]);
            d.cy[j] = static_cast<D>(s.cy[j]); d.iy[j] = static_cast<D>(s.iy[j]);
            d.py[j] = static_cast<D>(s.py[j]); d.ry[j] = static_cast<D>(s.ry[j]);
            d.ds[j] = static_cast<D>(s.ds[j]);
        } else {
            const int32_t r = row_off[p] + (i - n);
            d.cz[r] = static_cast<D>(s.cz[r]); d.iz[r] = static_cast<D>(s.iz[r]);
            d.pz[r] = static_cast<D>(s.pz[r]); d.rz[r] = static_cast<D>(s.rz[r]);
        }
    }
};

__global__ void set_mode_kernel(InstState* st, int p, int32_t mode) { st[p].mode = mode; }

// Save every instance's status and mark it running (timing runs), or restore it.
__global__ void swap_status_kernel(InstState* st, int32_t* saved, int K, int restore) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= K) return;
    if (restore) {
        st[p].status = saved[p];
    } else {
        saved[p] = st[p].status;
        st[p].status = ST_RUNNING;
    }
}

// ---- the projector ----------------------------------------------------------------------

template <typename T>
static IterVecs<T> alloc_vecs(DeviceArena& ar, int64_t N, int64_t M) {
    IterVecs<T> v{};
    T** nv[] = {&v.cx, &v.ix, &v.px, &v.rx, &v.cy, &v.iy, &v.py, &v.ry, &v.ds, &v.lb, &v.ub, &v.xt, &v.w};
    for (T** q : nv) *q = ar.alloc<T>(N);
    T** mv[] = {&v.cz, &v.iz, &v.pz, &v.rz, &v.b};
    for (T** q : mv) *q = ar.alloc<T>(M);
    return v;
}

Projector::Projector(const std::vector<ProblemData>& probs, int precision) : precision_(precision) {
    int dev = 0;
    PDFP_CK(cudaGetDevice(&dev));
    PDFP_CK(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev));
    PDFP_CK(cudaDeviceGetAttribute(&max_smem_sm_, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    PDFP_CK(cudaDeviceGetAttribute(&max_smem_block_, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    PDFP_CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    std::vector<ProblemIn> in;
    for (const ProblemData& p : probs)
        in.push_back(ProblemIn{p.m, p.n, p.rp, p.ci, p.v, p.is_eq});
    std::string msg = build_layout(in, true, M_.L);
    if (!msg.empty()) throw Error(E_INVALID, msg);
    const HostLayout& L = M_.L;
    K_ = L.K;
    // FP32 iterates pay only where the step kernels move enough bytes to be
    // memory-bound; below kMixedMinNnz nonzeros (PDFP_MIXED_MIN_NNZ overrides)
    // every launch is latency-bound and a mixed handle computes in FP64.
    if (precision_ == PDFP_MIXED) {
        const char* mm = std::getenv("PDFP_MIXED_MIN_NNZ");
        const int64_t min_nnz = mm ? std::atoll(mm) : kMixedMinNnz;
        if (L.NNZ < min_nnz) precision_ = PDFP_FP64;
    }
    M_.upload(ar_, precision_ == PDFP_MIXED);
    // Small members (every one at most kTinyMaxDim rows + columns and
    // kTinyMaxNnz nonzeros; PDFP_TINY=0 switches this off): the minor steps of a
    // window run in one launch, one block per member.
    {
        const char* te = std::getenv("PDFP_TINY");
        tiny_ = !(te && te[0] == '0') && K_ <= 65535;
        for (int p = 0; p < K_ && tiny_; ++p) {
            const int64_t dim = (L.row_off[p + 1] - L.row_off[p]) + (L.col_off[p + 1] - L.col_off[p]);
            const int64_t nz = L.A.rp[L.row_off[p + 1]] - L.A.rp[L.row_off[p]];
            if (dim > kTinyMaxDim || nz > kTinyMaxNnz) tiny_ = false;
        }
    }

    // PDFP_MEDIUM=1: the minor steps of a window run in one cooperative launch, one
    // block per SM over nonzero-balanced row ranges.  Off by default: on a 500k-
    // nonzero handle it measured within run-to-run noise of the per-step launches.
    {
        const char* me = std::getenv("PDFP_MEDIUM");
        medium_ = me && me[0] == '1';
        if (medium_ && tiny_) medium_ = false;
        if (medium_) {
            int coop = 0, dev = 0;
            PDFP_CK(cudaGetDevice(&dev));
            PDFP_CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
            if (!coop) medium_ = false;
        }
        if (medium_) {
            const int G = num_sms_;
            // each block's share: nonzeros + 4 per row (the epilogue), contiguous rows
            auto split = [&](const std::vector<int32_t>& rp, int64_t rows) {
                std::vector<int32_t> part(G + 1, 0);
                const double total = static_cast<double>(rp[rows]) + 4.0 * static_cast<double>(rows);
                int64_t r = 0;
                for (int g = 1; g < G; ++g) {
                    const double want = total * g / G;
                    while (r < rows && static_cast<double>(rp[r + 1]) + 4.0 * static_cast<double>(r + 1) <= want) ++r;
                    part[g] = static_cast<int32_t>(r);
                }
                part[G] = static_cast<int32_t>(rows);
                return part;
            };
            part_t_ = ar_.upload(split(L.At.rp, L.N));
            part_a_ = ar_.upload(split(L.A.rp, L.M));
            gbar_ = ar_.alloc<unsigned>(4);
        }
    }

    // tilings of the evaluation passes (the step kernels' tilings are tuned below)
    StageGeom gev{8, 8, 8, 0, 2, 32 * 1024, 2048};
    ev_t_ = M_.make_tiling(ar_, true, gev);
    ev_a_ = M_.make_tiling(ar_, false, gev);

    // vectors
    v64_ = alloc_vecs<double>(ar_, L.N, L.M);
    v64_.val_t = M_.v64_t;
    v64_.val_a = M_.v64_a;
    if (precision_ == PDFP_MIXED) {
        v32_ = alloc_vecs<float>(ar_, L.N, L.M);
        v32_.val_t = M_.v32_t;
        v32_.val_a = M_.v32_a;
    }
    row_unscale_ = nullptr;
    part_col_ = ar_.alloc<double>(8 * static_cast<size_t>(std::max(ev_t_.dev.n_tiles, 1)));
    part_row_ = ar_.alloc<double>(4 * static_cast<size_t>(std::max(ev_a_.dev.n_tiles, 1)));
    st_ = ar_.alloc<InstState>(K_);
    flags_ = ar_.alloc<InstFlags>(K_ + 1);
    err_ = ar_.alloc<int32_t>(4);
    nan_seen_ = ar_.alloc<int32_t>(1);
    has_col_scale_.assign(K_, false);
    sp_ = ar_.alloc<SolveParams>(K_);
    stage_ = ar_.alloc<double>(std::max<int64_t>(std::max(M_.max_m, M_.max_n), 1));
    flags_h_ = static_cast<InstFlags*>(pinned_take(sizeof(InstFlags) * (K_ + 1)));
    st_h_ = static_cast<InstState*>(pinned_take(sizeof(InstState) * K_));
    host_total_.assign(K_, 0);
    last_running_.assign(K_, 0);
    any_stop_ = ar_.alloc<int32_t>(4);
    nan_seen_h_ = static_cast<int32_t*>(pinned_take(sizeof(int32_t)));
    vec_mode_.assign(K_, precision_ == PDFP_MIXED ? MODE_FP32 : MODE_FP64);

    // per-instance data vectors (permuted into packed order)
    bool any_unscale = false;
    for (const ProblemData& p : probs) any_unscale = any_unscale || p.row_unscale;
    if (any_unscale) row_unscale_ = ar_.alloc<double>(L.M);
    std::vector<InstState> hs(K_);
    std::vector<double> hb(L.M), hlb(L.N), hub(L.N), hw(L.N), hru(any_unscale ? L.M : 0);
    for (int p = 0; p < K_; ++p) {
        const ProblemData& P = probs[p];
        const int32_t c0 = L.col_off[p], r0 = L.row_off[p];
        for (int32_t j = 0; j < P.n; ++j) {
            const int32_t o = L.col_orig[c0 + j];
            if (std::isnan(P.lb[o]) || std::isnan(P.ub[o]) || std::isnan(P.w[o]))
                throw Error(E_INVALID, "NaN in var_lb, var_ub or w");
            hlb[c0 + j] = P.lb[o];
            hub[c0 + j] = P.ub[o];
            hw[c0 + j] = P.is_int[o] ? std::fabs(P.w[o]) : -1.0;
        }
        double bsq = 0.0, bosq = 0.0;
        for (int32_t i = 0; i < P.m; ++i) {
            const int32_t o = L.row_orig[r0 + i];
            if (!std::isfinite(P.b[o])) throw Error(E_INVALID, "non-finite right-hand side");
            hb[r0 + i] = P.b[o];
            bsq += P.b[o] * P.b[o];
            if (P.row_unscale) {
                hru[r0 + i] = P.row_unscale[o];
                const double t = P.b[o] * P.row_unscale[o];  // b ./ D_r  (src/pdfp.jl:87)
                bosq += t * t;
            } else if (any_unscale) {
                hru[r0 + i] = 1.0;
            }
        }
        InstState& s = hs[p];
        std::memset(&s, 0, sizeof(s));
        s.max_sv = NAN;
        s.primal_weight = 1.0;
        s.best_primal_weight = 1.0;
        s.best_gap = INFINITY;
        s.fpe = INFINITY;
        s.initial_fpe = INFINITY;
        s.last_trial_fpe = INFINITY;
        s.rel_p = s.rel_d = s.rel_gap = INFINITY;
        s.dual_den = 1.0;
        s.gap_den = 1.0;
        s.b_norm = P.row_unscale ? std::sqrt(bosq) : std::sqrt(bsq);
        s.nnz_zero = (P.m == 0 || P.rp[P.m] == 0) ? 1 : 0;
        s.mode = vec_mode_[p];
        s.status = ST_RUNNING;
        has_unscale_.push_back(P.row_unscale != nullptr);
    }
    auto up = [&](double* d, const std::vector<double>& h) {
        if (!h.empty()) PDFP_CK(cudaMemcpy(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    };
    up(v64_.b, hb);
    up(v64_.lb, hlb);
    up(v64_.ub, hub);
    up(v64_.w, hw);
    if (any_unscale) up(row_unscale_, hru);
    if (precision_ == PDFP_MIXED) {
        auto cast = [&](float* d, const std::vector<double>& h) {
            std::vector<float> f(h.size());
            for (size_t i = 0; i < h.size(); ++i) f[i] = static_cast<float>(h[i]);
            if (!f.empty()) PDFP_CK(cudaMemcpy(d, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice));
        };
        cast(v32_.b, hb);
        cast(v32_.lb, hlb);
        cast(v32_.ub, hub);
        cast(v32_.w, hw);
    }
    PDFP_CK(cudaMemcpy(st_, hs.data(), sizeof(InstState) * K_, cudaMemcpyHostToDevice));

    ed_.xt = v64_.xt;
    ed_.w = v64_.w;
    ed_.b = v64_.b;
    ed_.row_unscale = row_unscale_;
    ed_.val_t = M_.v64_t;
    ed_.val_a = M_.v64_a;
    ed_.part_col = part_col_;
    ed_.part_row = part_row_;
    for (auto& e : sev_) PDFP_CK(cudaEventCreate(&e));
    PDFP_CK(cudaDeviceSynchronize());
    // The autotuner pays for itself only where a step kernel takes longer than its
    // launch: below 256K nonzeros every candidate times the same few microseconds.
    // PDFP_AUTOTUNE=0 / =1 switches it off / on regardless of size.
    // PDFP_STEP_ENGINE=tile / =flat / =flat1 / =vec fixes the step engine (flat1: one
    // quad per thread and tile; vec: the FP32 steps only, the FP64 steps keep the
    // tile engine) and skips the tuner.
    // The step kernels stream the matrix under an L2 evict-first policy, so the
    // gathered vector and the iterates stay in L2 (zipf-lp: 1% more iterations/s);
    // PDFP_STREAM_EVICT_FIRST=0 / =1 switches it off / on.
    if (const char* ef = std::getenv("PDFP_STREAM_EVICT_FIRST")) evict_first_ = ef[0] == '1';
    // PDFP_STEP_OVERLAP=1 lets consecutive step launches of a window overlap one's
    // drain with the next one's staging (programmatic dependent launch).  Off by
    // default: on zipf-lp it cost ~14 us per iteration (4,785 -> 4,485 it/s) while
    // the kernels themselves took as long as before.
    if (const char* ov = std::getenv("PDFP_STEP_OVERLAP")) overlap_ = ov[0] == '1';
    const char* at = std::getenv("PDFP_AUTOTUNE");
    const char* se = std::getenv("PDFP_STEP_ENGINE");
    const int forced = !se ? -1
                       : std::strcmp(se, "tile") == 0 ? 0
                       : std::strcmp(se, "flat") == 0 || std::strcmp(se, "flat1") == 0 ? 1
                       : std::strcmp(se, "vec") == 0 ? 2 : -1;
    if (forced >= 0) {
        const int qpt = std::strcmp(se, "flat1") == 0 ? 1 : 2;
        for (StepSide* q : {&p32_, &d32_, &p64_, &d64_}) {
            if (forced == 2 && (q == &p64_ || q == &d64_)) continue;
            q->engine = forced;
            q->qpt = qpt;
        }
    }
    // The A side's long rows by column segment (seg_spmv.cuh), FP32 steps on the tile
    // engine: PDFP_SEG="n,l" regroups the rows of at least l nonzeros into n column
    // segments; PDFP_SEG=tune lets the autotuner try a few such forms against the
    // plain tile engine; unset or 0, the long rows stay on the step engine (on the
    // zipf-lp matrices measured so far the form was slower, and building its
    // candidates costs about a second per large handle).
    // Optional after them: the partials' stage bytes, threads per role and stages.
    if (const char* sg = std::getenv("PDFP_SEG")) {
        int n = 0, l = 0, sb = d32_.seg_stage, nt = d32_.seg_nt, ns = d32_.seg_stages, bps = 1;
        const int got = std::sscanf(sg, "%d,%d,%d,%d,%d,%d", &n, &l, &sb, &nt, &ns, &bps);
        if (std::strcmp(sg, "tune") == 0) {
            seg_mode_ = -1;
        } else if (got == 1 && n == 0) {
            seg_mode_ = 0;
        } else if ((got == 2 || got == 5 || got == 6) && n > 0 && n <= 65536 && l > 0 &&
                   sb >= 8192 && sb <= 49152 && sb % 128 == 0 && (nt == 128 || nt == 256) &&
                   ns >= 2 && ns <= 4 && bps >= 1 && bps <= 8) {
            seg_mode_ = n;
            seg_long_ = l;
            seg_cfg_[0] = sb;
            seg_cfg_[1] = nt;
            seg_cfg_[2] = ns;
            seg_cfg_[3] = bps;
        } else {
            throw Error(E_INVALID, "PDFP_SEG must read 0, tune or segments,long_row_threshold"
                                   "[,stage_bytes,threads,stages[,blocks_per_segment]]");
        }
    }
    if (seg_mode_ > 0 && precision_ == PDFP_MIXED) {
        d32_.seg_nseg = seg_mode_;
        d32_.seg_long = seg_long_;
        d32_.seg_stage = seg_cfg_[0];
        d32_.seg_nt = seg_cfg_[1];
        d32_.seg_stages = seg_cfg_[2];
        d32_.seg_bps = seg_cfg_[3];
    }
    // PDFP_TUNING="s,t,l,s,t,l" pins both sides' step kernels of this precision
    // (A' then A: stage bytes, threads per role -- 0: flat engine, whose stage
    // bytes tell its variant; 32: vec engine, whose "stage bytes" are its nonzeros
    // per lane, FP32 steps only -- and the L2-only gather flag), as pdfp_get_tuning
    // reports them; the tuner does not run.
    bool pinned = false;
    if (const char* pt = std::getenv("PDFP_TUNING")) {
        int v[12] = {0, 0, 0, 0, 0, 0, 4, 4, 0, 0, 0, 0};
        const int got = std::sscanf(pt, "%d,%d,%d,%d,%d,%d,%d,%d,%d,%d,%d,%d", &v[0], &v[1], &v[2],
                                    &v[3], &v[4], &v[5], &v[6], &v[7], &v[8], &v[9], &v[10], &v[11]);
        if (got != 6 && got != 8 && got != 10 && got != 12)
            throw Error(E_INVALID, "PDFP_TUNING must read stage,threads,l2,stage,threads,l2"
                                   "[,stages,stages[,blocks,blocks[,reducers,reducers]]]");
        if (v[6] < 2 || v[6] > 4 || v[7] < 2 || v[7] > 4)
            throw Error(E_INVALID, "PDFP_TUNING: stages must be 2, 3 or 4");
        if (v[8] < 0 || v[8] > 8 || v[9] < 0 || v[9] > 8)
            throw Error(E_INVALID, "PDFP_TUNING: blocks per SM must be 0 (as many as fit) to 8");
        StepSide* sides[2][2] = {{&p32_, &d32_}, {&p64_, &d64_}};
        for (int k = 0; k < 2; ++k)
            for (int f = 0; f < 2; ++f) {
                StepSide& q = *sides[f][k];
                const int* c = v + 3 * k;
                if (c[1] != 0 && c[1] != 32 && c[1] != 128 && c[1] != 256)
                    throw Error(E_INVALID, "PDFP_TUNING: threads per role must be 0, 32, 128 or 256");
                if (c[1] == 32) {  // the vec engine: FP32 steps; the FP64 steps keep their default
                    if (c[0] != 1 && c[0] != 2 && c[0] != 4 && c[0] != 8)
                        throw Error(E_INVALID, "PDFP_TUNING: the vec engine's nonzeros per lane must "
                                               "be 1, 2, 4 or 8");
                    if (c[2] < 0 || c[2] > 1)
                        throw Error(E_INVALID, "PDFP_TUNING: the vec engine's gather policy must be 0 or 1");
                    if (v[10 + k] != 0)
                        throw Error(E_INVALID, "PDFP_TUNING: the vec engine has no reducers (0)");
                    if (f == 1) continue;
                    q.engine = 2;
                    q.lane_nnz = c[0];
                    q.gather_l2 = c[2];
                    continue;
                }
                if (c[1] != 0 && (c[0] < 8192 || c[0] > 49152 || c[0] % 128 != 0))
                    throw Error(E_INVALID, "PDFP_TUNING: tile-engine stage bytes must be a multiple "
                                           "of 128 in [8192, 49152]");
                q.engine = c[1] == 0 ? 1 : 0;
                q.qpt = c[0] == 0 || c[0] == flat_stage_bytes(4, 1024) || c[0] == flat_stage_bytes(8, 1024) ? 1 : 2;
                q.stage_bytes = c[0] > 0 ? c[0] : q.stage_bytes;
                q.nt = c[1] == 0 ? 256 : c[1];
                if (c[2] < 0 || c[2] > 2) throw Error(E_INVALID, "PDFP_TUNING: gather policy must be 0, 1 or 2");
                q.gather_l2 = c[2];
                q.stages = v[6 + k];
                q.max_blocks = v[8 + k];
                const int red = v[10 + k];
                if (red != 0 && red != c[1] && !(c[1] != 0 && red == c[1] / 2))
                    throw Error(E_INVALID, "PDFP_TUNING: reducers must be 0, the threads per role "
                                           "or half of them");
                q.half_red = c[1] != 0 && red == c[1] / 2;
            }
        pinned = true;
    }
    const bool tune = forced >= 0 || pinned ? false
                      : at && at[0] == '0' ? false
                      : (at && at[0] == '1' ? true : M_.L.NNZ >= (1 << 18));
    if (precision_ == PDFP_MIXED) {
        if (tune) autotune(true); else { prepare_side(p32_, true, true); prepare_side(d32_, false, true); }
    }
    if (tune && precision_ == PDFP_FP64) {
        autotune(false);
    } else {
        prepare_side(p64_, true, false);
        prepare_side(d64_, false, false);
    }
    // PDFP_VEC_WINDOW=1: when both sides of the FP32 steps run on the vec engine and
    // neither has long-row pieces, a window's minor steps run in one cooperative launch
    // (vec_window_kernel) instead of two launches per step
    {
        const char* vw = std::getenv("PDFP_VEC_WINDOW");
        vecwin_ = vw && vw[0] == '1' && precision_ == PDFP_MIXED && !tiny_ && p32_.engine == 2 &&
                  d32_.engine == 2 && p32_.vec.n_slots == 0 && d32_.vec.n_slots == 0;
        if (vecwin_) {
            int coop = 0, dev = 0, per_sm = 0;
            PDFP_CK(cudaGetDevice(&dev));
            PDFP_CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
            PDFP_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, vec_window_kernel<PrimalOp<float, false, kFlatThreads>, DualOp<float, false, kFlatThreads>>,
                kVecThreads, 0));
            if (!coop || per_sm < 1) {
                vecwin_ = false;
            } else {
                vecwin_grid_ = per_sm * num_sms_;
                if (!gbar_) gbar_ = ar_.alloc<unsigned>(4);
            }
        }
    }
}

template <>
IterVecs<float>& Projector::vecs<float>() { return v32_; }
template <>
IterVecs<double>& Projector::vecs<double>() { return v64_; }

template <typename T, bool MAJOR>
void Projector::launch_primal(const StepSide& s, int k, bool overlap) {
    const int mode = std::is_same<T, float>::value ? MODE_FP32 : MODE_FP64;
    if constexpr (std::is_same<T, float>::value)
        if (s.engine == 2) {
            launch_vec(s.vec, PrimalOp<T, MAJOR, kFlatThreads>{vecs<T>(), st_, k, mode, err_, s.gather_l2}, s.grid, stream_);
            return;
        }
    if (s.engine == 1)
        launch_flat(s.tiling.dev, PrimalOp<T, MAJOR, kFlatThreads>{vecs<T>(), st_, k, mode, err_, s.gather_l2}, s.qpt, s.grid, stream_);
    else if (s.nt == 256)
        launch_tile(s.tiling.dev, PrimalOp<T, MAJOR, 256>{vecs<T>(), st_, k, mode, err_, s.gather_l2}, s.grid, stream_, overlap, s.carveout, s.half_red);
    else
        launch_tile(s.tiling.dev, PrimalOp<T, MAJOR, 128>{vecs<T>(), st_, k, mode, err_, s.gather_l2}, s.grid, stream_, overlap, s.carveout, s.half_red);
}

template <typename T, bool MAJOR>
void Projector::launch_dual(const StepSide& s, int k, bool overlap) {
    const int mode = std::is_same<T, float>::value ? MODE_FP32 : MODE_FP64;
    if constexpr (std::is_same<T, float>::value) {
        if (s.engine == 2) {
            launch_vec(s.vec, DualOp<T, MAJOR, kFlatThreads>{vecs<T>(), st_, M_.row_off, M_.n_eq, k, mode, err_, s.gather_l2}, s.grid, stream_);
            return;
        }
        if (s.seg_nseg > 0) {  // the long rows first; the tile launch then follows no step launch
            launch_seg(s.segt.dev, s.segd, s.seg_nt, s.seg_bps,
                       DualOp<T, MAJOR, kFlatThreads>{vecs<T>(), st_, M_.row_off, M_.n_eq, k, mode, err_, s.gather_l2},
                       stream_);
            overlap = false;
        }
    }
    if (s.engine == 1)
        launch_flat(s.tiling.dev, DualOp<T, MAJOR, kFlatThreads>{vecs<T>(), st_, M_.row_off, M_.n_eq, k, mode, err_, s.gather_l2}, s.qpt, s.grid, stream_);
    else if (s.nt == 256)
        launch_tile(s.tiling.dev, DualOp<T, MAJOR, 256>{vecs<T>(), st_, M_.row_off, M_.n_eq, k, mode, err_, s.gather_l2}, s.grid, stream_, overlap, s.carveout, s.half_red);
    else
        launch_tile(s.tiling.dev, DualOp<T, MAJOR, 128>{vecs<T>(), st_, M_.row_off, M_.n_eq, k, mode, err_, s.gather_l2}, s.grid, stream_, overlap, s.carveout, s.half_red);
}

// Grid of a step Op family for a tiling (sets the shared-memory attribute of
// both the MAJOR and the minor kernel).
template <template <typename, bool, int> class OpT, typename T>
static int step_grid(const SideDev& d, int nt, int sms, bool async, bool half_red) {
    if (nt == 256) {
        tile_grid<OpT<T, false, 256>>(d, sms, async, half_red);
        return tile_grid<OpT<T, true, 256>>(d, sms, async, half_red);
    }
    tile_grid<OpT<T, false, 128>>(d, sms, async, half_red);
    return tile_grid<OpT<T, true, 128>>(d, sms, async, half_red);
}

void Projector::prepare_side(StepSide& s, bool primal, bool f32) {
    const int e = f32 ? 4 : 8;
    if (s.engine != 0) s.seg_nseg = 0;  // segmented long rows: tile engine only
    if (s.engine == 2) {
        if (!f32) throw Error(E_INVALID, "internal: the vec engine runs the FP32 steps only");
        // The A' side (short, even rows on the zipf-lp matrix: 68 us against 72 us a
        // launch) takes larger items while they leave at least two per warp of a full
        // grid; on the A side (Zipf-skewed rows) larger items measured slower.
        s.vec = M_.make_vec(ar_, primal, s.lane_nnz,
                            primal ? int64_t(2) * num_sms_ * kVecMinBlocks * (kVecThreads / 32) : 0);
        s.stage_bytes = s.lane_nnz;
        s.nt = 32;
        s.half_red = false;
        if (s.gather_l2 == 2) s.gather_l2 = 1;
        // both the MAJOR and the minor kernel: the grid is the smaller of the two
        const int g0 = primal ? vec_grid<PrimalOp<float, false, kFlatThreads>>(s.vec, num_sms_)
                              : vec_grid<DualOp<float, false, kFlatThreads>>(s.vec, num_sms_);
        const int g1 = primal ? vec_grid<PrimalOp<float, true, kFlatThreads>>(s.vec, num_sms_)
                              : vec_grid<DualOp<float, true, kFlatThreads>>(s.vec, num_sms_);
        s.grid = std::min(g0, g1);
        return;
    }
    if (s.engine == 1) {
        const int cap = s.qpt * 4 * kFlatThreads;
        s.stage_bytes = flat_stage_bytes(e, cap);
        s.nt = 0;
        StageGeom g{e, e, e, 0, 1, s.stage_bytes, kFlatMaxRows};
        s.tiling = M_.make_tiling(ar_, primal, g);
        if (!flat_tiling_fits(s.tiling.host, cap))
            throw Error(E_INVALID, "internal: a flat-engine tile exceeds the kernel's caps");
        if (primal)
            s.grid = f32 ? flat_grid<PrimalOp<float, false, kFlatThreads>>(s.tiling.dev, s.qpt, num_sms_)
                         : flat_grid<PrimalOp<double, false, kFlatThreads>>(s.tiling.dev, s.qpt, num_sms_);
        else
            s.grid = f32 ? flat_grid<DualOp<float, false, kFlatThreads>>(s.tiling.dev, s.qpt, num_sms_)
                         : flat_grid<DualOp<double, false, kFlatThreads>>(s.tiling.dev, s.qpt, num_sms_);
        return;
    }
    StageGeom g{e, e, e, primal ? 8 : 3, 1, s.stage_bytes, 2048};
    std::vector<uint8_t> is_long;
    const std::vector<uint8_t>* skip = nullptr;
    if (s.seg_nseg > 0) {
        if (primal || !f32) throw Error(E_INVALID, "internal: segmented long rows are an FP32 A-side form");
        const StageGeom gs{4, 4, 4, 0, 1, s.seg_stage, 2048};
        const DualOp<float, false, kFlatThreads> dop{v32_, st_, M_.row_off, M_.n_eq, 0, MODE_FP32, err_, 0};
        bool ok = M_.make_seg(ar_, s.seg_nseg, s.seg_long, gs, s.segd, s.segt, is_long);
        if (ok) {
            s.segt.dev.stages = s.seg_stages;
            s.segt.dev.evict_first = evict_first_ ? 1 : 0;
            ok = s.seg_nt == 256 ? seg_attr<256>(s.segt.dev, s.segd, dop, max_smem_block_)
                                 : seg_attr<128>(s.segt.dev, s.segd, dop, max_smem_block_);
        }
        if (ok)
            skip = &is_long;
        else
            s.seg_nseg = 0;  // no row qualifies, or a segment does not fit a block
    }
    s.tiling = M_.make_tiling(ar_, primal, g, skip);
    s.tiling.dev.stages = s.stages;
    s.tiling.dev.evict_first = evict_first_ ? 1 : 0;
    const bool async = s.gather_l2 == 2;
    if (!f32 || async) s.half_red = false;  // half-size reducers: FP32 register-gather steps only
    if (primal)
        s.grid = f32 ? step_grid<PrimalOp, float>(s.tiling.dev, s.nt, num_sms_, async, s.half_red)
                     : step_grid<PrimalOp, double>(s.tiling.dev, s.nt, num_sms_, async, false);
    else
        s.grid = f32 ? step_grid<DualOp, float>(s.tiling.dev, s.nt, num_sms_, async, s.half_red)
                     : step_grid<DualOp, double>(s.tiling.dev, s.nt, num_sms_, async, false);
    // A cap on resident blocks per SM: fewer blocks than shared memory allows, with
    // the unified L1 / shared split asking only for their shared memory, so that
    // the rest stays L1 (the gathers' in-flight misses live there).
    s.carveout = -1;
    if (s.max_blocks > 0 && s.grid > 0) {
        s.grid = std::min(s.grid, s.max_blocks * num_sms_);
        const SideDev& d = s.tiling.dev;
        const int mx = max_smem_sm_;
        if (s.nt == 256)
            s.carveout = primal ? (f32 ? tile_carveout<PrimalOp<float, false, 256>>(d, s.max_blocks, mx)
                                       : tile_carveout<PrimalOp<double, false, 256>>(d, s.max_blocks, mx))
                                : (f32 ? tile_carveout<DualOp<float, false, 256>>(d, s.max_blocks, mx)
                                       : tile_carveout<DualOp<double, false, 256>>(d, s.max_blocks, mx));
        else
            s.carveout = primal ? (f32 ? tile_carveout<PrimalOp<float, false, 128>>(d, s.max_blocks, mx)
                                       : tile_carveout<PrimalOp<double, false, 128>>(d, s.max_blocks, mx))
                                : (f32 ? tile_carveout<DualOp<float, false, 128>>(d, s.max_blocks, mx)
                                       : tile_carveout<DualOp<double, false, 128>>(d, s.max_blocks, mx));
    }
}

// The autotuner: times the minor step kernel of each side for every candidate
// (engine, shared-memory stage size x threads per role x gather cache policy, and
// for the FP32 A side a few segmentations of its long rows) on this handle's
// matrix, each launch right after one of the other side's step, twice, and keeps
// the fastest.  Runs at creation on the all-zero state, which it resets afterwards.
void Projector::autotune(bool f32) {
    struct Cand {
        int engine, stage, nt, l2, qpt, stages;
        int max_blocks = 0;  // resident blocks per SM (0: as many as fit)
        int half_red = 0;    // 1: nt / 2 reducer threads
    };
    // tile engine, 4 stages per block: 12-16 KB stages give 3-4 blocks per SM, 24 KB
    // two, 32-48 KB one; 128-thread roles with 2-3 larger stages, 3 blocks per SM;
    // then the flat engine with both gather cache policies
    static const Cand cands[] = {
        {0, 12 * 1024, 128, 0, 0, 4}, {0, 16 * 1024, 128, 0, 0, 4}, {0, 16 * 1024, 256, 0, 0, 4},
        {0, 24 * 1024, 256, 0, 0, 4}, {0, 32 * 1024, 256, 0, 0, 4}, {0, 48 * 1024, 256, 0, 0, 4},
        {0, 16 * 1024, 256, 1, 0, 4}, {0, 24 * 1024, 256, 1, 0, 4}, {0, 32 * 1024, 256, 1, 0, 4},
        {0, 24 * 1024, 128, 1, 0, 3}, {0, 32 * 1024, 128, 1, 0, 2}, {0, 24 * 1024, 128, 0, 0, 3},
        {0, 12 * 1024, 128, 0, 0, 3}, {0, 12 * 1024, 128, 0, 0, 2}, {0, 16 * 1024, 128, 0, 0, 3},
        {0, 16 * 1024, 128, 1, 0, 3}, {0, 20 * 1024, 128, 1, 0, 3}, {0, 20 * 1024, 128, 0, 0, 3},
        {0, 24 * 1024, 128, 1, 0, 2}, {0, 28 * 1024, 128, 1, 0, 2}, {0, 16 * 1024, 128, 0, 0, 2},
        {0, 14 * 1024, 128, 0, 0, 3}, {0, 18 * 1024, 128, 0, 0, 3}, {0, 32 * 1024, 128, 1, 0, 3},
        {0, 20 * 1024, 128, 1, 0, 2}, {0, 26 * 1024, 128, 1, 0, 2}, {0, 24 * 1024, 128, 0, 0, 2},
        {0, 12 * 1024, 128, 1, 0, 4}, {0, 14 * 1024, 128, 1, 0, 3},
        {1, 0, 0, 0, 2, 4},           {1, 0, 0, 0, 1, 4},           {1, 0, 0, 1, 2, 4},
        // fewer resident blocks than fit, the rest of the unified memory left as L1
        {0, 24 * 1024, 128, 1, 0, 2, 3}, {0, 20 * 1024, 128, 1, 0, 2, 3}, {0, 16 * 1024, 128, 1, 0, 3, 3},
        {0, 20 * 1024, 128, 1, 0, 3, 3}, {0, 12 * 1024, 128, 0, 0, 3, 3}, {0, 16 * 1024, 128, 0, 0, 2, 3},
        {0, 12 * 1024, 128, 0, 0, 4, 3}, {0, 28 * 1024, 128, 1, 0, 2, 2}, {0, 24 * 1024, 128, 1, 0, 3, 2},
        {0, 16 * 1024, 128, 0, 0, 3, 3}, {0, 22 * 1024, 128, 1, 0, 2, 3}, {0, 26 * 1024, 128, 1, 0, 2, 3},
        {0, 18 * 1024, 128, 1, 0, 3, 3},
        // 256 gatherers with 128 reducers
        {0, 24 * 1024, 256, 0, 0, 2, 0, 1}, {0, 32 * 1024, 256, 1, 0, 2, 0, 1},
        // gather policy 2: per-thread async copies into the stage (FP32 steps)
        {0, 12 * 1024, 128, 2, 0, 3}, {0, 20 * 1024, 128, 2, 0, 3}, {0, 24 * 1024, 128, 2, 0, 3},
        {0, 32 * 1024, 256, 2, 0, 4},
        // the vec engine (FP32 steps): nonzeros per lane x gather cache policy
        {2, 1, 32, 0, 0, 4}, {2, 1, 32, 1, 0, 4}, {2, 2, 32, 0, 0, 4}, {2, 2, 32, 1, 0, 4},
        {2, 4, 32, 0, 0, 4}, {2, 4, 32, 1, 0, 4}, {2, 8, 32, 0, 0, 4}, {2, 8, 32, 1, 0, 4}};
    constexpr int NC = sizeof(cands) / sizeof(cands[0]);
    cudaEvent_t e0, e1;
    PDFP_CK(cudaEventCreate(&e0));
    PDFP_CK(cudaEventCreate(&e1));
    // Mean time of one minor step launch of a side (1e30 if it cannot launch), each
    // launch timed right after one of the other side's step (`partner`), as a PDHG
    // iteration runs them: the partner has just streamed its matrix through L2, so
    // the candidate finds the cache as it will in the solves (timed back to back
    // against itself, a candidate would find its own per-row vectors still in L2).
    auto run_side = [&](const StepSide& q, bool pr, int k) {
        if (pr) {
            if (f32) launch_primal<float, false>(q, k); else launch_primal<double, false>(q, k);
        } else {
            if (f32) launch_dual<float, false>(q, k); else launch_dual<double, false>(q, k);
        }
    };
    auto time_side = [&](const StepSide& s, bool primal, const StepSide& partner) -> float {
        run_side(s, primal, 2);
        run_side(s, primal, 3);
        if (cudaGetLastError() != cudaSuccess) return 1e30f;  // candidate cannot launch
        const int reps = 8;
        float total = 0.f;
        for (int r = 0; r < reps; ++r) {
            run_side(partner, !primal, 4 + r);
            PDFP_CK(cudaEventRecord(e0, stream_));
            run_side(s, primal, 4 + r);
            PDFP_CK(cudaEventRecord(e1, stream_));
            PDFP_CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            PDFP_CK(cudaEventElapsedTime(&ms, e0, e1));
            total += ms;
        }
        PDFP_CK(cudaGetLastError());
        return total / reps;
    };
    // the A side's partner while A' is tuned: a tile configuration that does well on
    // large matrices (then A is tuned against the chosen A' side)
    StepSide dual0;
    dual0.stage_bytes = 24 * 1024;
    dual0.nt = 128;
    dual0.gather_l2 = 1;
    dual0.stages = 2;
    dual0.max_blocks = 3;
    prepare_side(dual0, false, f32);
    tune_table_.clear();
    for (int side = 0; side < 2; ++side) {
        const bool primal = side == 0;
        std::vector<StepSide> sides(NC);
        std::vector<float> best_ms(NC, 1e30f);
        bool empty_side = false;
        for (int i = 0; i < NC; ++i) {
            sides[i].engine = cands[i].engine;
            sides[i].stages = cands[i].stages;
            if (cands[i].engine == 1) sides[i].qpt = cands[i].qpt;
            sides[i].stage_bytes = cands[i].stage;
            sides[i].nt = cands[i].nt;
            sides[i].gather_l2 = cands[i].l2;
            sides[i].max_blocks = cands[i].max_blocks;
            sides[i].half_red = cands[i].half_red != 0;
            if (cands[i].engine == 2) {
                if (!f32) continue;  // FP32 steps only
                sides[i].lane_nnz = cands[i].stage;
            }
            prepare_side(sides[i], primal, f32);
            if (sides[i].grid <= 0) empty_side = true;
        }
        StepSide& dst = primal ? (f32 ? p32_ : p64_) : (f32 ? d32_ : d64_);
        if (empty_side) {  // nothing to time (no rows on this side)
            dst = sides[2];
            continue;
        }
        for (int sweep = 0; sweep < 2; ++sweep) {
            for (int i = 0; i < NC; ++i) {
                if (cands[i].l2 == 2 && !f32) continue;  // FP64 steps have no async policy
                if (cands[i].engine == 2 && !f32) continue;
                best_ms[i] = std::min(best_ms[i], time_side(sides[i], primal,
                                                            primal ? dual0 : (f32 ? p32_ : p64_)));
            }
        }
        int bi = 0;
        for (int i = 0; i < NC; ++i) {
            tune_table_.push_back(TuneRow{side, sides[i].stage_bytes, cands[i].nt, cands[i].l2, cands[i].stages,
                                          cands[i].max_blocks,
                                          cands[i].engine == 2 ? 0
                                          : sides[i].half_red ? cands[i].nt / 2 : cands[i].nt,
                                          best_ms[i]});
            if (best_ms[i] < best_ms[bi]) bi = i;
        }
        dst = sides[bi];
        dst.tuned_ms = best_ms[bi];
        // the A side of the FP32 steps with its long rows by column segment, on the
        // chosen tile configuration for the rest
        if (f32 && !primal && dst.engine == 0 && seg_mode_ != 0) {
            struct SegCand {
                int nseg, lmin, stage, nt, stages, bps;
            };
            std::vector<SegCand> sc;
            if (seg_mode_ > 0)
                sc.push_back({seg_mode_, seg_long_, seg_cfg_[0], seg_cfg_[1], seg_cfg_[2], seg_cfg_[3]});
            else if (M_.L.NNZ >= (int64_t(1) << 22))
                sc = {{num_sms_, 512, 24 * 1024, 256, 3, 1},     {num_sms_, 1024, 16 * 1024, 128, 3, 2},
                      {num_sms_, 512, 16 * 1024, 128, 3, 2},     {2 * num_sms_, 1024, 16 * 1024, 128, 3, 1},
                      {2 * num_sms_, 512, 12 * 1024, 128, 2, 2}, {num_sms_, 512, 32 * 1024, 256, 3, 1}};
            const StepSide keep = dst;
            for (const SegCand& q : sc) {
                StepSide c = keep;
                c.seg_nseg = q.nseg;
                c.seg_long = q.lmin;
                c.seg_stage = q.stage;
                c.seg_nt = q.nt;
                c.seg_stages = q.stages;
                c.seg_bps = q.bps;
                prepare_side(c, false, true);
                if (c.seg_nseg == 0) continue;  // not applicable to this matrix
                float ms = 1e30f;
                for (int sweep = 0; sweep < 2; ++sweep) ms = std::min(ms, time_side(c, false, p32_));
                tune_table_.push_back(TuneRow{2, q.nseg, q.lmin, c.gather_l2, q.stages, q.stage,
                                              q.nt, ms});
                if (seg_mode_ > 0 || ms < dst.tuned_ms) {
                    dst = c;
                    dst.tuned_ms = ms;
                }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // the timing runs advanced the (all-zero) iterates: reset them
    const HostLayout& L = M_.L;
    const size_t es = f32 ? sizeof(float) : sizeof(double);
    void* nvec[] = {f32 ? (void*)v32_.cx : (void*)v64_.cx, f32 ? (void*)v32_.cy : (void*)v64_.cy,
                    f32 ? (void*)v32_.rx : (void*)v64_.rx};
    for (void* q : nvec) PDFP_CK(cudaMemsetAsync(q, 0, es * L.N, stream_));
    PDFP_CK(cudaMemsetAsync(f32 ? (void*)v32_.cz : (void*)v64_.cz, 0, es * L.M, stream_));
    PDFP_CK(cudaStreamSynchronize(stream_));
}

int Projector::tuning_table(float* ms, int32_t* cfg, int cap) const {
    const int n = static_cast<int>(tune_table_.size());
    for (int i = 0; i < n && i < cap; ++i) {
        ms[i] = tune_table_[i].ms;
        cfg[7 * i + 0] = tune_table_[i].side;
        cfg[7 * i + 1] = tune_table_[i].stage;
        cfg[7 * i + 2] = tune_table_[i].nt;
        cfg[7 * i + 3] = tune_table_[i].l2;
        cfg[7 * i + 4] = tune_table_[i].stages;
        cfg[7 * i + 5] = tune_table_[i].max_blocks;
        cfg[7 * i + 6] = tune_table_[i].reducers;
    }
    return n;
}

void Projector::tuning_stages(int32_t* out) const {
    const bool f32 = precision_ == PDFP_MIXED;
    out[0] = (f32 ? p32_ : p64_).stages;
    out[1] = (f32 ? d32_ : d64_).stages;
}

void Projector::tuning_blocks(int32_t* out) const {
    const bool f32 = precision_ == PDFP_MIXED;
    out[0] = (f32 ? p32_ : p64_).max_blocks;
    out[1] = (f32 ? d32_ : d64_).max_blocks;
}

void Projector::tuning_seg(int32_t* out) const {
    const StepSide& d = precision_ == PDFP_MIXED ? d32_ : d64_;
    out[0] = d.seg_nseg;
    out[1] = d.seg_nseg > 0 ? d.seg_long : 0;
}

void Projector::tuning_reducers(int32_t* out) const {
    const bool f32 = precision_ == PDFP_MIXED;
    const StepSide& p = f32 ? p32_ : p64_;
    const StepSide& d = f32 ? d32_ : d64_;
    out[0] = p.engine != 0 ? 0 : (p.half_red ? p.nt / 2 : p.nt);
    out[1] = d.engine != 0 ? 0 : (d.half_red ? d.nt / 2 : d.nt);
}

void Projector::tuning(int32_t* out) const {
    const bool f32 = precision_ == PDFP_MIXED;
    const StepSide& p = f32 ? p32_ : p64_;
    const StepSide& d = f32 ? d32_ : d64_;
    out[0] = p.stage_bytes;
    out[1] = p.nt;
    out[2] = p.engine == 2 ? p.vec.n_items : p.tiling.dev.n_tiles;
    out[3] = d.stage_bytes;
    out[4] = d.nt;
    out[5] = d.engine == 2 ? d.vec.n_items : d.tiling.dev.n_tiles;
    out[6] = p.gather_l2;
    out[7] = d.gather_l2;
}

Projector::~Projector() {
    for (auto& e : tev_) if (e) cudaEventDestroy(e);
    for (auto& e : sev_) if (e) cudaEventDestroy(e);
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
    pinned_give(flags_h_, sizeof(InstFlags) * (K_ + 1));
    pinned_give(st_h_, sizeof(InstState) * K_);
    pinned_give(nan_seen_h_, sizeof(int32_t));
    if (host_stage_ev_) cudaEventSynchronize(host_stage_ev_);
    pinned_give(host_stage_, host_stage_bytes_);
    if (host_stage_ev_) cudaEventDestroy(host_stage_ev_);
    if (stream_) cudaStreamDestroy(stream_);
}

void Projector::set_polish(int32_t stall_evaluations, double fp32_floor) {
    if (stall_evaluations < 0) throw Error(E_INVALID, "stall_evaluations must be >= 0");
    if (!(fp32_floor > 0.0) || !(fp32_floor < 1.0))
        throw Error(E_INVALID, "fp32_floor must lie in (0, 1)");
    stall_limit_ = stall_evaluations;
    fp32_floor_ = fp32_floor;
}

// The timing mode's events are made the first time it is switched on.
void Projector::set_kernel_timing(bool on) {
    if (on && !tev_[0])
        for (auto& e : tev_) PDFP_CK(cudaEventCreate(&e));
    timing_ = on;
}

void Projector::check_instance(int p) const {
    if (p < 0 || p >= K_) throw Error(E_INVALID, "instance index out of range");
}

// Stage the caller's column vector of instance p (n values) and raise E_INVALID,
// before anything is written, when it holds a NaN: a short vector is checked on the
// host (no round trip to the device), a long one on the device.
void Projector::stage_cols(int p, const double* src, const char* what) {
    const int32_t n = M_.L.col_off[p + 1] - M_.L.col_off[p];
    if (n <= kHostNanScanMax) {
        for (int32_t j = 0; j < n; ++j)
            if (std::isnan(src[j])) throw Error(E_INVALID, std::string("NaN in the ") + what);
        // through the handle's own page-locked buffer, so that the caller's may be reused
        // when this returns; its previous copy must have left it first
        if (!host_stage_) {
            host_stage_bytes_ = sizeof(double) * static_cast<size_t>(std::max(M_.max_n, 1));
            host_stage_ = static_cast<double*>(pinned_take(host_stage_bytes_));
            PDFP_CK(cudaEventCreateWithFlags(&host_stage_ev_, cudaEventDisableTiming));
        } else {
            PDFP_CK(cudaEventSynchronize(host_stage_ev_));
        }
        std::memcpy(host_stage_, src, sizeof(double) * n);
        PDFP_CK(cudaMemcpyAsync(stage_, host_stage_, sizeof(double) * n, cudaMemcpyHostToDevice, stream_));
        PDFP_CK(cudaEventRecord(host_stage_ev_, stream_));
        return;
    }
    PDFP_CK(cudaMemcpyAsync(stage_, src, sizeof(double) * n, cudaMemcpyHostToDevice, stream_));
    PDFP_CK(cudaMemsetAsync(nan_seen_, 0, sizeof(int32_t), stream_));
    launch_elem(K_, n, NanScan{stage_, M_.col_off, p, nan_seen_}, stream_);
    PDFP_CK(cudaGetLastError());
    PDFP_CK(cudaMemcpyAsync(nan_seen_h_, nan_seen_, sizeof(int32_t), cudaMemcpyDeviceToHost, stream_));
    PDFP_CK(cudaStreamSynchronize(stream_));
    if (*nan_seen_h_) throw Error(E_INVALID, std::string("NaN in the ") + what);
}

// Write the staged vector into dst (and dst2) in packed order: as given, or divided by D_c.
template <typename T>
void Projector::load_cols(int p, T* dst, T* dst2, bool unscaled) {
    const int32_t n = M_.L.col_off[p + 1] - M_.L.col_off[p];
    if (unscaled)
        launch_elem(K_, n, ScaleIn<T>{dst, dst2, stage_, col_scale_, M_.col_off, M_.col_orig, p}, stream_);
    else
        launch_elem(K_, n, PermuteIn<T>{dst, dst2, stage_, M_.col_off, M_.col_orig, p}, stream_);
    PDFP_CK(cudaGetLastError());
}

void Projector::check_unscaled(int p) const {
    if (!has_col_scale_[p]) throw Error(E_INVALID, "no column scale set for this instance");
}

void Projector::set_col_scale(int p, const double* dc) {
    check_instance(p);
    const int32_t n = cols(p);
    for (int32_t j = 0; j < n; ++j)
        if (!(dc[j] > 0.0) || !std::isfinite(dc[j]))
            throw Error(E_INVALID, "column scale entries must be positive and finite");
    if (!col_scale_) col_scale_ = ar_.alloc<double>(std::max<int64_t>(M_.L.N, 1));
    if (n > 0) {
        PDFP_CK(cudaMemcpyAsync(stage_, dc, sizeof(double) * n, cudaMemcpyHostToDevice, stream_));
        load_cols<double>(p, col_scale_, nullptr, false);
        PDFP_CK(cudaStreamSynchronize(stream_));
    }
    has_col_scale_[p] = true;
}

void Projector::set_x(int p, const double* x, bool unscaled) {
    check_instance(p);
    if (unscaled) check_unscaled(p);
    if (cols(p) == 0) return;
    stage_cols(p, x, "start point");
    if (vec_mode_[p] == MODE_FP32)
        load_cols<float>(p, v32_.cx, v32_.ix, unscaled);
    else
        load_cols<double>(p, v64_.cx, v64_.ix, unscaled);
}

void Projector::set_target(int p, const double* xt, bool unscaled) {
    check_instance(p);
    if (unscaled) check_unscaled(p);
    if (cols(p) > 0) {
        stage_cols(p, xt, "target");
        load_cols<double>(p, v64_.xt, nullptr, unscaled);
        if (precision_ == PDFP_MIXED) load_cols<float>(p, v32_.xt, nullptr, unscaled);
    }
    warm_start(p);
}

void Projector::warm_start(int p) {
    check_instance(p);
    const HostLayout& L = M_.L;
    const int64_t len = (L.col_off[p + 1] - L.col_off[p]) + (L.row_off[p + 1] - L.row_off[p]);
    if (vec_mode_[p] == MODE_FP32)
        launch_elem(K_, len, WarmStartCopy<float>{v32_, M_.col_off, M_.row_off, p}, stream_);
    else
        launch_elem(K_, len, WarmStartCopy<double>{v64_, M_.col_off, M_.row_off, p}, stream_);
    warm_start_state_kernel<<<1, 1, 0, stream_>>>(st_, p);
    host_total_[p] = 0;
    last_running_[p] = 0;  // a new projection: it starts afresh, it does not resume
    PDFP_CK(cudaGetLastError());  // stream-ordered before the next solve; no host wait
}

void Projector::get_vector(int p, int which, double* out, bool unscaled) {
    check_instance(p);
    const HostLayout& L = M_.L;
    const bool rowvec = (which == PDFP_VEC_PDHG_Z || which == PDFP_VEC_CURRENT_Z);
    if (unscaled) {
        check_unscaled(p);
        if (rowvec || which == PDFP_VEC_CURRENT_Y || which == PDFP_VEC_PDHG_Y || which == PDFP_VEC_DUAL_SLACK)
            throw Error(E_INVALID, "only primal column vectors have an unscaled form");
    }
    const int32_t len = rowvec ? L.row_off[p + 1] - L.row_off[p] : L.col_off[p + 1] - L.col_off[p];
    if (len == 0) return;
    auto pick = [&](auto& v) -> decltype(v.px) {
        switch (which) {
            case PDFP_VEC_PDHG_X: return v.px;
            case PDFP_VEC_PDHG_Y: return v.py;
            case PDFP_VEC_PDHG_Z: return v.pz;
            case PDFP_VEC_CURRENT_X: return v.cx;
            case PDFP_VEC_CURRENT_Y: return v.cy;
            case PDFP_VEC_CURRENT_Z: return v.cz;
            case PDFP_VEC_DUAL_SLACK: return v.ds;
            case PDFP_VEC_REFLECTED_X: return v.rx;
            default: throw Error(E_INVALID, "unknown vector");
        }
    };
    const int32_t* off = rowvec ? M_.row_off : M_.col_off;
    const int32_t* orig = rowvec ? M_.row_orig : M_.col_orig;
    if (unscaled && vec_mode_[p] == MODE_FP32)
        launch_elem(K_, len, ScaleOut<float>{stage_, pick(v32_), col_scale_, off, orig, p}, stream_);
    else if (unscaled)
        launch_elem(K_, len, ScaleOut<double>{stage_, pick(v64_), col_scale_, off, orig, p}, stream_);
    else if (vec_mode_[p] == MODE_FP32)
        launch_elem(K_, len, PermuteOut<float>{stage_, pick(v32_), off, orig, p}, stream_);
    else
        launch_elem(K_, len, PermuteOut<double>{stage_, pick(v64_), off, orig, p}, stream_);
    PDFP_CK(cudaGetLastError());
    PDFP_CK(cudaMemcpyAsync(out, stage_, sizeof(double) * len, cudaMemcpyDeviceToHost, stream_));
    PDFP_CK(cudaStreamSynchronize(stream_));
}

void Projector::ensure_step_sizes(int32_t sv_max_iterations, double sv_tolerance) {
    if (sv_ready_) return;  // every instance has its estimate: no state read-back
    std::vector<InstState> hs(K_);
    PDFP_CK(cudaMemcpy(hs.data(), st_, sizeof(InstState) * K_, cudaMemcpyDeviceToHost));
    std::vector<int> run(K_, 0);
    bool any = false;
    for (int p = 0; p < K_; ++p) {
        run[p] = (!hs[p].nnz_zero && std::isnan(hs[p].max_sv)) ? 1 : 0;  // cached per run (src/pdfp.jl:225-229)
        any = any || run[p];
    }
    if (!any) {
        sv_ready_ = true;
        return;
    }
    std::vector<double> sv = power_iteration(M_, ar_, ev_a_, ev_t_, run, sv_max_iterations,
                                             sv_tolerance, stream_, num_sms_, err_, nullptr);
    bool all = true;
    for (int p = 0; p < K_; ++p) all = all && (!run[p] || !std::isnan(sv[p]));
    sv_ready_ = all;
    DeviceArena tmp;
    double* d = tmp.alloc<double>(K_);
    PDFP_CK(cudaMemcpy(d, sv.data(), sizeof(double) * K_, cudaMemcpyHostToDevice));
    set_max_sv_kernel<<<(K_ + 127) / 128, 128, 0, stream_>>>(st_, d, K_);
    PDFP_CK(cudaGetLastError());
    PDFP_CK(cudaStreamSynchronize(stream_));
}

template <typename T>
void Projector::launch_tiny_steps(int i0, int i1) {
    const int mode = std::is_same<T, float>::value ? MODE_FP32 : MODE_FP64;
    tiny_steps_kernel<PrimalOp<T, false, kTinyThreads>, DualOp<T, false, kTinyThreads>>
        <<<K_, kTinyThreads, 0, stream_>>>(
        PrimalOp<T, false, kTinyThreads>{vecs<T>(), st_, 0, mode, err_, 0},
        DualOp<T, false, kTinyThreads>{vecs<T>(), st_, M_.row_off, M_.n_eq, 0, mode, err_, 0},
        M_.rp_t, M_.ci_t, M_.rp_a, M_.ci_a, M_.col_off, M_.row_off, i0, i1);
    PDFP_CK(cudaGetLastError());
}

template <typename T>
void Projector::launch_medium_steps(int i0, int i1) {
    const int mode = std::is_same<T, float>::value ? MODE_FP32 : MODE_FP64;
    using POp = PrimalOp<T, false, kMediumThreads>;
    using DOp = DualOp<T, false, kMediumThreads>;
    // gathers read L2 (policy 1): the gathered vectors were written by other blocks
    const POp pop{vecs<T>(), st_, 0, mode, err_, 1};
    const DOp dop{vecs<T>(), st_, M_.row_off, M_.n_eq, 0, mode, err_, 1};
    const GridBar bar{gbar_, gbar_ + 1, gbar_ + 2};
    PDFP_CK(cudaMemsetAsync(gbar_, 0, sizeof(unsigned) * 4, stream_));  // count, generation, abort
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(num_sms_));
    cfg.blockDim = dim3(kMediumThreads);
    cfg.stream = stream_;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    PDFP_CK(cudaLaunchKernelEx(&cfg, medium_steps_kernel<POp, DOp>, pop, dop, M_.rp_t, M_.ci_t, M_.rp_a,
                               M_.ci_a, M_.col_off, M_.row_off, K_, static_cast<const int32_t*>(part_t_),
                               static_cast<const int32_t*>(part_a_), bar, static_cast<int32_t>(i0),
                               static_cast<int32_t>(i1)));
}

void Projector::launch_vec_window(int i0, int i1) {
    using POp = PrimalOp<float, false, kFlatThreads>;
    using DOp = DualOp<float, false, kFlatThreads>;
    // gathers read L2 (policy 1): the gathered vectors were written by other blocks
    const POp pop{v32_, st_, 0, MODE_FP32, err_, 1};
    const DOp dop{v32_, st_, M_.row_off, M_.n_eq, 0, MODE_FP32, err_, 1};
    const GridBar bar{gbar_, gbar_ + 1, gbar_ + 2};
    PDFP_CK(cudaMemsetAsync(gbar_, 0, sizeof(unsigned) * 4, stream_));  // count, generation, abort
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(vecwin_grid_));
    cfg.blockDim = dim3(kVecThreads);
    cfg.stream = stream_;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    PDFP_CK(cudaLaunchKernelEx(&cfg, vec_window_kernel<POp, DOp>, p32_.vec, d32_.vec, pop, dop, bar,
                               static_cast<int32_t>(i0), static_cast<int32_t>(i1)));
}

// Timing mode's plan for a window of `freq` steps: the RUN, minor steps
// [run_a, run_b) in the middle half of steps 2 .. freq-1, is bracketed by two events
// and nothing else, so it times the average step as the other windows run it; up to
// kSplitSteps single minor steps outside it (evenly spread, half before and half
// after) get events around each kernel, and only the share of each kernel in them is
// used, to split the run's step time between the two kernels.
Projector::TimingPlan Projector::timing_plan(int freq) {
    TimingPlan t{};
    const int M = freq - 2;  // minor steps
    if (M < 8) return t;
    t.run_a = 2 + M / 4;
    t.run_b = t.run_a + M / 2;
    auto spread = [&](int a, int b) {  // up to kSplitSteps / 2 steps of [a, b)
        const int len = b - a, want = kSplitSteps / 2;
        const int every = std::max(1, len / want);
        for (int i = a; i < b && t.n_split < kSplitSteps && (i - a) / every < want; i += every)
            t.split[t.n_split++] = i;
    };
    spread(2, t.run_a);
    spread(t.run_b + 1, freq);  // step run_b carries the run's closing event
    return t;
}

void Projector::record_window(int freq, bool with32, bool with64) {
    const int mode32 = MODE_FP32, mode64 = MODE_FP64;
    // a step launch directly after another step launch may overlap its drain
    // (tile engine; see tile_spmv.cuh); after anything else it waits in full
    bool after_step = false;
    auto step = [&](auto launch) {
        launch(overlap_ && after_step);
        after_step = true;
    };
    auto prim32 = [&](int k, bool major) {
        step([&](bool o) { if (major) launch_primal<float, true>(p32_, k, o); else launch_primal<float, false>(p32_, k, o); });
    };
    auto dual32 = [&](int k, bool major) {
        step([&](bool o) { if (major) launch_dual<float, true>(d32_, k, o); else launch_dual<float, false>(d32_, k, o); });
    };
    auto prim64 = [&](int k, bool major) {
        step([&](bool o) { if (major) launch_primal<double, true>(p64_, k, o); else launch_primal<double, false>(p64_, k, o); });
    };
    auto dual64 = [&](int k, bool major) {
        step([&](bool o) { if (major) launch_dual<double, true>(d64_, k, o); else launch_dual<double, false>(d64_, k, o); });
    };
    auto evals = [&](int which) {
        if (with32) {
            launch_tile(ev_t_.dev, EvalColOp<float, NT_EVAL>{v32_, ed_, st_, which, mode32, err_}, g_.ec, stream_);
            launch_tile(ev_a_.dev, EvalRowOp<float, NT_EVAL>{v32_, ed_, st_, M_.row_off, M_.n_eq, which, mode32, err_}, g_.er, stream_);
        }
        if (with64) {
            launch_tile(ev_t_.dev, EvalColOp<double, NT_EVAL>{v64_, ed_, st_, which, mode64, err_}, g_.ec, stream_);
            launch_tile(ev_a_.dev, EvalRowOp<double, NT_EVAL>{v64_, ed_, st_, M_.row_off, M_.n_eq, which, mode64, err_}, g_.er, stream_);
        }
    };
    // timing mode (see timing_plan): a run of minor steps between two events, and
    // single minor steps with events around each kernel for the split between them
    const TimingPlan plan = timing_plan(freq);
    const bool sample = timing_ && plan.run_b > plan.run_a && (with32 != with64);
    int n_split = 0;
    for (int i = 1; i <= freq; ++i) {
        const bool major = (i == 1 || i == freq);
        if (tiny_ && !sample && i == 2 && freq > 2) {
            // steps 2 .. freq-1 in one launch per precision
            if (with32) launch_tiny_steps<float>(2, freq);
            if (with64) launch_tiny_steps<double>(2, freq);
            after_step = false;
            i = freq - 1;
            continue;
        }
        if (vecwin_ && with32 && !with64 && !sample && i == 2 && freq > 2) {
            // steps 2 .. freq-1 of the FP32 steps on the vec engine in one cooperative launch
            launch_vec_window(2, freq);
            after_step = false;
            i = freq - 1;
            continue;
        }
        if (medium_ && !sample && i == 2 && freq > 2) {
            // steps 2 .. freq-1 in one cooperative launch per precision
            if (with32) launch_medium_steps<float>(2, freq);
            if (with64) launch_medium_steps<double>(2, freq);
            after_step = false;
            i = freq - 1;
            continue;
        }
        if (sample && n_split < plan.n_split && i == plan.split[n_split]) {
            cudaEvent_t* e = &tev_[2 + 3 * n_split];
            after_step = false;
            PDFP_CK(cudaEventRecordWithFlags(e[0], stream_, cudaEventRecordExternal));
            if (with32) prim32(i, major); else prim64(i, major);
            after_step = false;
            PDFP_CK(cudaEventRecordWithFlags(e[1], stream_, cudaEventRecordExternal));
            if (with32) dual32(i, major); else dual64(i, major);
            after_step = false;
            PDFP_CK(cudaEventRecordWithFlags(e[2], stream_, cudaEventRecordExternal));
            ++n_split;
            continue;
        }
        if (sample && i == plan.run_a) {
            after_step = false;
            PDFP_CK(cudaEventRecordWithFlags(tev_[0], stream_, cudaEventRecordExternal));
        }
        if (sample && i == plan.run_b) {
            after_step = false;
            PDFP_CK(cudaEventRecordWithFlags(tev_[1], stream_, cudaEventRecordExternal));
        }
        if (with32) { prim32(i, major); dual32(i, major); }
        if (with64) { prim64(i, major); dual64(i, major); }
        if (i == 1) {
            after_step = false;
            evals(EVAL_AFTER_RESTART);
            launch_finalize(K_, Controller{ev_t_.inst_tile0, part_col_, ev_a_.inst_tile0, part_row_, st_, flags_, PHASE_AFTER_FIRST, polish_enabled_}, stream_);
        }
    }
    evals(EVAL_FULL);
    launch_finalize(K_, Controller{ev_t_.inst_tile0, part_col_, ev_a_.inst_tile0, part_row_, st_, flags_, PHASE_EVAL, polish_enabled_}, stream_);
    const int64_t maxlen = static_cast<int64_t>(M_.max_m) + M_.max_n;
    if (with32) launch_elem(K_, maxlen, RestartCopy<float>{v32_, st_, M_.col_off, M_.row_off, mode32}, stream_);
    if (with64) launch_elem(K_, maxlen, RestartCopy<double>{v64_, st_, M_.col_off, M_.row_off, mode64}, stream_);
}

// persistent grid sizes and shared-memory attributes of the evaluation kernels
// (outside any capture)
void Projector::prepare_window() {
    if (precision_ == PDFP_MIXED) {
        tile_grid<EvalColOp<float, NT_EVAL>>(ev_t_.dev, num_sms_);
        tile_grid<EvalRowOp<float, NT_EVAL>>(ev_a_.dev, num_sms_);
    }
    g_.ec = tile_grid<EvalColOp<double, NT_EVAL>>(ev_t_.dev, num_sms_);
    g_.er = tile_grid<EvalRowOp<double, NT_EVAL>>(ev_a_.dev, num_sms_);
}

// Evaluation windows on the stream: a small handle runs up to kTinyWindowsPerLaunch
// windows of every member in one launch per precision (tiny_solve_kernel); any other
// handle replays one window's captured graph.
void Projector::run_window(int freq, bool with32, bool with64) {
    if (tiny_ && !timing_) {
        const int32_t rowsum_len = 2 * std::max(M_.max_m, M_.max_n);
        if (!window_ready_) {
            // the staged form when every member's copy fits next to the row sums
            // (PDFP_TINY_STAGE=0 switches it off)
            const char* ts = std::getenv("PDFP_TINY_STAGE");
            const bool want = !(ts && ts[0] == '0');
            const HostLayout& L = M_.L;
            size_t s32 = 0, s64 = 0;
            for (int p = 0; p < K_; ++p) {
                const int64_t nc = L.col_off[p + 1] - L.col_off[p], nr = L.row_off[p + 1] - L.row_off[p];
                const int64_t nzt = L.At.rp[L.col_off[p + 1]] - L.At.rp[L.col_off[p]];
                const int64_t nza = L.A.rp[L.row_off[p + 1]] - L.A.rp[L.row_off[p]];
                const bool un = row_unscale_ != nullptr;
                s32 = std::max(s32, tiny_stage_bytes<float>(nc, nr, nzt, nza, un));
                s64 = std::max(s64, tiny_stage_bytes<double>(nc, nr, nzt, nza, un));
            }
            const size_t base = sizeof(double) * static_cast<size_t>(rowsum_len);
            const size_t cap = static_cast<size_t>(max_smem_sm_) - 8 * 1024;
            tiny_smem32_ = want && base + s32 <= cap ? base + s32 : base;
            tiny_smem64_ = want && base + s64 <= cap ? base + s64 : base;
            tiny_staged32_ = tiny_smem32_ > base;
            tiny_staged64_ = tiny_smem64_ > base;
            auto attr = [&](auto kern, size_t bytes) {
                if (bytes > 48 * 1024)
                    PDFP_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 static_cast<int>(bytes)));
            };
            if (tiny_staged32_) attr(tiny_solve_kernel<float, true>, tiny_smem32_);
            else attr(tiny_solve_kernel<float, false>, tiny_smem32_);
            if (tiny_staged64_) attr(tiny_solve_kernel<double, true>, tiny_smem64_);
            else attr(tiny_solve_kernel<double, false>, tiny_smem64_);
            window_ready_ = true;
        }
        (void)freq;  // each member's own evaluation frequency (its state) drives the kernel
        auto launch = [&](auto kern, auto& vecs, size_t bytes) {
            kern<<<K_, kTinyThreads, bytes, stream_>>>(vecs, ed_, st_, flags_, M_.rp_t, M_.ci_t, M_.rp_a,
                                                       M_.ci_a, M_.col_off, M_.row_off, M_.n_eq, err_,
                                                       kTinyWindowsPerLaunch, polish_enabled_, rowsum_len,
                                                       any_stop_cur_);
        };
        if (with32) {
            if (tiny_staged32_) launch(tiny_solve_kernel<float, true>, v32_, tiny_smem32_);
            else launch(tiny_solve_kernel<float, false>, v32_, tiny_smem32_);
        }
        if (with64) {
            if (tiny_staged64_) launch(tiny_solve_kernel<double, true>, v64_, tiny_smem64_);
            else launch(tiny_solve_kernel<double, false>, v64_, tiny_smem64_);
        }
        PDFP_CK(cudaGetLastError());
        return;
    }
    PDFP_CK(cudaGraphLaunch(window_graph(freq, with32, with64), stream_));
}

cudaGraphExec_t Projector::window_graph(int freq, bool with32, bool with64) {
    const int key = freq * 8 + (with32 ? 1 : 0) + (with64 ? 2 : 0) + (timing_ ? 4 : 0);
    auto it = graphs_.find(key);
    if (it != graphs_.end()) return it->second;
    prepare_window();
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    PDFP_CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    try {
        record_window(freq, with32, with64);
    } catch (...) {  // leave the stream out of capture mode before reporting
        cudaGraph_t partial = nullptr;
        cudaStreamEndCapture(stream_, &partial);
        if (partial) cudaGraphDestroy(partial);
        cudaGetLastError();
        throw;
    }
    cudaError_t e = cudaStreamEndCapture(stream_, &graph);
    if (e != cudaSuccess) throw Error(E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    PDFP_CK(cudaGraphInstantiate(&exec, graph, 0));
    cudaGraphDestroy(graph);
    graphs_[key] = exec;
    return exec;
}

void Projector::solve(const pdfp_params* params, const double* primal_weights, pdfp_result* results,
                      const uint8_t* resume, bool any) {
    auto wall0 = std::chrono::steady_clock::now();
    for (int p = 0; p < K_ && resume; ++p)
        if (resume[p] && !last_running_[p])
            throw Error(E_INVALID, "instance " + std::to_string(p) +
                                       " cannot resume: it is not running from an earlier call");
    // validate and stage the parameters
    std::vector<SolveParams> sp(K_);
    int freq = -1;
    int32_t sv_it = 5000;
    double sv_tol = 1e-4;
    double max_time = 0.0;
    for (int p = 0; p < K_; ++p) {
        const pdfp_params& q = params[p];
        if (q.termination_evaluation_frequency < 1)
            throw Error(E_INVALID, "termination_evaluation_frequency must be >= 1");
        if (freq < 0) freq = q.termination_evaluation_frequency;
        if (q.termination_evaluation_frequency != freq)
            throw Error(E_INVALID, "batch members must share termination_evaluation_frequency");
        if (!(primal_weights[p] > 0.0) || !std::isfinite(primal_weights[p]))
            throw Error(E_INVALID, "primal_weight must be positive and finite");
        SolveParams& s = sp[p];
        s.eps_opt = q.eps_optimal_relative;
        s.eps_feas = q.eps_feasible_relative;
        s.time_limit = q.time_limit;
        s.omega = q.reflection_coefficient;
        s.art = q.artificial_restart_threshold;
        s.suff = q.sufficient_reduction_for_restart;
        s.nec = q.necessary_reduction_for_restart;
        s.kp = q.k_p;
        s.ki = q.k_i;
        s.kd = q.k_d;
        s.ismooth = q.i_smooth;
        s.primal_weight = primal_weights[p];
        s.iter_limit = q.iteration_limit;
        s.freq = q.termination_evaluation_frequency;
        // A mixed handle starts every instance in FP32.  FP32 iterates carry about
        // seven significant digits: an instance whose tolerance asks for more than
        // the FP32 floor gets there through the FP64 polish (see the controller);
        // with the polish switched off it runs in FP64 from the start instead.
        const bool tight = std::min(q.eps_optimal_relative, q.eps_feasible_relative) < fp32_floor_;
        s.mode = precision_ == PDFP_MIXED && (stall_limit_ > 0 || !tight) ? MODE_FP32 : MODE_FP64;
        s.stall_limit = stall_limit_;
        s.fp32_floor = fp32_floor_;
        s.resume = resume && resume[p] ? 1 : 0;
        if (s.resume) s.mode = vec_mode_[p];  // it keeps its form (FP32 or the polish)
        sv_it = q.sv_max_iterations;
        sv_tol = q.sv_tolerance;
        max_time = std::max(max_time, q.time_limit);
    }
    PDFP_CK(cudaEventRecord(sev_[0], stream_));
    PDFP_CK(cudaMemcpyAsync(sp_, sp.data(), sizeof(SolveParams) * K_, cudaMemcpyHostToDevice, stream_));
    solve_begin_kernel<<<(K_ + 127) / 128, 128, 0, stream_>>>(st_, sp_, K_);
    PDFP_CK(cudaGetLastError());
    ensure_step_sizes(sv_it, sv_tol);
    // a mixed handle starts each instance in the mode chosen above: convert the
    // iterates of instances whose vectors are in the other form
    bool with32 = false, with64 = false;
    for (int p = 0; p < K_; ++p) (sp[p].mode == MODE_FP32 ? with32 : with64) = true;
    if (precision_ == PDFP_MIXED) {
        const HostLayout& L = M_.L;
        for (int p = 0; p < K_; ++p) {
            if (vec_mode_[p] == sp[p].mode) continue;
            const int64_t len = (L.col_off[p + 1] - L.col_off[p]) + (L.row_off[p + 1] - L.row_off[p]);
            if (sp[p].mode == MODE_FP32)
                launch_elem(K_, len, ConvertVecs<double, float>{v64_, v32_, M_.col_off, M_.row_off, p}, stream_);
            else
                launch_elem(K_, len, ConvertVecs<float, double>{v32_, v64_, M_.col_off, M_.row_off, p}, stream_);
            vec_mode_[p] = sp[p].mode;
        }
    }
    solve_init_kernel<<<(K_ + 127) / 128, 128, 0, stream_>>>(st_, flags_, sp_, K_);
    launch_rows(ev_t_.dev, DenRows{v64_.w, v64_.xt, part_col_}, stream_);
    launch_finalize(K_, DenFin{ev_t_.inst_tile0, part_col_, nullptr, nullptr, st_}, stream_);
    PDFP_CK(cudaGetLastError());
    PDFP_CK(cudaMemsetAsync(err_, 0, sizeof(int32_t) * 4, stream_));

    // Which instances start running (iteration_limit > total): solve_init_kernel's
    // rule, evaluated on the host from the totals it tracks, so that no first poll
    // is needed; after a call that advanced the state otherwise, read it back.
    if (totals_known_) {
        for (int p = 0; p < K_; ++p)
            flags_h_[p] = InstFlags{sp[p].resume || host_total_[p] < sp[p].iter_limit ? ST_RUNNING
                                                                                     : ST_ITERATION_LIMIT,
                                    sp[p].mode, 0, 0};
    } else {
        PDFP_CK(cudaMemcpyAsync(flags_h_, flags_, sizeof(InstFlags) * K_, cudaMemcpyDeviceToHost, stream_));
        PDFP_CK(cudaStreamSynchronize(stream_));
    }
    bool polled = false;  // st_h_ holds the state after the last window
    int32_t dev_err = 0;
    double kp_sum = 0.0, kd_sum = 0.0;
    int64_t k_samples = 0;
    const TimingPlan plan = timing_plan(freq);
    // any: return at the first window boundary after an instance that was running
    // has stopped; the whole-window kernel's blocks leave at theirs too (any_stop)
    std::vector<uint8_t> started(K_);
    for (int p = 0; p < K_; ++p) started[p] = flags_h_[p].status == ST_RUNNING;
    if (any) PDFP_CK(cudaMemsetAsync(any_stop_, 0, sizeof(int32_t), stream_));
    any_stop_cur_ = any ? any_stop_ : nullptr;
    for (;;) {
        bool running = false;
        for (int p = 0; p < K_; ++p) running = running || flags_h_[p].status == ST_RUNNING;
        if (!running) break;
        run_window(freq, with32, with64);
        PDFP_CK(cudaMemcpyAsync(flags_h_, flags_, sizeof(InstFlags) * K_, cudaMemcpyDeviceToHost, stream_));
        PDFP_CK(cudaMemcpyAsync(&flags_h_[K_].status, err_, sizeof(int32_t), cudaMemcpyDeviceToHost, stream_));
        // the states too, and the end event: the poll that finds every instance
        // done then needs no further round trip
        PDFP_CK(cudaMemcpyAsync(st_h_, st_, sizeof(InstState) * K_, cudaMemcpyDeviceToHost, stream_));
        PDFP_CK(cudaEventRecord(sev_[1], stream_));
        PDFP_CK(cudaStreamSynchronize(stream_));
        polled = true;
        dev_err = flags_h_[K_].status;
        if (dev_err) throw Error(E_TIMEOUT, "a bounded device wait gave up (bulk copy did not complete)");
        if (timing_ && plan.run_b > plan.run_a && (with32 != with64)) {
            float run = 0.f, sp = 0.f, sd = 0.f;
            PDFP_CK(cudaEventElapsedTime(&run, tev_[0], tev_[1]));
            for (int t = 0; t < plan.n_split; ++t) {
                float a = 0.f, b = 0.f;
                PDFP_CK(cudaEventElapsedTime(&a, tev_[2 + 3 * t], tev_[3 + 3 * t]));
                PDFP_CK(cudaEventElapsedTime(&b, tev_[3 + 3 * t], tev_[4 + 3 * t]));
                sp += a;
                sd += b;
            }
            const double share = sp + sd > 0.f ? static_cast<double>(sp) / (sp + sd) : 0.5;
            kp_sum += share * run;
            kd_sum += (1.0 - share) * run;
            k_samples += plan.run_b - plan.run_a;
        }
        // FP64 polish for instances whose FP32 progress stalled
        for (int p = 0; p < K_; ++p) {
            if (flags_h_[p].polish_request && flags_h_[p].status == ST_RUNNING && vec_mode_[p] == MODE_FP32) {
                const HostLayout& L = M_.L;
                const int64_t len = (L.col_off[p + 1] - L.col_off[p]) + (L.row_off[p + 1] - L.row_off[p]);
                launch_elem(K_, len, ConvertVecs<float, double>{v32_, v64_, M_.col_off, M_.row_off, p}, stream_);
                set_mode_kernel<<<1, 1, 0, stream_>>>(st_, p, MODE_FP64);
                PDFP_CK(cudaGetLastError());
                vec_mode_[p] = MODE_FP64;
                with64 = true;
                polished_.insert(p);
                polled = false;
            }
        }
        const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
        if (wall > max_time + 120.0) {
            any_stop_cur_ = nullptr;
            throw Error(E_TIMEOUT, "solve exceeded its time limit by 120 s on the host clock");
        }
        if (any) {
            bool stopped = false;
            for (int p = 0; p < K_; ++p) stopped = stopped || (started[p] && flags_h_[p].status != ST_RUNNING);
            if (stopped) break;
        }
    }
    any_stop_cur_ = nullptr;
    if (!polled) {
        PDFP_CK(cudaMemcpyAsync(st_h_, st_, sizeof(InstState) * K_, cudaMemcpyDeviceToHost, stream_));
        PDFP_CK(cudaEventRecord(sev_[1], stream_));
        PDFP_CK(cudaStreamSynchronize(stream_));
    }
    const InstState* hs = st_h_;
    float solve_ms = 0.f;
    PDFP_CK(cudaEventElapsedTime(&solve_ms, sev_[0], sev_[1]));
    for (int p = 0; p < K_; ++p) {
        const InstState& s = hs[p];
        pdfp_result& r = results[p];
        std::memset(&r, 0, sizeof(r));
        r.status = s.status;
        r.restarts = s.restarts;
        r.total_count = s.total;
        r.rel_primal = s.rel_p;
        r.rel_dual = s.rel_d;
        r.rel_gap = s.rel_gap;
        r.primal_weight = s.primal_weight;
        r.step_size = s.step_size;
        r.max_singular_value = s.max_sv;
        r.fixed_point_error = s.fpe;
        r.objective_value = s.l1;
        r.polished = polished_.count(p) ? 1 : 0;
        r.fp64_iterations = s.fp64_iters;
        r.precision = s.mode == MODE_FP32 ? PDFP_MIXED : PDFP_FP64;
        r.device_ms = solve_ms;
        r.kernel_ms_primal = k_samples ? kp_sum / k_samples : 0.0;  // the runs' step time, split
        r.kernel_ms_dual = k_samples ? kd_sum / k_samples : 0.0;
        r.kernel_samples = k_samples;
        vec_mode_[p] = s.mode;
        host_total_[p] = s.total;
        last_running_[p] = s.status == ST_RUNNING ? 1 : 0;
    }
    totals_known_ = true;
    for (int p = 0; p < K_; ++p)  // a polished instance that keeps running stays marked
        if (!last_running_[p]) polished_.erase(p);
}

void Projector::profile_step(int iterations, float* ms_primal, float* ms_dual, double* bytes_primal,
                             double* bytes_dual) {
    totals_known_ = false;  // the next solve reads the instance states back first
    // Times the two fused step kernels (minor steps) over `iterations` steps of
    // every running instance, with events around each launch on the stream.
    const bool mixed = precision_ == PDFP_MIXED;
    window_graph(200, mixed, !mixed);  // sets grid sizes and smem attributes
    DeviceArena tmp;
    int32_t* saved = tmp.alloc<int32_t>(K_);
    swap_status_kernel<<<(K_ + 127) / 128, 128, 0, stream_>>>(st_, saved, K_, 0);
    PDFP_CK(cudaGetLastError());
    cudaEvent_t e[3];
    for (auto& x : e) PDFP_CK(cudaEventCreate(&x));
    float tp = 0.f, td = 0.f;
    for (int i = 0; i < iterations; ++i) {
        const int k = 2 + (i % 150);
        PDFP_CK(cudaEventRecord(e[0], stream_));
        if (mixed) launch_primal<float, false>(p32_, k); else launch_primal<double, false>(p64_, k);
        PDFP_CK(cudaEventRecord(e[1], stream_));
        if (mixed) launch_dual<float, false>(d32_, k); else launch_dual<double, false>(d64_, k);
        PDFP_CK(cudaEventRecord(e[2], stream_));
        PDFP_CK(cudaEventSynchronize(e[2]));
        float a = 0.f, b = 0.f;
        PDFP_CK(cudaEventElapsedTime(&a, e[0], e[1]));
        PDFP_CK(cudaEventElapsedTime(&b, e[1], e[2]));
        tp += a;
        td += b;
    }
    for (auto& x : e) cudaEventDestroy(x);
    swap_status_kernel<<<(K_ + 127) / 128, 128, 0, stream_>>>(st_, saved, K_, 1);
    PDFP_CK(cudaGetLastError());
    PDFP_CK(cudaStreamSynchronize(stream_));
    *ms_primal = iterations > 0 ? tp / iterations : 0.f;
    *ms_dual = iterations > 0 ? td / iterations : 0.f;
    const HostLayout& L = M_.L;
    const double sv = mixed ? 4.0 : 8.0;
    // algorithmic bytes: A' (values + indices + row pointers), 8 n-vectors read,
    // 3 written, z gathered once / A, 3 m-vectors read, 1 written, x_bar gathered once
    *bytes_primal = L.NNZ * (sv + 4.0) + 4.0 * (L.N + 1) + sv * (11.0 * L.N) + sv * L.M;
    *bytes_dual = L.NNZ * (sv + 4.0) + 4.0 * (L.M + 1) + sv * (4.0 * L.M) + sv * L.N;
}

}  // namespace pdfp
