// precond.cu -- the diagonal preconditioner on the device.
//
// scale_problem, src/preconditioner.jl:26-99: ten Ruiz rounds (1/sqrt of the
// largest |a| per row and column), one Pock-Chambolle pass (1/sqrt of the sum
// of |a|^alpha per row, |a|^(2-alpha) per column), then the scaled bounds and
// the optional bound/objective rescaling.  Row maxima and row sums are taken by
// one thread per row of A (and of A'), summing in ascending index order, so the
// scaling factors and scaled values are bit-identical to the reference's CPU
// arithmetic (Julia walks its CSC matrix column by column, which gives each row
// sum its terms in ascending column order and each column sum in ascending row
// order).  The scaled bounds, costs and the optional bound/objective rescaling
// (two sequential norms, as the reference's loops) run on the device too.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "device.hpp"
#include "kernels.cuh"
#include "power.cuh"
#include "solvers.hpp"

namespace pdfp {

static constexpr double SCALING_EPSILON = 1e-12;  // src/preconditioner.jl:11

// scale[i] = 1/sqrt(max_p |v_p|) over row i (1 if below SCALING_EPSILON)
__global__ void ruiz_scale_kernel(const int32_t* __restrict__ rp, const double* __restrict__ v,
                                  int32_t rows, double* __restrict__ scale) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        double mx = 0.0;
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            const double a = fabs(v[p]);
            if (a > mx) mx = a;
        }
        scale[i] = mx < SCALING_EPSILON ? 1.0 : 1.0 / sqrt(mx);
    }
}

// Pock-Chambolle: scale[i] = 1/sqrt(sum_p |v_p|^e), terms in ascending order
__global__ void pc_scale_kernel(const int32_t* __restrict__ rp, const double* __restrict__ v,
                                int32_t rows, double e, double* __restrict__ scale) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            const double a = fabs(v[p]);
            s = __dadd_rn(s, e == 1.0 ? a : pow(a, e));
        }
        scale[i] = s < SCALING_EPSILON ? 1.0 : 1.0 / sqrt(s);
    }
}

// v_p *= rs[row] * cs[col]  for one side (rows of this side use `rs_row`)
__global__ void apply_scale_kernel(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                   double* __restrict__ v, int32_t rows,
                                   const double* __restrict__ row_scale,
                                   const double* __restrict__ col_scale, int transpose) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            // A: r = row_scale[i], c = col_scale[ci];  A': r = row_scale[ci], c = col_scale[i]
            const double r = transpose ? row_scale[ci[p]] : row_scale[i];
            const double c = transpose ? col_scale[i] : col_scale[ci[p]];
            v[p] = __dmul_rn(v[p], __dmul_rn(r, c));
        }
    }
}

__global__ void mul_inplace_kernel(double* __restrict__ d, const double* __restrict__ s, int32_t n) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        d[i] = __dmul_rn(d[i], s[i]);
}

// scaled bounds and costs, src/preconditioner.jl:66-70:
// c_s = c .* D_c; var bounds / D_c and row bounds .* D_r where finite
__global__ void scale_vectors_kernel(const double* __restrict__ c, const double* __restrict__ lb,
                                     const double* __restrict__ ub, const double* __restrict__ D_c,
                                     int32_t n, const double* __restrict__ clb,
                                     const double* __restrict__ cub, const double* __restrict__ D_r,
                                     int32_t m, double* __restrict__ c_s, double* __restrict__ lb_s,
                                     double* __restrict__ ub_s, double* __restrict__ clb_s,
                                     double* __restrict__ cub_s) {
    for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        c_s[j] = __dmul_rn(c[j], D_c[j]);
        lb_s[j] = isfinite(lb[j]) ? lb[j] / D_c[j] : lb[j];
        ub_s[j] = isfinite(ub[j]) ? ub[j] / D_c[j] : ub[j];
    }
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        clb_s[i] = isfinite(clb[i]) ? __dmul_rn(clb[i], D_r[i]) : clb[i];
        cub_s[i] = isfinite(cub[i]) ? __dmul_rn(cub[i], D_r[i]) : cub[i];
    }
}

// bound/objective rescaling, src/preconditioner.jl:72-96: the two squared
// norms (sequential sums, as the reference's loops), then the scaling
__global__ void rescale_norms_kernel(const double* __restrict__ clb, const double* __restrict__ cub,
                                     const double* __restrict__ clb_s,
                                     const double* __restrict__ cub_s, int32_t m,
                                     const double* __restrict__ c_s, int32_t n,
                                     double* __restrict__ out /* bound_sq, c_sq */) {
    if (threadIdx.x == 0) {
        double bound_sq = 0.0;
        for (int32_t i = 0; i < m; ++i) {
            const bool flo = isfinite(clb[i]), fhi = isfinite(cub[i]);
            const double lo = clb_s[i], hi = cub_s[i];
            if (flo && (!fhi || fabs(lo - hi) > SCALING_EPSILON)) bound_sq = __dadd_rn(bound_sq, __dmul_rn(lo, lo));
            if (fhi) bound_sq = __dadd_rn(bound_sq, __dmul_rn(hi, hi));
        }
        out[0] = bound_sq;
    }
    if (threadIdx.x == 32) {
        double c_sq = 0.0;
        for (int32_t j = 0; j < n; ++j) c_sq = __dadd_rn(c_sq, __dmul_rn(c_s[j], c_s[j]));
        out[1] = c_sq;
    }
}

__global__ void rescale_apply_kernel(const double* __restrict__ lb, const double* __restrict__ ub,
                                     int32_t n, const double* __restrict__ clb,
                                     const double* __restrict__ cub, int32_t m,
                                     const double* __restrict__ sq, double* __restrict__ c_s,
                                     double* __restrict__ lb_s, double* __restrict__ ub_s,
                                     double* __restrict__ clb_s, double* __restrict__ cub_s,
                                     double* __restrict__ scales /* bound, objective */) {
    const double bs = 1.0 / (sqrt(sq[0]) + 1.0);
    const double os = 1.0 / (sqrt(sq[1]) + 1.0);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        scales[0] = bs;
        scales[1] = os;
    }
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        if (isfinite(clb[i])) clb_s[i] = __dmul_rn(clb_s[i], bs);
        if (isfinite(cub[i])) cub_s[i] = __dmul_rn(cub_s[i], bs);
    }
    for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        if (isfinite(lb[j])) lb_s[j] = __dmul_rn(lb_s[j], bs);
        if (isfinite(ub[j])) ub_s[j] = __dmul_rn(ub_s[j], bs);
        c_s[j] = __dmul_rn(c_s[j], os);
    }
}

// Small matrices (at most kScaleTinyMaxDim rows + columns and kScaleTinyMaxNnz
// nonzeros): every Ruiz round and the Pock-Chambolle pass in one launch of one
// block -- the same per-row and per-entry operations as the kernels above, in the
// same order (no value depends on how rows are shared among threads), with block
// barriers where those kernels end.
constexpr int64_t kScaleTinyMaxDim = 4096;
constexpr int64_t kScaleTinyMaxNnz = 65536;
constexpr int kScaleTinyThreads = 1024;

__global__ void __launch_bounds__(kScaleTinyThreads)
    scale_tiny_kernel(const int32_t* __restrict__ rp_a, const int32_t* __restrict__ ci_a,
                      double* __restrict__ v_a, const int32_t* __restrict__ rp_t,
                      const int32_t* __restrict__ ci_t, double* __restrict__ v_t, int32_t m,
                      int32_t n, int32_t ruiz_iterations, double alpha, double* __restrict__ rs,
                      double* __restrict__ cs, double* __restrict__ D_r, double* __restrict__ D_c) {
    const int t = threadIdx.x;
    for (int32_t it = 0; it <= ruiz_iterations; ++it) {
        const bool pc = it == ruiz_iterations;  // the last pass: Pock-Chambolle
        for (int32_t i = t; i < m; i += kScaleTinyThreads) {
            if (pc) {
                double sum = 0.0;
                for (int32_t p = rp_a[i]; p < rp_a[i + 1]; ++p) {
                    const double a = fabs(v_a[p]);
                    sum = __dadd_rn(sum, alpha == 1.0 ? a : pow(a, alpha));
                }
                rs[i] = sum < SCALING_EPSILON ? 1.0 : 1.0 / sqrt(sum);
            } else {
                double mx = 0.0;
                for (int32_t p = rp_a[i]; p < rp_a[i + 1]; ++p) {
                    const double a = fabs(v_a[p]);
                    if (a > mx) mx = a;
                }
                rs[i] = mx < SCALING_EPSILON ? 1.0 : 1.0 / sqrt(mx);
            }
        }
        for (int32_t j = t; j < n; j += kScaleTinyThreads) {
            if (pc) {
                const double e = 2.0 - alpha;
                double sum = 0.0;
                for (int32_t p = rp_t[j]; p < rp_t[j + 1]; ++p) {
                    const double a = fabs(v_t[p]);
                    sum = __dadd_rn(sum, e == 1.0 ? a : pow(a, e));
                }
                cs[j] = sum < SCALING_EPSILON ? 1.0 : 1.0 / sqrt(sum);
            } else {
                double mx = 0.0;
                for (int32_t p = rp_t[j]; p < rp_t[j + 1]; ++p) {
                    const double a = fabs(v_t[p]);
                    if (a > mx) mx = a;
                }
                cs[j] = mx < SCALING_EPSILON ? 1.0 : 1.0 / sqrt(mx);
            }
        }
        __syncthreads();
        for (int32_t i = t; i < m; i += kScaleTinyThreads)
            for (int32_t p = rp_a[i]; p < rp_a[i + 1]; ++p)
                v_a[p] = __dmul_rn(v_a[p], __dmul_rn(rs[i], cs[ci_a[p]]));
        for (int32_t j = t; j < n; j += kScaleTinyThreads)
            for (int32_t p = rp_t[j]; p < rp_t[j + 1]; ++p)
                v_t[p] = __dmul_rn(v_t[p], __dmul_rn(rs[ci_t[p]], cs[j]));
        for (int32_t i = t; i < m; i += kScaleTinyThreads) D_r[i] = __dmul_rn(D_r[i], rs[i]);
        for (int32_t j = t; j < n; j += kScaleTinyThreads) D_c[j] = __dmul_rn(D_c[j], cs[j]);
        __syncthreads();
    }
}

static int blocks_for(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 8192))); }

__global__ void fill_kernel(double* __restrict__ d, int64_t n, double v) {
    for (int64_t i = blockIdx.x * 256 + threadIdx.x; i < n; i += int64_t(gridDim.x) * 256) d[i] = v;
}

void scale_uploaded(const DeviceMatrix& M, DeviceArena& ar, int32_t ruiz_iterations, double alpha,
                    bool rescale, const double* const vin[5], double* const vout[5], double* D_r,
                    double* D_c, double* scales, cudaStream_t st) {
    const int32_t m = static_cast<int32_t>(M.L.M), n = static_cast<int32_t>(M.L.N);
    double* rs = ar.alloc<double>(m);
    double* cs = ar.alloc<double>(n);
    const int bm = blocks_for(m), bn = blocks_for(n);
    if (m) fill_kernel<<<bm, 256, 0, st>>>(D_r, m, 1.0);
    if (n) fill_kernel<<<bn, 256, 0, st>>>(D_c, n, 1.0);
    fill_kernel<<<1, 256, 0, st>>>(scales, 2, 1.0);
    auto apply = [&]() {
        if (m) apply_scale_kernel<<<bm, 256, 0, st>>>(M.rp_a, M.ci_a, M.v64_a, m, rs, cs, 0);
        if (n) apply_scale_kernel<<<bn, 256, 0, st>>>(M.rp_t, M.ci_t, M.v64_t, n, rs, cs, 1);
        if (m) mul_inplace_kernel<<<bm, 256, 0, st>>>(D_r, rs, m);
        if (n) mul_inplace_kernel<<<bn, 256, 0, st>>>(D_c, cs, n);
    };
    const char* te = std::getenv("PDFP_TINY");
    const bool tiny = !(te && te[0] == '0') && static_cast<int64_t>(m) + n <= kScaleTinyMaxDim &&
                      M.L.NNZ <= kScaleTinyMaxNnz && m > 0 && n > 0;
    if (tiny) {  // every round in one launch
        scale_tiny_kernel<<<1, kScaleTinyThreads, 0, st>>>(M.rp_a, M.ci_a, M.v64_a, M.rp_t, M.ci_t,
                                                           M.v64_t, m, n, std::max(ruiz_iterations, 0),
                                                           alpha, rs, cs, D_r, D_c);
    } else {
        for (int32_t it = 0; it < ruiz_iterations; ++it) {  // src/preconditioner.jl:36-49
            if (m) ruiz_scale_kernel<<<bm, 256, 0, st>>>(M.rp_a, M.v64_a, m, rs);
            if (n) ruiz_scale_kernel<<<bn, 256, 0, st>>>(M.rp_t, M.v64_t, n, cs);
            apply();
        }
        // Pock-Chambolle, src/preconditioner.jl:51-64
        if (m) pc_scale_kernel<<<bm, 256, 0, st>>>(M.rp_a, M.v64_a, m, alpha, rs);
        if (n) pc_scale_kernel<<<bn, 256, 0, st>>>(M.rp_t, M.v64_t, n, 2.0 - alpha, cs);
        apply();
    }
    // the scaled vectors and the optional bound/objective rescaling
    double* sq = ar.alloc<double>(2);
    const int bb = blocks_for(std::max(m, n));
    scale_vectors_kernel<<<bb, 256, 0, st>>>(vin[0], vin[1], vin[2], D_c, n, vin[3], vin[4], D_r, m,
                                             vout[0], vout[1], vout[2], vout[3], vout[4]);
    if (rescale) {
        rescale_norms_kernel<<<1, 64, 0, st>>>(vin[3], vin[4], vout[3], vout[4], m, vout[0], n, sq);
        rescale_apply_kernel<<<bb, 256, 0, st>>>(vin[1], vin[2], n, vin[3], vin[4], m, sq, vout[0],
                                                 vout[1], vout[2], vout[3], vout[4], scales);
    }
    PDFP_CK(cudaGetLastError());
}

void scale_problem_device(const pdfp_csr& A, const double* c, const double* var_lb,
                          const double* var_ub, const double* con_lb, const double* con_ub,
                          int32_t ruiz_iterations, double alpha, bool rescale, double* val_out,
                          double* c_out, double* var_lb_out, double* var_ub_out, double* con_lb_out,
                          double* con_ub_out, double* D_r_out, double* D_c_out, double* bound_scale,
                          double* objective_scale) {
    static const int32_t zero_rp = 0;
    const int32_t m = A.m, n = A.n;
    ProblemIn in{m, n, m > 0 ? A.row_ptr : &zero_rp, A.col_idx, A.val, nullptr};
    DeviceMatrix M;
    std::string msg = build_layout({in}, false, M.L);
    if (!msg.empty()) throw Error(E_INVALID, msg);
    DeviceArena ar;
    M.upload(ar, false);
    // inputs in one block: c, lb, ub (n each), con_lb, con_ub (m each), then the outputs,
    // D_c, D_r and the two scales
    const int64_t tot = 3 * int64_t(n) + 2 * int64_t(m);
    std::vector<double> hin(std::max<int64_t>(tot, 1));
    const double* src[5] = {c, var_lb, var_ub, con_lb, con_ub};
    const int64_t len[5] = {n, n, n, m, m};
    double* const din = ar.alloc<double>(hin.size());
    double* const dout = ar.alloc<double>(tot + n + m + 2);
    const double* vin[5];
    double* vout[5];
    int64_t off = 0;
    for (int k = 0; k < 5; ++k) {
        if (len[k]) std::copy(src[k], src[k] + len[k], hin.begin() + off);
        vin[k] = din + off;
        vout[k] = dout + off;
        off += len[k];
    }
    double* D_c = dout + tot;
    double* D_r = D_c + n;
    double* scales = D_r + m;
    if (tot) PDFP_CK(cudaMemcpy(din, hin.data(), sizeof(double) * tot, cudaMemcpyHostToDevice));
    scale_uploaded(M, ar, ruiz_iterations, alpha, rescale, vin, vout, D_r, D_c, scales, 0);
    PDFP_CK(cudaDeviceSynchronize());
    std::vector<double> hout(tot + n + m + 2);
    PDFP_CK(cudaMemcpy(hout.data(), dout, sizeof(double) * hout.size(), cudaMemcpyDeviceToHost));
    if (M.L.NNZ) PDFP_CK(cudaMemcpy(val_out, M.v64_a, sizeof(double) * M.L.NNZ, cudaMemcpyDeviceToHost));
    double* dst[5] = {c_out, var_lb_out, var_ub_out, con_lb_out, con_ub_out};
    off = 0;
    for (int k = 0; k < 5; ++k) {
        if (len[k]) std::copy(hout.begin() + off, hout.begin() + off + len[k], dst[k]);
        off += len[k];
    }
    if (n) std::copy(hout.begin() + tot, hout.begin() + tot + n, D_c_out);
    if (m) std::copy(hout.begin() + tot + n, hout.begin() + tot + n + m, D_r_out);
    *bound_scale = hout[tot + n + m];
    *objective_scale = hout[tot + n + m + 1];
}

double estimate_sv_device(const pdfp_csr& A, int32_t max_iterations, double tolerance,
                          int32_t* iterations) {
    static const int32_t zero_rp = 0;
    ProblemIn in{A.m, A.n, A.m > 0 ? A.row_ptr : &zero_rp, A.col_idx, A.val, nullptr};
    DeviceMatrix M;
    std::string msg = build_layout({in}, false, M.L);
    if (!msg.empty()) throw Error(E_INVALID, msg);
    DeviceArena ar;
    M.upload(ar, false);
    StageGeom gev{8, 8, 8, 0, 2, 32 * 1024, 2048};
    DeviceMatrix::Tiling ta = M.make_tiling(ar, false, gev);
    DeviceMatrix::Tiling tt = M.make_tiling(ar, true, gev);
    int dev = 0, sms = 148;
    PDFP_CK(cudaGetDevice(&dev));
    PDFP_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaStream_t s;
    PDFP_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    int32_t* err = ar.alloc<int32_t>(4);
    std::vector<int32_t> its;
    std::vector<double> r;
    try {
        r = power_iteration(M, ar, ta, tt, {1}, max_iterations, tolerance, s, sms, err, &its);
    } catch (...) {
        cudaStreamDestroy(s);
        throw;
    }
    cudaStreamDestroy(s);
    if (iterations) *iterations = its.empty() ? 0 : its[0];
    return r[0];
}

}  // namespace pdfp
