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
// order).  The two norms of the optional rescaling are tree reductions.
#include <algorithm>
#include <cmath>
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

static int blocks_for(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 8192))); }

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
    double* D_r = ar.alloc<double>(m);
    double* D_c = ar.alloc<double>(n);
    double* rs = ar.alloc<double>(m);
    double* cs = ar.alloc<double>(n);
    std::vector<double> ones_m(m, 1.0), ones_n(n, 1.0);
    if (m) PDFP_CK(cudaMemcpy(D_r, ones_m.data(), sizeof(double) * m, cudaMemcpyHostToDevice));
    if (n) PDFP_CK(cudaMemcpy(D_c, ones_n.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    const int bm = blocks_for(m), bn = blocks_for(n);
    auto apply = [&]() {
        if (m) apply_scale_kernel<<<bm, 256>>>(M.rp_a, M.ci_a, M.v64_a, m, rs, cs, 0);
        if (n) apply_scale_kernel<<<bn, 256>>>(M.rp_t, M.ci_t, M.v64_t, n, rs, cs, 1);
        if (m) mul_inplace_kernel<<<bm, 256>>>(D_r, rs, m);
        if (n) mul_inplace_kernel<<<bn, 256>>>(D_c, cs, n);
    };
    for (int32_t it = 0; it < ruiz_iterations; ++it) {  // src/preconditioner.jl:36-49
        if (m) ruiz_scale_kernel<<<bm, 256>>>(M.rp_a, M.v64_a, m, rs);
        if (n) ruiz_scale_kernel<<<bn, 256>>>(M.rp_t, M.v64_t, n, cs);
        apply();
    }
    // Pock-Chambolle, src/preconditioner.jl:51-64
    if (m) pc_scale_kernel<<<bm, 256>>>(M.rp_a, M.v64_a, m, alpha, rs);
    if (n) pc_scale_kernel<<<bn, 256>>>(M.rp_t, M.v64_t, n, 2.0 - alpha, cs);
    apply();
    PDFP_CK(cudaGetLastError());
    PDFP_CK(cudaDeviceSynchronize());

    const int64_t nnz = M.L.NNZ;
    std::vector<double> hDr(m), hDc(n);
    if (m) PDFP_CK(cudaMemcpy(hDr.data(), D_r, sizeof(double) * m, cudaMemcpyDeviceToHost));
    if (n) PDFP_CK(cudaMemcpy(hDc.data(), D_c, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (nnz) PDFP_CK(cudaMemcpy(val_out, M.v64_a, sizeof(double) * nnz, cudaMemcpyDeviceToHost));
    // scaled vectors, src/preconditioner.jl:66-70
    for (int32_t j = 0; j < n; ++j) {
        c_out[j] = c[j] * hDc[j];
        var_lb_out[j] = std::isfinite(var_lb[j]) ? var_lb[j] / hDc[j] : var_lb[j];
        var_ub_out[j] = std::isfinite(var_ub[j]) ? var_ub[j] / hDc[j] : var_ub[j];
        D_c_out[j] = hDc[j];
    }
    for (int32_t i = 0; i < m; ++i) {
        con_lb_out[i] = std::isfinite(con_lb[i]) ? con_lb[i] * hDr[i] : con_lb[i];
        con_ub_out[i] = std::isfinite(con_ub[i]) ? con_ub[i] * hDr[i] : con_ub[i];
        D_r_out[i] = hDr[i];
    }
    double bs = 1.0, os = 1.0;
    if (rescale) {  // src/preconditioner.jl:72-96
        double bound_sq = 0.0;
        for (int32_t i = 0; i < m; ++i) {
            const bool flo = std::isfinite(con_lb[i]), fhi = std::isfinite(con_ub[i]);
            const double lo = con_lb_out[i], hi = con_ub_out[i];
            if (flo && (!fhi || std::fabs(lo - hi) > SCALING_EPSILON)) bound_sq += lo * lo;
            if (fhi) bound_sq += hi * hi;
        }
        double csq = 0.0;
        for (int32_t j = 0; j < n; ++j) csq += c_out[j] * c_out[j];
        bs = 1.0 / (std::sqrt(bound_sq) + 1.0);
        os = 1.0 / (std::sqrt(csq) + 1.0);
        for (int32_t i = 0; i < m; ++i) {
            if (std::isfinite(con_lb[i])) con_lb_out[i] *= bs;
            if (std::isfinite(con_ub[i])) con_ub_out[i] *= bs;
        }
        for (int32_t j = 0; j < n; ++j) {
            if (std::isfinite(var_lb[j])) var_lb_out[j] *= bs;
            if (std::isfinite(var_ub[j])) var_ub_out[j] *= bs;
            c_out[j] *= os;
        }
    }
    *bound_scale = bs;
    *objective_scale = os;
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
