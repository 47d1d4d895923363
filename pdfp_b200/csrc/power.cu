// power.cu -- host driver of the batched power iteration.
#include <algorithm>
#include <cmath>
#include <cstdlib>

#include "power.cuh"

namespace pdfp {

static uint64_t splitmix64(uint64_t& state) {
    uint64_t z = (state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void normal_vector(uint64_t seed, int64_t m, double* out) {
    uint64_t st = seed;
    const double two_pi = 6.283185307179586;
    for (int64_t i = 0; i < m; ++i) {
        double u1 = (static_cast<double>(splitmix64(st) >> 11) + 0.5) * 0x1.0p-53;
        double u2 = (static_cast<double>(splitmix64(st) >> 11) + 0.5) * 0x1.0p-53;
        out[i] = std::sqrt(-2.0 * std::log(u1)) * std::cos(two_pi * u2);
    }
}

std::vector<double> power_iteration(const DeviceMatrix& M, DeviceArena& ar,
                                    const DeviceMatrix::Tiling& ta,
                                    const DeviceMatrix::Tiling& tt, const std::vector<int>& run,
                                    int32_t max_iterations, double tolerance,
                                    cudaStream_t stream, int num_sms, int32_t* err_d,
                                    std::vector<int32_t>* iters_out) {
    const HostLayout& L = M.L;
    const int K = L.K;
    std::vector<double> result(K, NAN);
    bool any = false;
    for (int p = 0; p < K; ++p) any = any || run[p];
    if (!any) return result;

    DeviceArena tmp;
    PowerBufs b;
    b.eig = tmp.alloc<double>(L.M);
    b.nxt = tmp.alloc<double>(L.M);
    b.dual = tmp.alloc<double>(L.N);
    b.part = tmp.alloc<double>(2 * static_cast<size_t>(std::max(ta.dev.n_tiles, 1)));
    b.ps = tmp.alloc<PowerState>(K);

    // start vectors in the caller's row order, permuted to packed order
    std::vector<double> start(L.M, 0.0);
    std::vector<double> buf;
    for (int p = 0; p < K; ++p) {
        const int32_t r0 = L.row_off[p], m = L.row_off[p + 1] - r0;
        buf.assign(m, 0.0);
        normal_vector(20240517ull, m, buf.data());
        for (int32_t i = 0; i < m; ++i) start[r0 + i] = buf[L.row_orig[r0 + i]];
    }
    if (L.M) PDFP_CK(cudaMemcpyAsync(b.eig, start.data(), sizeof(double) * L.M, cudaMemcpyHostToDevice, stream));
    std::vector<PowerState> ps(K);
    for (int p = 0; p < K; ++p) {
        ps[p] = PowerState{};
        ps[p].tol = tolerance;
        ps[p].max_it = max_iterations;
        ps[p].done = run[p] ? 0 : 1;
        ps[p].sigma_sq = 1.0;
    }
    PDFP_CK(cudaMemcpyAsync(b.ps, ps.data(), sizeof(PowerState) * K, cudaMemcpyHostToDevice, stream));

    // small instances: one launch for the whole iteration (power_tiny_kernel)
    bool tiny = true;
    int64_t smem_doubles = 1;
    for (int p = 0; p < K && tiny; ++p) {
        const int64_t mp = L.row_off[p + 1] - L.row_off[p], np = L.col_off[p + 1] - L.col_off[p];
        const int64_t nz = L.A.rp[L.row_off[p + 1]] - L.A.rp[L.row_off[p]];
        if (mp + np > kPowerTinyMaxDim || nz > kPowerTinyMaxNnz) tiny = false;
        smem_doubles = std::max<int64_t>(smem_doubles, 2 * mp + np);
    }
    if (const char* te = std::getenv("PDFP_TINY")) tiny = tiny && te[0] != '0';
    if (tiny) {
        const size_t smem = sizeof(double) * static_cast<size_t>(smem_doubles);
        PDFP_CK(cudaFuncSetAttribute(power_tiny_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem)));
        power_tiny_kernel<<<K, kPowerTinyThreads, smem, stream>>>(b, M.rp_t, M.ci_t, M.v64_t, M.rp_a,
                                                                   M.ci_a, M.v64_a, M.row_off, M.col_off);
        PDFP_CK(cudaGetLastError());
        std::vector<PowerState> hs(K);
        PDFP_CK(cudaMemcpyAsync(hs.data(), b.ps, sizeof(PowerState) * K, cudaMemcpyDeviceToHost, stream));
        PDFP_CK(cudaStreamSynchronize(stream));
        if (iters_out) iters_out->assign(K, 0);
        for (int p = 0; p < K; ++p) {
            if (!run[p]) continue;
            const double s2 = hs[p].sigma_sq;
            result[p] = std::isnan(s2) ? s2 : std::sqrt(s2 > 0.0 ? s2 : 0.0);
            if (iters_out) (*iters_out)[p] = hs[p].it;
        }
        return result;
    }

    launch_rows(ta.dev, PiInitRows{b}, stream);
    launch_finalize(K, PiInitFin{ta.inst_tile0, b.part, nullptr, nullptr, b}, stream);

    constexpr int NT = 256;
    PiColOp<NT> col{b, M.v64_t, err_d};
    PiRowOp<NT> row{b, M.v64_a, err_d};
    const int gcol = tile_grid<PiColOp<NT>>(tt.dev, num_sms);
    const int grow = tile_grid<PiRowOp<NT>>(ta.dev, num_sms);
    PiNormalize nrm{b, M.row_off};

    // windows of W iterations, captured once as a graph
    const int W = 25;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    PDFP_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    for (int w = 0; w < W; ++w) {
        launch_elem(K, M.max_m, nrm, stream);
        launch_tile(tt.dev, col, gcol, stream);
        launch_tile(ta.dev, row, grow, stream);
        launch_finalize(K, PiDotFin{ta.inst_tile0, b.part, nullptr, nullptr, b}, stream);
        launch_rows(ta.dev, PiResRows{b}, stream);
        launch_finalize(K, PiResFin{ta.inst_tile0, b.part, nullptr, nullptr, b}, stream);
    }
    PDFP_CK(cudaStreamEndCapture(stream, &graph));
    PDFP_CK(cudaGraphInstantiate(&exec, graph, 0));
    std::vector<PowerState> hs(K);
    const int max_windows = max_iterations / W + 2;
    for (int wi = 0; wi < max_windows; ++wi) {
        PDFP_CK(cudaGraphLaunch(exec, stream));
        PDFP_CK(cudaMemcpyAsync(hs.data(), b.ps, sizeof(PowerState) * K, cudaMemcpyDeviceToHost, stream));
        PDFP_CK(cudaStreamSynchronize(stream));
        bool all = true;
        for (int p = 0; p < K; ++p) all = all && hs[p].done;
        if (all) break;
    }
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    PDFP_CK(cudaMemcpyAsync(hs.data(), b.ps, sizeof(PowerState) * K, cudaMemcpyDeviceToHost, stream));
    PDFP_CK(cudaStreamSynchronize(stream));
    if (iters_out) iters_out->assign(K, 0);
    for (int p = 0; p < K; ++p) {
        if (!run[p]) continue;
        double s2 = hs[p].sigma_sq;
        // sqrt(max(sigma_sq, 0)) with Julia's max (NaN propagates)
        result[p] = std::isnan(s2) ? s2 : std::sqrt(s2 > 0.0 ? s2 : 0.0);
        if (iters_out) (*iters_out)[p] = hs[p].it;
    }
    return result;
}

}  // namespace pdfp
