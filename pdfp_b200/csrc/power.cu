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

// ---- small instances: the whole power iteration in one launch --------------------
//
// When every instance has at most kPowerTinyMaxDim rows + columns and
// kPowerTinyMaxNnz nonzeros, each iteration's six launches would be latency-bound:
// instead one block per instance runs every iteration, with eig, nxt and dual in
// shared memory, the same steps in the same order (PiInitFin, then PiNormalize,
// PiColOp, PiRowOp, PiDotFin, PiResRows, PiResFin per iteration), rows summed
// sequentially in storage order and the dot products reduced in a fixed order.
// The loop ends by the instance's own test or its iteration cap.
constexpr int kPowerTinyThreads = 256;
constexpr int64_t kPowerTinyMaxDim = 4096;
constexpr int64_t kPowerTinyMaxNnz = 65536;

// Sums (a, c) over the block (fixed order); every thread gets the totals.
__device__ __forceinline__ void power_block_sum2(double& a, double& c, double* red) {
    for (int o = 16; o > 0; o >>= 1) {
        a = add_rn(a, __shfl_xor_sync(0xffffffffu, a, o));
        c = add_rn(c, __shfl_xor_sync(0xffffffffu, c, o));
    }
    __syncthreads();  // the previous sum's readers are done with red
    if ((threadIdx.x & 31) == 0) {
        red[2 * (threadIdx.x >> 5)] = a;
        red[2 * (threadIdx.x >> 5) + 1] = c;
    }
    __syncthreads();
    a = 0.0;
    c = 0.0;
    for (int w = 0; w < kPowerTinyThreads / 32; ++w) {
        a = add_rn(a, red[2 * w]);
        c = add_rn(c, red[2 * w + 1]);
    }
}

__global__ void __launch_bounds__(kPowerTinyThreads)
    power_tiny_kernel(PowerBufs b, const int32_t* __restrict__ rp_t, const int32_t* __restrict__ ci_t,
                      const double* __restrict__ v_t, const int32_t* __restrict__ rp_a,
                      const int32_t* __restrict__ ci_a, const double* __restrict__ v_a,
                      const int32_t* __restrict__ row_off, const int32_t* __restrict__ col_off) {
    extern __shared__ double sm[];  // eig[m], nxt[m], dual[n] of this instance
    __shared__ double red[2 * (kPowerTinyThreads / 32)];
    __shared__ PowerState st;
    const int p = blockIdx.x;
    if (threadIdx.x == 0) st = b.ps[p];
    __syncthreads();
    if (st.done) return;  // block-uniform
    const int32_t r0 = row_off[p], m = row_off[p + 1] - r0;
    const int32_t c0 = col_off[p], n = col_off[p + 1] - c0;
    double* eig = sm;
    double* nxt = sm + m;
    double* dual = sm + 2 * m;
    const int t = threadIdx.x;

    // PiInitRows / PiInitFin
    double a = 0.0, c = 0.0;
    for (int32_t i = t; i < m; i += kPowerTinyThreads) {
        const double e = b.eig[r0 + i];
        eig[i] = e;
        a += e * e;
    }
    power_block_sum2(a, c, red);
    if (t == 0) {
        st.nrm = sqrt(a);
        st.it = 0;
        st.sigma_sq = 1.0;
        if (st.max_it <= 0 || st.nrm == 0.0) st.done = 1;
    }
    __syncthreads();
    while (!st.done) {
        for (int32_t i = t; i < m; i += kPowerTinyThreads) nxt[i] = eig[i] / st.nrm;  // PiNormalize
        __syncthreads();
        for (int32_t j = t; j < n; j += kPowerTinyThreads) {  // PiColOp: dual = A' nxt
            const int32_t row = c0 + j;
            double sum = 0.0;
            for (int32_t k = rp_t[row]; k < rp_t[row + 1]; ++k)
                sum = add_rn(sum, mul_rn(v_t[k], nxt[ci_t[k] - r0]));
            dual[j] = sum;
        }
        __syncthreads();
        a = 0.0;
        c = 0.0;
        for (int32_t i = t; i < m; i += kPowerTinyThreads) {  // PiRowOp: eig = A dual, <nxt, eig>
            const int32_t row = r0 + i;
            double sum = 0.0;
            for (int32_t k = rp_a[row]; k < rp_a[row + 1]; ++k)
                sum = add_rn(sum, mul_rn(v_a[k], dual[ci_a[k] - c0]));
            eig[i] = sum;
            a += nxt[i] * sum;
        }
        power_block_sum2(a, c, red);
        const double sigma_sq = a;  // PiDotFin
        a = 0.0;
        c = 0.0;
        for (int32_t i = t; i < m; i += kPowerTinyThreads) {  // PiResRows
            const double e = eig[i];
            const double v = sub_rn(e, mul_rn(sigma_sq, nxt[i]));
            nxt[i] = v;
            a += v * v;
            c += e * e;
        }
        power_block_sum2(a, c, red);
        if (t == 0) {  // PiResFin
            st.sigma_sq = sigma_sq;
            st.it += 1;
            st.res_sq = a;
            if (sqrt(a) < st.tol) {
                st.done = 1;
            } else if (st.it >= st.max_it) {
                st.done = 1;
            } else {
                st.nrm = sqrt(c);
                if (st.nrm == 0.0) st.done = 1;
            }
        }
        __syncthreads();
    }
    if (t == 0) b.ps[p] = st;
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
