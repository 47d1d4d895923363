// power.cuh -- estimate_max_singular_value (src/preconditioner.jl:108-125) on the device.
//
// Power iteration on A A' in the row space, batched over the instances of a
// packed matrix, every instance with its own convergence test.  One iteration
// is: nxt = eig / ||eig||; dual = A' nxt; eig = A dual; sigma^2 = <nxt, eig>;
// nxt = eig - sigma^2 nxt; stop when ||nxt|| < tolerance.  The sparse products
// run on the tile engine in FP64 and sum each row in ascending storage order.
#pragma once
#include "device.hpp"
#include "kernels.cuh"

namespace pdfp {

struct PowerBufs {
    double *eig, *nxt, *dual;
    double* part;  // A-eval tiles x 2
    PowerState* ps;
};

struct PiNormalize {  // nxt = eig / nrm
    PowerBufs b;
    const int32_t* row_off;
    __device__ bool active(int p) const { return !b.ps[p].done; }
    __device__ int32_t begin(int p) const { return row_off[p]; }
    __device__ int32_t end(int p) const { return row_off[p + 1]; }
    __device__ void elem(int p, int32_t i) const { b.nxt[i] = b.eig[i] / b.ps[p].nrm; }
};

template <int NTHREADS>
struct PiColOp {  // dual = A' nxt
    using MT = double;
    using VT = double;
    using AT = double;
    using GT = double;
    struct TileP {
        int32_t d;
    };
    static constexpr int NT = NTHREADS, NV = 1, NVEC = 0, NP = 0;
    PowerBufs b;
    const double* val;
    int32_t* errp;
    __device__ const double* values() const { return val; }
    __device__ const double* staged(int) const { return nullptr; }
    __device__ int32_t* err() const { return errp; }
    __device__ bool active(int p) const { return !b.ps[p].done; }
    __device__ TileP tile_params(int) const { return TileP{0}; }
    __device__ void gather(int32_t c, double (&g)[1]) const { g[0] = b.nxt[c]; }
    __device__ void row(int32_t j, int32_t, int, const TileP&, const double* const*,
                        const double (&s)[1], double*) const {
        b.dual[j] = s[0];
    }
    __device__ void write_partials(int32_t, const double*) const {}
};

template <int NTHREADS>
struct PiRowOp {  // eig = A dual; partial <nxt, eig>
    using MT = double;
    using VT = double;
    using AT = double;
    using GT = double;
    struct TileP {
        int32_t d;
    };
    static constexpr int NT = NTHREADS, NV = 1, NVEC = 0, NP = 1;
    PowerBufs b;
    const double* val;
    int32_t* errp;
    __device__ const double* values() const { return val; }
    __device__ const double* staged(int) const { return nullptr; }
    __device__ int32_t* err() const { return errp; }
    __device__ bool active(int p) const { return !b.ps[p].done; }
    __device__ TileP tile_params(int) const { return TileP{0}; }
    __device__ void gather(int32_t c, double (&g)[1]) const { g[0] = b.dual[c]; }
    __device__ void row(int32_t i, int32_t, int, const TileP&, const double* const*,
                        const double (&s)[1], double* acc) const {
        b.eig[i] = s[0];
        acc[0] += b.nxt[i] * s[0];
    }
    __device__ void write_partials(int32_t t, const double* acc) const {
        b.part[t * 2] = acc[0];
        b.part[t * 2 + 1] = 0.0;
    }
};

struct PiDotFin {
    static constexpr int NA = 2, NB = 0;
    const int32_t* ta0;
    const double* pa;
    const int32_t* tb0;
    const double* pb;
    PowerBufs b;
    __device__ bool active(int p) const { return !b.ps[p].done; }
    __device__ void finalize(int p, const double* a) const { b.ps[p].sigma_sq = a[0]; }
};

struct PiResRows {  // nxt = eig - sigma^2 nxt; partials ||nxt||^2, ||eig||^2
    static constexpr int NP = 2;
    PowerBufs b;
    __device__ bool active(int p) const { return !b.ps[p].done; }
    __device__ void row(int32_t i, int p, double* acc) const {
        const double e = b.eig[i];
        const double v = sub_rn(e, mul_rn(b.ps[p].sigma_sq, b.nxt[i]));
        b.nxt[i] = v;
        acc[0] += v * v;
        acc[1] += e * e;
    }
    __device__ void write_partials(int32_t t, const double* acc) const {
        b.part[t * 2] = acc[0];
        b.part[t * 2 + 1] = acc[1];
    }
};

struct PiResFin {
    static constexpr int NA = 2, NB = 0;
    const int32_t* ta0;
    const double* pa;
    const int32_t* tb0;
    const double* pb;
    PowerBufs b;
    __device__ bool active(int p) const { return !b.ps[p].done; }
    __device__ void finalize(int p, const double* a) const {
        PowerState& s = b.ps[p];
        s.it += 1;
        s.res_sq = a[0];
        if (sqrt(a[0]) < s.tol) {
            s.done = 1;
        } else if (s.it >= s.max_it) {
            s.done = 1;
        } else {
            s.nrm = sqrt(a[1]);
            if (s.nrm == 0.0) s.done = 1;
        }
    }
};

struct PiInitRows {  // partial ||eig||^2 of the start vector
    static constexpr int NP = 2;
    PowerBufs b;
    __device__ bool active(int p) const { return !b.ps[p].done; }
    __device__ void row(int32_t i, int, double* acc) const { acc[0] += b.eig[i] * b.eig[i]; }
    __device__ void write_partials(int32_t t, const double* acc) const {
        b.part[t * 2] = acc[0];
        b.part[t * 2 + 1] = 0.0;
    }
};

struct PiInitFin {
    static constexpr int NA = 2, NB = 0;
    const int32_t* ta0;
    const double* pa;
    const int32_t* tb0;
    const double* pb;
    PowerBufs b;
    __device__ bool active(int p) const { return !b.ps[p].done; }
    __device__ void finalize(int p, const double* a) const {
        PowerState& s = b.ps[p];
        s.nrm = sqrt(a[0]);
        s.it = 0;
        s.sigma_sq = 1.0;
        if (s.max_it <= 0 || s.nrm == 0.0) s.done = 1;
    }
};

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

// Host driver: estimates ||A_p||_2 for every instance p with run[p] != 0 and
// returns the estimates (NaN where not run).  `start` holds the start vectors
// in packed row order.  Uses the A and A' eval tilings given.
std::vector<double> power_iteration(const DeviceMatrix& M, DeviceArena& ar,
                                    const DeviceMatrix::Tiling& ta,
                                    const DeviceMatrix::Tiling& tt,
                                    const std::vector<int>& run, int32_t max_iterations,
                                    double tolerance, cudaStream_t stream, int num_sms,
                                    int32_t* err_d, std::vector<int32_t>* iters_out);

// Deterministic start vector: SplitMix64 stream from `seed`, two uniforms per
// entry, Box-Muller cosine branch (stands in for randn(MersenneTwister(seed), m)).
void normal_vector(uint64_t seed, int64_t m, double* out);

}  // namespace pdfp
