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
