// projector.hpp -- the PDFP projector handle (host side).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <set>
#include <vector>

#include "../../include/pdfp_b200.h"
#include "device.hpp"
#include "pdfp_ops.cuh"
#include "state.hpp"

namespace pdfp {

// One projection problem in the caller's numbering (scaled data).
struct ProblemData {
    int32_t m, n;
    const int32_t* rp;
    const int32_t* ci;
    const double* v;
    const double* b;
    const uint8_t* is_eq;
    const uint8_t* is_int;
    const double* lb;
    const double* ub;
    const double* w;
    const double* row_unscale;
};

class Projector {
  public:
    Projector(const std::vector<ProblemData>& probs, int precision);
    ~Projector();
    Projector(const Projector&) = delete;
    Projector& operator=(const Projector&) = delete;

    int instances() const { return K_; }
    int rows(int p) const { return M_.L.row_off[p + 1] - M_.L.row_off[p]; }
    int cols(int p) const { return M_.L.col_off[p + 1] - M_.L.col_off[p]; }

    void set_x(int p, const double* x);
    void set_target(int p, const double* xt);
    void warm_start(int p);
    void solve(const pdfp_params* params, const double* primal_weights, pdfp_result* results);
    void get_vector(int p, int which, double* out);
    void profile_step(int iterations, float* ms_primal, float* ms_dual, double* bytes_primal,
                      double* bytes_dual);
    void set_polish(bool on) { polish_enabled_ = on ? 1 : 0; }

  private:
    void check_instance(int p) const;
    void ensure_step_sizes(int32_t sv_max_iterations, double sv_tolerance);
    void record_window(int freq, bool with32, bool with64);
    cudaGraphExec_t window_graph(int freq, bool with32, bool with64);

    int precision_;
    int K_ = 0;
    int num_sms_ = 148;
    cudaStream_t stream_ = nullptr;
    DeviceArena ar_;
    DeviceMatrix M_;
    DeviceMatrix::Tiling it_t_, it_a_, it64_t_, it64_a_, ev_t_, ev_a_;
    IterVecs<double> v64_{};
    IterVecs<float> v32_{};
    EvalData ed_{};
    double* row_unscale_ = nullptr;
    double *part_col_ = nullptr, *part_row_ = nullptr;
    InstState* st_ = nullptr;
    InstFlags* flags_ = nullptr;
    InstFlags* flags_h_ = nullptr;
    int32_t* err_ = nullptr;
    SolveParams* sp_ = nullptr;
    double* stage_ = nullptr;
    std::vector<int> vec_mode_;
    std::vector<bool> has_unscale_;
    std::set<int> polished_;
    int32_t polish_enabled_ = 1;
    struct Grids {
        int p32 = 0, d32 = 0, p64 = 0, d64 = 0, ec = 0, er = 0;
    } g_;
    std::map<int, cudaGraphExec_t> graphs_;
};

}  // namespace pdfp
