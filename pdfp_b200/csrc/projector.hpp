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

    // unscaled = true: the vector is in the caller's original units and the
    // device applies the instance's column scale D_c (set_col_scale) itself
    void set_col_scale(int p, const double* dc);
    void set_x(int p, const double* x, bool unscaled = false);
    void set_target(int p, const double* xt, bool unscaled = false);
    void warm_start(int p);
    // any = false: until every instance has stopped.  any = true: until at least one
    // instance that was running has stopped (at a window boundary); the others keep
    // running, and a later call with resume[p] set continues instance p from there
    // (its parameters and counters as they were; params[p] is then not read).
    void solve(const pdfp_params* params, const double* primal_weights, pdfp_result* results,
               const uint8_t* resume = nullptr, bool any = false);
    void get_vector(int p, int which, double* out, bool unscaled = false);
    void profile_step(int iterations, float* ms_primal, float* ms_dual, double* bytes_primal,
                      double* bytes_dual);
    // Mixed precision: the FP32 phase of an instance ends, and the FP64 polish takes
    // over, after stall_evaluations evaluations without a 10% KKT improvement while
    // above tolerance (0: never), or once its residuals reach fp32_floor (relative)
    // while the requested tolerance is tighter.
    void set_polish(int32_t stall_evaluations, double fp32_floor);
    // Chosen step-kernel configurations: {stage_bytes, threads, tiles} for the
    // A'-side and the A-side kernel of the handle's base precision.
    void tuning(int32_t* out) const;
    void tuning_stages(int32_t* out) const;
    void tuning_blocks(int32_t* out) const;
    void tuning_reducers(int32_t* out) const;
    // The A-side step of the FP32 steps with its long rows by column segment:
    // {segments, long-row threshold}, {0, 0} when it has none.
    void tuning_seg(int32_t* out) const;
    // 0: per-step launches (graph), 1: cooperative row passes, 2: cooperative vec
    // window, 3: whole windows per small member in one launch
    int32_t window_form() const { return tiny_ ? 3 : vecwin_ ? 2 : medium_ ? 1 : 0; }
    // Every autotuner measurement: ms[i] and cfg[7i..7i+6] = {side (0: A', 1: A),
    // stage bytes, gatherer threads, gather policy, stages, blocks per SM cap,
    // reducer threads}; side 2: the A side with its long rows by column segment,
    // {2, segments, long-row threshold, gather policy of the other rows, the
    // partials' stages, stage bytes and threads per role}; returns the count.
    int tuning_table(float* ms, int32_t* cfg, int cap) const;
    void set_kernel_timing(bool on);

  private:
    // One side of the PDHG step: its tile geometry, block size and tiling.
    struct StepSide {
        int engine = 0;  // 0: tile engine (tile_spmv.cuh), 1: flat engine (flat_spmv.cuh),
                         // 2: vec engine (vec_spmv.cuh; FP32 steps)
        int qpt = 2;     // flat engine: quads (4 nonzeros) per thread and tile, 1 or 2
        int lane_nnz = 4;  // vec engine: target nonzeros per lane of a row
        VecDev vec{};      // vec engine: its items
        // A side, FP32, tile engine: rows of at least seg_long nonzeros regrouped by
        // column segment (seg_spmv.cuh; seg_nseg segments, 0: off); the tiling then
        // covers the other rows
        int seg_nseg = 0, seg_long = 0;
        int seg_stage = 16 * 1024, seg_nt = 128, seg_stages = 3;  // the partials' tile engine
        int seg_bps = 1;  // its blocks per segment
        SegDev segd{};
        DeviceMatrix::Tiling segt;  // tiling of the (segment, long row) pairs
        int stages = 4;  // tile engine: shared-memory stages per block, 2..4
        int max_blocks = 0;  // tile engine: resident blocks per SM cap (0: as many as fit)
        int carveout = -1;   // preferred shared-memory share of L1 for that cap (percent)
        bool half_red = false;  // tile engine: nt / 2 reducer threads (FP32 steps)
        int stage_bytes = 32 * 1024;
        int nt = 256;
        DeviceMatrix::Tiling tiling;
        int grid = 0;
        int gather_l2 = 0;
        float tuned_ms = 0.f;
    };
    struct TuneRow {
        int side, stage, nt, l2;  // nt = 0: the flat engine; nt = 32: the vec engine (stage = lane_nnz)
        int stages;
        int max_blocks;
        int reducers;
        float ms;
    };
    std::vector<TuneRow> tune_table_;
    template <typename T>
    IterVecs<T>& vecs();
    template <typename T, bool MAJOR>
    void launch_primal(const StepSide& s, int k, bool overlap = false);
    template <typename T, bool MAJOR>
    void launch_dual(const StepSide& s, int k, bool overlap = false);
    void prepare_side(StepSide& s, bool primal, bool f32);
    void autotune(bool f32);
    void check_instance(int p) const;
    void check_unscaled(int p) const;
    void stage_cols(int p, const double* src, const char* what);
    template <typename T>
    void load_cols(int p, T* dst, T* dst2, bool unscaled);
    void ensure_step_sizes(int32_t sv_max_iterations, double sv_tolerance);
    void record_window(int freq, bool with32, bool with64);
    static constexpr int kSplitSteps = 8;  // timing mode: single steps timed per kernel per window
    struct TimingPlan {
        int run_a = 0, run_b = 0;  // the timed run of minor steps [run_a, run_b)
        int split[kSplitSteps] = {};
        int n_split = 0;
    };
    static TimingPlan timing_plan(int freq);
    template <typename T>
    void launch_tiny_steps(int i0, int i1);
    template <typename T>
    void launch_medium_steps(int i0, int i1);
    cudaGraphExec_t window_graph(int freq, bool with32, bool with64);
    void prepare_window();
    void run_window(int freq, bool with32, bool with64);
    bool window_ready_ = false;  // the whole-window kernels' launch shape is set
    size_t tiny_smem32_ = 0, tiny_smem64_ = 0;      // their dynamic shared memory
    bool tiny_staged32_ = false, tiny_staged64_ = false;  // members copied into shared memory

    int precision_;
    int K_ = 0;
    int num_sms_ = 148;
    int max_smem_sm_ = 233472;  // unified L1 / shared memory usable as shared, per SM
    int max_smem_block_ = 232448;  // shared memory one block may opt in to
    int seg_mode_ = 0;  // segmented long rows: -1 autotuned, 0 off, > 0 that many segments
    int seg_long_ = 0;   // with seg_mode_ > 0: the long-row threshold
    int seg_cfg_[4] = {16 * 1024, 128, 3, 1};  // and the partials' stage bytes, threads, stages,
                                               // blocks per segment
    cudaStream_t stream_ = nullptr;
    DeviceArena ar_;
    DeviceMatrix M_;
    DeviceMatrix::Tiling ev_t_, ev_a_;
    StepSide p32_, d32_, p64_, d64_;
    IterVecs<double> v64_{};
    IterVecs<float> v32_{};
    EvalData ed_{};
    double* row_unscale_ = nullptr;
    double *part_col_ = nullptr, *part_row_ = nullptr;
    InstState* st_ = nullptr;
    InstFlags* flags_ = nullptr;
    InstFlags* flags_h_ = nullptr;
    InstState* st_h_ = nullptr;       // page-locked copy of the states, read with each poll
    std::vector<int64_t> host_total_;  // PDHG iterations per instance as of the last solve
    std::vector<uint8_t> last_running_;  // still running when the last solve returned
    int32_t* any_stop_ = nullptr;      // device flag: an instance stopped (any-solves)
    int32_t* any_stop_cur_ = nullptr;  // any_stop_ during an any-solve, else null
    bool totals_known_ = true;         // host_total_ matches the device
    int32_t* err_ = nullptr;
    SolveParams* sp_ = nullptr;
    double* stage_ = nullptr;
    double* host_stage_ = nullptr;         // page-locked copy of a short caller vector
    size_t host_stage_bytes_ = 0;
    cudaEvent_t host_stage_ev_ = nullptr;  // its last copy to stage_ has left it
    double* col_scale_ = nullptr;  // D_c in packed column order, once set_col_scale ran
    std::vector<bool> has_col_scale_;
    int32_t* nan_seen_ = nullptr;
    int32_t* nan_seen_h_ = nullptr;
    std::vector<int> vec_mode_;
    std::vector<bool> has_unscale_;
    std::set<int> polished_;
    int32_t polish_enabled_ = 1;
    int32_t stall_limit_ = 10;   // evaluations without 10% KKT progress before the FP64 polish
    double fp32_floor_ = 1e-6;  // relative residual the FP32 phase aims for under a tighter tolerance
    struct Grids {
        int ec = 0, er = 0;
    } g_;
    std::map<int, cudaGraphExec_t> graphs_;
    bool timing_ = false;
    bool sv_ready_ = false;  // every instance holds its ||A||_2 estimate
    bool evict_first_ = true;  // step kernels stream the matrix L2 evict-first
    bool overlap_ = false;     // consecutive step launches overlap (programmatic launch)
    bool tiny_ = false;  // every member small: a window's minor steps run in one launch
    bool medium_ = false;  // a mid-sized handle: the minor steps in one cooperative launch
    int32_t *part_t_ = nullptr, *part_a_ = nullptr;  // each block's rows of A' and of A
    unsigned* gbar_ = nullptr;                          // the grid barrier's words
    bool vecwin_ = false;  // FP32 minor steps of a window in one cooperative vec launch
    int vecwin_grid_ = 0;  // its blocks (all resident)
    void launch_vec_window(int i0, int i1);
    cudaEvent_t tev_[2 + 3 * kSplitSteps] = {};  // timing mode: the run's two, then 3 per split step
    cudaEvent_t sev_[2] = {nullptr, nullptr};              // whole solve
};

}  // namespace pdfp
