// api.cu -- the extern "C" entry points of libpdfp_b200.so (include/pdfp_b200.h).
//
// Every entry point catches the library's exceptions and returns a status
// code; the message is kept per thread for pdfp_last_error().
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>

#include "../../include/pdfp_b200.h"
#include "device.hpp"
#include "projector.hpp"
#include "mps.hpp"
#include "solvers.hpp"

namespace pdfp {
const char* last_error_cstr();
}

struct pdfp_handle {
    std::unique_ptr<pdfp::Projector> proj;
};

namespace {

template <class F>
int guarded(F&& f) {
    try {
        pdfp::set_last_error("");
        f();
        return PDFP_OK;
    } catch (const pdfp::Error& e) {
        pdfp::set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        pdfp::set_last_error("host allocation failed");
        return PDFP_E_NOMEM;
    } catch (const std::exception& e) {
        pdfp::set_last_error(e.what());
        return PDFP_E_INVALID;
    }
}

void require_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) throw pdfp::Error(PDFP_E_NODEVICE, "no CUDA device available");
}

void check_csr(const pdfp_csr* A) {
    if (!A) throw pdfp::Error(PDFP_E_INVALID, "null matrix");
    if (A->m < 0 || A->n < 0) throw pdfp::Error(PDFP_E_INVALID, "negative dimension");
    if (A->m > 0 && !A->row_ptr) throw pdfp::Error(PDFP_E_INVALID, "null row_ptr");
    if (A->m > 0 && A->row_ptr[A->m] > 0 && (!A->col_idx || !A->val))
        throw pdfp::Error(PDFP_E_INVALID, "null col_idx or val");
}

pdfp::ProblemData to_data(const pdfp_problem& p) {
    check_csr(&p.A);
    if ((p.A.m > 0 && (!p.b)) || (p.A.n > 0 && (!p.is_int || !p.var_lb || !p.var_ub || !p.w)))
        throw pdfp::Error(PDFP_E_INVALID, "null problem vector");
    static const int32_t zero_rp = 0;
    return pdfp::ProblemData{p.A.m, p.A.n, p.A.m > 0 ? p.A.row_ptr : &zero_rp, p.A.col_idx, p.A.val,
                             p.b, p.is_eq, p.is_int, p.var_lb, p.var_ub, p.w, p.row_unscale};
}

}  // namespace

extern "C" {

void pdfp_default_params(pdfp_params* p) {
    if (!p) return;
    p->eps_optimal_relative = 1e-4;
    p->eps_feasible_relative = 1e-4;
    p->iteration_limit = 100000;
    p->time_limit = 3600.0;
    p->termination_evaluation_frequency = 200;
    p->sv_max_iterations = 5000;
    p->reflection_coefficient = 1.0;
    p->sv_tolerance = 1e-4;
    p->artificial_restart_threshold = 0.36;
    p->sufficient_reduction_for_restart = 0.2;
    p->necessary_reduction_for_restart = 0.5;
    p->k_p = 0.99;
    p->k_i = 0.01;
    p->k_d = 0.0;
    p->i_smooth = 0.3;
}

const char* pdfp_last_error(void) { return pdfp::last_error_cstr(); }

const char* pdfp_version(void) { return "pdfp_b200 0.1.0 (sm_100a)"; }

int pdfp_set_device(int32_t device) {
    return guarded([&] {
        int count = 0;
        PDFP_CK(cudaGetDeviceCount(&count));
        if (device < 0 || device >= count) throw pdfp::Error(PDFP_E_INVALID, "device index out of range");
        PDFP_CK(cudaSetDevice(device));
    });
}

int pdfp_device_name(char* buf, int32_t len) {
    return guarded([&] {
        require_device();
        int dev = 0;
        PDFP_CK(cudaGetDevice(&dev));
        cudaDeviceProp prop;
        PDFP_CK(cudaGetDeviceProperties(&prop, dev));
        if (buf && len > 0) {
            std::strncpy(buf, prop.name, static_cast<size_t>(len) - 1);
            buf[len - 1] = '\0';
        }
    });
}

int pdfp_create(const pdfp_csr* A, const double* b, const uint8_t* is_eq, const uint8_t* is_int,
                const double* var_lb, const double* var_ub, const double* w,
                const double* row_unscale, int32_t precision, pdfp_handle** out) {
    if (!A || !out) {
        pdfp::set_last_error("null argument");
        return PDFP_E_INVALID;
    }
    pdfp_problem p{*A, b, is_eq, is_int, var_lb, var_ub, w, row_unscale};
    return pdfp_create_batch(1, &p, precision, out);
}

int pdfp_create_batch(int32_t k, const pdfp_problem* problems, int32_t precision, pdfp_handle** out) {
    return guarded([&] {
        if (!out || !problems || k < 1) throw pdfp::Error(PDFP_E_INVALID, "null argument or k < 1");
        *out = nullptr;
        if (precision != PDFP_FP64 && precision != PDFP_MIXED)
            throw pdfp::Error(PDFP_E_INVALID, "precision must be PDFP_FP64 or PDFP_MIXED");
        require_device();
        std::vector<pdfp::ProblemData> data;
        for (int32_t i = 0; i < k; ++i) data.push_back(to_data(problems[i]));
        std::unique_ptr<pdfp_handle> h(new pdfp_handle);
        h->proj.reset(new pdfp::Projector(data, precision));
        *out = h.release();
    });
}

int pdfp_set_x(pdfp_handle* h, int32_t instance, const double* x) {
    return guarded([&] {
        if (!h || !x) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        h->proj->set_x(instance, x);
    });
}

int pdfp_set_target(pdfp_handle* h, int32_t instance, const double* x_tilde) {
    return guarded([&] {
        if (!h || !x_tilde) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        h->proj->set_target(instance, x_tilde);
    });
}

int pdfp_warm_start(pdfp_handle* h, int32_t instance) {
    return guarded([&] {
        if (!h) throw pdfp::Error(PDFP_E_INVALID, "null handle");
        h->proj->warm_start(instance);
    });
}

int pdfp_solve(pdfp_handle* h, const pdfp_params* p, double primal_weight, pdfp_result* r) {
    return guarded([&] {
        if (!h || !p || !r) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        const int K = h->proj->instances();
        std::vector<pdfp_params> ps(K, *p);
        std::vector<double> pw(K, primal_weight);
        std::vector<pdfp_result> rs(K);
        h->proj->solve(ps.data(), pw.data(), rs.data());
        *r = rs[0];
    });
}

int pdfp_solve_batch(pdfp_handle* h, const pdfp_params* params, const double* primal_weights,
                     pdfp_result* results) {
    return guarded([&] {
        if (!h || !params || !primal_weights || !results) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        h->proj->solve(params, primal_weights, results);
    });
}

int pdfp_solve_batch_any(pdfp_handle* h, const pdfp_params* params, const double* primal_weights,
                         const uint8_t* resume, pdfp_result* results) {
    return guarded([&] {
        if (!h || !params || !primal_weights || !results) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        h->proj->solve(params, primal_weights, results, resume, true);
    });
}

int pdfp_get_vector(pdfp_handle* h, int32_t instance, int32_t which, double* out) {
    return guarded([&] {
        if (!h || !out) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        h->proj->get_vector(instance, which, out);
    });
}

int pdfp_get_x(pdfp_handle* h, int32_t instance, double* x_scaled) {
    return pdfp_get_vector(h, instance, PDFP_VEC_PDHG_X, x_scaled);
}

int pdfp_set_col_scale(pdfp_handle* h, int32_t instance, const double* D_c) {
    return guarded([&] {
        if (!h || !D_c) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        h->proj->set_col_scale(instance, D_c);
    });
}

int pdfp_set_x_unscaled(pdfp_handle* h, int32_t instance, const double* x) {
    return guarded([&] {
        if (!h || !x) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        h->proj->set_x(instance, x, true);
    });
}

int pdfp_set_target_unscaled(pdfp_handle* h, int32_t instance, const double* x_tilde) {
    return guarded([&] {
        if (!h || !x_tilde) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        h->proj->set_target(instance, x_tilde, true);
    });
}

int pdfp_get_vector_unscaled(pdfp_handle* h, int32_t instance, int32_t which, double* out) {
    return guarded([&] {
        if (!h || !out) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        h->proj->get_vector(instance, which, out, true);
    });
}

int pdfp_get_x_unscaled(pdfp_handle* h, int32_t instance, double* x) {
    return pdfp_get_vector_unscaled(h, instance, PDFP_VEC_PDHG_X, x);
}

int pdfp_host_alloc(int64_t bytes, void** out) {
    return guarded([&] {
        if (!out || bytes < 0) throw pdfp::Error(PDFP_E_INVALID, "bad argument");
        *out = nullptr;
        PDFP_CK(cudaMallocHost(out, static_cast<size_t>(std::max<int64_t>(bytes, 1))));
    });
}

int pdfp_host_free(void* p) {
    return guarded([&] {
        if (p) PDFP_CK(cudaFreeHost(p));
    });
}

int pdfp_shape(const pdfp_handle* h, int32_t instance, int32_t* k, int32_t* m, int32_t* n) {
    return guarded([&] {
        if (!h) throw pdfp::Error(PDFP_E_INVALID, "null handle");
        const int K = h->proj->instances();
        if (k) *k = K;
        if (instance < 0 || instance >= K) throw pdfp::Error(PDFP_E_INVALID, "instance index out of range");
        if (m) *m = h->proj->rows(instance);
        if (n) *n = h->proj->cols(instance);
    });
}

int pdfp_destroy(pdfp_handle* h) {
    return guarded([&] { delete h; });
}

int pdfp_set_kernel_timing(pdfp_handle* h, int32_t on) {
    return guarded([&] {
        if (!h) throw pdfp::Error(PDFP_E_INVALID, "null handle");
        h->proj->set_kernel_timing(on != 0);
    });
}

int pdfp_set_polish(pdfp_handle* h, int32_t stall_evaluations, double fp32_floor) {
    return guarded([&] {
        if (!h) throw pdfp::Error(PDFP_E_INVALID, "null handle");
        h->proj->set_polish(stall_evaluations, fp32_floor);
    });
}

int pdfp_get_tuning(const pdfp_handle* h, int32_t* out) {
    return guarded([&] {
        if (!h || !out) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        h->proj->tuning(out);
    });
}

int pdfp_get_tuning_stages(const pdfp_handle* h, int32_t* out) {
    return guarded([&] {
        if (!h || !h->proj || !out) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        h->proj->tuning_stages(out);
    });
}

int pdfp_get_tuning_blocks(const pdfp_handle* h, int32_t* out) {
    return guarded([&] {
        if (!h || !h->proj || !out) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        h->proj->tuning_blocks(out);
    });
}

int pdfp_get_tuning_reducers(const pdfp_handle* h, int32_t* out) {
    return guarded([&] {
        if (!h || !h->proj || !out) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        h->proj->tuning_reducers(out);
    });
}

int pdfp_get_tuning_seg(const pdfp_handle* h, int32_t* out) {
    return guarded([&] {
        if (!h || !h->proj || !out) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        h->proj->tuning_seg(out);
    });
}

int pdfp_get_window_form(const pdfp_handle* h, int32_t* out) {
    return guarded([&] {
        if (!h || !h->proj || !out) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        *out = h->proj->window_form();
    });
}

int pdfp_get_tuning_table(const pdfp_handle* h, float* ms, int32_t* cfg, int32_t cap,
                          int32_t* count) {
    return guarded([&] {
        if (!h || !count || (cap > 0 && (!ms || !cfg))) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        *count = h->proj->tuning_table(ms, cfg, cap);
    });
}

int pdfp_profile_step(pdfp_handle* h, int32_t iterations, float* ms_primal, float* ms_dual,
                      double* bytes_primal, double* bytes_dual) {
    return guarded([&] {
        if (!h || !ms_primal || !ms_dual || !bytes_primal || !bytes_dual)
            throw pdfp::Error(PDFP_E_INVALID, "null argument");
        h->proj->profile_step(iterations, ms_primal, ms_dual, bytes_primal, bytes_dual);
    });
}

int pdfp_scale_problem(const pdfp_csr* A, const double* c, const double* var_lb,
                       const double* var_ub, const double* con_lb, const double* con_ub,
                       int32_t ruiz_iterations, double pock_chambolle_alpha,
                       int32_t bound_objective_rescaling, double* val_out, double* c_out,
                       double* var_lb_out, double* var_ub_out, double* con_lb_out,
                       double* con_ub_out, double* D_r, double* D_c, double* bound_scale,
                       double* objective_scale) {
    return guarded([&] {
        check_csr(A);
        require_device();
        pdfp::scale_problem_device(*A, c, var_lb, var_ub, con_lb, con_ub, ruiz_iterations,
                                   pock_chambolle_alpha, bound_objective_rescaling != 0, val_out,
                                   c_out, var_lb_out, var_ub_out, con_lb_out, con_ub_out, D_r, D_c,
                                   bound_scale, objective_scale);
    });
}

int pdfp_mps_read(const char* path, pdfp_mps** out) {
    return guarded([&] {
        if (!path || !out) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        *out = nullptr;
        *out = reinterpret_cast<pdfp_mps*>(pdfp::read_mps_file(path));
    });
}

int pdfp_mps_dims(const pdfp_mps* p, int32_t* m, int32_t* n, int64_t* nnz, int32_t* n_int) {
    return guarded([&] {
        if (!p || !m || !n || !nnz || !n_int) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        const pdfp::MpsModel& M = *reinterpret_cast<const pdfp::MpsModel*>(p);
        *m = M.m;
        *n = M.n;
        *nnz = static_cast<int64_t>(M.ci.size());
        *n_int = static_cast<int32_t>(M.int_idx.size());
    });
}

int pdfp_mps_get(const pdfp_mps* p, double* c, double* c0, int32_t* row_ptr, int32_t* col_idx,
                 double* val, double* b, uint8_t* is_eq, double* l, double* u, int32_t* int_idx) {
    return guarded([&] {
        if (!p || !c0 || !row_ptr) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        const pdfp::MpsModel& M = *reinterpret_cast<const pdfp::MpsModel*>(p);
        auto put = [](auto* dst, const auto& src) {
            if (src.empty()) return;
            if (!dst) throw pdfp::Error(PDFP_E_INVALID, "null output array");
            std::memcpy(dst, src.data(), sizeof(src[0]) * src.size());
        };
        *c0 = M.c0;
        put(c, M.c);
        put(row_ptr, M.rp);
        put(col_idx, M.ci);
        put(val, M.v);
        put(b, M.b);
        put(is_eq, M.is_eq);
        put(l, M.l);
        put(u, M.u);
        put(int_idx, M.int_idx);
    });
}

int pdfp_mps_destroy(pdfp_mps* p) {
    pdfp::mps_destroy(reinterpret_cast<pdfp::MpsModel*>(p));
    return PDFP_OK;
}

int pdfp_checker_create(const pdfp_csr* A, const double* b, const uint8_t* is_eq,
                        pdfp_checker** out) {
    return guarded([&] {
        if (!A || !out) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        *out = nullptr;
        require_device();
        *out = reinterpret_cast<pdfp_checker*>(pdfp::checker_create(*A, b, is_eq));
    });
}

int pdfp_checker_max_violation(pdfp_checker* c, const double* x, double* violation) {
    return guarded([&] {
        if (!c || !violation) throw pdfp::Error(PDFP_E_INVALID, "null argument");
        *violation = pdfp::checker_max_violation(*reinterpret_cast<pdfp::Checker*>(c), x);
    });
}

int pdfp_checker_destroy(pdfp_checker* c) {
    pdfp::checker_destroy(reinterpret_cast<pdfp::Checker*>(c));
    return PDFP_OK;
}

int pdfp_estimate_max_singular_value(const pdfp_csr* A, int32_t max_iterations, double tolerance,
                                     double* sigma, int32_t* iterations) {
    return guarded([&] {
        check_csr(A);
        if (!sigma) throw pdfp::Error(PDFP_E_INVALID, "null output");
        require_device();
        int32_t it = 0;
        *sigma = pdfp::estimate_sv_device(*A, max_iterations, tolerance, &it);
        if (iterations) *iterations = it;
    });
}

int pdlp_solve_relaxation(const pdfp_csr* A, const double* c, const double* l, const double* u,
                          const double* b, const uint8_t* is_le, double tolerance,
                          double time_limit, int32_t cupdlpx_termination, int32_t precision,
                          double* x_out, double* dual_slack_out, pdfp_result* r) {
    return guarded([&] {
        check_csr(A);
        if (!x_out || !dual_slack_out || !r) throw pdfp::Error(PDFP_E_INVALID, "null output");
        require_device();
        pdfp::solve_lp_relaxation_device(*A, c, l, u, b, is_le, tolerance, time_limit,
                                         cupdlpx_termination != 0, precision, x_out,
                                         dual_slack_out, r);
    });
}

}  // extern "C"

int pdfp_rounder_create(const pdfp_csr* A, const double* b, const uint8_t* is_le, const double* l,
                        const double* u, const uint8_t* is_int, pdfp_rounder** out) {
    return guarded([&] {
        if (!A || !out || (A->m > 0 && (!b || !is_le || !A->row_ptr)) || (A->n > 0 && (!l || !u || !is_int)))
            throw pdfp::Error(PDFP_E_INVALID, "null argument");
        if (A->m < 0 || A->n < 0) throw pdfp::Error(PDFP_E_INVALID, "negative dimension");
        *out = reinterpret_cast<pdfp_rounder*>(pdfp::rounder_create(A, b, is_le, l, u, is_int));
    });
}

int pdfp_rounder_round(const pdfp_rounder* r, const double* x_star, const int32_t* first,
                       int32_t n_first, int32_t batch_phase, const int32_t* batch, int32_t n_batch,
                       const int32_t* after, int32_t n_after, const int32_t* int_idx, int32_t n_int,
                       const uint8_t* direction, int64_t max_pops, double* xt, int32_t* infeasible) {
    return guarded([&] {
        if (!r || !x_star || !xt || !infeasible || n_first < 0 || n_batch < 0 || n_after < 0 ||
            n_int < 0 || (n_first && !first) || (n_batch && !batch) || (n_after && !after) ||
            (n_int && !int_idx))
            throw pdfp::Error(PDFP_E_INVALID, "bad argument");
        pdfp::rounder_round(*reinterpret_cast<const pdfp::Rounder*>(r), x_star, first, n_first,
                            batch_phase, batch, n_batch, after, n_after, int_idx, n_int, direction,
                            max_pops, xt, infeasible);
    });
}

int pdfp_rounder_destroy(pdfp_rounder* r) {
    pdfp::rounder_destroy(reinterpret_cast<pdfp::Rounder*>(r));
    return PDFP_OK;
}
