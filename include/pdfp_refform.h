/* pdfp_refform.h -- the reference's GPU projector step, as written, for comparison.
 *
 * libpdfp_refform.so runs the plain FP64 PDHG step the way the reference runs it
 * on a CuVector state: per step a cuSPARSE SpMV with A', the primal kernel, the
 * dual_y kernel, a cuSPARSE SpMV with A and the dual_z kernel
 * (src/pdfp_kernels.jl:4-86, src/pdfp.jl:158-163), on FP64 CSR copies of A and
 * A' with int32 indices (src/pdlp.jl:79-80).  It is not part of the drop-in: the
 * benchmark and the tests use it as the "plain FP64 GPU form" the fused
 * projector of libpdfp_b200.so is measured against.  Status codes and the
 * pdfp_csr struct are those of pdfp_b200.h.
 */
#ifndef PDFP_REFFORM_H
#define PDFP_REFFORM_H

#include "pdfp_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Message of the last failing call on this thread. */
PDFP_API const char* pdfp_refform_last_error(void);

/* PDFPState(A, b, is_eq, is_int, var_lb, var_ub, w; use_gpu = true)
 * (src/pdfp.jl:60-76): device copies of A, A' and the vectors. */
PDFP_API int pdfp_refform_create(const pdfp_csr* A, const double* b, const uint8_t* is_eq,
                                 const uint8_t* is_int, const double* var_lb,
                                 const double* var_ub, const double* w, void** out);

/* copyto!(current_x, x0); copyto!(initial_x, x0); set_target!(x_tilde)
 * (src/pump.jl:305-306, src/pdfp.jl:98-114); y and z restart from zero. */
PDFP_API int pdfp_refform_reset(void* h, const double* x_tilde, const double* x0);

/* `count` calls of pdhg_step! (src/pdfp.jl:158-163) with k_offset = k0, k0+1, ...
 * at inner count 0, step size eta and primal weight; *ms = their device time. */
PDFP_API int pdfp_refform_steps(void* h, double step_size, double primal_weight, int32_t k0,
                                int32_t count, float* ms);

/* which: 0 pdhg_x, 1 current_x (n values); 2 pdhg_z, 3 current_z (m values). */
PDFP_API int pdfp_refform_get(void* h, int32_t which, double* out);

PDFP_API int pdfp_refform_destroy(void* h);

#ifdef __cplusplus
}
#endif

#endif /* PDFP_REFFORM_H */
