/* pdfp_bench.h -- libpdfp_bench.so: measurement support for the benchmark and
 * the tests (no counterpart in the reference; not part of the drop-in).
 * Status codes are those of pdfp_b200.h. */
#ifndef PDFP_BENCH_H
#define PDFP_BENCH_H

#include "pdfp_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Message of the last failing call on this thread. */
PDFP_API const char* pdfp_bench_last_error(void);

/* The rate, in gathers per second, at which this GPU serves `nnz` independent
 * random 4-byte loads from an m-entry FP32 vector when indices and values
 * stream in coalesced -- the ceiling of a sparse step whose column indices are
 * scattered, measured with the simplest kernel that reaches it (best of
 * `repeats` launches in a few launch shapes).  nnz: a positive multiple of 4
 * below 2^31.  Allocates and frees its own test data. */
PDFP_API int pdfp_measure_gather_rate(int64_t nnz, int32_t m, int32_t repeats,
                                      double* gathers_per_s);

#ifdef __cplusplus
}
#endif
#endif
