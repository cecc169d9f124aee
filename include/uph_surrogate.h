/*
 * uph_surrogate.h -- C ABI of the learned surrogate's building blocks.
 *
 * The reference has no learned part; everything declared here is a project
 * addition.  All pointers are device pointers; every call is asynchronous on
 * `stream` (a cudaStream_t, NULL for the default stream) and reports
 * argument errors through uph_status.  Device-side failures (a bounded wait
 * that gave up) set bits in the caller's error word `err`.
 */
#ifndef UPH_SURROGATE_H
#define UPH_SURROGATE_H

#include <stdint.h>

#include "uph.h"

#ifdef __cplusplus
extern "C" {
#endif

/* C[M x N] = A[M x K] . B[N x K]^T on the tcgen05 tensor cores: BF16
 * inputs (row-major, K contiguous), FP32 accumulation in TMEM.  K must be a
 * multiple of 64, N of 128, leading dimensions of 8.
 *   splits == 1: optional bias[N] and ReLU, then FP32 and/or BF16 output;
 *   splits  > 1: K is split across CTAs, FP32 partials (splits * M * N
 *                floats in `partials`) are summed in a fixed order into
 *                c_f32 (dense, ldc == N), added to its contents when
 *                accumulate != 0. */
uph_status uph_tc_gemm_bf16(const void *A, int32_t lda, const void *B, int32_t ldb, int32_t M, int32_t N,
                            int32_t K, const float *bias, int32_t relu, float *c_f32, void *c_bf16, int32_t ldc,
                            int32_t splits, float *partials, int32_t accumulate, unsigned *err, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* UPH_SURROGATE_H */
