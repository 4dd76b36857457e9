/*
 * grrt_surrogate.h — the learned transfer-function surrogate of libgrrt.so.
 *
 * No counterpart in the reference. A small MLP maps (image-plane alpha, beta,
 * spin, inclination) to the quantities a thin-disk pixel's colour is made of;
 * it is trained on the GPU on geodesics the plain FP64 integrator traces, by
 * the library's own BF16 tensor-core (tcgen05) kernels with FP32 accumulation.
 * The plain integrator stays the fallback and the judge: samples the network
 * cannot decide to its calibrated accuracy are re-traced exactly.
 */
#ifndef GRRT_SURROGATE_H
#define GRRT_SURROGATE_H

#include "grrt_api.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The surrogate's BF16 GEMM, exposed for verification: C = A * B^T with
 * A [M x K] and B [N x K] row-major BF16 device matrices (pitches lda, ldb in
 * elements), FP32 accumulation, then per element
 *   v = acc (+ bias[col]) (* silu'(gate_z[row * ld_gate + col]))
 *   out_f32[split * M * ld_f32 + row * ld_f32 + col] = v       (if out_f32)
 *   out_bf16[row * ld_bf16 + col] = bf16(act ? silu(v) : v)    (if out_bf16)
 * splits > 1 splits K and writes raw FP32 partials only (bias, gate_z and
 * out_bf16 must be NULL). Requires 16 <= N <= 256, N % 16 == 0, K % 64 == 0,
 * pitches % 8 == 0 and 16-byte aligned pointers. Returns 0, or -1 on a bad
 * shape, a launch error, or a device-side timeout. Synchronises `stream`. */
GRRT_EXPORT int grrt_surrogate_gemm_bf16(const void* A, int lda, const void* B, int ldb, int M, int N, int K,
                                         int splits, const float* bias, const float* gate_z, int ld_gate, int act,
                                         float* out_f32, int ld_f32, void* out_bf16, int ld_bf16, void* stream);

#ifdef __cplusplus
}
#endif

#endif
