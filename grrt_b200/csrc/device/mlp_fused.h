// Fused tensor-core inference of the surrogate MLP (mlp_fused.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstddef>

namespace grrt_b200 {
namespace surr {

// out[n x 16] = network(X[n x 4]); params: the FP32 parameter array (layer 1
// and the biases are read from it), wb[0..2]: BF16 W2..W4 [256 x 256],
// w5b: BF16 W5 [16 x 256]. X and out 16-byte aligned. *d_err gets a non-zero
// code if a CTA timed out. With d_n, the row count is min(n, *d_n), read on
// the device (a count written by an earlier kernel on the stream); n sizes the grid.
cudaError_t launch_mlp_fused(const float* X, long long n, const float* params, __nv_bfloat16* const* wb,
                             const __nv_bfloat16* w5b, float* out, int* d_err, cudaStream_t s,
                             const unsigned* d_n = nullptr);
size_t mlp_fused_smem_bytes();

}  // namespace surr
}  // namespace grrt_b200
