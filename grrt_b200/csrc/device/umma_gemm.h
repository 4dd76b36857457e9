// BF16 tensor-core GEMM of the learned surrogate (umma_gemm.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstddef>

namespace grrt_b200 {

enum : int { kActNone = 0, kActSilu = 1 };

// Epilogue of C = A * B^T (per output element, in this order):
//   v = acc (+ bias[col]) (* silu'(gate_z[row][col]))
//   out_f32[split * split_stride + row * ld_f32 + col] = v
//   out_bf16[row * ld_bf16 + col] = bf16(act(v))
// Null pointers skip their step. Split-K (splits > 1) allows out_f32 only.
struct GemmEpilogue {
    const float* bias = nullptr;
    const float* gate_z = nullptr;
    int ld_gate = 0;
    float* out_f32 = nullptr;
    int ld_f32 = 0;
    size_t split_stride = 0;
    __nv_bfloat16* out_bf16 = nullptr;
    int ld_bf16 = 0;
    int act = kActNone;
};

// A: [M x K] row-major BF16 (pitch lda), B: [N x K] row-major BF16 (pitch ldb).
// Requires 16 <= N <= 256, N % 16 == 0, K % 64 == 0, pitches % 8 == 0,
// 16-byte aligned bases. M is arbitrary (rows past M read as zero and are not
// written). *d_err (device int) receives a non-zero code if a CTA timed out.
cudaError_t umma_gemm_bf16(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K,
                           int splits, const GemmEpilogue& ep, int* d_err, cudaStream_t stream);
size_t umma_gemm_smem_bytes(int N);

}  // namespace grrt_b200
