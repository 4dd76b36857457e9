// Exported entry points of the learned surrogate (include/grrt_surrogate.h).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/grrt_surrogate.h"
#include "device/umma_gemm.h"

using namespace grrt_b200;

extern "C" GRRT_EXPORT int grrt_surrogate_gemm_bf16(const void* A, int lda, const void* B, int ldb, int M, int N,
                                                    int K, int splits, const float* bias, const float* gate_z,
                                                    int ld_gate, int act, float* out_f32, int ld_f32, void* out_bf16,
                                                    int ld_bf16, void* stream) {
    if (!A || !B || (!out_f32 && !out_bf16)) return -1;
    auto s = static_cast<cudaStream_t>(stream);
    int* d_err = nullptr;
    if (cudaMallocAsync(reinterpret_cast<void**>(&d_err), sizeof(int), s) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    cudaMemsetAsync(d_err, 0, sizeof(int), s);
    GemmEpilogue ep;
    ep.bias = bias;
    ep.gate_z = gate_z;
    ep.ld_gate = ld_gate;
    ep.out_f32 = out_f32;
    ep.ld_f32 = ld_f32;
    ep.split_stride = static_cast<size_t>(M) * static_cast<size_t>(ld_f32);
    ep.out_bf16 = static_cast<__nv_bfloat16*>(out_bf16);
    ep.ld_bf16 = ld_bf16;
    ep.act = act;
    cudaError_t e = umma_gemm_bf16(static_cast<const __nv_bfloat16*>(A), lda, static_cast<const __nv_bfloat16*>(B),
                                   ldb, M, N, K, splits, ep, d_err, s);
    int h_err = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFreeAsync(d_err, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return h_err == 0 ? 0 : -1;
}
