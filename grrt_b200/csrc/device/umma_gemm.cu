// BF16 GEMM on the sm_100a tensor cores for the learned surrogate:
//   C[M x N] = A[M x K] * B[N x K]^T   (A, B row-major BF16, i.e. K-major),
// FP32 accumulation in tensor memory, with a fused epilogue (bias, SiLU,
// SiLU-derivative gating, FP32/BF16 outputs, split-K partials).
//
// One CTA computes a 128-row tile and all N (<= 256) columns:
//   warp 0 lane 0: TMA producer (A and B K-blocks of 64 into a 4-stage ring,
//                  SWIZZLE_128B, completion on per-stage mbarriers);
//   warp 1 lane 0: MMA issuer (4 x tcgen05.mma K=16 per stage, commit frees
//                  the stage, a final commit signals the epilogue);
//   warps 0-3:     epilogue, each warp reads its 32 TMEM lanes (= tile rows).
// Every mbarrier wait is bounded; on timeout the CTA records an error code in
// *err, waits (bounded) for its TMA copies in flight, frees its tensor memory
// and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "launch_cache.h"
#include "sm100.cuh"
#include "umma_gemm.h"

namespace grrt_b200 {

namespace {

constexpr int kBM = 128;
constexpr int kBK = 64;
constexpr int kStages = 4;
constexpr int kThreads = 128;
constexpr uint32_t kWaitLimit = 1u << 22;  // polls; a healthy wait needs a handful

struct GemmSmem {
    uint64_t full[kStages];
    uint64_t empty[kStages];
    uint64_t done;
    uint32_t tmem_base;
    int failed;
};

__device__ __forceinline__ float silu(float z) { return sm100::silu_fast(z); }
__device__ __forceinline__ float silu_grad(float z) { return sm100::silu_grad_fast(z); }

__global__ void __launch_bounds__(kThreads, 1)
umma_gemm_kernel(const __grid_constant__ CUtensorMap tmap_a, const __grid_constant__ CUtensorMap tmap_b,
                 const GemmEpilogue ep, int M, int N, int k_blocks_per_split, int k_blocks_total, int* err) {
    extern __shared__ unsigned char smem_raw[];
    // 1024-byte alignment for the swizzle atoms
    const uint32_t raw = sm100::smem_u32(smem_raw);
    unsigned char* tiles = smem_raw + ((1024u - (raw & 1023u)) & 1023u);
    const uint32_t a_bytes = kBM * kBK * 2, b_bytes = static_cast<uint32_t>(N) * kBK * 2;
    const uint32_t stage_bytes = a_bytes + b_bytes;
    GemmSmem* sh = reinterpret_cast<GemmSmem*>(tiles + kStages * stage_bytes);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kBM;
    const int split = blockIdx.y;
    const int kb0 = split * k_blocks_per_split;
    int kb1 = kb0 + k_blocks_per_split;
    if (kb1 > k_blocks_total) kb1 = k_blocks_total;
    const int nk = kb1 - kb0;
    // TMEM columns: a power of two >= 32 covering N
    uint32_t tcols = 32;
    while (tcols < static_cast<uint32_t>(N)) tcols <<= 1;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            sm100::mbar_init(&sh->full[s], 1);
            sm100::mbar_init(&sh->empty[s], 1);
        }
        sm100::mbar_init(&sh->done, 1);
        sh->failed = 0;
        sm100::fence_mbar_init();
        sm100::tma_prefetch_desc(&tmap_a);
        sm100::tma_prefetch_desc(&tmap_b);
    }
    if (warp == 0) {
        sm100::tmem_alloc(&sh->tmem_base, tcols);
        sm100::tmem_relinquish();
    }
    sm100::tc_fence_before();
    __syncthreads();
    sm100::tc_fence_after();
    const uint32_t tmem = sh->tmem_base;
    const uint32_t idesc = sm100::idesc_bf16_f32(kBM, N);

    int issued = 0;  // producer: stages handed to TMA
    if (warp == 0 && lane == 0 && nk > 0) {
        for (int i = 0; i < nk; ++i) {
            const int s = i % kStages;
            if (i >= kStages && !sm100::mbar_wait(&sh->empty[s], ((i / kStages) - 1) & 1, kWaitLimit)) {
                atomicCAS(&sh->failed, 0, 1);
                break;
            }
            unsigned char* a_dst = tiles + s * stage_bytes;
            unsigned char* b_dst = a_dst + a_bytes;
            sm100::mbar_arrive_expect_tx(&sh->full[s], stage_bytes);
            const int kx = (kb0 + i) * kBK;
            sm100::tma_load_2d(a_dst, &tmap_a, &sh->full[s], kx, m0);
            sm100::tma_load_2d(b_dst, &tmap_b, &sh->full[s], kx, 0);
            ++issued;
        }
    } else if (warp == 1 && lane == 0) {
        for (int i = 0; i < nk; ++i) {
            const int s = i % kStages;
            if (!sm100::mbar_wait(&sh->full[s], (i / kStages) & 1, kWaitLimit) ||
                *reinterpret_cast<volatile int*>(&sh->failed)) {
                atomicCAS(&sh->failed, 0, 2);
                break;
            }
            sm100::tc_fence_after();
            const uint32_t a_addr = sm100::smem_u32(tiles + s * stage_bytes);
            const uint32_t b_addr = a_addr + a_bytes;
            const uint64_t da = sm100::desc_kmajor_sw128(a_addr), db = sm100::desc_kmajor_sw128(b_addr);
#pragma unroll
            for (int k = 0; k < kBK / 16; ++k) {
                // +32 bytes along K per step: start-address field counts 16-byte units
                sm100::umma_f16(tmem, da + 2 * k, db + 2 * k, idesc, (i > 0 || k > 0) ? 1u : 0u);
            }
            sm100::umma_commit(&sh->empty[s]);
        }
        sm100::umma_commit(&sh->done);  // also completes when nothing was issued
    }
    __syncwarp();

    // epilogue: wait for the accumulator
    bool ok = sm100::mbar_wait(&sh->done, 0, kWaitLimit);
    if (!ok) atomicCAS(&sh->failed, 0, 3);
    sm100::tc_fence_after();
    __syncthreads();
    const bool good = (*reinterpret_cast<volatile int*>(&sh->failed) == 0);
    const int row = m0 + warp * 32 + lane;
    if (good) {
        const uint32_t t_row = tmem + (static_cast<uint32_t>(warp * 32) << 16);
        const size_t zoff = ep.split_stride * static_cast<size_t>(split);
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            sm100::tmem_ld16(t_row + static_cast<uint32_t>(c0), v);
            if (nk <= 0) {
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = 0.0f;
            }
            if (row >= M) continue;
            if (ep.bias) {
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] += ep.bias[c0 + j];
            }
            if (ep.gate_z) {  // backward through SiLU: v *= silu'(z)
                const float* z = ep.gate_z + static_cast<size_t>(row) * ep.ld_gate + c0;
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] *= silu_grad(z[j]);
            }
            if (ep.out_f32) {
                float* o = ep.out_f32 + zoff + static_cast<size_t>(row) * ep.ld_f32 + c0;
#pragma unroll
                for (int j = 0; j < 16; j += 4) *reinterpret_cast<float4*>(o + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
            }
            if (ep.out_bf16) {
                __nv_bfloat16* o = ep.out_bf16 + static_cast<size_t>(row) * ep.ld_bf16 + c0;
                alignas(16) __nv_bfloat162 h[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    float x0 = v[2 * j], x1 = v[2 * j + 1];
                    if (ep.act == kActSilu) {
                        x0 = silu(x0);
                        x1 = silu(x1);
                    }
                    h[j] = __floats2bfloat162_rn(x0, x1);
                }
                *reinterpret_cast<uint4*>(o) = *reinterpret_cast<const uint4*>(&h[0]);
                *reinterpret_cast<uint4*>(o + 8) = *reinterpret_cast<const uint4*>(&h[4]);
            }
        }
    }
    if (!good && threadIdx.x == 0) {
        atomicExch(err, sh->failed);
    }
    // a failed producer may still have copies in flight: wait for them (bounded)
    if (!good && warp == 0 && lane == 0) {
        for (int i = 0; i < issued; ++i) sm100::mbar_wait(&sh->full[i % kStages], (i / kStages) & 1, kWaitLimit);
    }
    sm100::tc_fence_before();
    __syncthreads();
    if (warp == 0) sm100::tmem_dealloc(tmem, tcols);
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Row-major BF16 matrix [rows x cols] with row pitch ld (elements), box
// [box_rows x 64], SWIZZLE_128B; out-of-range elements read as zero.
bool make_tmap(CUtensorMap* m, const void* base, int rows, int cols, int ld, int box_rows) {
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld) * 2};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(kBK), static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

size_t umma_gemm_smem_bytes(int N) {
    return 1024 + static_cast<size_t>(kStages) * (kBM * kBK * 2 + static_cast<size_t>(N) * kBK * 2) + sizeof(GemmSmem);
}

cudaError_t umma_gemm_bf16(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K,
                           int splits, const GemmEpilogue& ep, int* d_err, cudaStream_t stream) {
    // shapes the kernel supports; everything else is a caller error
    if (M <= 0 || N < 16 || N > 256 || (N % 16) != 0 || K <= 0 || (K % kBK) != 0 || splits < 1) return cudaErrorInvalidValue;
    if ((lda % 8) != 0 || (ldb % 8) != 0 || lda < K || ldb < K) return cudaErrorInvalidValue;
    if ((reinterpret_cast<uintptr_t>(A) & 15) || (reinterpret_cast<uintptr_t>(B) & 15)) return cudaErrorInvalidValue;
    if (ep.out_bf16 && ((ep.ld_bf16 % 8) != 0 || (reinterpret_cast<uintptr_t>(ep.out_bf16) & 15))) return cudaErrorInvalidValue;
    if (ep.out_f32 && ((ep.ld_f32 % 4) != 0 || (reinterpret_cast<uintptr_t>(ep.out_f32) & 15))) return cudaErrorInvalidValue;
    if (splits > 1 && (ep.out_bf16 || ep.bias || ep.gate_z || !ep.out_f32 || ep.split_stride == 0))
        return cudaErrorInvalidValue;  // split-K writes raw FP32 partials only
    CUtensorMap ta, tb;
    if (!make_tmap(&ta, A, M, K, lda, kBM) || !make_tmap(&tb, B, N, K, ldb, N)) return cudaErrorInvalidValue;
    const int kbt = K / kBK;
    const int per = (kbt + splits - 1) / splits;
    splits = (kbt + per - 1) / per;  // every split gets at least one K-block
    const size_t smem = umma_gemm_smem_bytes(N);
    // the shared-memory attribute is set once per device, with that device current
    struct Attr {
        cudaError_t err = cudaSuccess;
    };
    const Attr& attr = per_device_shape<Attr>([](int) {
        Attr a;
        a.err = cudaFuncSetAttribute(umma_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(umma_gemm_smem_bytes(256)));
        return a;
    });
    if (attr.err != cudaSuccess) return attr.err;
    dim3 grid((M + kBM - 1) / kBM, splits);
    umma_gemm_kernel<<<grid, kThreads, smem, stream>>>(ta, tb, ep, M, N, per, kbt, d_err);
    return cudaGetLastError();
}

}  // namespace grrt_b200
