// Fused inference of the surrogate MLP on the sm_100a tensor cores: one
// persistent kernel computes out[n x 16] = network(X[n x 4]) with the hidden
// activations kept in shared memory between layers.
//
// Per 128-row tile:
//   layer 1 (K = 4): the epilogue warps on the CUDA cores, written as BF16
//     straight into the A operand buffer (K-major, 128-byte swizzle: the layout
//     a TMA SWIZZLE_128B load produces);
//   layers 2-4 (256 x 256) and 5 (16 x 256): one thread issues tcgen05.mma
//     (kind::f16, BF16 x BF16 -> FP32 in tensor memory) over the A buffer and
//     weight K-blocks that a TMA producer thread streams through a 4-stage
//     ring; the epilogue warps read the accumulator (tcgen05.ld), add the
//     bias, apply SiLU and overwrite the A buffer with the next layer's input.
// Roles: warps 0-7 epilogue (warp w: rows 32 (w % 4).., columns half w / 4),
// warp 8 TMA producer, warp 9 MMA issuer. Handshakes: per-stage full/empty
// mbarriers (weights), act_ready (epilogue -> MMA, 256 arrivals) and
// acc_ready (MMA commit -> epilogue). Every wait is bounded; on a timeout the
// CTA records an error, waits (bounded) for its copies in flight, frees its
// tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstddef>
#include <cstdint>
#include <mutex>

#include "mlp_fused.h"
#include "sm100.cuh"
#include "surrogate.h"

namespace grrt_b200 {
namespace surr {

namespace {

constexpr int kRows = 128;
constexpr int kStages = 4;
constexpr int kEpiWarps = 8;
constexpr int kThreads = (kEpiWarps + 2) * 32;
constexpr uint32_t kActBytes = 4 * kRows * 128;  // 4 K-blocks of 128 rows x 64 BF16
constexpr uint32_t kStageBytes = kHidden * 128;  // 256 rows x 64 BF16
constexpr uint32_t kWaitLimit = 1u << 22;

// FusedSmem also holds a per-CTA copy of the small parameters the epilogue
// reads for every value (W1, b1, b2..b4, b5).
struct FusedSmem {
    uint64_t full[kStages];
    uint64_t empty[kStages];
    uint64_t act_ready;
    uint64_t acc_ready;
    uint32_t tmem_base;
    int failed;
    alignas(16) float w1[kHidden * kIn];  // read as float4 per hidden unit
    float b1[kHidden];
    float bh[3][kHidden];
    float b5[kOutPad];
};

static_assert(offsetof(FusedSmem, w1) % 16 == 0, "float4 reads of W1");

struct FusedMaps {
    CUtensorMap w[4];  // W2, W3, W4 (256 x 256), W5 (16 x 256)
};

// the same SiLU as the training kernels
__device__ __forceinline__ float silu_f(float z) { return sm100::silu_fast(z); }

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sm100::smem_u32(bar)) : "memory");
}

// byte offset of the 16-byte chunk holding columns [k, k + 8) of row r in the
// swizzled K-major A buffer
__device__ __forceinline__ uint32_t act_offset(int r, int k) {
    const int kb = k >> 6, c = (k & 63) >> 3;
    return static_cast<uint32_t>(kb) * (kRows * 128) + static_cast<uint32_t>(r) * 128 +
           (static_cast<uint32_t>(c ^ (r & 7)) << 4);
}

__device__ __forceinline__ uint4 pack8(const float* v) {
    uint4 u;
    __nv_bfloat162 h0 = __floats2bfloat162_rn(v[0], v[1]), h1 = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 h2 = __floats2bfloat162_rn(v[4], v[5]), h3 = __floats2bfloat162_rn(v[6], v[7]);
    u.x = *reinterpret_cast<uint32_t*>(&h0);
    u.y = *reinterpret_cast<uint32_t*>(&h1);
    u.z = *reinterpret_cast<uint32_t*>(&h2);
    u.w = *reinterpret_cast<uint32_t*>(&h3);
    return u;
}

__global__ void __launch_bounds__(kThreads, 1)
mlp_fused_kernel(const __grid_constant__ FusedMaps maps, const float* __restrict__ X, long long n_cap,
                 const unsigned* __restrict__ n_dev, const float* __restrict__ params, float* __restrict__ out,
                 int* err) {
    // the row count: n_cap, or the device count a previous kernel wrote (at most n_cap)
    const long long n = n_dev ? (static_cast<long long>(*n_dev) < n_cap ? static_cast<long long>(*n_dev) : n_cap)
                              : n_cap;
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = sm100::smem_u32(smem_raw);
    unsigned char* act = smem_raw + ((1024u - (raw & 1023u)) & 1023u);
    unsigned char* ring = act + kActBytes;
    FusedSmem* sh = reinterpret_cast<FusedSmem*>(ring + kStages * kStageBytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long n_tiles = (n + kRows - 1) / kRows;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            sm100::mbar_init(&sh->full[s], 1);
            sm100::mbar_init(&sh->empty[s], 1);
        }
        sm100::mbar_init(&sh->act_ready, kEpiWarps * 32);
        sm100::mbar_init(&sh->acc_ready, 1);
        sh->failed = 0;
        sm100::fence_mbar_init();
    }
    for (int i = threadIdx.x; i < kHidden * kIn; i += blockDim.x) sh->w1[i] = params[ParamLayout::w1 + i];
    for (int i = threadIdx.x; i < kHidden; i += blockDim.x) {
        sh->b1[i] = params[ParamLayout::b1 + i];
        for (int l = 0; l < 3; ++l) sh->bh[l][i] = params[ParamLayout::b(l + 2) + i];
    }
    for (int i = threadIdx.x; i < kOutPad; i += blockDim.x) sh->b5[i] = params[ParamLayout::b5 + i];
    if (warp == kEpiWarps) {
        if (lane == 0)
            for (int l = 0; l < 4; ++l) sm100::tma_prefetch_desc(&maps.w[l]);
        sm100::tmem_alloc(&sh->tmem_base, 256);
        sm100::tmem_relinquish();
    }
    sm100::tc_fence_before();
    __syncthreads();
    sm100::tc_fence_after();
    const uint32_t tmem = sh->tmem_base;
    volatile int* failed = &sh->failed;

    if (warp == kEpiWarps) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            uint32_t it = 0;
            for (long long t = blockIdx.x; t < n_tiles && !*failed; t += gridDim.x) {
                for (int l = 0; l < 4 && !*failed; ++l) {
                    const uint32_t bytes = (l < 3) ? kStageBytes : static_cast<uint32_t>(kOutPad) * 128;
                    for (int kb = 0; kb < 4; ++kb, ++it) {
                        const int s = static_cast<int>(it % kStages);
                        if (it >= kStages &&
                            !sm100::mbar_wait(&sh->empty[s], ((it / kStages) - 1) & 1, kWaitLimit)) {
                            atomicCAS(&sh->failed, 0, 1);
                            break;
                        }
                        sm100::mbar_arrive_expect_tx(&sh->full[s], bytes);
                        sm100::tma_load_2d(ring + s * kStageBytes, &maps.w[l], &sh->full[s], kb * 64, 0);
                    }
                }
            }
            // copies still in flight complete before the CTA may exit
            const uint32_t last = it;
            for (uint32_t k = (last > kStages ? last - kStages : 0); k < last; ++k)
                sm100::mbar_wait(&sh->full[k % kStages], (k / kStages) & 1, kWaitLimit);
        }
    } else if (warp == kEpiWarps + 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            uint32_t it = 0, n_act = 0;
            const uint32_t id_hidden = sm100::idesc_bf16_f32(kRows, kHidden);
            const uint32_t id_out = sm100::idesc_bf16_f32(kRows, kOutPad);
            const uint32_t a_base = sm100::smem_u32(act);
            for (long long t = blockIdx.x; t < n_tiles && !*failed; t += gridDim.x) {
                for (int l = 0; l < 4; ++l) {
                    if (!sm100::mbar_wait(&sh->act_ready, n_act & 1, kWaitLimit)) {
                        atomicCAS(&sh->failed, 0, 2);
                        break;
                    }
                    ++n_act;
                    sm100::tc_fence_after();
                    bool ok = true;
                    for (int kb = 0; kb < 4; ++kb, ++it) {
                        const int s = static_cast<int>(it % kStages);
                        if (!sm100::mbar_wait(&sh->full[s], (it / kStages) & 1, kWaitLimit)) {
                            atomicCAS(&sh->failed, 0, 3);
                            ok = false;
                            break;
                        }
                        sm100::tc_fence_after();
                        const uint64_t da = sm100::desc_kmajor_sw128(a_base + kb * kRows * 128);
                        const uint64_t db = sm100::desc_kmajor_sw128(sm100::smem_u32(ring + s * kStageBytes));
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            sm100::umma_f16(tmem, da + 2 * k, db + 2 * k, l < 3 ? id_hidden : id_out,
                                            (kb > 0 || k > 0) ? 1u : 0u);
                        sm100::umma_commit(&sh->empty[s]);
                    }
                    sm100::umma_commit(&sh->acc_ready);
                    if (!ok || *failed) break;
                }
            }
        }
    } else {
        // ---------------- epilogue warps ----------------
        const int quad = warp & 3, half = warp >> 2;
        const int r = quad * 32 + lane;
        const int c0 = half * (kHidden / 2);
        const uint32_t t_row = tmem + (static_cast<uint32_t>(quad * 32) << 16);
        uint32_t n_acc = 0;
        for (long long t = blockIdx.x; t < n_tiles && !*failed; t += gridDim.x) {
            const long long row = t * kRows + r;
            // layer 1 on the CUDA cores
            float x0 = 0.f, x1 = 0.f, x2 = 0.f, x3 = 0.f;
            if (row < n) {
                const float4 xv = *reinterpret_cast<const float4*>(X + row * kIn);
                x0 = xv.x;
                x1 = xv.y;
                x2 = xv.z;
                x3 = xv.w;
            }
            for (int k = c0; k < c0 + kHidden / 2; k += 8) {
                float v[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float4 w = *reinterpret_cast<const float4*>(&sh->w1[(k + j) * kIn]);
                    const float z = sh->b1[k + j] + w.x * x0 + w.y * x1 + w.z * x2 + w.w * x3;
                    v[j] = silu_f(z);
                }
                *reinterpret_cast<uint4*>(act + act_offset(r, k)) = pack8(v);
            }
            fence_proxy_async();
            mbar_arrive(&sh->act_ready);
            for (int l = 2; l <= 5; ++l) {
                if (!sm100::mbar_wait(&sh->acc_ready, n_acc & 1, kWaitLimit)) {
                    atomicCAS(&sh->failed, 0, 4);
                    break;
                }
                ++n_acc;
                sm100::tc_fence_after();
                if (l < 5) {
                    const float* bias = sh->bh[l - 2];
                    for (int k = c0; k < c0 + kHidden / 2; k += 32) {
                        float v[32];
                        sm100::tmem_ld32(t_row + static_cast<uint32_t>(k), v);
#pragma unroll
                        for (int j = 0; j < 32; ++j) v[j] = silu_f(v[j] + bias[k + j]);
#pragma unroll
                        for (int j = 0; j < 32; j += 8)
                            *reinterpret_cast<uint4*>(act + act_offset(r, k + j)) = pack8(v + j);
                    }
                    sm100::tc_fence_before();
                    fence_proxy_async();
                    mbar_arrive(&sh->act_ready);
                } else {
                    float v[16];
                    sm100::tmem_ld16(t_row, v);  // every warp of the quadrant loads (aligned), half 0 stores
                    sm100::tc_fence_before();
                    if (half == 0 && row < n) {
                        float* o = out + row * kOutPad;
#pragma unroll
                        for (int j = 0; j < 16; j += 4)
                            *reinterpret_cast<float4*>(o + j) = make_float4(v[j] + sh->b5[j], v[j + 1] + sh->b5[j + 1],
                                                                            v[j + 2] + sh->b5[j + 2],
                                                                            v[j + 3] + sh->b5[j + 3]);
                    }
                }
            }
        }
    }
    sm100::tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && sh->failed) atomicExch(err, 100 + sh->failed);
    if (warp == kEpiWarps) sm100::tmem_dealloc(tmem, 256);
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

bool weight_map(CUtensorMap* m, const __nv_bfloat16* w, int rows) {
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(kHidden), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(kHidden) * 2};
    const cuuint32_t box[2] = {64, static_cast<cuuint32_t>(rows)};
    const cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(w), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

size_t mlp_fused_smem_bytes() { return 1024 + kActBytes + kStages * kStageBytes + sizeof(FusedSmem); }

cudaError_t launch_mlp_fused(const float* X, long long n, const float* params, __nv_bfloat16* const* wb,
                             const __nv_bfloat16* w5b, float* out, int* d_err, cudaStream_t s,
                             const unsigned* d_n) {
    if (n <= 0) return cudaSuccess;
    if ((reinterpret_cast<uintptr_t>(X) & 15) || (reinterpret_cast<uintptr_t>(out) & 15)) return cudaErrorInvalidValue;
    FusedMaps maps;
    for (int l = 0; l < 3; ++l)
        if (!weight_map(&maps.w[l], wb[l], kHidden)) return cudaErrorInvalidValue;
    if (!weight_map(&maps.w[3], w5b, kOutPad)) return cudaErrorInvalidValue;
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    static int sms = 0;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(mlp_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(mlp_fused_smem_bytes()));
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    });
    if (attr != cudaSuccess) return attr;
    const long long tiles = (n + kRows - 1) / kRows;
    const int grid = static_cast<int>(tiles < sms ? tiles : sms);
    mlp_fused_kernel<<<grid, kThreads, mlp_fused_smem_bytes(), s>>>(maps, X, n, d_n, params, out, d_err);
    return cudaGetLastError();
}

}  // namespace surr
}  // namespace grrt_b200
