// Fused inference of the surrogate MLP on the sm_100a tensor cores: one
// persistent kernel computes out[n x 16] = network(X[n x 4]) with the hidden
// activations kept in shared memory between layers.
//
// Per 128-row tile:
//   layer 1 (K = 4): the epilogue warps on the CUDA cores, written as BF16
//     straight into the tile's A operand buffer (K-major, 128-byte swizzle:
//     the layout a TMA SWIZZLE_128B load produces);
//   layers 2-4 (256 x 256) and 5 (16 x 256): one thread issues tcgen05.mma
//     (kind::f16, BF16 x BF16 -> FP32 in tensor memory) over the A buffer and
//     weight K-blocks that a TMA producer thread streams through a 3-stage
//     ring; the epilogue warps read the accumulator (tcgen05.ld), add the
//     bias, apply SiLU and overwrite the A buffer with the next layer's input.
// Two tiles are in flight (slots 0 and 1, each with its A buffer and a
// 256-column accumulator: all 512 columns of tensor memory), and all three
// roles walk the slots' steps in the same alternating order. The MMAs of one
// slot then run while the epilogue works on the other slot, so the tensor
// pipe and the epilogue's special-function work overlap instead of taking
// turns.
// Roles: warps 0-15 epilogue (warp w: rows 32 (w % 4).., columns
// 64 (w / 4)..; four warps per scheduler hide the tensor-memory and
// special-function latencies), warp 16 TMA producer, warp 17 MMA issuer.
// Handshakes: per-stage full/empty mbarriers (weights), per slot act_ready
// (epilogue -> MMA, 512 arrivals) and
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

#include "launch_cache.h"
#include "mlp_fused.h"
#include "sm100.cuh"
#include "surrogate.h"

namespace grrt_b200 {
namespace surr {

namespace {

constexpr int kRows = 128;
constexpr int kStages = 3;
constexpr int kSlots = 2;
constexpr int kEpiWarps = 16;                // 4 per tensor-memory lane quadrant
constexpr int kColGroups = kEpiWarps / 4;     // column groups per row
constexpr int kColsPerThread = kHidden / kColGroups;
constexpr int kThreads = (kEpiWarps + 2) * 32;
constexpr uint32_t kActBytes = 4 * kRows * 128;  // 4 K-blocks of 128 rows x 64 BF16
constexpr uint32_t kStageBytes = kHidden * 128;  // 256 rows x 64 BF16
constexpr uint32_t kWaitLimit = 1u << 22;

// Barriers and the tensor-memory address (the small parameters, W1 and the
// biases, are read through the L1 cache: shared memory holds the two A
// buffers and the weight ring).
// float4 reads of the biases: every bias block starts on a 16-byte boundary
static_assert(ParamLayout::b1 % 4 == 0 && ParamLayout::b2 % 4 == 0 && ParamLayout::b3 % 4 == 0 &&
                  ParamLayout::b4 % 4 == 0 && ParamLayout::b5 % 4 == 0,
              "bias offsets");

struct FusedSmem {
    uint64_t full[kStages];
    uint64_t empty[kStages];
    uint64_t act_ready[kSlots];
    uint64_t acc_ready[kSlots];
    uint32_t tmem_base;
    int failed;
};

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

// Tiles of slot u: blockIdx.x + (2 j + u) gridDim.x, j = 0, 1, ...
__device__ __forceinline__ long long slot_tiles(long long n_tiles, int u) {
    const long long first = blockIdx.x + static_cast<long long>(u) * gridDim.x;
    if (first >= n_tiles) return 0;
    return (n_tiles - 1 - first) / (2ll * gridDim.x) + 1;
}
__device__ __forceinline__ long long slot_tile(int u, long long j) {
    return blockIdx.x + (2 * j + u) * static_cast<long long>(gridDim.x);
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
    unsigned char* act0 = smem_raw + ((1024u - (raw & 1023u)) & 1023u);
    unsigned char* ring = act0 + kSlots * kActBytes;
    FusedSmem* sh = reinterpret_cast<FusedSmem*>(ring + kStages * kStageBytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long n_tiles = (n + kRows - 1) / kRows;
    const long long tiles_of[kSlots] = {slot_tiles(n_tiles, 0), slot_tiles(n_tiles, 1)};
    // steps per slot: 4 MMA layers, or 5 epilogue stages, per tile
    const long long rounds_mma = 4 * tiles_of[0], rounds_epi = 5 * tiles_of[0];

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            sm100::mbar_init(&sh->full[s], 1);
            sm100::mbar_init(&sh->empty[s], 1);
        }
        for (int u = 0; u < kSlots; ++u) {
            sm100::mbar_init(&sh->act_ready[u], kEpiWarps * 32);
            sm100::mbar_init(&sh->acc_ready[u], 1);
        }
        sh->failed = 0;
        sm100::fence_mbar_init();
    }
    if (warp == kEpiWarps) {
        if (lane == 0)
            for (int l = 0; l < 4; ++l) sm100::tma_prefetch_desc(&maps.w[l]);
        sm100::tmem_alloc(&sh->tmem_base, 512);
        sm100::tmem_relinquish();
    }
    sm100::tc_fence_before();
    __syncthreads();
    sm100::tc_fence_after();
    const uint32_t tmem = sh->tmem_base;
    volatile int* failed = &sh->failed;

    if (warp == kEpiWarps) {
        // ---------------- TMA producer: the MMA's weight stream, in its order ----------------
        if (lane == 0) {
            uint32_t it = 0;
            for (long long r = 0; r < rounds_mma && !*failed; ++r) {
                for (int u = 0; u < kSlots && !*failed; ++u) {
                    if (r >= 4 * tiles_of[u]) continue;
                    const int l = static_cast<int>(r % 4);
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
            uint32_t it = 0, n_act[kSlots] = {0, 0};
            const uint32_t id_hidden = sm100::idesc_bf16_f32(kRows, kHidden);
            const uint32_t id_out = sm100::idesc_bf16_f32(kRows, kOutPad);
            for (long long r = 0; r < rounds_mma && !*failed; ++r) {
                for (int u = 0; u < kSlots && !*failed; ++u) {
                    if (r >= 4 * tiles_of[u]) continue;
                    const int l = static_cast<int>(r % 4);
                    if (!sm100::mbar_wait(&sh->act_ready[u], n_act[u] & 1, kWaitLimit)) {
                        atomicCAS(&sh->failed, 0, 2);
                        break;
                    }
                    ++n_act[u];
                    sm100::tc_fence_after();
                    const uint32_t a_base = sm100::smem_u32(act0 + u * kActBytes);
                    const uint32_t acc = tmem + static_cast<uint32_t>(u * kHidden);
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
                            sm100::umma_f16(acc, da + 2 * k, db + 2 * k, l < 3 ? id_hidden : id_out,
                                            (kb > 0 || k > 0) ? 1u : 0u);
                        sm100::umma_commit(&sh->empty[s]);
                    }
                    sm100::umma_commit(&sh->acc_ready[u]);
                    if (!ok) break;
                }
            }
        }
    } else {
        // ---------------- epilogue warps ----------------
        const int quad = warp & 3, group = warp >> 2;
        const int r_in_tile = quad * 32 + lane;
        const int c0 = group * kColsPerThread;
        uint32_t n_acc[kSlots] = {0, 0};
        for (long long rr = 0; rr < rounds_epi && !*failed; ++rr) {
            for (int u = 0; u < kSlots && !*failed; ++u) {
                if (rr >= 5 * tiles_of[u]) continue;
                const int stage = static_cast<int>(rr % 5);  // 0: layer 1; 1-3: hidden layers 2-4; 4: output
                const long long row = slot_tile(u, rr / 5) * kRows + r_in_tile;
                unsigned char* act = act0 + u * kActBytes;
                if (stage == 0) {
                    // layer 1 on the CUDA cores
                    float x0 = 0.f, x1 = 0.f, x2 = 0.f, x3 = 0.f;
                    if (row < n) {
                        const float4 xv = *reinterpret_cast<const float4*>(X + row * kIn);
                        x0 = xv.x;
                        x1 = xv.y;
                        x2 = xv.z;
                        x3 = xv.w;
                    }
                    const float4* w1 = reinterpret_cast<const float4*>(params + ParamLayout::w1);
                    const float4* b1 = reinterpret_cast<const float4*>(params + ParamLayout::b1);
                    for (int k = c0; k < c0 + kColsPerThread; k += 8) {
                        float v[8];
                        const float4 ba = __ldg(b1 + k / 4), bb = __ldg(b1 + k / 4 + 1);
                        const float bv[8] = {ba.x, ba.y, ba.z, ba.w, bb.x, bb.y, bb.z, bb.w};
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const float4 w = __ldg(w1 + k + j);
                            const float z = bv[j] + w.x * x0 + w.y * x1 + w.z * x2 + w.w * x3;
                            v[j] = silu_f(z);
                        }
                        *reinterpret_cast<uint4*>(act + act_offset(r_in_tile, k)) = pack8(v);
                    }
                    fence_proxy_async();
                    mbar_arrive(&sh->act_ready[u]);
                    continue;
                }
                if (!sm100::mbar_wait(&sh->acc_ready[u], n_acc[u] & 1, kWaitLimit)) {
                    atomicCAS(&sh->failed, 0, 4);
                    break;
                }
                ++n_acc[u];
                sm100::tc_fence_after();
                const uint32_t t_row = tmem + static_cast<uint32_t>(u * kHidden) +
                                       (static_cast<uint32_t>(quad * 32) << 16);
                if (stage < 4) {
                    const float* bias = params + ParamLayout::b(stage + 1);
#pragma unroll 1
                    for (int k = c0; k < c0 + kColsPerThread; k += 32) {
                        float v[32];
                        sm100::tmem_ld32(t_row + static_cast<uint32_t>(k), v);
                        const float4* b4 = reinterpret_cast<const float4*>(bias + k);  // one address per warp
#pragma unroll
                        for (int j = 0; j < 32; j += 4) {
                            const float4 b = __ldg(b4 + j / 4);
                            v[j] = silu_f(v[j] + b.x);
                            v[j + 1] = silu_f(v[j + 1] + b.y);
                            v[j + 2] = silu_f(v[j + 2] + b.z);
                            v[j + 3] = silu_f(v[j + 3] + b.w);
                        }
#pragma unroll
                        for (int j = 0; j < 32; j += 8)
                            *reinterpret_cast<uint4*>(act + act_offset(r_in_tile, k + j)) = pack8(v + j);
                    }
                    sm100::tc_fence_before();
                    fence_proxy_async();
                    mbar_arrive(&sh->act_ready[u]);
                } else {
                    float v[16];
                    sm100::tmem_ld16(t_row, v);  // every warp of the quadrant loads (aligned), group 0 stores
                    sm100::tc_fence_before();
                    if (group == 0 && row < n) {
                        const float* b5 = params + ParamLayout::b5;
                        float* o = out + row * kOutPad;
#pragma unroll
                        for (int j = 0; j < 16; j += 4)
                            *reinterpret_cast<float4*>(o + j) =
                                make_float4(v[j] + __ldg(b5 + j), v[j + 1] + __ldg(b5 + j + 1),
                                            v[j + 2] + __ldg(b5 + j + 2), v[j + 3] + __ldg(b5 + j + 3));
                    }
                }
            }
        }
    }
    sm100::tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && sh->failed) atomicExch(err, 100 + sh->failed);
    if (warp == kEpiWarps) sm100::tmem_dealloc(tmem, 512);
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

size_t mlp_fused_smem_bytes() { return 1024 + kSlots * kActBytes + kStages * kStageBytes + sizeof(FusedSmem); }

cudaError_t launch_mlp_fused(const float* X, long long n, const float* params, __nv_bfloat16* const* wb,
                             const __nv_bfloat16* w5b, float* out, int* d_err, cudaStream_t s,
                             const unsigned* d_n) {
    if (n <= 0) return cudaSuccess;
    if ((reinterpret_cast<uintptr_t>(X) & 15) || (reinterpret_cast<uintptr_t>(out) & 15)) return cudaErrorInvalidValue;
    FusedMaps maps;
    for (int l = 0; l < 3; ++l)
        if (!weight_map(&maps.w[l], wb[l], kHidden)) return cudaErrorInvalidValue;
    if (!weight_map(&maps.w[3], w5b, kOutPad)) return cudaErrorInvalidValue;
    struct Shape {
        cudaError_t attr = cudaSuccess;
        int sms = 0;
    };
    // the shared-memory attribute is set once per device, with that device current
    const Shape& sh = per_device_shape<Shape>([](int dev) {
        Shape v;
        v.attr = cudaFuncSetAttribute(mlp_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(mlp_fused_smem_bytes()));
        cudaDeviceGetAttribute(&v.sms, cudaDevAttrMultiProcessorCount, dev);
        return v;
    });
    if (sh.attr != cudaSuccess) return sh.attr;
    const int sms = sh.sms;
    const long long tiles = (n + kRows - 1) / kRows;
    const int grid = static_cast<int>(tiles < sms ? tiles : sms);
    mlp_fused_kernel<<<grid, kThreads, mlp_fused_smem_bytes(), s>>>(maps, X, n, d_n, params, out, d_err);
    return cudaGetLastError();
}

}  // namespace surr
}  // namespace grrt_b200
