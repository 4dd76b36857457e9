// Tone mapping on the device, in place on a linear-HDR RGBA float frame: the
// reference's ToneMapper::apply_all (src/tonemapper.cpp:7-71), i.e.
// log-average auto exposure (key 0.18, lit above luminance 1e-10), extended
// Reinhard with the white point at the frame's brightest pixel, and gamma 2.2.
//
// Pass 1: per block, the sum of log(1e-6 + L) over the lit pixels, their count
// and the largest L (grid-stride, warp and block reductions in a fixed
// order). Pass 2 (one block): the block partials combined in block order
// (deterministic), then the exposure and the white point. Pass 3: the per-pixel
// map. The host version sums the logs pixel by pixel with the C library's
// log/exp/pow; here the sum is grouped by blocks and the functions are CUDA's,
// so the two agree to a few float ulp, not bit for bit.
#include <cuda_runtime.h>

#include <cstdint>

#include "render_launch.h"

namespace grrt_b200 {

namespace {

constexpr int kTmThreads = 256;
constexpr unsigned kAll = 0xffffffffu;
constexpr double kKey = 0.18, kDelta = 1e-6, kLit = 1e-10;

struct TmPartial {
    double log_sum;
    double l_max;
    unsigned long long count;
};

struct TmParams {
    double exposure;
    double white2;  // (L_max * exposure)^2
    int active;     // 0: an all-black frame, left as it is
};

__device__ __forceinline__ double luminance(const float4 p, double& R, double& G, double& B) {
    R = fmax(0.0, static_cast<double>(p.x));
    G = fmax(0.0, static_cast<double>(p.y));
    B = fmax(0.0, static_cast<double>(p.z));
    return 0.2126 * R + 0.7152 * G + 0.0722 * B;
}

__global__ void __launch_bounds__(kTmThreads) tm_stats_kernel(const float4* __restrict__ px, long long n,
                                                              TmPartial* __restrict__ part) {
    double s = 0.0, m = 0.0;
    unsigned long long c = 0;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        double R, G, B;
        const double L = luminance(px[i], R, G, B);
        if (L > kLit) {
            s += log(kDelta + L);
            ++c;
        }
        if (L > m) m = L;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(kAll, s, o);
        c += __shfl_xor_sync(kAll, c, o);
        m = fmax(m, __shfl_xor_sync(kAll, m, o));
    }
    __shared__ double ss[kTmThreads / 32], sm[kTmThreads / 32];
    __shared__ unsigned long long sc[kTmThreads / 32];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        ss[w] = s;
        sm[w] = m;
        sc[w] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        TmPartial p{0.0, 0.0, 0};
        for (int k = 0; k < kTmThreads / 32; ++k) {
            p.log_sum += ss[k];
            p.count += sc[k];
            p.l_max = fmax(p.l_max, sm[k]);
        }
        part[blockIdx.x] = p;
    }
}

__global__ void __launch_bounds__(kTmThreads) tm_params_kernel(const TmPartial* __restrict__ part, int nparts,
                                                               TmParams* __restrict__ prm) {
    __shared__ double ss[kTmThreads], sm[kTmThreads];
    __shared__ unsigned long long sc[kTmThreads];
    double s = 0.0, m = 0.0;
    unsigned long long c = 0;
    for (int k = threadIdx.x; k < nparts; k += blockDim.x) {
        s += part[k].log_sum;
        c += part[k].count;
        m = fmax(m, part[k].l_max);
    }
    ss[threadIdx.x] = s;
    sm[threadIdx.x] = m;
    sc[threadIdx.x] = c;
    __syncthreads();
    for (int h = kTmThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            ss[threadIdx.x] += ss[threadIdx.x + h];
            sc[threadIdx.x] += sc[threadIdx.x + h];
            sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        TmParams p{0.0, 0.0, 0};
        if (sm[0] > 0.0 && sc[0] > 0) {
            const double l_avg = exp(ss[0] / static_cast<double>(sc[0]));
            p.exposure = kKey / l_avg;
            const double lw = sm[0] * p.exposure;
            p.white2 = lw * lw;
            p.active = 1;
        }
        *prm = p;
    }
}

__device__ __forceinline__ float gamma_encode(double v) {
    return static_cast<float>(pow(fmin(fmax(v, 0.0), 1.0), 1.0 / 2.2));
}

__global__ void __launch_bounds__(kTmThreads) tm_map_kernel(float4* __restrict__ px, long long n,
                                                            const TmParams* __restrict__ prm) {
    const TmParams p = *prm;
    if (!p.active) return;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        float4 v = px[i];
        double R, G, B;
        const double L = luminance(v, R, G, B);
        if (L <= 0.0) {
            v.x = v.y = v.z = 0.0f;
        } else {
            const double ls = L * p.exposure;
            const double lm = fmin(fmax(ls * (1.0 + ls / p.white2) / (1.0 + ls), 0.0), 1.0);
            const double scale = lm / L;
            v.x = gamma_encode(R * scale);
            v.y = gamma_encode(G * scale);
            v.z = gamma_encode(B * scale);
        }
        px[i] = v;
    }
}

}  // namespace

cudaError_t launch_tonemap(float* d_rgba, int width, int height, cudaStream_t stream) {
    const long long n = static_cast<long long>(width) * height;
    if (n <= 0) return cudaSuccess;
    if (reinterpret_cast<uintptr_t>(d_rgba) & 15) return cudaErrorInvalidValue;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    long long want = (n + kTmThreads - 1) / kTmThreads;
    const int nparts = static_cast<int>(want < 4LL * sms ? want : 4LL * sms);
    void* scratch = nullptr;
    e = cudaMallocAsync(&scratch, sizeof(TmPartial) * nparts + sizeof(TmParams), stream);
    if (e != cudaSuccess) return e;
    auto* part = static_cast<TmPartial*>(scratch);
    auto* prm = reinterpret_cast<TmParams*>(part + nparts);
    auto* px = reinterpret_cast<float4*>(d_rgba);
    tm_stats_kernel<<<nparts, kTmThreads, 0, stream>>>(px, n, part);
    tm_params_kernel<<<1, kTmThreads, 0, stream>>>(part, nparts, prm);
    tm_map_kernel<<<nparts, kTmThreads, 0, stream>>>(px, n, prm);
    e = cudaGetLastError();
    const cudaError_t f = cudaFreeAsync(scratch, stream);
    return e != cudaSuccess ? e : f;
}

}  // namespace grrt_b200
