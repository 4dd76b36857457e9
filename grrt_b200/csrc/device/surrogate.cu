// Device side of the learned surrogate: training data traced by the FP64
// integrator, the MLP's non-GEMM training kernels (the GEMMs are
// umma_gemm.cu, inference is mlp_fused.cu), and the surrogate render's
// prepare / shade passes.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "integrate.cuh"
#include "mixed_spec.cuh"
#include "shading.cuh"
#include "sm100.cuh"
#include "surrogate.h"
#include "surrogate_geom.cuh"

namespace grrt_b200 {
namespace surr {

namespace {

constexpr unsigned kMask = 0xffffffffu;
constexpr int kTraceThreads = 128;

__device__ __forceinline__ unsigned fetch_work(bool want, unsigned* counter, unsigned total) {
    const int lane = threadIdx.x & 31;
    const unsigned m = __ballot_sync(kMask, want);
    unsigned base = 0;
    if (m) {
        const int leader = __ffs(m) - 1;
        if (lane == leader) base = atomicAdd(counter, static_cast<unsigned>(__popc(m)));
        base = __shfl_sync(kMask, base, leader);
    }
    if (!want) return ~0u;
    const unsigned q = base + __popc(m & ((1u << lane) - 1u));
    return q < total ? q : ~0u;
}

// the same SiLU as the tensor-core epilogues (umma_gemm.cu, mlp_fused.cu)
__device__ __forceinline__ float silu(float z) { return sm100::silu_fast(z); }

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// Camera sample at fractional pixel (x, y): the image-plane angles (both
// scaled by the width, as the reference camera) and the covariant momentum.
__device__ void pixel_ray(const DevScene& S, double x, double y, double p[4], double& alpha, double& beta) {
    alpha = (x - S.width / 2.0) * S.fov / S.width;
    beta = (y - S.height / 2.0) * S.fov / S.width;
    camera_momentum(S, x, y, p);
}

// Closed-form margins of a camera ray (capture > 0 = falls in).
__device__ void ray_margins(const DevScene& S, const double p[4], float& cap, float& graze) {
    const RayConstants rc = constants(S.a, S.cam_pos[2], p);
    const double r_h = S.r_stop - 0.01;
    // an outgoing camera ray (p_r > 0) never turns back inside the camera radius
    cap = (p[1] < 0.0) ? static_cast<float>(capture_margin(S.M, S.a, rc, r_h, S.observer_r)) : -1.0f;
    graze = static_cast<float>(graze_margin(S.a, rc));
}

// Targets of a finished trace (network space).
__device__ void finish_targets(const DevScene& S, int term, int nc, int n_extra, double r1, double r2,
                               const Vec5<double>& y, double pt, double pph, float* Yq) {
    // u = M / r, saturated at the relevance cut: a crossing that moves into the
    // hole and one that never happens before capture give the same u_cut
    const double u_cut = S.M / (kRelevant * S.r_in);
    const double none = (term == kTermEscaped) ? 0.0 : u_cut;
    Yq[kOutU1] = static_cast<float>(nc >= 1 ? fmin(S.M / r1, u_cut) : none);
    Yq[kOutU2] = static_cast<float>(nc >= 2 ? fmin(S.M / r2, u_cut) : none);
    if (term == kTermEscaped) {
        const Vec5<double> d = kerr_rhs<double>(S.M, S.a, pt, pph, y);
        const Vec5<float> k{static_cast<float>(d.r), static_cast<float>(d.th), static_cast<float>(d.ph),
                            static_cast<float>(d.pr), static_cast<float>(d.pth)};
        const mixed::EscapeArc e = mixed::escape_arc(S.r_escape, y, k);
        double th = e.th0, ph = e.ph0;
        const bool flip = mixed::fold_sky(th, ph);
        const double cth = (d.r > 0.0 ? y.r * y.r * d.th / d.r : 0.0) * (flip ? -1.0 : 1.0);
        double sp, cp;
        sincos(ph, &sp, &cp);
        Yq[kOutCosTh] = static_cast<float>(cos(th));
        Yq[kOutSinPh] = static_cast<float>(sp);
        Yq[kOutCosPh] = static_cast<float>(cp);
        Yq[kOutCTh] = static_cast<float>(cth * kCThScale);
    } else {
        Yq[kOutCosTh] = Yq[kOutSinPh] = Yq[kOutCosPh] = Yq[kOutCTh] = 0.0f;
    }
    Yq[6] = static_cast<float>(term);
    Yq[7] = static_cast<float>(n_extra);
}

}  // namespace

// ---------------------------------------------------------------------------
// training data: the plain FP64 method (as the thin-disk kernel) recording the
// first two equatorial crossings, the number of later ones outside
// kRelevant * r_in, and the escape direction
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kTraceThreads, 4)
surr_trace_kernel(const DevScene* __restrict__ scenes, int n_cams, int n_side, int jitter_s, float* __restrict__ X,
                  float* __restrict__ Y, unsigned* queue, DevStats* stats) {
    const unsigned per_cam = static_cast<unsigned>(n_side) * n_side;
    const unsigned total = per_cam * static_cast<unsigned>(n_cams);
    unsigned long long n_att = 0, n_acc = 0;
    unsigned q = ~0u;
    bool live = false, exhausted = false;
    const DevScene* S = scenes;
    Vec5<double> y, k1;  // k1 = f(y), kept from the previous attempt when k1_ok
    bool k1_ok = false;
    double pt = 0, pph = 0, dl = 0, r1 = 0, r2 = 0;
    int retry = 0, step = 0, nc = 0, n_extra = 0;
    while (true) {
        const bool want = !live && !exhausted;
        const unsigned nq = fetch_work(want, queue, total);
        if (want) {
            if (nq == ~0u) {
                exhausted = true;
            } else {
                q = nq;
                S = scenes + q / per_cam;
                const unsigned pix = q % per_cam;
                const int i = static_cast<int>(pix % n_side), j = static_cast<int>(pix / n_side);
                const double xs = i + pixel_hash(i, j, jitter_s, 0), ys = j + pixel_hash(i, j, jitter_s, 1);
                double p[4], alpha, beta;
                pixel_ray(*S, xs, ys, p, alpha, beta);
                y = Vec5<double>{S->cam_pos[1], S->cam_pos[2], S->cam_pos[3], p[1], p[2]};
                pt = p[0];
                pph = p[3];
                float in[4];
                encode_inputs(alpha, beta, S->a, S->cam_pos[2], in);
#pragma unroll
                for (int k = 0; k < 4; ++k) X[4 * static_cast<size_t>(q) + k] = in[k];
                float cap, graze;
                ray_margins(*S, p, cap, graze);
                Y[kYCols * static_cast<size_t>(q) + 8] = cap;
                Y[kYCols * static_cast<size_t>(q) + 9] = graze;
                dl = S->dl0;
                retry = 0;
                step = 0;
                nc = 0;
                n_extra = 0;
                r1 = r2 = 0.0;
                k1_ok = false;
                live = true;
            }
        }
        if (!__any_sync(kMask, live)) break;
        int term = -1;
        if (live && retry == 0) {
            if (step >= S->max_steps) term = kTermMaxSteps;
            else if (y.r < S->r_stop) term = kTermHorizon;
            else if (y.r > S->r_escape) term = kTermEscaped;
        }
        if (live && term < 0) {
            if (!k1_ok) {
                k1 = kerr_rhs<double>(S->M, S->a, pt, pph, y);
                k1_ok = true;
            }
            Vec5<double> y5, k7;
            const double err = dp45_attempt_k1<double>(S->M, S->a, pt, pph, y, dl, k1, y5, k7);
            ++n_att;
            const StepDecision d = pi_control(err, S->tol, dl, retry, y5.r);
            if (d.accept) {
                ++n_acc;
                const double d_prev = y.th - kHalfPi, d_new = y5.th - kHalfPi;
                if (d_prev * d_new < 0.0 && fabs(d_prev - d_new) > 1e-12) {
                    // crossings in time order at any radius (a crossing that goes
                    // to infinity or into the hole leaves its slot continuously);
                    // later ones only matter where a disk can emit
                    const double rc = y.r + (-d_prev / (d_new - d_prev)) * (y5.r - y.r);
                    if (nc == 0) r1 = rc;
                    else if (nc == 1) r2 = rc;
                    else if (rc >= kRelevant * S->r_in) ++n_extra;
                    ++nc;
                }
                y = y5;
                k1 = k7;
                dl = d.next;
                retry = 0;
                ++step;
            } else {
                dl = d.next;
                ++retry;
            }
        }
        if (live && term >= 0) {
            live = false;
            finish_targets(*S, term, nc, n_extra, r1, r2, y, pt, pph, Y + kYCols * static_cast<size_t>(q));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n_att += __shfl_xor_sync(kMask, n_att, o);
        n_acc += __shfl_xor_sync(kMask, n_acc, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&stats->attempts, n_att);
        atomicAdd(&stats->accepted, n_acc);
        atomicAdd(&stats->fp64_attempts, n_att);
    }
}

cudaError_t launch_trace_dataset(const DevScene* d_scenes, int n_cams, int n_side, int jitter_s, float* X, float* Y,
                                 unsigned* queue, DevStats* stats, cudaStream_t s) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, surr_trace_kernel, kTraceThreads, 0);
    if (per < 1) per = 1;
    cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    surr_trace_kernel<<<sms * per, kTraceThreads, 0, s>>>(d_scenes, n_cams, n_side, jitter_s, X, Y, queue, stats);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// training-step kernels
// ---------------------------------------------------------------------------
__global__ void gather_kernel(const float* __restrict__ X, const float* __restrict__ Y, size_t n_data, int batch,
                              const unsigned* step, float* __restrict__ Xb, float* __restrict__ Yb) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= batch) return;
    const uint64_t h = splitmix64((static_cast<uint64_t>(*step) << 32) ^ static_cast<uint64_t>(r));
    const size_t q = static_cast<size_t>(h % n_data);
#pragma unroll
    for (int k = 0; k < kIn; ++k) Xb[static_cast<size_t>(r) * kIn + k] = X[q * kIn + k];
#pragma unroll
    for (int k = 0; k < kYCols; ++k) Yb[static_cast<size_t>(r) * kYCols + k] = Y[q * kYCols + k];
}

cudaError_t launch_gather(const float* X, const float* Y, size_t n_data, int batch, const unsigned* step, float* Xb,
                          float* Yb, cudaStream_t s) {
    gather_kernel<<<(batch + 255) / 256, 256, 0, s>>>(X, Y, n_data, batch, step, Xb, Yb);
    return cudaGetLastError();
}

// one thread per hidden unit, blocks stride over rows
__global__ void __launch_bounds__(kHidden)
layer1_fwd_kernel(const float* __restrict__ Xb, int rows, const float* __restrict__ params, float* __restrict__ Z1,
                  __nv_bfloat16* __restrict__ H1) {
    const int f = threadIdx.x;
    const float* W = params + ParamLayout::w1 + static_cast<size_t>(f) * kIn;
    const float w0 = W[0], w1 = W[1], w2 = W[2], w3 = W[3], b = params[ParamLayout::b1 + f];
    for (int r = blockIdx.x; r < rows; r += gridDim.x) {
        const float* x = Xb + static_cast<size_t>(r) * kIn;
        const float z = b + w0 * x[0] + w1 * x[1] + w2 * x[2] + w3 * x[3];
        if (Z1) Z1[static_cast<size_t>(r) * kHidden + f] = z;
        H1[static_cast<size_t>(r) * kHidden + f] = __float2bfloat16_rn(silu(z));
    }
}

cudaError_t launch_layer1_fwd(const float* Xb, int rows, const float* params, float* Z1, __nv_bfloat16* H1,
                              cudaStream_t s) {
    int grid = rows < 148 * 16 ? rows : 148 * 16;
    if (grid < 1) grid = 1;
    layer1_fwd_kernel<<<grid, kHidden, 0, s>>>(Xb, rows, params, Z1, H1);
    return cudaGetLastError();
}

// Masked weighted MSE over the six outputs; dO = d(loss)/dO as BF16 [rows x 64]
// (columns 6..15 written as zero, 16..63 left as they are: zero).
__global__ void loss_kernel(const float* __restrict__ O, const float* __restrict__ Yb, int rows, LossWeights w,
                            __nv_bfloat16* __restrict__ dO, float* loss) {
    __shared__ float red[8];
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (r < rows) {
        const float* o = O + static_cast<size_t>(r) * kOutPad;
        const float* y = Yb + static_cast<size_t>(r) * kYCols;
        const int term = static_cast<int>(y[6]);
        // rays near the critical curve, grazing the plane, or with three or more
        // crossings are re-traced exactly at render time: not fitted
        const bool fit = fabsf(y[8]) >= kFitCapture && y[9] >= kFitGraze && y[7] == 0.0f;
        const bool u_ok = fit && (term == kTermHorizon || term == kTermEscaped);
        const bool esc = fit && term == kTermEscaped;
        const float inv = 1.0f / rows;
        __nv_bfloat16* g = dO + static_cast<size_t>(r) * kDOutPad;
#pragma unroll
        for (int j = 0; j < kOutPad; ++j) {
            float gj = 0.0f;
            if (j < kTargets) {
                float wt = 0.0f;
                if (j < 2) wt = u_ok ? w.u : 0.0f;
                else if (j < 5) wt = esc ? w.dir : 0.0f;
                else wt = esc ? w.cth : 0.0f;
                const float d = o[j] - y[j];
                l += wt * d * d;
                gj = 2.0f * wt * d * inv;
            } else if (j < kOutLogSigDir && u_ok) {
                // log-sigma head of u slot j - kTargets: NLL with the residual fixed
                const float d = o[j - kTargets] - y[j - kTargets];
                const float s = fminf(fmaxf(o[j], -12.0f), 4.0f);
                const float e = __expf(-2.0f * s);
                l += w.sig * 0.5f * (d * d * e + 2.0f * s);
                gj = w.sig * (1.0f - d * d * e) * inv;
            } else if (j == kOutLogSigDir && esc) {
                // direction head: isotropic 3-d residual of outputs 2-4
                float d2 = 0.0f;
#pragma unroll
                for (int c = kOutCosTh; c <= kOutCosPh; ++c) d2 += (o[c] - y[c]) * (o[c] - y[c]);
                const float s = fminf(fmaxf(o[j], -12.0f), 4.0f);
                const float e = __expf(-2.0f * s);
                l += w.sig * 0.5f * (d2 * e + 6.0f * s);
                gj = w.sig * (3.0f - d2 * e) * inv;
            }
            g[j] = __float2bfloat16_rn(gj);
        }
        l *= inv;
    }
#pragma unroll
    for (int k = 16; k > 0; k >>= 1) l += __shfl_xor_sync(kMask, l, k);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int k = 0; k < static_cast<int>(blockDim.x >> 5); ++k) t += red[k];
        atomicAdd(loss, t);
    }
}

cudaError_t launch_loss(const float* O, const float* Yb, int rows, LossWeights w, __nv_bfloat16* dO, float* loss,
                        cudaStream_t s) {
    loss_kernel<<<(rows + 255) / 256, 256, 0, s>>>(O, Yb, rows, w, dO, loss);
    return cudaGetLastError();
}

// 32x32 tiles through shared memory; out[c][r] = in[r][c]
__global__ void transpose_kernel(const __nv_bfloat16* __restrict__ in, int rows, int cols, int ld_in,
                                 __nv_bfloat16* __restrict__ out, int ld_out) {
    __shared__ __nv_bfloat16 tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        tile[k][threadIdx.x] =
            (r < rows && c < cols) ? in[static_cast<size_t>(r) * ld_in + c] : __float2bfloat16_rn(0.0f);
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (c < cols && r < rows) out[static_cast<size_t>(c) * ld_out + r] = tile[threadIdx.x][k];
    }
}

cudaError_t launch_transpose(const __nv_bfloat16* in, int rows, int cols, int ld_in, __nv_bfloat16* out, int ld_out,
                             cudaStream_t s) {
    dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
    transpose_kernel<<<grid, block, 0, s>>>(in, rows, cols, ld_in, out, ld_out);
    return cudaGetLastError();
}

// partials[g][c] = sum of rows g, g + G, ... of column c
__global__ void colsum_kernel(const __nv_bfloat16* __restrict__ A, int rows, int cols, int ld,
                              float* __restrict__ partials) {
    const int c = threadIdx.x;
    if (c >= cols) return;
    float acc = 0.0f;
    for (int r = blockIdx.x; r < rows; r += gridDim.x) acc += __bfloat162float(A[static_cast<size_t>(r) * ld + c]);
    partials[static_cast<size_t>(blockIdx.x) * cols + c] = acc;
}

__global__ void reduce_rows_kernel(const float* __restrict__ part, int parts, size_t n, float* __restrict__ out) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    float acc = 0.0f;
    for (int p = 0; p < parts; ++p) acc += part[static_cast<size_t>(p) * n + i];
    out[i] = acc;
}

cudaError_t launch_colsum(const __nv_bfloat16* A, int rows, int cols, int ld, float* partials, int grid_parts,
                          float* out, cudaStream_t s) {
    colsum_kernel<<<grid_parts, 256, 0, s>>>(A, rows, cols, ld, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    reduce_rows_kernel<<<(cols + 255) / 256, 256, 0, s>>>(partials, grid_parts, static_cast<size_t>(cols), out);
    return cudaGetLastError();
}

// dW1[f][i] = sum_r dZ1[r][f] X[r][i], db1[f] = sum_r dZ1[r][f]: partials per
// row group [g][f][4] and [g][b1 f], reduced into grad (W1 block, then b1).
__global__ void __launch_bounds__(kHidden)
layer1_bwd_kernel(const __nv_bfloat16* __restrict__ dZ1, const float* __restrict__ Xb, int rows,
                  float* __restrict__ partials) {
    const int f = threadIdx.x;
    float a0 = 0, a1 = 0, a2 = 0, a3 = 0, ab = 0;
    for (int r = blockIdx.x; r < rows; r += gridDim.x) {
        const float g = __bfloat162float(dZ1[static_cast<size_t>(r) * kHidden + f]);
        const float* x = Xb + static_cast<size_t>(r) * kIn;
        a0 += g * x[0];
        a1 += g * x[1];
        a2 += g * x[2];
        a3 += g * x[3];
        ab += g;
    }
    float* p = partials + static_cast<size_t>(blockIdx.x) * (kHidden * 5);
    p[f * 4 + 0] = a0;
    p[f * 4 + 1] = a1;
    p[f * 4 + 2] = a2;
    p[f * 4 + 3] = a3;
    p[kHidden * 4 + f] = ab;
}

cudaError_t launch_layer1_bwd(const __nv_bfloat16* dZ1, const float* Xb, int rows, float* partials, int grid_parts,
                              float* grad, cudaStream_t s) {
    layer1_bwd_kernel<<<grid_parts, kHidden, 0, s>>>(dZ1, Xb, rows, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    static_assert(ParamLayout::b1 == ParamLayout::w1 + kHidden * kIn, "W1 and b1 are contiguous");
    reduce_rows_kernel<<<(kHidden * 5 + 255) / 256, 256, 0, s>>>(partials, grid_parts, kHidden * 5,
                                                                  grad + ParamLayout::w1);
    return cudaGetLastError();
}

cudaError_t launch_reduce_splits(const float* part, int splits, size_t n, float* out, cudaStream_t s) {
    reduce_rows_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(part, splits, n, out);
    return cudaGetLastError();
}

__global__ void adam_begin_kernel(unsigned* step) { *step += 1; }

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, size_t n, const unsigned* step, float lr, float b1, float b2,
                            float eps) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const float t = static_cast<float>(*step);
    const float c1 = 1.0f - powf(b1, t), c2 = 1.0f - powf(b2, t);
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

cudaError_t launch_adam(float* params, const float* grad, float* m, float* v, size_t n, unsigned* step, float lr,
                        float beta1, float beta2, float eps, cudaStream_t s) {
    adam_begin_kernel<<<1, 1, 0, s>>>(step);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    adam_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(params, grad, m, v, n, step, lr, beta1, beta2,
                                                                       eps);
    return cudaGetLastError();
}

__global__ void record_loss_kernel(const float* loss, const unsigned* step, float* hist, int cap) {
    const unsigned t = *step;  // already advanced by this step's optimiser update
    if (t >= 1 && static_cast<int>(t - 1) < cap) hist[t - 1] = *loss;
}

cudaError_t launch_record_loss(const float* loss, const unsigned* step, float* hist, int cap, cudaStream_t s) {
    record_loss_kernel<<<1, 1, 0, s>>>(loss, step, hist, cap);
    return cudaGetLastError();
}

struct CastTargets {
    __nv_bfloat16* wb[3];
    __nv_bfloat16* wt[3];
    __nv_bfloat16* w5b;
    __nv_bfloat16* w5t;
};

__global__ void cast_kernel(const float* __restrict__ params, CastTargets t) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;  // over 3 * 256 * 256 + 16 * 256
    constexpr int kSq = kHidden * kHidden;
    if (idx < 3 * kSq) {
        const int l = idx / kSq, e = idx % kSq;
        const int o = e / kHidden, i = e % kHidden;
        const __nv_bfloat16 v = __float2bfloat16_rn(params[ParamLayout::w(l + 2) + e]);
        t.wb[l][e] = v;
        t.wt[l][static_cast<size_t>(i) * kHidden + o] = v;
    } else if (idx < 3 * kSq + kOutPad * kHidden) {
        const int e = idx - 3 * kSq;
        const int o = e / kHidden, i = e % kHidden;
        const __nv_bfloat16 v = __float2bfloat16_rn(params[ParamLayout::w5 + e]);
        t.w5b[e] = v;
        t.w5t[static_cast<size_t>(i) * kDOutPad + o] = v;
    }
}

cudaError_t launch_cast_weights(const float* params, __nv_bfloat16* const* wb, __nv_bfloat16* const* wt,
                                __nv_bfloat16* w5b, __nv_bfloat16* w5t, cudaStream_t s) {
    CastTargets t;
    for (int l = 0; l < 3; ++l) {
        t.wb[l] = wb[l];
        t.wt[l] = wt[l];
    }
    t.w5b = w5b;
    t.w5t = w5t;
    const int n = 3 * kHidden * kHidden + kOutPad * kHidden;
    cast_kernel<<<(n + 255) / 256, 256, 0, s>>>(params, t);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// render: prepare (inputs + closed-form margins), shade (colour or re-trace)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void sample_coords(const DevScene& S, const DevTile& tile, size_t q, double& x, double& yy) {
    const int g2 = S.grid * S.grid;
    const int pix = static_cast<int>(q / g2), s = static_cast<int>(q % g2);
    const int i = tile.x0 + pix % tile.w, j = tile.y0 + (pix / tile.w) * tile.row_step;
    const int sy = s / S.grid, sx = s % S.grid;
    x = i + (sx + pixel_hash(i, j, s, 0)) * S.cell;
    yy = j + (sy + pixel_hash(i, j, s, 1)) * S.cell;
}

__global__ void prepare_kernel(const __grid_constant__ DevScene S, const DevTile tile, size_t q0, size_t nq,
                               double settle_radius, float* __restrict__ X, SampleAux* __restrict__ aux,
                               unsigned* __restrict__ count, unsigned* __restrict__ total, DevMixedBuffers mb,
                               DevStats* stats) {
    // whole warps stay together for the ballots
    const size_t k = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    const int lane = threadIdx.x & 31;
    bool keep = false, settled = false;
    double p[4] = {0, 0, 0, 0}, alpha = 0, beta = 0;
    const unsigned q = static_cast<unsigned>(q0 + k);
    if (k < nq) {
        double x, yy;
        sample_coords(S, tile, q0 + k, x, yy);
        pixel_ray(S, x, yy, p, alpha, beta);
        // black sky: never near the disk, the hole or a photon orbit (closed
        // form): colour 0 and escaped, as the FP64 method gives it
        settled = settle_radius > 0.0 &&
                  camera_ray_clears(S.M, S.a, S.r_stop - 0.01, S.cam_pos[1], S.cam_pos[2], p, settle_radius);
        keep = !settled;
        if (settled) {
            mb.sample_rgb[3 * static_cast<size_t>(q) + 0] = 0.0;
            mb.sample_rgb[3 * static_cast<size_t>(q) + 1] = 0.0;
            mb.sample_rgb[3 * static_cast<size_t>(q) + 2] = 0.0;
            mb.sample_fate[q] = static_cast<unsigned>(kTermEscaped);
        }
    }
    const unsigned m = __ballot_sync(kMask, keep);
    const unsigned ns = __popc(__ballot_sync(kMask, settled));
    if (lane == 0 && ns) atomicAdd(&stats->rays, static_cast<unsigned long long>(ns));
    if (!m) return;
    const int leader = __ffs(m) - 1;
    unsigned base = 0;
    if (lane == leader) {
        base = atomicAdd(count, static_cast<unsigned>(__popc(m)));
        atomicAdd(total, static_cast<unsigned>(__popc(m)));
    }
    base = __shfl_sync(kMask, base, leader);
    if (!keep) return;
    const unsigned j = base + __popc(m & ((1u << lane) - 1u));
    float in[4];
    encode_inputs(alpha, beta, S.a, S.cam_pos[2], in);
    *reinterpret_cast<float4*>(X + 4 * static_cast<size_t>(j)) = make_float4(in[0], in[1], in[2], in[3]);
    SampleAux a;
    a.pt = p[0];
    a.pph = p[3];
    ray_margins(S, p, a.capture_margin, a.graze_margin);
    a.q = q;
    aux[j] = a;
}

cudaError_t launch_prepare(const DevScene& S, const DevTile& tile, size_t q0, size_t nq, double settle_radius,
                           float* X, SampleAux* aux, unsigned* count, unsigned* total, const DevMixedBuffers& mb,
                           DevStats* stats, cudaStream_t s) {
    if (nq == 0) return cudaSuccess;
    prepare_kernel<<<static_cast<unsigned>((nq + 127) / 128), 128, 0, s>>>(S, tile, q0, nq, settle_radius, X, aux,
                                                                          count, total, mb, stats);
    return cudaGetLastError();
}

__device__ __forceinline__ void add_emission(const DevScene& S, double r, double pt, double pph, double c[3]) {
    double e0, e1, e2;
    disk_emission(S, r, pt, pph, e0, e1, e2);
    c[0] += e0;
    c[1] += e1;
    c[2] += e2;
}

// append sample q to a list (warp-aggregated over the lanes that want to)
__device__ __forceinline__ void append(bool want, unsigned q, unsigned* count, unsigned* list) {
    const int lane = threadIdx.x & 31;
    const unsigned m = __ballot_sync(kMask, want);
    if (!m) return;
    const int leader = __ffs(m) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(count, static_cast<unsigned>(__popc(m)));
    base = __shfl_sync(kMask, base, leader);
    if (want) list[base + __popc(m & ((1u << lane) - 1u))] = q;
}

__global__ void shade_kernel(const __grid_constant__ DevScene S, const DevTile tile, const unsigned* count,
                             size_t cap, const float* __restrict__ O, const SampleAux* __restrict__ aux,
                             RenderBands bands, DevMixedBuffers mb, DevStats* stats) {
    // whole warps stay together for the ballots in append
    const size_t k = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    const size_t nq = *count < cap ? *count : cap;
    bool exact = false;    // colour depends on the FP64 steps: re-trace
    bool uncertain = false;  // the network cannot rule out the disk: FP32 speculation decides
    unsigned q = 0;
    if (k < nq) {
        const SampleAux a = aux[k];
        q = a.q;
        const float* o = O + k * kOutPad;
        if (fabsf(a.capture_margin) < bands.capture || a.graze_margin < bands.graze) exact = true;
        const bool captured = a.capture_margin > 0.0f;
        double col[3] = {0.0, 0.0, 0.0};
        int nc = 0;
        if (!exact && S.disk_on) {
            if (!(o[0] == o[0]) || !(o[1] == o[1])) exact = true;  // NaN
            for (int c = 0; c < 2 && !exact; ++c) {
                const double u = o[c];
                // this sample's u error band: the calibrated multiple of its predicted sigma
                const double du = bands.du * exp(fmin(fmax(static_cast<double>(o[kOutLogSig1 + c]), -12.0), 4.0));
                if (!(u + du > 0.0)) continue;  // no crossing: escapes first
                const double r = S.M / fmax(u, 1e-12);
                // radius band: r in [M/(u+du), M/(u-du)]
                const double r_lo = S.M / (u + du);
                const double r_hi = (u > du) ? S.M / (u - du) : 1e30;
                if (r_hi < S.r_in || r_lo > S.r_out) continue;  // surely outside the disk
                if (r_lo <= S.r_in || r_hi >= S.r_out) {
                    // may cross an edge: lit or dark is the FP32 speculation's call
                    // when the predicted radius lies outside the disk, else exact
                    if (r < S.r_in || r > S.r_out) uncertain = true;
                    else exact = true;
                    break;
                }
                double cm[3] = {0, 0, 0}, lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
                add_emission(S, r, a.pt, a.pph, cm);
                add_emission(S, r_lo, a.pt, a.pph, lo);
                add_emission(S, r_hi, a.pt, a.pph, hi);
                for (int ch = 0; ch < 3; ++ch) {
                    const double ref = fabs(cm[ch]);
                    if (fabs(lo[ch] - cm[ch]) > bands.tol_rel * ref || fabs(hi[ch] - cm[ch]) > bands.tol_rel * ref)
                        exact = true;
                }
                if (!(cm[0] > 0.0 || cm[1] > 0.0 || cm[2] > 0.0)) exact = true;  // at an emission threshold
                col[0] += cm[0];
                col[1] += cm[1];
                col[2] += cm[2];
                ++nc;
            }
        }
        if (!exact && !uncertain && !captured && S.stars_on) {
            const float ct = o[kOutCosTh], sp = o[kOutSinPh], cp = o[kOutCosPh];
            const float nrm = sp * sp + cp * cp;
            // a star possibly in reach: the speculative pass, whose FP32
            // trajectory gives the sky arc far more precisely, decides
            if (!(fabsf(ct) < 0.999f) || !(nrm > 0.5f && nrm < 2.0f)) {
                uncertain = true;
            } else {
                mixed::EscapeArc e;
                e.th0 = acos(static_cast<double>(ct));
                e.ph0 = atan2(static_cast<double>(sp), static_cast<double>(cp));
                const double s_th = sin(e.th0);
                const double E = -a.pt;
                const double du = 1.0 / S.r_escape - 1.0 / (7.0 * S.r_escape);
                // far field: c_theta learned, c_phi = r^2 dphi/dr -> L / (E sin^2 theta)
                const double cth = o[kOutCTh] / kCThScale;
                const double cph = a.pph / (E * s_th * s_th);
                e.dth = static_cast<float>(cth * du);
                e.dph = static_cast<float>(cph * du);
                const double dir_band =
                    bands.dir * exp(fmin(fmax(static_cast<double>(o[kOutLogSigDir]), -12.0), 4.0));
                if (mixed::star_in_reach(S.stars, e, 1e-4 + dir_band)) uncertain = true;
            }
        }
        if (exact) uncertain = false;
        if (!exact && !uncertain) {
            mb.sample_rgb[3 * static_cast<size_t>(q) + 0] = col[0];
            mb.sample_rgb[3 * static_cast<size_t>(q) + 1] = col[1];
            mb.sample_rgb[3 * static_cast<size_t>(q) + 2] = col[2];
            mb.sample_fate[q] =
                static_cast<unsigned>(captured ? kTermHorizon : kTermEscaped) | (static_cast<unsigned>(nc) << 2);
        }
    }
    append(exact, q, mb.retrace_count, mb.retrace_list);
    append(uncertain, q, mb.spec_count, mb.spec_list);
    const unsigned live = __ballot_sync(kMask, k < nq);
    if ((threadIdx.x & 31) == 0 && live) atomicAdd(&stats->rays, static_cast<unsigned long long>(__popc(live)));
}

cudaError_t launch_shade(const DevScene& S, const DevTile& tile, const unsigned* count, size_t cap, const float* O,
                         const SampleAux* aux, const RenderBands& bands, const DevMixedBuffers& mb, DevStats* stats,
                         cudaStream_t s) {
    const size_t nq = cap;
    if (nq == 0) return cudaSuccess;
    shade_kernel<<<static_cast<unsigned>((nq + 127) / 128), 128, 0, s>>>(S, tile, count, cap, O, aux, bands, mb,
                                                                        stats);
    return cudaGetLastError();
}

__global__ void eval_errors_kernel(const float* __restrict__ O, const float* __restrict__ Y, size_t n,
                                   float* __restrict__ err) {
    const size_t q = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (q >= n) return;
    const float* o = O + q * kOutPad;
    const float* y = Y + q * kYCols;
    const int term = static_cast<int>(y[6]);
    float* e = err + q * 4;
    const bool u_ok = term == kTermHorizon || term == kTermEscaped;
    e[0] = u_ok ? fabsf(o[0] - y[0]) * __expf(-fminf(fmaxf(o[kOutLogSig1], -12.0f), 4.0f)) : -1.0f;
    e[1] = u_ok ? fabsf(o[1] - y[1]) * __expf(-fminf(fmaxf(o[kOutLogSig2], -12.0f), 4.0f)) : -1.0f;
    if (term == kTermEscaped) {
        // angle between the predicted and true arc-start directions
        const float st_p = sqrtf(fmaxf(0.0f, 1.0f - o[2] * o[2])), st_t = sqrtf(fmaxf(0.0f, 1.0f - y[2] * y[2]));
        const float np = rsqrtf(fmaxf(o[3] * o[3] + o[4] * o[4], 1e-12f));
        const float px = st_p * o[4] * np, py = st_p * o[3] * np, pz = o[2];
        const float tx = st_t * y[4], ty = st_t * y[3], tz = y[2];
        const float dx = px - tx, dy = py - ty, dz = pz - tz;
        const float inv_sig = __expf(-fminf(fmaxf(o[kOutLogSigDir], -12.0f), 4.0f));
        e[2] = 2.0f * asinf(fminf(1.0f, 0.5f * sqrtf(dx * dx + dy * dy + dz * dz))) * inv_sig;
        e[3] = fabsf(o[5] - y[5]) / static_cast<float>(kCThScale) * inv_sig;
    } else {
        e[2] = e[3] = -1.0f;
    }
}

cudaError_t launch_eval_errors(const float* O, const float* Y, size_t n, float* err, cudaStream_t s) {
    eval_errors_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(O, Y, n, err);
    return cudaGetLastError();
}

}  // namespace surr
}  // namespace grrt_b200
