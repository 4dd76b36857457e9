// Device side of the learned surrogate (surrogate.cu): data generation with
// the FP64 integrator, the MLP's training kernels, and the surrogate render's
// prepare / shade passes.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "render_launch.h"
#include "scene.h"

namespace grrt_b200 {
namespace surr {

constexpr int kIn = 4;
constexpr int kHidden = 256;
constexpr int kTargets = 6;   // fitted quantities (u1, u2, cos theta, sin phi, cos phi, c_theta)
constexpr int kUsedOut = 9;   // outputs: the targets, then log sigma of the u1, u2 and direction errors
constexpr int kOutPad = 16;   // output layer rows computed by the GEMM (kUsedOut used)
constexpr int kDOutPad = 64;  // K of the output layer's backward GEMM
constexpr int kYCols = 10;    // 6 targets, termination, later crossings, capture margin, graze margin
// Targets u1, u2: u = M / r of the first and second equatorial crossing in
// time order, saturated at M / (kRelevant r_in) (no disk emits inside); 0 when
// the ray escapes first, the saturation value when it falls in first. Later
// crossings count only outside kRelevant * r_in (record column 7).
constexpr double kRelevant = 0.9;

// Offsets (floats) of the parameters in one FP32 array.
struct ParamLayout {
    static constexpr size_t w1 = 0, b1 = w1 + kHidden * kIn;
    static constexpr size_t w2 = b1 + kHidden, b2 = w2 + kHidden * kHidden;
    static constexpr size_t w3 = b2 + kHidden, b3 = w3 + kHidden * kHidden;
    static constexpr size_t w4 = b3 + kHidden, b4 = w4 + kHidden * kHidden;
    static constexpr size_t w5 = b4 + kHidden, b5 = w5 + kOutPad * kHidden;
    static constexpr size_t total = b5 + kOutPad;
    __host__ __device__ static constexpr size_t w(int l) {
        return l == 2 ? w2 : l == 3 ? w3 : l == 4 ? w4 : l == 5 ? w5 : w1;
    }
    __host__ __device__ static constexpr size_t b(int l) {
        return l == 2 ? b2 : l == 3 ? b3 : l == 4 ? b4 : l == 5 ? b5 : b1;
    }
};

// Loss weights: squared error of the six targets, and the Gaussian negative
// log-likelihood of the log-sigma heads with the residual held fixed (the
// heads learn the error, not the value): 0.5 (d^2 exp(-2 s) + 2 s) for u1 and
// u2, 0.5 (|d|^2 exp(-2 s) + 6 s) for the three direction outputs.
struct LossWeights {
    float u = 16.0f, dir = 0.5f, cth = 0.25f, sig = 0.1f;
};
// Samples fitted: capture margin |m| >= kFitCapture, graze margin >=
// kFitGraze, no relevant crossing after the second (the rest is the exact
// path's; the calibrated bands never fall below these).
constexpr float kFitCapture = 0.05f;
constexpr float kFitGraze = 0.02f;

// Data: every sample of n_cams cameras x (n_side x n_side) pixels, jittered by
// the reference's pixel hash with sample index `jitter_s` (0 train, 1 validation).
// X[q][4] network inputs; Y[q][10] the six targets, termination, number of
// crossings after the second outside kRelevant * r_in, capture margin, graze
// margin.
cudaError_t launch_trace_dataset(const DevScene* d_scenes, int n_cams, int n_side, int jitter_s, float* X, float* Y,
                                 unsigned* queue, DevStats* stats, cudaStream_t s);

// Training-step pieces.
cudaError_t launch_gather(const float* X, const float* Y, size_t n_data, int batch, const unsigned* step,
                          float* Xb, float* Yb, cudaStream_t s);
cudaError_t launch_layer1_fwd(const float* Xb, int rows, const float* params, float* Z1, __nv_bfloat16* H1,
                              cudaStream_t s);
cudaError_t launch_loss(const float* O, const float* Yb, int rows, LossWeights w, __nv_bfloat16* dO, float* loss,
                        cudaStream_t s);
cudaError_t launch_transpose(const __nv_bfloat16* in, int rows, int cols, int ld_in, __nv_bfloat16* out, int ld_out,
                             cudaStream_t s);
// Column sums of a BF16 matrix into out[cols] (partials: grid_parts x cols floats).
cudaError_t launch_colsum(const __nv_bfloat16* A, int rows, int cols, int ld, float* partials, int grid_parts,
                          float* out, cudaStream_t s);
cudaError_t launch_layer1_bwd(const __nv_bfloat16* dZ1, const float* Xb, int rows, float* partials, int grid_parts,
                              float* grad, cudaStream_t s);
cudaError_t launch_reduce_splits(const float* part, int splits, size_t n, float* out, cudaStream_t s);
cudaError_t launch_adam(float* params, const float* grad, float* m, float* v, size_t n, unsigned* step, float lr,
                        float beta1, float beta2, float eps, cudaStream_t s);
cudaError_t launch_record_loss(const float* loss, const unsigned* step, float* hist, int cap, cudaStream_t s);
// BF16 copies of the GEMM layers: wb[l] [out x in] and wt[l] [in x out]
// (l = 2..4), w5b [16 x 256], w5t [256 x 64] (columns >= 16 left zero).
cudaError_t launch_cast_weights(const float* params, __nv_bfloat16* const* wb, __nv_bfloat16* const* wt,
                                __nv_bfloat16* w5b, __nv_bfloat16* w5t, cudaStream_t s);

// Render: per sample of the tile, the camera ray's network inputs and
// closed-form margins; then, from the network outputs, the colour or a
// place in the exact re-trace queue.
struct RenderBands {
    double du = 4.0;           // u error band = du * sigma (the sample's predicted error)
    double dir = 4.0;          // direction error band (rad) = dir * sigma_dir
    double capture = 0.15;     // |capture margin| below this: exact
    double graze = 0.02;       // graze margin below this: exact
    double tol_rel = 1e-3;     // colour sensitivity budget (relative)
};
struct SampleAux {
    double pt, pph;
    float capture_margin, graze_margin;
    unsigned q;  // the sample
};
// Samples q0 .. q0 + nq - 1 of the tile. With settle_radius > 0 (a black
// sky), a sample whose closed-form smallest radius exceeds it is final at
// once (colour 0, escaped, written to mb) and skips the network; the others
// are appended to X / aux, *count of them (zeroed by the caller), and added
// to *total (the render's network samples).
cudaError_t launch_prepare(const DevScene& S, const DevTile& tile, size_t q0, size_t nq, double settle_radius,
                           float* X, SampleAux* aux, unsigned* count, unsigned* total, const DevMixedBuffers& mb,
                           DevStats* stats, cudaStream_t s);
// Shades the *count prepared samples (at most cap) from the network outputs O.
cudaError_t launch_shade(const DevScene& S, const DevTile& tile, const unsigned* count, size_t cap, const float* O,
                         const SampleAux* aux, const RenderBands& bands, const DevMixedBuffers& mb, DevStats* stats,
                         cudaStream_t s);

// Validation: per sample, errors of the network outputs against the targets
// (err[q][0] = |du1| / sigma1, [1] = |du2| / sigma2, [2] = arc-start direction
// error (rad) / sigma_dir, [3] = |c_theta error| / sigma_dir; -1 where the
// target does not apply).
cudaError_t launch_eval_errors(const float* O, const float* Y, size_t n, float* err, cudaStream_t s);

}  // namespace surr
}  // namespace grrt_b200
