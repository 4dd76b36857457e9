/*
 * grrt_surrogate.h — the learned transfer-function surrogate of libgrrt.so.
 *
 * No counterpart in the reference. A small MLP maps (image-plane alpha, beta,
 * spin, inclination) to the quantities a thin-disk pixel's colour is made of;
 * it is trained on the GPU on geodesics the plain FP64 integrator traces, by
 * the library's own BF16 tensor-core (tcgen05) kernels with FP32 accumulation.
 * The plain integrator stays the fallback and the arbiter: samples the network
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

/* ---- the surrogate object ------------------------------------------------
 * Network: inputs (alpha, beta) (image-plane angles, radians, both scaled by
 * the width as in the reference camera), spin, inclination, each mapped to
 * [-1, 1]; hidden 4 x 256 SiLU; outputs
 *   0, 1: u = M / r of the first and second equatorial crossing in time
 *         order, saturated at M / (0.9 r_in) (no disk emits inside); 0 when
 *         the ray escapes first, the saturation value when it falls in first
 *   2-4:  cos(theta), sin(phi), cos(phi) of the sky position at r = 1000 M
 *         (folded as the star lookup folds it)
 *   5:    c_theta / 32 with c_theta = r^2 dtheta/dr there (far-field bending)
 *   6, 7: log sigma of the network's own error on outputs 0 and 1, and
 *   8:    on the direction (outputs 2-4), trained by a Gaussian likelihood on
 *         the residual; a sample's u and direction bands are calibrated
 *         multiples of its sigmas.
 * The redshift factor g is not learned: at a crossing radius it follows in
 * closed form from the ray's constants (p_t, p_phi), as in the plain form. */
typedef struct GRRTSurrogate GRRTSurrogate;

/* New network (uniform init, variance 1/fan_in, from `seed`) on the current
 * device. NULL on failure; the reason from grrt_surrogate_error(NULL). */
GRRT_EXPORT GRRTSurrogate* grrt_surrogate_create(unsigned seed);
GRRT_EXPORT void grrt_surrogate_destroy(GRRTSurrogate* s);
GRRT_EXPORT const char* grrt_surrogate_error(const GRRTSurrogate* s);

/* Training set: every camera (its GRRTParams, thin disk) at n_side x n_side
 * pixels, 1 sample per pixel jittered by the reference's pixel hash, traced by
 * the plain FP64 integrator on the GPU. Replaces any previous set. */
GRRT_EXPORT int grrt_surrogate_generate(GRRTSurrogate* s, const GRRTParams* cams, int n_cams, int n_side);
/* Number of samples in the training set; with buffers of `capacity` samples,
 * copies inputs (float[4] each) and records (float[10] each: the six targets,
 * termination, crossings after the second outside 0.9 r_in, capture margin,
 * graze margin). */
GRRT_EXPORT long long grrt_surrogate_dataset(GRRTSurrogate* s, float* x_out, float* y_out, long long capacity);

/* `steps` Adam steps (beta 0.9 / 0.999) on random batches of `batch` samples
 * (a multiple of 128): rate lr for the first half of the run, then halved at
 * every further eighth. loss_out (float[steps] or NULL) gets each step's
 * loss. Each step runs as a replayed CUDA graph of the library's kernels. */
GRRT_EXPORT int grrt_surrogate_train(GRRTSurrogate* s, int steps, int batch, double lr, float* loss_out);

/* Calibrates the fallback bands on a fresh validation set of the given
 * cameras (jitter sample 1). Critical band: covers every sample whose
 * closed-form fate disagrees with the integrator's (x2) and every sample with
 * a crossing outside 0.9 r_in after the second that does not graze (x1.2), at
 * least 0.05.
 * Graze band: turning point within mu = 0.02 of the equator. u band: the
 * `quantile` of |u error| / sigma over the samples outside both bands, times
 * `safety` (a multiple of each sample's predicted sigma); direction band: the
 * same for the direction error over sigma_dir. report8 (or NULL): u band
 * multiple, direction band, capture band, graze band, validation samples,
 * fate disagreements, fraction of samples in the bands, median |u error| /
 * sigma outside them. */
GRRT_EXPORT int grrt_surrogate_calibrate(GRRTSurrogate* s, const GRRTParams* cams, int n_cams, int n_side,
                                         double quantile, double safety, double* report8);
GRRT_EXPORT int grrt_surrogate_set_bands(GRRTSurrogate* s, double du, double dir, double capture, double graze,
                                         double tol_rel);
/* out5: du (multiple of sigma), dir, capture, graze, tol_rel. Returns 1 if
 * calibrated or set, 0 if default. */
GRRT_EXPORT int grrt_surrogate_get_bands(const GRRTSurrogate* s, double* out5);

/* FP32 parameters: W1[256x4], b1, W2..W4[256x256], b2..b4, W5[16x256]
 * (rows 9..15 zero), b5[16]. Returns the count; copies when capacity allows. */
GRRT_EXPORT long long grrt_surrogate_params(GRRTSurrogate* s, float* out, long long capacity);
GRRT_EXPORT int grrt_surrogate_set_params(GRRTSurrogate* s, const float* in, long long n);
/* Network outputs float[n][16] for device inputs float[n][4] (the fused
 * tensor-core inference kernel; both pointers 16-byte aligned). */
GRRT_EXPORT int grrt_surrogate_forward(GRRTSurrogate* s, const float* d_in, long long n, float* d_out);
/* One forward + backward pass on host data (n a multiple of 128; records as
 * in grrt_surrogate_dataset; termination 2 masks a row): the loss and the
 * gradient of every parameter, without an update. */
GRRT_EXPORT int grrt_surrogate_gradients(GRRTSurrogate* s, const float* h_in, const float* h_y, int n, float* h_grad,
                                         double* loss);

/* Renders the context's thin-disk frame (as grrt_render_device: d_rgba,
 * d_rgb64, d_fate may be NULL) with the surrogate: closed-form fate, network
 * crossings and escape direction; the mixed form's FP32 speculation for the
 * samples whose error band reaches the disk from outside it or whose sky arc
 * (widened by the direction band) could reach a star; exact FP64
 * re-trace of the samples inside the bands, whose colour is sensitive beyond
 * tol_rel, or that the speculation queues. grrt_get_stats and
 * grrt_get_phase_ms of the context report the render (phases: network +
 * shading, speculation + star pass, exact re-trace, resolve). */
GRRT_EXPORT int grrt_surrogate_render_device(GRRTSurrogate* s, GRRTContext* ctx, float* d_rgba, double* d_rgb64,
                                             unsigned int* d_fate, void* stream);
GRRT_EXPORT int grrt_surrogate_render(GRRTSurrogate* s, GRRTContext* ctx, float* framebuffer);
/* Samples re-traced exactly and samples in the last render. */
GRRT_EXPORT int grrt_surrogate_last_exact(const GRRTSurrogate* s, long long* exact, long long* samples);
/* The same, plus the samples sent to the FP32 speculation and the samples the
 * network evaluated (the rest were settled in closed form on a black sky);
 * speculated and network may be NULL. */
GRRT_EXPORT int grrt_surrogate_last_counts(const GRRTSurrogate* s, long long* exact, long long* speculated,
                                           long long* network, long long* samples);

GRRT_EXPORT int grrt_surrogate_save(const GRRTSurrogate* s, const char* path);
GRRT_EXPORT int grrt_surrogate_load(GRRTSurrogate* s, const char* path);

#ifdef __cplusplus
}
#endif

#endif
