/*
 * grrt_b200.h — entry points libgrrt.so adds beside the drop-in C API.
 *
 * Nothing here changes a reference signature; these are additive exports for
 * callers that keep data on the GPU, choose the precision form, read the work
 * counters, or inspect the host-built tables. None has a counterpart in the
 * reference's C API (include/grrt/api.h); each comment names the reference
 * code whose behaviour the call exposes.
 *
 * Device pointers are CUDA device memory of the context's device; `stream` is
 * a cudaStream_t (NULL = the legacy default stream). The *_device calls only
 * enqueue work and return; the caller synchronises the stream.
 */
#ifndef GRRT_B200_EXT_H
#define GRRT_B200_EXT_H

#include "grrt_api.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Precision forms. FP64: the reference method (Dormand-Prince 5(4) + PI
 * control, src/rk4.cpp:87-136) in double throughout. MIXED: FP32 right-hand
 * sides while the ray is far from the hole, FP64 state and FP64 near it. */
#define GRRT_FORM_FP64 0
#define GRRT_FORM_MIXED 1

/* Work counters of the last render call (summed over its launches). */
typedef struct {
    unsigned long long attempts;      /* Dormand-Prince attempts, accepted + rejected */
    unsigned long long accepted;      /* accepted outer steps */
    unsigned long long crossings;     /* thin-disk emission events */
    unsigned long long rays;          /* camera samples traced */
    unsigned long long horizon;       /* samples ending at the horizon */
    unsigned long long escaped;       /* samples ending beyond the escape radius */
    unsigned long long max_steps;     /* samples ending on the step budget */
    unsigned long long clamp_evals;   /* volumetric step-clamp evaluations */
    unsigned long long march_steps;   /* volumetric RK4 steps */
    unsigned long long physics_steps; /* volumetric steps inside matter */
    unsigned long long bin_updates;   /* per-frequency transfer updates */
    unsigned long long fp64_attempts; /* attempts evaluated in FP64 */
    double kernel_ms;                 /* device time of the render kernels (CUDA events) */
} GRRTStats;

/* Select the precision form for later renders (src/geodesic_tracer.cpp:100 is
 * the FP64 call it replaces). Returns 0, or -1 for an unknown form. */
GRRT_EXPORT int grrt_set_precision(GRRTContext* ctx, int form);
GRRT_EXPORT int grrt_get_precision(const GRRTContext* ctx);

/* Mixed-form knobs: outer steps that start at r > r_factor * r_horizon use
 * FP32 right-hand sides controlled against tol_fp32; defaults 3.0 and 1e-6. */
GRRT_EXPORT int grrt_set_mixed_params(GRRTContext* ctx, double r_factor, double tol_fp32);

/* RGB render into device memory (the loop of Renderer::render,
 * src/renderer.cpp:30-82). d_rgba: float[W*H*4] or NULL; d_rgb64: the
 * spp-averaged double colour, double[W*H*3] or NULL; d_fate: per sample
 * (pixel*grid^2 + s) termination | (disk crossings << 2), or NULL.
 * W, H are the context's width and height. Returns 0 or -1. */
GRRT_EXPORT int grrt_render_device(GRRTContext* ctx, float* d_rgba, double* d_rgb64,
                                   unsigned int* d_fate, void* stream);

/* Spectral render into device memory (Renderer::render_spectral,
 * src/renderer.cpp:84-138): d_spec double[width*height*bins]. */
GRRT_EXPORT int grrt_render_spectral_device(GRRTContext* ctx, double* d_spec, int width, int height,
                                            unsigned int* d_fate, void* stream);

/* Spectral render that allocates no device memory. No counterpart in the
 * reference (its renders run on host threads and allocate host buffers).
 *
 * For callers that may not allocate device memory while they render: a host
 * application that gives the renderer a fixed memory budget and forbids
 * driver allocations during a frame, work recorded into a CUDA graph
 * (cudaMalloc cannot be captured), or a process near the device memory limit
 * where an allocation could fail mid-frame. Instead of cudaMalloc'd scratch it
 * uses a fixed array compiled into the library (about 19.4 MB on every GPU that
 * loads it, held until the process exits). The caller passes the inputs and
 * outputs: d_freqs (num_bins observer-frame frequencies in Hz, device memory)
 * and d_spec (double[width*height*num_bins], device memory); the scene comes
 * from the context, which must already hold it on the device (any earlier
 * render call on the context uploads it). Same output as
 * grrt_render_spectral_device, enqueued on `stream`.
 *
 * Limits: num_bins <= 32, otherwise -1 with grrt_error set. The first call on
 * each device looks up the array's device address; make that first call before
 * any stream capture. All calls share the array and it keeps the last call's
 * contents, so calls that overlap on the GPU race and must be serialised by
 * the caller. It does not update grrt_get_stats and does not poll grrt_cancel. */
GRRT_EXPORT int grrt_render_spectral_device_noalloc(GRRTContext* ctx, const double* d_freqs, int num_bins,
                                                    double* d_spec, int width, int height, void* stream);

/* Counters of the last render; synchronises the context's device. */
GRRT_EXPORT int grrt_get_stats(GRRTContext* ctx, GRRTStats* out);

/* Copy a host-built table (the same values the reference builds) into out.
 * Names: "flux", "flux_meta" {flux_max, r_inner, r_outer, peak_T},
 * "spectrum_color", "spectrum_lum", "stars" (theta, phi, brightness per star),
 * "star_cells" (cell offsets), "star_items", "camera" {pos[4], e0..e3, g[16], fov,
 * width, height}, "scalars" {M, a, r_horizon, isco, observer_r, tol, max_steps, spp},
 * and with a volumetric disk "vol_H", "vol_zmax", "vol_rho_mid", "vol_T_eff",
 * "vol_rho_prof", "vol_T_prof", "vol_perm", "vol_scalars", "op_kabs", "op_kes",
 * "op_kross", "op_mu", "op_scalars". Returns the element count (even when out is
 * NULL or capacity is too small, in which case nothing is copied), -1 if the
 * name is unknown or the table absent. */
GRRT_EXPORT long long grrt_scene_table(const GRRTContext* ctx, const char* name, double* out,
                                       long long capacity);

/* Initial covariant state of a camera sample at fractional pixel (x, y) —
 * Camera::ray_for_pixel (src/camera.cpp:69-96) evaluated on the host.
 * out[8] = (t, r, theta, phi, p_t, p_r, p_theta, p_phi). */
GRRT_EXPORT int grrt_camera_ray(const GRRTContext* ctx, double x, double y, double* out);

#ifdef __cplusplus
}
#endif

#endif /* GRRT_B200_EXT_H */
