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
 * control, src/rk4.cpp:87-136) in double throughout. MIXED, thin disk: every
 * sample is integrated first with FP32 right-hand sides (FP64 state); samples
 * whose colour depends on the FP64 step sequence (emitting crossings, grazes,
 * near-critical orbits, escapes with a star in reach, the step budget) are
 * re-traced with the FP64 method, all others are exactly 0. MIXED, volumetric
 * disk: samples whose FP32 trajectory provably stays away from the volume are
 * finished by that pass (escape or horizon, no emission); every other sample
 * is re-traced in FP64, so the output equals the FP64 form's bit for bit. */
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
    double hamiltonian_max;           /* with GRRT_DIAG_HAMILTONIAN, thin-disk FP64 form: max over
                                         the samples that do not end at the horizon of |H| / p_t^2
                                         at the final state, H = 1/2 g^{mu nu} p_mu p_nu (0 on the
                                         light cone; near the horizon its evaluation cancels);
                                         0 where not measured */
} GRRTStats;

/* Diagnostics of later renders (flags, 0 = none). GRRT_DIAG_HAMILTONIAN: the
 * thin-disk FP64 form runs its diagnostic instantiation, which also measures
 * the Hamiltonian constraint at every sample's final state
 * (GRRTStats.hamiltonian_max); the render itself is unchanged. No counterpart
 * in the reference (its README says the constraint is monitored). Returns 0,
 * or -1 for unknown flags. */
#define GRRT_DIAG_HAMILTONIAN 1
GRRT_EXPORT int grrt_set_diagnostics(GRRTContext* ctx, int flags);

/* Select the precision form for later renders (src/geodesic_tracer.cpp:100 is
 * the FP64 call it replaces). Returns 0, or -1 for an unknown form. */
GRRT_EXPORT int grrt_set_precision(GRRTContext* ctx, int form);
GRRT_EXPORT int grrt_get_precision(const GRRTContext* ctx);

/* Mixed-form knobs. Thin disk: every sample is first integrated with FP32
 * right-hand sides against tol_fp32; a sample that sweeps more than 3 rad
 * inside r_near = max(r_factor * r_horizon, 1.25 x the outermost photon orbit)
 * (near-critical) is among those re-traced in FP64. Volumetric disk: the same
 * speculation, with the volume's reach in place of the disk test. Defaults 3.0
 * and 3e-6; r_factor must lie in [1, 100] and tol_fp32 in [1e-9, 1e-2], else
 * -1. */
GRRT_EXPORT int grrt_set_mixed_params(GRRTContext* ctx, double r_factor, double tol_fp32);

/* Device time (ms, CUDA events on the render stream) of each kernel phase of
 * the last render: the mixed thin-disk form has 4 (FP32 speculation, star
 * pass, FP64 re-trace, resolve), the thin-disk FP64 form 2 (FP64 trace,
 * resolve), the volumetric mixed forms 3 (FP32 speculation, FP64 re-trace,
 * resolve); every other render has 1. Writes at most capacity values; returns
 * the number of phases, or -1. Waits for the render. */
GRRT_EXPORT int grrt_get_phase_ms(GRRTContext* ctx, double* out, int capacity);

/* RGB render into device memory (the loop of Renderer::render,
 * src/renderer.cpp:30-82). d_rgba: float[W*H*4] or NULL; d_rgb64: the
 * spp-averaged double colour, double[W*H*3] or NULL; d_fate: per sample
 * (pixel*grid^2 + s) termination | (disk crossings << 2), or NULL.
 * W, H are the context's width and height. Returns 0 or -1. */
GRRT_EXPORT int grrt_render_device(GRRTContext* ctx, float* d_rgba, double* d_rgb64,
                                   unsigned int* d_fate, void* stream);

/* The same for the n_rows image rows row0, row0 + row_step, ... at full width,
 * written densely (output row k = image row row0 + k * row_step): a rank's
 * share of a frame split across GPUs by interleaved rows. Each pixel is
 * computed exactly as in the full render. -1 when a row lies outside the image. */
GRRT_EXPORT int grrt_render_rows_device(GRRTContext* ctx, int row0, int row_step, int n_rows, float* d_rgba,
                                        double* d_rgb64, unsigned int* d_fate, void* stream);

/* Tone mapping of a device RGBA float frame in place (the reference's
 * grrt_tonemap: log-average auto exposure, extended Reinhard, gamma 2.2),
 * enqueued on `stream`. d_rgba 16-byte aligned. Agrees with grrt_tonemap on
 * the host to a few float ulp (the log sum is grouped by blocks). 0 or -1. */
GRRT_EXPORT int grrt_tonemap_device(float* d_rgba, int width, int height, void* stream);

/* Spectral render into device memory (Renderer::render_spectral,
 * src/renderer.cpp:84-138): d_spec double[width*height*bins]. */
GRRT_EXPORT int grrt_render_spectral_device(GRRTContext* ctx, double* d_spec, int width, int height,
                                            unsigned int* d_fate, void* stream);

/* The same for the n_rows image rows row0, row0 + row_step, ... at full width,
 * written densely (output row k = image row row0 + k * row_step; d_spec is
 * double[n_rows*W*nb], d_fate one word per sample or NULL): a rank's share of
 * a spectral frame split across GPUs by interleaved rows. Each pixel is
 * computed exactly as in the full render. -1 when a row lies outside the image
 * or no bins are set. */
GRRT_EXPORT int grrt_render_spectral_rows_device(GRRTContext* ctx, int row0, int row_step, int n_rows,
                                                 double* d_spec, unsigned int* d_fate, void* stream);

/* The same for the w x h tile at image pixel (x, y) (the spectral counterpart
 * of grrt_render_tile, api.cpp:215-218 in the reference, whose CPU version
 * is a stub): d_spec is double[w*h*nb], row-major over the tile. -1 when the
 * tile leaves the image or no bins are set. */
GRRT_EXPORT int grrt_render_spectral_tile_device(GRRTContext* ctx, int x, int y, int w, int h, double* d_spec,
                                                 unsigned int* d_fate, void* stream);

/* Spectral render that allocates no device memory. No counterpart in the
 * reference (its renders run on host threads and allocate host buffers).
 *
 * For callers that may not allocate device memory while they render: a host
 * application that gives the renderer a fixed memory budget and forbids
 * driver allocations during a frame, or a process near the device memory
 * limit where an allocation could fail mid-frame. Instead of cudaMalloc'd scratch it
 * uses a fixed array compiled into the library (about 19.4 MB on every GPU that
 * loads it, held until the process exits). The caller passes the inputs and
 * outputs: d_freqs (num_bins observer-frame frequencies in Hz, device memory)
 * and d_spec (double[width*height*num_bins], device memory); the scene comes
 * from the context, which must already hold it on the device (any earlier
 * render call on the context uploads it). Same output as
 * grrt_render_spectral_device, enqueued on `stream`; a context without a
 * volumetric disk gets all-zero spectra, as there.
 *
 * Limits: num_bins <= 32, otherwise -1 with grrt_error set. The first call on
 * each device looks up the array's device address; make that first call before
 * any stream capture. All calls share the array and it keeps the last call's
 * contents, so calls that overlap on the GPU race and must be serialised by
 * the caller. It does not update grrt_get_stats and does not poll grrt_cancel. */
GRRT_EXPORT int grrt_render_spectral_device_noalloc(GRRTContext* ctx, const double* d_freqs, int num_bins,
                                                    double* d_spec, int width, int height, void* stream);

/* ---- Batched form: many thin-disk cameras in one persistent launch ----
 * No counterpart in the reference (it renders one camera per grrt_create).
 * Each camera is described by its own GRRTParams and keeps the reference's
 * per-camera semantics exactly (tables, jitter, spp). All pixels of all
 * cameras go through one device work queue, so long rays of one camera
 * overlap with short rays of the others; the launch is replayed as a CUDA
 * graph. A batch holds either thin-disk cameras (RGB renders, FP64 or mixed
 * form) or volumetric cameras (spectral renders, FP64 form; each camera with
 * its own frequency bins), not both. */
typedef struct GRRTBatch GRRTBatch;

/* Chunk orders of the schedule: all chunks of camera 0, then camera 1, ...;
 * or chunk k of every camera before chunk k+1. GRRT_BATCH_ORDER_SAMPLES (FP64
 * thin-disk batches): every camera's samples in camera order, traced by
 * samples with the warp staging of the single FP64 render, then resolved into
 * pixels; the chunk size and the threads per block do not apply (other
 * batches take it as camera-major). */
#define GRRT_BATCH_ORDER_CAMERA_MAJOR 0
#define GRRT_BATCH_ORDER_ROUND_ROBIN 1
#define GRRT_BATCH_ORDER_SAMPLES 2

/* params: count cameras. NULL on failure with the reason in grrt_batch_error(NULL). */
GRRT_EXPORT GRRTBatch* grrt_batch_create(const GRRTParams* params, int count);
GRRT_EXPORT void grrt_batch_destroy(GRRTBatch* batch);
GRRT_EXPORT const char* grrt_batch_error(const GRRTBatch* batch);
GRRT_EXPORT int grrt_batch_set_precision(GRRTBatch* batch, int form);
/* Work is cut into chunks of chunk_size consecutive pixels of one camera;
 * blocks_per_sm 0 = as many as fit. */
GRRT_EXPORT int grrt_batch_set_schedule(GRRTBatch* batch, int chunk_size, int order, int blocks_per_sm);
GRRT_EXPORT int grrt_batch_get_schedule(const GRRTBatch* batch, int* chunk_size, int* order, int* blocks_per_sm);
/* Threads per block of the FP64 thin-disk batch kernel (64, 128 or 256, at the
 * same 128 registers per thread) and the mixed form's FP32 tolerance and
 * r_factor (as grrt_set_mixed_params) for every camera. Defaults 128, 3e-6, 3. */
GRRT_EXPORT int grrt_batch_set_tuning(GRRTBatch* batch, int block, double tol_fp32, double r_factor);
GRRT_EXPORT int grrt_batch_get_tuning(const GRRTBatch* batch, int* block, double* tol_fp32, double* r_factor);
/* Times candidate settings on the batch itself and keeps the fastest:
 * FP64 thin-disk batches: chunk 64..4096 x both orders x two occupancies, then
 * 64/128/256 threads per block; spectral batches: chunk x order x occupancy;
 * mixed batches: two occupancies x tol_fp32 {1e-6, 3e-6, 1e-5} x r_factor
 * {3, 4}, each candidate held to the mixed form's bar against the batch's
 * FP64 render (every pixel within 1e-4 relative) and dropped if it misses it.
 * cache_path (may be NULL) stores and reuses the choice for an identical
 * batch. best_ms may be NULL. */
GRRT_EXPORT int grrt_batch_autotune(GRRTBatch* batch, const char* cache_path, double* best_ms);
/* framebuffers[i]: float[W_i*H_i*4] host buffer of camera i (NULL skips it). */
GRRT_EXPORT int grrt_batch_render(GRRTBatch* batch, float* const* framebuffers);
/* d_rgba: device float4 buffer of sum(W_i*H_i) pixels, camera i at the prefix
 * offset sum_{k<i} W_k*H_k. Enqueued on stream. */
GRRT_EXPORT int grrt_batch_render_device(GRRTBatch* batch, float* d_rgba, void* stream);
GRRT_EXPORT int grrt_batch_get_stats(GRRTBatch* batch, GRRTStats* out);

/* Volumetric batches. Bins (observer-frame Hz) of one camera, or of every
 * camera with camera = -1; each camera needs bins before the first render
 * (as grrt_set_frequency_bins for one context). */
GRRT_EXPORT int grrt_batch_set_frequency_bins(GRRTBatch* batch, int camera, const double* frequencies_hz,
                                              int num_bins);
/* Element offset of camera i's cube in the batch output (i = count gives the
 * total size); -1 for a thin-disk batch. */
GRRT_EXPORT long long grrt_batch_spectral_offset(GRRTBatch* batch, int camera);
/* d_spec: device doubles, camera i's cube double[W_i*H_i*nb_i] (index
 * (j*W_i + x)*nb_i + k, as grrt_render_spectral) at grrt_batch_spectral_offset(i).
 * Each camera's cube is bit-identical to its own grrt_render_spectral_device. */
GRRT_EXPORT int grrt_batch_render_spectral_device(GRRTBatch* batch, double* d_spec, void* stream);
/* cubes[i]: double[W_i*H_i*nb_i] host buffer of camera i (NULL skips it). */
GRRT_EXPORT int grrt_batch_render_spectral(GRRTBatch* batch, double* const* cubes);

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

/* Single-ray debug trace: the FP64 trace of the camera sample at fractional
 * pixel (x, y), run on the device, as the records of the lines
 * GeodesicTracer::trace_debug prints (src/geodesic_tracer.cpp:339-493);
 * grrt_debug_pixel prints them in that layout for the pixel centre.
 *   START      v: r, theta, phi, p_t, p_r, p_theta, p_phi (the device's initial state)
 *   STEP       one accepted outer step (step = its loop index); v: r, theta,
 *              z, next dlambda, H, z_max, phi (H and z_max NaN without a
 *              volumetric disk); event: GRRT_DEBUG_EVENT_* (volumetric)
 *   THIN_HIT   an emitting thin-disk crossing; v: r_cross, emission r, g, b
 *   MARCH_ENTRY a ray-march starts; v: r, z of its first state
 *   MARCH_EXIT the ray-march ended; aux: its RK4 steps; v: the volume's colour
 *              so far (J nu^3 per channel), r, z of its last state
 *   END        event: termination (0 horizon, 1 escaped, 2 step budget);
 *              aux: emitting crossings or ray-march entries; v: r, theta, phi,
 *              colour r, g, b (disk and volume only: no sky), attempts. */
#define GRRT_DEBUG_START 0
#define GRRT_DEBUG_STEP 1
#define GRRT_DEBUG_THIN_HIT 2
#define GRRT_DEBUG_MARCH_ENTRY 3
#define GRRT_DEBUG_MARCH_EXIT 4
#define GRRT_DEBUG_END 5
#define GRRT_DEBUG_EVENT_NONE 0
#define GRRT_DEBUG_EVENT_CROSS 1
#define GRRT_DEBUG_EVENT_INSIDE 2
#define GRRT_DEBUG_EVENT_NEAR 3

typedef struct {
    int kind;   /* GRRT_DEBUG_* */
    int step;
    int event;
    int aux;
    double v[7];
} GRRTDebugRecord;

/* Run the debug trace; copies the first min(n, capacity) records into
 * records (when n > capacity the last slot holds the END record) and returns
 * n, the number of records of the trace, or -1 on an error (grrt_error).
 * Synchronises the context's stream. */
GRRT_EXPORT int grrt_debug_trace(GRRTContext* ctx, double x, double y, GRRTDebugRecord* records, int capacity);

#ifdef __cplusplus
}
#endif

#endif /* GRRT_B200_EXT_H */
