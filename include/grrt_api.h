/*
 * grrt_api.h — the drop-in C ABI of the GRRT renderer, served by libgrrt.so.
 *
 * Every declaration here replaces one symbol of the reference's public C API
 * with the same name, signature, ownership rules and return codes; the
 * citation beside each names the reference declaration (include/grrt/api.h)
 * and its behaviour (src/api.cpp). GRRTParams and the enums keep the
 * reference's field order and types (include/grrt/types.h:4-64) so the struct
 * is byte-identical and existing callers (the reference CLI, FFI bindings)
 * link against this library unchanged.
 *
 * Buffers are always caller-owned host memory:
 *   RGB:      float[width*height*4], row-major, row 0 = top, linear HDR, alpha = 1
 *   spectral: double[width*height*num_bins], index (j*width+i)*num_bins+k,
 *             erg s^-1 cm^-2 Hz^-1 sr^-1
 * The pixel work runs on the GPU (sm_100a); there is no CPU fallback.
 */
#ifndef GRRT_B200_API_H
#define GRRT_B200_API_H

#if defined(_WIN32)
#define GRRT_EXPORT __declspec(dllexport)
#else
#define GRRT_EXPORT __attribute__((visibility("default")))
#endif

/* include/grrt/types.h:4-7 */
typedef enum {
    GRRT_METRIC_SCHWARZSCHILD = 0,
    GRRT_METRIC_KERR = 1
} GRRTMetricType;

/* include/grrt/types.h:9-12. Both values select the GPU path here. */
typedef enum {
    GRRT_BACKEND_CPU = 0,
    GRRT_BACKEND_CUDA = 1
} GRRTBackend;

/* include/grrt/types.h:14-18. GRRT_BG_TEXTURE is accepted and, like the
 * reference, renders as black. */
typedef enum {
    GRRT_BG_BLACK = 0,
    GRRT_BG_STARS = 1,
    GRRT_BG_TEXTURE = 2
} GRRTBackgroundType;

/* include/grrt/types.h:20-64 — same members, same order, same types.
 * A zero value means "use the default" for the fields the reference defaults
 * in grrt_create (src/api.cpp:47-52, 57, 72-75, 124, 141). */
typedef struct {
    int width;
    int height;

    GRRTMetricType metric_type;
    double mass;                 /* M (default 1) */
    double spin;                 /* a/M; with KERR, <= 0 selects 0.998 */

    double observer_r;           /* default 50 */
    double observer_theta;       /* radians, default 1.396 */
    double observer_phi;         /* radians */
    double fov;                  /* horizontal field of view, radians, default 1.047 */

    double cam_yaw;              /* unused, as in the reference */
    double cam_pitch;            /* unused */
    double cam_roll;             /* unused */

    int disk_enabled;
    double disk_inner;           /* 0 = ISCO */
    double disk_outer;           /* 0 = 20 (thin) / 30 (volumetric) */
    double disk_temperature;     /* peak temperature in K, 0 = 1e7 or derived */

    int disk_volumetric;         /* 0 = thin disk, 1 = volumetric */
    double disk_alpha;           /* Shakura-Sunyaev viscosity */
    double disk_turbulence;      /* fBm density amplitude */
    int disk_seed;               /* noise permutation seed */
    double disk_noise_scale;     /* noise feature size in M, 0 = 2 H(peak) */
    int disk_noise_octaves;      /* fBm octaves */

    double mass_solar;           /* M in solar masses (derives peak temperature) */
    double eddington_fraction;   /* accretion rate / Eddington */

    GRRTBackgroundType background_type;
    const char* background_texture_path;  /* unused, as in the reference */

    double integrator_tolerance; /* default 1e-8 */
    int integrator_max_steps;    /* default 10000 */

    int samples_per_pixel;       /* rounded down to a square grid */
    int thread_count;            /* unused, as in the reference */
    GRRTBackend backend;

    int num_frequency_bins;          /* widens the opacity table range at create */
    const double* frequency_bins_hz;
} GRRTParams;

typedef struct GRRTContext GRRTContext;

/* Progress callback: fraction in [0,1]. Called from the calling host thread. */
typedef void (*grrt_progress_fn)(float fraction, void* user_data);

#ifdef __cplusplus
extern "C" {
#endif

/* api.h:11 / api.cpp:43-173. Builds every table on the host and uploads the
 * scene to the current CUDA device. NULL on failure, reason in grrt_last_error(). */
GRRT_EXPORT GRRTContext* grrt_create(const GRRTParams* params);
/* api.h:12 / api.cpp:175-183 */
GRRT_EXPORT void grrt_destroy(GRRTContext* ctx);
/* api.h:13 / api.cpp:185-187: copies the parameters, rebuilds nothing. */
GRRT_EXPORT void grrt_update_params(GRRTContext* ctx, const GRRTParams* params);

/* api.h:16 / api.cpp:189-191 */
GRRT_EXPORT int grrt_render(GRRTContext* ctx, float* framebuffer);
/* api.h:17-18 / api.cpp:193-213: 0 on success, non-zero with grrt_error(ctx) set. */
GRRT_EXPORT int grrt_render_cb(GRRTContext* ctx, float* framebuffer,
                               grrt_progress_fn progress, void* user_data);
/* api.h:19-20 / api.cpp:215-218: a stub returning 0 in the reference; here it
 * renders the requested tile of the full image into buffer
 * (tile_width*tile_height*4 floats) and returns 0, or -1 on a bad rectangle. */
GRRT_EXPORT int grrt_render_tile(GRRTContext* ctx, float* buffer,
                                 int x, int y, int tile_width, int tile_height);
/* api.h:21 / api.cpp:220-227: sets a flag the render loop polls between
 * launches; an interrupted render returns non-zero with grrt_error "cancelled". */
GRRT_EXPORT void grrt_cancel(GRRTContext* ctx);
/* api.h:22 / api.cpp:229-231: fraction of the last render completed. */
GRRT_EXPORT float grrt_progress(const GRRTContext* ctx);
/* api.h:23 / api.cpp:233-235: NULL when there is no error. */
GRRT_EXPORT const char* grrt_error(const GRRTContext* ctx);
/* api.h:24 / api.cpp:237-243: 1 when an sm_100 device is usable. */
GRRT_EXPORT int grrt_cuda_available(void);
/* api.h:25 / api.cpp:245-247: thread-local message of the last failed create. */
GRRT_EXPORT const char* grrt_last_error(void);

/* api.h:28 / src/tonemapper.cpp:7-71: auto-exposure + extended Reinhard +
 * gamma 2.2, in place on RGBA floats (a host post-process). */
GRRT_EXPORT void grrt_tonemap(float* framebuffer, int width, int height);

/* api.h:32 / api.cpp:339-348: traces one pixel centre and prints per-step
 * diagnostics to stdout. */
GRRT_EXPORT void grrt_debug_pixel(GRRTContext* ctx, int px, int py);

/* api.h:35-37 / api.cpp:249-257: copies the observer-frame frequencies (Hz). */
GRRT_EXPORT void grrt_set_frequency_bins(GRRTContext* ctx,
                                         const double* frequencies_hz,
                                         int num_bins);
/* api.h:38-39 / api.cpp:259-262: -1 if no bins are set. */
GRRT_EXPORT int grrt_render_spectral(GRRTContext* ctx, double* spectral_buffer,
                                     int width, int height);
/* api.h:40-42 / api.cpp:264-281 */
GRRT_EXPORT int grrt_render_spectral_cb(GRRTContext* ctx, double* spectral_buffer,
                                        int width, int height,
                                        grrt_progress_fn progress, void* user_data);
/* api.h:47-51 / api.cpp:283-332: writes the cube to a FITS file (BITPIX -64,
 * big-endian, rows flipped; byte-identical to the reference's file). The
 * whole cube is rendered on the device first; then the GPU packs it into
 * FITS order in groups of frequency planes, and each group is written to the
 * file while the next groups cross the bus. Host memory: one pinned copy of
 * the cube, kept by the context. 0 on success, -1 with grrt_error(ctx) set. */
GRRT_EXPORT int grrt_render_spectral_to_fits_cb(GRRTContext* ctx,
                                                const char* output_path,
                                                int width, int height,
                                                grrt_progress_fn progress,
                                                void* user_data);

#ifdef __cplusplus
}
#endif

#endif /* GRRT_B200_API_H */
