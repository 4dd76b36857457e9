// The exported C API of libgrrt.so: the reference's drop-in surface
// (include/grrt_api.h) and the additive entry points (include/grrt_b200.h).
//
// grrt_create resolves the parameters exactly as src/api.cpp:43-173 does and
// builds every table on the host (bit-identical to the reference's). The
// tables move to the GPU at the first render; every pixel is then traced by
// the sm_100a kernels. There is no CPU render path: a render without a usable
// GPU fails with an error.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "context.h"
#include "device/render_launch.h"
#include "fits.h"
#include "host/tables.h"

using namespace grrt_b200;

namespace {
thread_local std::string g_last_error;
}  // namespace

// ---------------------------------------------------------------------------
// create / destroy
// ---------------------------------------------------------------------------
extern "C" GRRT_EXPORT GRRTContext* grrt_create(const GRRTParams* params) {
    if (!params) {
        g_last_error = "grrt_create: params is NULL";
        return nullptr;
    }
    if (params->width <= 0 || params->height <= 0) {
        g_last_error = "grrt_create: width and height must be positive";
        return nullptr;
    }
    auto ctx = std::make_unique<GRRTContext>();
    try {
        ctx->build(*params);
    } catch (const std::exception& e) {
        g_last_error = std::string("grrt_create: ") + e.what();
        return nullptr;
    }
    std::printf("grrt: created context (%dx%d, %s, M=%g, a=%g, r_obs=%g, disk=%s, stars=%s, backend=cuda-sm100)\n",
                params->width, params->height,
                params->metric_type == GRRT_METRIC_KERR ? "kerr" : "schwarzschild", ctx->mass, ctx->spin_a,
                ctx->observer_r, params->disk_enabled ? "on" : "off",
                params->background_type == GRRT_BG_STARS ? "on" : "off");
    return ctx.release();
}

extern "C" GRRT_EXPORT void grrt_destroy(GRRTContext* ctx) { delete ctx; }

extern "C" GRRT_EXPORT void grrt_update_params(GRRTContext* ctx, const GRRTParams* params) {
    // As the reference: copy only; tables, camera and scene stay as built.
    if (ctx && params) ctx->params = *params;
}

// ---------------------------------------------------------------------------
// RGB rendering
// ---------------------------------------------------------------------------
extern "C" GRRT_EXPORT int grrt_render(GRRTContext* ctx, float* framebuffer) {
    return grrt_render_cb(ctx, framebuffer, nullptr, nullptr);
}

extern "C" GRRT_EXPORT int grrt_render_cb(GRRTContext* ctx, float* framebuffer, grrt_progress_fn progress,
                                          void* user_data) {
    if (!ctx) return -1;
    if (!framebuffer) {
        ctx->error = "grrt_render: framebuffer is NULL";
        return -1;
    }
    const int W = ctx->params.width, H = ctx->params.height;
    DevTile tile;
    tile.x0 = 0;
    tile.y0 = 0;
    tile.w = W;
    tile.h = H;
    tile.out_pitch = W;
    const int rc = ctx->render_rgb_to_host(tile, framebuffer, progress, user_data);
    if (rc == 0) std::printf("grrt: rendered %dx%d frame (cuda)\n", W, H);
    return rc;
}

extern "C" GRRT_EXPORT int grrt_render_tile(GRRTContext* ctx, float* buffer, int x, int y, int tile_width,
                                            int tile_height) {
    if (!ctx) return -1;
    if (!buffer || tile_width <= 0 || tile_height <= 0 || x < 0 || y < 0 ||
        x + tile_width > ctx->params.width || y + tile_height > ctx->params.height) {
        ctx->error = "grrt_render_tile: tile outside the image or buffer is NULL";
        return -1;
    }
    DevTile tile;
    tile.x0 = x;
    tile.y0 = y;
    tile.w = tile_width;
    tile.h = tile_height;
    tile.out_pitch = tile_width;
    return ctx->render_rgb_to_host(tile, buffer, nullptr, nullptr);
}

extern "C" GRRT_EXPORT int grrt_render_rows_device(GRRTContext* ctx, int row0, int row_step, int n_rows,
                                                   float* d_rgba, double* d_rgb64, unsigned int* d_fate,
                                                   void* stream) {
    if (!ctx) return -1;
    if (row0 < 0 || row_step < 1 || n_rows < 1 ||
        static_cast<long long>(row0) + static_cast<long long>(n_rows - 1) * row_step >= ctx->params.height) {
        ctx->error = "grrt_render_rows_device: rows outside the image";
        return -1;
    }
    DevTile tile;
    tile.x0 = 0;
    tile.y0 = row0;
    tile.w = ctx->params.width;
    tile.h = n_rows;
    tile.out_pitch = ctx->params.width;
    tile.row_step = row_step;
    return ctx->render_rgb_device(tile, d_rgba, d_rgb64, d_fate, static_cast<cudaStream_t>(stream), true);
}

extern "C" GRRT_EXPORT int grrt_set_diagnostics(GRRTContext* ctx, int flags) {
    if (!ctx || (flags & ~GRRT_DIAG_HAMILTONIAN)) return -1;
    ctx->diagnostics = flags;
    return 0;
}

extern "C" GRRT_EXPORT void grrt_cancel(GRRTContext* ctx) {
    if (ctx) ctx->request_cancel();
}

extern "C" GRRT_EXPORT float grrt_progress(const GRRTContext* ctx) { return ctx ? ctx->progress : 0.0f; }

extern "C" GRRT_EXPORT const char* grrt_error(const GRRTContext* ctx) {
    if (!ctx || ctx->error.empty()) return nullptr;
    return ctx->error.c_str();
}

extern "C" GRRT_EXPORT int grrt_cuda_available(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return 0;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return 0;
    return prop.major >= 10 ? 1 : 0;
}

extern "C" GRRT_EXPORT const char* grrt_last_error(void) {
    return g_last_error.empty() ? nullptr : g_last_error.c_str();
}

// ---------------------------------------------------------------------------
// Spectral rendering
// ---------------------------------------------------------------------------
extern "C" GRRT_EXPORT void grrt_set_frequency_bins(GRRTContext* ctx, const double* f, int n) {
    if (!ctx) return;
    if (n > 0 && f)
        ctx->freq_bins.assign(f, f + n);
    else
        ctx->freq_bins.clear();
}

extern "C" GRRT_EXPORT int grrt_render_spectral(GRRTContext* ctx, double* buf, int width, int height) {
    return grrt_render_spectral_cb(ctx, buf, width, height, nullptr, nullptr);
}

extern "C" GRRT_EXPORT int grrt_render_spectral_cb(GRRTContext* ctx, double* buf, int width, int height,
                                                   grrt_progress_fn progress, void* user_data) {
    if (!ctx) return -1;
    if (ctx->freq_bins.empty()) {
        ctx->error = "No frequency bins set -- call grrt_set_frequency_bins first";
        return -1;
    }
    if (!buf || width <= 0 || height <= 0) {
        ctx->error = "grrt_render_spectral: bad buffer or size";
        return -1;
    }
    const int rc = ctx->render_spectral_to_host(width, height, buf, progress, user_data);
    if (rc == 0)
        std::printf("grrt: rendered %dx%d spectral frame (%zu bins, cuda)\n", width, height,
                    ctx->freq_bins.size());
    return rc;
}

extern "C" GRRT_EXPORT int grrt_render_spectral_to_fits_cb(GRRTContext* ctx, const char* path, int width,
                                                           int height, grrt_progress_fn progress,
                                                           void* user_data) {
    if (!ctx) return -1;
    if (ctx->freq_bins.empty()) {
        ctx->error = "No frequency bins set -- call grrt_set_frequency_bins first";
        return -1;
    }
    if (!path || path[0] == '\0') {
        ctx->error = "grrt_render_spectral_to_fits_cb: output_path is null or empty";
        return -1;
    }
    if (width <= 0 || height <= 0) {
        ctx->error = "grrt_render_spectral_to_fits_cb: bad size";
        return -1;
    }
    const int rc = ctx->render_spectral_to_fits(path, width, height, progress, user_data);
    if (rc == 0)
        std::printf("grrt: streamed %dx%d spectral frame (%zu bins) to '%s'\n", width, height,
                    ctx->freq_bins.size(), path);
    return rc;
}

// ---------------------------------------------------------------------------
// Tone mapping (src/tonemapper.cpp:7-71): a host post-process on the float
// framebuffer — log-average auto exposure, extended Reinhard, gamma 2.2.
// ---------------------------------------------------------------------------
extern "C" GRRT_EXPORT void grrt_tonemap(float* fb, int width, int height) {
    if (!fb || width <= 0 || height <= 0) return;
    const int n = width * height;
    constexpr double key = 0.18, delta = 1e-6, lit = 1e-10;
    auto lum = [&](int i, double& R, double& G, double& B) {
        R = std::max(0.0, static_cast<double>(fb[4 * i + 0]));
        G = std::max(0.0, static_cast<double>(fb[4 * i + 1]));
        B = std::max(0.0, static_cast<double>(fb[4 * i + 2]));
        return 0.2126 * R + 0.7152 * G + 0.0722 * B;
    };
    double log_sum = 0.0, L_max = 0.0;
    int count = 0;
    for (int i = 0; i < n; ++i) {
        double R, G, B;
        const double L = lum(i, R, G, B);
        if (L > lit) {
            log_sum += std::log(delta + L);
            ++count;
        }
        if (L > L_max) L_max = L;
    }
    if (L_max <= 0.0 || count == 0) return;
    const double L_avg = std::exp(log_sum / count);
    const double exposure = key / L_avg;
    const double Lw = L_max * exposure;
    const double Lw2 = Lw * Lw;
    auto gamma = [](double v) { return std::pow(std::clamp(v, 0.0, 1.0), 1.0 / 2.2); };
    for (int i = 0; i < n; ++i) {
        double R, G, B;
        const double L = lum(i, R, G, B);
        if (L <= 0.0) {
            fb[4 * i + 0] = fb[4 * i + 1] = fb[4 * i + 2] = 0.0f;
            continue;
        }
        const double Ls = L * exposure;
        double Lm = Ls * (1.0 + Ls / Lw2) / (1.0 + Ls);
        Lm = std::clamp(Lm, 0.0, 1.0);
        const double s = Lm / L;
        fb[4 * i + 0] = static_cast<float>(gamma(R * s));
        fb[4 * i + 1] = static_cast<float>(gamma(G * s));
        fb[4 * i + 2] = static_cast<float>(gamma(B * s));
    }
}

// The same on the device, in place on a device frame, enqueued on `stream`.
extern "C" GRRT_EXPORT int grrt_tonemap_device(float* d_rgba, int width, int height, void* stream) {
    if (!d_rgba || width <= 0 || height <= 0) return -1;
    const cudaError_t e = launch_tonemap(d_rgba, width, height, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return 0;
}

extern "C" GRRT_EXPORT void grrt_debug_pixel(GRRTContext* ctx, int px, int py) {
    if (!ctx) {
        std::printf("grrt_debug_pixel: context not ready\n");
        return;
    }
    std::printf("Debugging pixel (%d, %d) in %dx%d image\n", px, py, ctx->params.width, ctx->params.height);
    ctx->debug_pixel(px, py);
}

// ---------------------------------------------------------------------------
// Additive entry points (include/grrt_b200.h)
// ---------------------------------------------------------------------------
extern "C" GRRT_EXPORT int grrt_set_precision(GRRTContext* ctx, int form) {
    if (!ctx) return -1;
    if (form != GRRT_FORM_FP64 && form != GRRT_FORM_MIXED) {
        ctx->error = "grrt_set_precision: unknown form";
        return -1;
    }
    ctx->form = form;
    return 0;
}

extern "C" GRRT_EXPORT int grrt_get_precision(const GRRTContext* ctx) { return ctx ? ctx->form : -1; }

extern "C" GRRT_EXPORT int grrt_set_mixed_params(GRRTContext* ctx, double r_factor, double tol_fp32) {
    // r_near below the horizon would switch the near-critical test off; an FP32
    // tolerance outside [1e-9, 1e-2] is below its error estimate's noise floor
    // or too coarse for the speculative trajectory to be trusted
    if (!ctx || !(r_factor >= 1.0 && r_factor <= 100.0) || !(tol_fp32 >= 1e-9 && tol_fp32 <= 1e-2)) return -1;
    ctx->mixed_r_factor = r_factor;
    ctx->tol_fp32 = tol_fp32;
    return 0;
}

extern "C" GRRT_EXPORT int grrt_render_device(GRRTContext* ctx, float* d_rgba, double* d_rgb64,
                                              unsigned int* d_fate, void* stream) {
    if (!ctx) return -1;
    DevTile tile;
    tile.w = ctx->params.width;
    tile.h = ctx->params.height;
    tile.out_pitch = tile.w;
    return ctx->render_rgb_device(tile, d_rgba, d_rgb64, d_fate, static_cast<cudaStream_t>(stream), true);
}

extern "C" GRRT_EXPORT int grrt_render_spectral_device(GRRTContext* ctx, double* d_spec, int width, int height,
                                                       unsigned int* d_fate, void* stream) {
    if (!ctx) return -1;
    if (ctx->freq_bins.empty()) {
        ctx->error = "No frequency bins set -- call grrt_set_frequency_bins first";
        return -1;
    }
    return ctx->render_spectral_device(width, height, d_spec, d_fate, static_cast<cudaStream_t>(stream), true);
}

extern "C" GRRT_EXPORT int grrt_render_spectral_rows_device(GRRTContext* ctx, int row0, int row_step, int n_rows,
                                                            double* d_spec, unsigned int* d_fate, void* stream) {
    if (!ctx) return -1;
    if (ctx->freq_bins.empty()) {
        ctx->error = "No frequency bins set -- call grrt_set_frequency_bins first";
        return -1;
    }
    if (row0 < 0 || row_step < 1 || n_rows < 1 ||
        static_cast<long long>(row0) + static_cast<long long>(n_rows - 1) * row_step >= ctx->params.height) {
        ctx->error = "grrt_render_spectral_rows_device: rows outside the image";
        return -1;
    }
    DevTile tile;
    tile.y0 = row0;
    tile.w = ctx->params.width;
    tile.h = n_rows;
    tile.out_pitch = ctx->params.width;
    tile.row_step = row_step;
    return ctx->render_spectral_tile(tile, d_spec, d_fate, static_cast<cudaStream_t>(stream), true);
}

extern "C" GRRT_EXPORT int grrt_render_spectral_tile_device(GRRTContext* ctx, int x, int y, int w, int h,
                                                            double* d_spec, unsigned int* d_fate, void* stream) {
    if (!ctx) return -1;
    if (ctx->freq_bins.empty()) {
        ctx->error = "No frequency bins set -- call grrt_set_frequency_bins first";
        return -1;
    }
    if (x < 0 || y < 0 || w < 1 || h < 1 || static_cast<long long>(x) + w > ctx->params.width ||
        static_cast<long long>(y) + h > ctx->params.height) {
        ctx->error = "grrt_render_spectral_tile_device: tile outside the image";
        return -1;
    }
    DevTile tile;
    tile.x0 = x;
    tile.y0 = y;
    tile.w = w;
    tile.h = h;
    tile.out_pitch = w;
    return ctx->render_spectral_tile(tile, d_spec, d_fate, static_cast<cudaStream_t>(stream), true);
}

extern "C" GRRT_EXPORT int grrt_get_stats(GRRTContext* ctx, GRRTStats* out) {
    if (!ctx || !out) return -1;
    return ctx->read_stats(out);
}

extern "C" GRRT_EXPORT int grrt_get_phase_ms(GRRTContext* ctx, double* out, int capacity) {
    if (!ctx || (!out && capacity > 0) || capacity < 0) return -1;
    return ctx->phase_ms(out, capacity);
}

extern "C" GRRT_EXPORT long long grrt_scene_table(const GRRTContext* ctx, const char* name, double* out,
                                                  long long capacity) {
    if (!ctx || !name) return -1;
    std::vector<double> v;
    if (!ctx->export_table(name, v)) return -1;
    const long long n = static_cast<long long>(v.size());
    if (out && capacity >= n) std::memcpy(out, v.data(), sizeof(double) * v.size());
    return n;
}

extern "C" GRRT_EXPORT int grrt_camera_ray(const GRRTContext* ctx, double x, double y, double* out) {
    if (!ctx || !out) return -1;
    camera_ray(ctx->cam, x, y, out, out + 4);
    return 0;
}

extern "C" GRRT_EXPORT int grrt_debug_trace(GRRTContext* ctx, double x, double y, GRRTDebugRecord* records,
                                            int capacity) {
    if (!ctx || capacity < 0 || (capacity > 0 && !records)) return -1;
    return ctx->debug_trace(x, y, records, capacity);
}
