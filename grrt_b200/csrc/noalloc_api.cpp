// grrt_render_spectral_device_noalloc: the spectral render for callers that
// may not allocate device memory while rendering (see include/grrt_b200.h).
// It reads the scene the context already holds on the device and writes into
// caller-owned buffers; its scratch is a file-scope device array in
// device/vol_render.cu. It calls no cudaMalloc, cudaFree or allocating
// library routine.
#include <cuda_runtime.h>

#include <string>

#include "context.h"
#include "device/render_launch.h"

using namespace grrt_b200;

extern "C" GRRT_EXPORT int grrt_render_spectral_device_noalloc(GRRTContext* ctx, const double* d_freqs,
                                                               int num_bins, double* d_spec, int width,
                                                               int height, void* stream) {
    if (!ctx) return -1;
    const int max_bins = volume_spectral_noalloc_max_bins();
    if (num_bins < 1 || num_bins > max_bins) {
        ctx->error = "grrt_render_spectral_device_noalloc: num_bins must be 1.." + std::to_string(max_bins) +
                     " (the fixed scratch holds that many bins)";
        return -1;
    }
    if (!d_freqs || !d_spec || width <= 0 || height <= 0) {
        ctx->error = "grrt_render_spectral_device_noalloc: bad buffer or size";
        return -1;
    }
    if (!ctx->device_ready) {
        ctx->error = "grrt_render_spectral_device_noalloc: the scene is not on the device yet; the first "
                     "render call on this context (any other grrt_render* entry point) uploads it";
        return -1;
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        cudaGetLastError();
        ctx->error = "grrt_render_spectral_device_noalloc: cannot select the context's device";
        return -1;
    }
    if (!ctx->vol) {
        // No volumetric disk: all-zero spectra, as grrt_render_spectral_device
        // and the reference give (src/geodesic_tracer.cpp:503-505).
        const size_t bytes = sizeof(double) * static_cast<size_t>(width) * height * num_bins;
        const cudaError_t z = cudaMemsetAsync(d_spec, 0, bytes, static_cast<cudaStream_t>(stream));
        if (z != cudaSuccess) {
            ctx->error = std::string("grrt_render_spectral_device_noalloc: ") + cudaGetErrorString(z);
            cudaGetLastError();
            return -1;
        }
        return 0;
    }
    DevTile tile;
    tile.w = width;
    tile.h = height;
    tile.out_pitch = width;
    const cudaError_t e = launch_volume_spectral_noalloc(ctx->scene_for_launch(), tile, d_freqs, num_bins, d_spec,
                                                         ctx->form, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        ctx->error = std::string("grrt_render_spectral_device_noalloc: ") + cudaGetErrorString(e);
        cudaGetLastError();
        return -1;
    }
    return 0;
}
