// Host-side entry points of the render kernels (implemented in the .cu files).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "scene.h"

namespace grrt_b200 {

// Device outputs of an RGB launch; any pointer may be null.
struct ThinOutputs {
    float4* rgba = nullptr;     // linear HDR RGBA, tile.out_pitch pixels per row
    double* rgb64 = nullptr;    // the spp-averaged double colour (3 per pixel)
    uint32_t* fate = nullptr;   // per sample: termination | (disk crossings << 2)
};

// Device outputs of a spectral launch.
struct SpectralOutputs {
    double* spec = nullptr;     // [pixel][bin], pixel = qy*out_pitch + qx
    uint32_t* fate = nullptr;
};

// Scratch of the mixed-precision thin-disk form (see mixed_render.cu).
struct DevMixedBuffers {
    unsigned* queue = nullptr;          // phase-1 work counter
    unsigned* queue2 = nullptr;         // phase-2 work counter
    unsigned* retrace_count = nullptr;  // samples queued for the FP64 re-trace
    unsigned* retrace_list = nullptr;   // their sample indices
    // optional: the speculative pass traces spec_list[0 .. *spec_count) instead
    // of every sample of the tile (the surrogate's uncertain samples)
    unsigned* spec_list = nullptr;
    unsigned* spec_count = nullptr;
    double* sample_rgb = nullptr;       // 3 per sample
    uint32_t* sample_fate = nullptr;    // per sample
    double margin = 0.05;               // disk-radius margin of the re-trace test
    double r_near = 0.0;                // escapes after coming inside r_near are re-traced
};

// Scratch a launch uses beside its inputs and outputs.
struct LaunchResources {
    unsigned int* queue = nullptr;    // work counter (zeroed by the launcher)
    DevStats* stats = nullptr;        // accumulated counters
    const volatile int* cancel = nullptr;  // host-mapped cancel flag, may be null
    double* spectral_scratch = nullptr;    // spectral transfer state, see volume_spectral_scratch_elems
    size_t spectral_scratch_elems = 0;
    // thin-disk FP64 form: the diagnostic instantiation that also measures the
    // Hamiltonian constraint (DevStats::h_max_bits)
    bool diag_hamiltonian = false;
};

// Longest-first order of n work items (cost_order.cu): items (NULL: 0..n-1;
// the count may be on the device, n_dev, at most n) are pixels of the tile
// (is_sample false: keyed by each pixel's first sample) or samples
// pixel * grid^2 + s; out receives them ordered by the closed-form distance of
// their camera ray to the critical curve, nearest first. scratch:
// cost_order_scratch_bytes(n).
size_t cost_order_scratch_bytes(size_t n);
cudaError_t order_by_cost(const DevScene& S, const DevTile& tile, const unsigned* items, unsigned n,
                          const unsigned* n_dev, bool is_sample, unsigned* out, void* scratch, cudaStream_t stream);

// Doubles of spectral scratch a launch with nb bins needs on the current device.
size_t volume_spectral_scratch_elems(int nb);

// Thin-disk render, FP64 form, one lane per pixel (thin_render.cu): the
// diagnostic instantiation (res.diag_hamiltonian) and the batched form use it.
cudaError_t launch_thin(const DevScene& S, const DevTile& tile, const ThinOutputs& out,
                        const LaunchResources& res, cudaStream_t stream);
// Thin-disk render, FP64 form, by samples (mixed_render.cu): the FP64 trace of
// every sample into the per-sample buffers of a mixed scratch
// (mixed_scratch_bytes), then the resolve. The same arithmetic as launch_thin.
// phase_events: NULL, or kFp64Phases + 1 events (trace, resolve).
constexpr int kFp64Phases = 2;
cudaError_t launch_thin_fp64(const DevScene& S, const DevTile& tile, const ThinOutputs& out,
                             const LaunchResources& res, void* scratch, size_t scratch_bytes,
                             cudaEvent_t* phase_events, cudaStream_t stream);

// Volumetric RGB render, FP64 form; and its mixed form (FP32 speculation with
// the thin form's star pass, FP64 re-trace, resolve: scratch of
// mixed_scratch_bytes, phase_events NULL or kMixedPhases + 1 events).
cudaError_t launch_volume_rgb(const DevScene& S, const DevTile& tile, const ThinOutputs& out,
                              const LaunchResources& res, cudaStream_t stream);
cudaError_t launch_volume_rgb_mixed(const DevScene& S, const DevTile& tile, const ThinOutputs& out,
                                    const LaunchResources& res, void* scratch, size_t scratch_bytes, double reach_z,
                                    cudaEvent_t* phase_events, cudaStream_t stream);
// The mixed form's FP64 re-trace of mb.retrace_list (mb.queue2 zeroed).
cudaError_t launch_volume_rgb_retrace(const DevScene& S, const DevTile& tile, const DevMixedBuffers& mb,
                                      DevStats* stats, const volatile int* cancel, cudaStream_t stream);

// Spectral render, FP64 form (vol_spectral.cu: warp-cooperative transfer).
constexpr int kVolSpectralThreads = 128;
cudaError_t launch_volume_spectral(const DevScene& S, const DevTile& tile, const double* freqs, int nb,
                                   const SpectralOutputs& out, const LaunchResources& res, cudaStream_t stream);
// The same kernel on a caller-chosen grid of kVolSpectralThreads-thread blocks
// and scratch (4 * nb doubles per thread); *queue must be zero.
cudaError_t launch_vol_spectral_on(const DevScene& S, const DevTile& tile, const double* freqs, int nb,
                                   double* out_spec, uint32_t* out_fate, double* scratch, unsigned* queue,
                                   DevStats* stats, const volatile int* cancel, int blocks, cudaStream_t stream);
// Mixed form of the spectral render: FP32 speculation, FP64 re-trace of the
// samples that may reach the volume, resolve. reach_z = max over the radial
// tables of z_max + 6 H. Scratch: volume_mixed_scratch_bytes; res must hold
// the spectral scratch as for launch_volume_spectral. phase_events: NULL or
// kVolMixedPhases + 1 events (speculate, re-trace, resolve).
constexpr int kVolMixedPhases = 3;
size_t volume_mixed_scratch_bytes(const DevTile& tile, int g2, int nb);
cudaError_t launch_volume_spectral_mixed(const DevScene& S, const DevTile& tile, const double* freqs, int nb,
                                         const SpectralOutputs& out, const LaunchResources& res, void* scratch,
                                         size_t scratch_bytes, double reach_z, cudaEvent_t* phase_events,
                                         cudaStream_t stream);

// Mixed-precision thin-disk render: FP32 speculation, FP64 re-trace, resolve.
size_t mixed_scratch_bytes(const DevTile& tile, int g2);
// Room for ordering the re-trace list inside a mixed scratch of n_samples
// samples (order_sample_list's scratch).
void* mixed_order_scratch(void* scratch, size_t n_samples);
// phase_events: NULL, or kMixedPhases + 1 events recorded on the stream around
// the phases (speculate, stars, re-trace, resolve).
constexpr int kMixedPhases = 4;
cudaError_t launch_thin_mixed(const DevScene& S, const DevTile& tile, const ThinOutputs& out,
                              const LaunchResources& res, void* scratch, size_t scratch_bytes, double margin,
                              double r_near, cudaEvent_t* phase_events, cudaStream_t stream);

// The mixed form's buffers inside a scratch of mixed_scratch_bytes (queue is
// the caller's phase-1 counter; spec_list left unset), and its re-trace and
// resolve phases on their own: the re-trace traces
// retrace_list[0 .. *retrace_count) with the FP64 method into sample_rgb /
// sample_fate; the resolve sums samples into pixels. queue2, retrace_count and
// the speculation-list counter (scratch bytes 256..1023) must be zeroed first.
DevMixedBuffers mixed_buffers(void* scratch, size_t n_samples, unsigned* queue);
// The same with a speculation list (after the re-trace list; its counter at
// scratch byte 768).
DevMixedBuffers mixed_buffers_with_list(void* scratch, size_t n_samples, unsigned* queue);
// The speculative pass (over mb.spec_list when set; mb.queue zeroed first) and
// the star pass on their own.
cudaError_t launch_mixed_speculate(const DevScene& S, const DevTile& tile, const DevMixedBuffers& mb,
                                   DevStats* stats, cudaStream_t stream);
cudaError_t launch_mixed_stars(const DevScene& S, const DevTile& tile, const DevMixedBuffers& mb,
                               cudaStream_t stream);
// scratch: the mixed scratch the buffers were cut from (mixed_scratch_bytes);
// on a black sky the list is ordered longest first in its tail region.
cudaError_t launch_mixed_retrace(const DevScene& S, const DevTile& tile, const DevMixedBuffers& mb, DevStats* stats,
                                 void* scratch, cudaStream_t stream);
cudaError_t launch_mixed_resolve(const DevScene& S, const DevTile& tile, const DevMixedBuffers& mb,
                                 const ThinOutputs& out, DevStats* stats, cudaStream_t stream);

// Re-trace lists in sample order (list_order.cu): list[0 .. *count) holds
// distinct sample indices below n; they are rewritten in increasing order.
// scratch: order_list_scratch_bytes(n) bytes, 256-byte aligned.
size_t order_list_scratch_bytes(size_t n);
cudaError_t order_sample_list(unsigned* list, const unsigned* count, size_t n, void* scratch, cudaStream_t stream);

// In-place tone mapping of a device RGBA float frame (tonemap.cu; 16-byte aligned).
cudaError_t launch_tonemap(float* d_rgba, int width, int height, cudaStream_t stream);

// One record of the single-ray debug trace (debug_trace.cu); the layout and
// the codes are GRRTDebugRecord's and its GRRT_DEBUG_* values.
struct DevDebugRecord {
    int kind, step, event, aux;
    double v[7];
};
constexpr int kDebugStart = 0, kDebugStep = 1, kDebugThinHit = 2, kDebugMarchEntry = 3, kDebugMarchExit = 4,
              kDebugEnd = 5;
constexpr int kDebugNone = 0, kDebugCross = 1, kDebugInside = 2, kDebugNear = 3;
constexpr int kDebugMaxRecords = 1 << 20;
// Records a trace of at most max_steps outer steps can produce (bounded by kDebugMaxRecords).
int debug_trace_capacity(int max_steps);
// Trace the camera sample at fractional pixel (x, y) in FP64 into rec[0 .. cap)
// (the last slot holds the END record when the trace has more); *count
// receives the number of records the trace produced.
cudaError_t launch_debug_trace(const DevScene& S, double x, double y, DevDebugRecord* rec, int cap, int* count,
                               cudaStream_t stream);

// Batched thin-disk render over many cameras (see DevBatch), FP64 form, with
// blocks of `block` threads (64, 128 or 256; the same registers per thread).
cudaError_t launch_thin_batch(const DevBatch& B, float4* out_rgba, unsigned int* queue, DevStats* stats,
                              int blocks, int block, cudaStream_t stream);
int thin_batch_max_blocks_per_sm(int block);

// Batched mixed form: the four phases of launch_thin_mixed, each one launch
// over the samples of every item (B.n_items, n_samples, n_pixels and each
// item's sample0 set). Scratch: mixed_scratch_bytes_for(B.n_samples).
// any_stars: some scene has stars on. blocks_per_sm: 0 = as many as fit.
size_t mixed_scratch_bytes_for(size_t n_samples);
cudaError_t launch_thin_mixed_batch(const DevBatch& B, bool any_stars, float4* out_rgba, unsigned* queue,
                                    DevStats* stats, void* scratch, size_t scratch_bytes, int blocks_per_sm,
                                    cudaStream_t stream);
int mixed_batch_max_blocks_per_sm();
// Batched FP64 form by samples: the trace of launch_thin_fp64 over the
// samples of every item in item order, then the resolve (scratch and items as
// for launch_thin_mixed_batch).
cudaError_t launch_thin_fp64_batch(const DevBatch& B, float4* out_rgba, unsigned* queue, DevStats* stats,
                                   void* scratch, size_t scratch_bytes, int blocks_per_sm, cudaStream_t stream);
int fp64_batch_max_blocks_per_sm();

// Batched volumetric spectral render over many cameras, FP64 form: one
// persistent launch of the warp-cooperative spectral kernel over the batch's
// chunk table. Each item carries its bins (freqs, nb) and its output offset
// (spec_offset, in elements); nb_max is the largest nb (the per-lane row
// stride), scratch holds 4 * nb_max doubles per lane of `blocks` blocks of
// vol_spectral_batch_threads() threads.
cudaError_t launch_vol_spectral_batch(const DevBatch& B, int nb_max, double* out_spec, double* scratch,
                                      size_t scratch_elems, unsigned* queue, DevStats* stats, int blocks,
                                      cudaStream_t stream);
int vol_spectral_batch_max_blocks_per_sm();
int vol_spectral_batch_threads();

// Spectral render whose scratch is a file-scope device array (no allocation);
// see vol_render.cu. Returns cudaErrorInvalidValue when nb exceeds the limit.
cudaError_t launch_volume_spectral_noalloc(const DevScene& S, const DevTile& tile, const double* freqs, int nb,
                                           double* out_spec, int form, cudaStream_t stream);
int volume_spectral_noalloc_max_bins();
size_t volume_spectral_noalloc_bytes();

}  // namespace grrt_b200
