// GRRTContext: resolved parameters, host tables, the device copy of the scene
// and the per-context launch resources.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <memory>
#include <string>
#include <vector>

#include "../../include/grrt_b200.h"
#include "device/render_launch.h"
#include "device/scene.h"
#include "host/tables.h"

// Chunks of the pipelined device-to-host copy (copy_to_host).
constexpr int kCopyChunks = 4;

struct GRRTContext {
    GRRTParams params{};

    // Resolved parameters (src/api.cpp:47-59, 72-75, 124, 141).
    double mass = 1.0, spin_a = 0.0, observer_r = 50.0, observer_theta = 1.396, fov = 1.047;
    double tolerance = 1e-8;
    int max_steps = 10000, spp = 1;
    double r_horizon = 2.0, isco = 6.0;

    grrt_b200::CameraFrame cam{};
    grrt_b200::SpectrumTable spectrum;
    bool has_disk = false;
    grrt_b200::FluxTable flux;
    bool has_stars = false;
    grrt_b200::StarCatalogue stars;
    std::unique_ptr<grrt_b200::VolumetricTables> vol;
    std::vector<double> ln_kabs;  // ln(max(kappa_abs, 1e-100)), precomputed for the device
    std::vector<double> freq_bins;

    // Precision form and its knobs.
    int form = GRRT_FORM_FP64;
    int diagnostics = 0;  // GRRT_DIAG_* flags
    double mixed_r_factor = 3.0;
    double tol_fp32 = 3e-6;
    double mixed_margin = 0.05;  // disk-radius margin (M) of the mixed form's re-trace test
    double vol_reach_z = 0.0;    // volumetric: max over r of z_max + 6 H (the mixed form's speculation bound)

    std::string error;
    float progress = 0.0f;
    // work counters of the last launch that progress reports read: the work
    // counter (d_queue) runs to progress_total; the mixed forms also have a
    // scratch header with the re-trace counter (+256) and list length (+512)
    unsigned progress_total = 0;
    const unsigned char* progress_header = nullptr;
    // volumetric kernels also count finished items (d_queue[1], header + 260),
    // which progress reads instead of the items taken (their long rays finish
    // long after the last item is taken)
    bool progress_done = false;

    // Device state (created at the first render).
    int device = -1;
    bool device_ready = false;
    void* d_arena = nullptr;
    grrt_b200::DevScene dev{};
    unsigned int* d_queue = nullptr;
    grrt_b200::DevStats* d_stats = nullptr;
    int* h_cancel = nullptr;   // host-mapped: [0] the cancel flag, [1] the value a cancel writes to work counters
    int* d_cancel = nullptr;   // device alias of the flag
    // work counters of the launch in flight that a cancel pushes past every
    // work index (the launch's counter; the mixed forms' re-trace counter),
    // through a host-to-device copy on cancel_stream: the copy engine writes
    // them while the kernels run, and lanes then take no new work
    std::atomic<unsigned*> cancel_q1{nullptr}, cancel_q2{nullptr};
    cudaStream_t cancel_stream = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // per-kernel phases of the last render (thin mixed form: speculate, stars,
    // re-trace, resolve; volumetric spectral mixed form: speculate, re-trace,
    // resolve; otherwise the one render kernel)
    cudaEvent_t ev_phase[grrt_b200::kMixedPhases + 1] = {};
    int n_phases = 0;
    double last_kernel_ms = 0.0;
    // cached device outputs for the host-buffer entry points
    void* d_out = nullptr;
    size_t d_out_bytes = 0;
    // pinned staging of the host-buffer entry points' device-to-host copy
    void* h_stage = nullptr;
    size_t h_stage_bytes = 0;
    cudaEvent_t ev_copy[kCopyChunks] = {};
    double* d_freqs = nullptr;
    size_t d_freqs_n = 0;
    double* d_spec_scratch = nullptr;
    size_t d_spec_scratch_n = 0;
    void* d_mixed_scratch = nullptr;
    size_t d_mixed_scratch_bytes = 0;

    GRRTContext() = default;
    ~GRRTContext();
    GRRTContext(const GRRTContext&) = delete;
    GRRTContext& operator=(const GRRTContext&) = delete;

    void build(const GRRTParams& p);
    bool ensure_device();
    grrt_b200::DevScene scene_for_launch() const;
    double mixed_r_near() const;

    int render_rgb_device(const grrt_b200::DevTile& tile, float* d_rgba, double* d_rgb64, unsigned* d_fate,
                          cudaStream_t s, bool reset_stats);
    int render_rgb_to_host(const grrt_b200::DevTile& tile, float* host, grrt_progress_fn cb, void* user);
    int render_spectral_device(int width, int height, double* d_spec, unsigned* d_fate, cudaStream_t s,
                               bool reset_stats);
    int render_spectral_tile(const grrt_b200::DevTile& tile, double* d_spec, unsigned* d_fate, cudaStream_t s,
                             bool reset_stats);
    int render_spectral_to_host(int width, int height, double* host, grrt_progress_fn cb, void* user);
    int render_spectral_to_fits(const char* path, int width, int height, grrt_progress_fn cb, void* user);
    int read_stats(GRRTStats* out);
    int phase_ms(double* out, int cap);
    bool export_table(const std::string& name, std::vector<double>& out) const;
    int debug_trace(double x, double y, GRRTDebugRecord* out, int capacity);
    void debug_pixel(int px, int py);
    void request_cancel();

    // helpers
    bool fail_cuda(cudaError_t e, const char* what);
    void* scratch_output(size_t bytes);
    bool stage_pinned(size_t bytes);
    int copy_to_host(void* host, const void* d, size_t bytes, cudaStream_t s);
    int wait_with_progress(cudaStream_t s, grrt_progress_fn cb, void* user);
};
