// Device-side scene description shared by the host launcher and the kernels.
//
// One DevScene is passed by value to every render kernel (it lives in the
// kernel parameter bank, so every field is a uniform, broadcast load). Tables
// are device pointers into one arena allocated at grrt_create.
#pragma once

#include <cstdint>

namespace grrt_b200 {

enum : int { kTermHorizon = 0, kTermEscaped = 1, kTermMaxSteps = 2 };

// Precision forms.
enum : int { kFormFP64 = 0, kFormMixed = 1 };

struct DevStars {
    const double* theta = nullptr;
    const double* phi = nullptr;
    const double* brightness = nullptr;
    const int* cell_start = nullptr;  // 180*360 + 1
    const int* cell_items = nullptr;
    double tol2 = 0.0;                // angular tolerance squared
};

struct DevVolume {
    double M = 1, a = 0;  // the disk's own mass and spin (raw create parameters)
    double r_min = 0, r_outer = 0, r_isco = 0, r_horizon = 0, taper_width = 0;
    double E_isco = 0, L_isco = 0, rho_scale = 1, noise_scale = 1, turbulence = 0;
    double inv_taper_w2 = 0;
    int octaves = 2, n_r = 500, n_z = 128;
    const double* H = nullptr;        // n_r
    const double* z_max = nullptr;    // n_r
    const double* rho_mid = nullptr;  // n_r
    const double* rho_prof = nullptr; // n_r*n_z
    const double* T_prof = nullptr;   // n_r*n_z
    const int* perm = nullptr;        // 512
    // opacity tables
    int n_nu = 0, n_rho = 100, n_T = 100;
    double log_nu_min = 0, log_nu_max = 0, log_rho_min = 0, log_rho_max = 0, log_T_min = 0, log_T_max = 0;
    const double* ln_kabs = nullptr;  // ln(max(kappa_abs, 1e-100)), [n_nu][n_rho][n_T]
    const double* kes = nullptr;      // [n_rho][n_T]
    double ut_obs = 1;                // 1/sqrt(1 - 2/r_obs), the ray-march observer normalisation
};

struct DevScene {
    // spacetime and integrator
    double M = 1, a = 0;
    double r_stop = 0;      // horizon radius + 0.01 (termination)
    double r_escape = 1000; // escape radius
    double tol = 1e-8;
    double dl0 = 0.5;       // 0.01 * observer_r
    double observer_r = 50;
    int max_steps = 10000;

    // camera
    double cam_pos[4] = {0, 0, 0, 0};
    double e0[4] = {0, 0, 0, 0}, e1[4] = {0, 0, 0, 0}, e2[4] = {0, 0, 0, 0}, e3[4] = {0, 0, 0, 0};
    double g[16] = {};      // covariant metric at the camera, row-major
    double fov = 1.047;
    int width = 0, height = 0;
    int grid = 1;           // floor(sqrt(spp))
    double cell = 1.0;      // 1/grid
    double inv_spp = 1.0;   // 1/grid^2

    // thin disk
    int disk_on = 0;
    double r_in = 0, r_out = 0, flux_max = 0, peak_T = 0, u_t_obs = 1;
    int flux_n = 0;
    const double* flux = nullptr;

    // blackbody chromaticity table
    double t_min = 1000, t_max = 100000;
    int spec_n = 0;
    const double* spec_color = nullptr;  // 3*spec_n

    int stars_on = 0;
    DevStars stars;

    int vol_on = 0;
    DevVolume vol;

    // mixed forms (speculative FP32 pass, then FP64 re-trace): the FP32
    // tolerance; r_near_mixed = max(r_factor x r_horizon, 1.25 x the outermost
    // photon orbit radius), inside which a
    // near-critical sweep sends a sample to the re-trace (and beyond which,
    // on a black sky, a certain escape is final); mixed_margin, the disk-radius
    // margin of the re-trace test
    double r_near_mixed = 0;
    double tol_fp32 = 3e-6;
    double mixed_margin = 0.05;
};

// Which pixels a launch covers: columns [x0, x0+w) of the h image rows
// y0, y0 + row_step, ..., y0 + (h-1) row_step (row_step 1: a rectangle),
// written densely into an output of row pitch `out_pitch` pixels.
struct DevTile {
    int x0 = 0, y0 = 0, w = 0, h = 0;
    int out_pitch = 0;
    int row_step = 1;
};

// Batched form: one launch over many cameras. Items are camera images (or
// tiles of them); the work is cut into chunks of consecutive pixels of one
// item, and the chunk table fixes the order lanes take them in.
struct DevBatchItem {
    int scene = 0;               // index into DevBatch::scenes
    int x0 = 0, y0 = 0, w = 0, h = 0;
    int out_pitch = 0;           // output row pitch in pixels
    size_t out_offset = 0;       // first output pixel of this item
    size_t sample0 = 0;          // first sample of this item (mixed form: samples of all items in item order)
    // spectral batches: the item's observer-frame frequencies (device), their
    // count, and the item's first output element (its cube is [w*h][nb])
    const double* freqs = nullptr;
    int nb = 0;
    size_t spec_offset = 0;
};
struct DevBatchChunk {
    int item = 0;
    int start = 0;               // first pixel (row-major within the item)
    int count = 0;               // pixels in this chunk (<= chunk_size)
};
struct DevBatch {
    const DevScene* scenes = nullptr;
    const DevBatchItem* items = nullptr;
    const DevBatchChunk* chunks = nullptr;
    int n_chunks = 0;
    int chunk_size = 1;
    // mixed form: the items in order (ascending out_offset and sample0)
    int n_items = 0;
    unsigned n_samples = 0;      // sum over items of w * h * grid^2
    size_t n_pixels = 0;         // sum over items of w * h
};

// Per-launch counters (summed over all threads with one atomic per warp).
struct DevStats {
    unsigned long long attempts;      // DP45 attempts
    unsigned long long accepted;      // accepted outer steps
    unsigned long long crossings;     // thin-disk emission events
    unsigned long long rays;          // camera samples completed
    unsigned long long horizon;       // terminations by kind
    unsigned long long escaped;
    unsigned long long max_steps;
    unsigned long long clamp_evals;   // volumetric pre-step derivative evaluations
    unsigned long long march_steps;   // volumetric RK4 steps
    unsigned long long physics_steps; // volumetric steps with matter
    unsigned long long bin_updates;   // per-frequency transfer updates
    unsigned long long fp64_attempts; // mixed form: attempts taken in FP64
    unsigned long long cancelled;     // launches that observed the cancel flag
    // max over FP64-traced samples of |H| / p_t^2 at the final state, as the
    // bits of a non-negative double (integer order = value order)
    unsigned long long h_max_bits;
    unsigned long long pad[2];
};

}  // namespace grrt_b200
