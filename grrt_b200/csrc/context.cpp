// GRRTContext implementation: parameter resolution and table build
// (src/api.cpp:43-173), device upload, kernel launches with progress polling
// and cancellation, FITS streaming, table export.
#include "context.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <thread>

#include "fits.h"

using namespace grrt_b200;

namespace {

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Host staging for the device arena: appends tables at 256-byte offsets.
struct ArenaBuilder {
    std::vector<unsigned char> bytes;
    size_t add(const void* src, size_t n) {
        const size_t off = align_up(bytes.size(), 256);
        bytes.resize(off + n);
        if (n) std::memcpy(bytes.data() + off, src, n);
        return off;
    }
    template <typename T>
    size_t add(const std::vector<T>& v) {
        return add(v.data(), v.size() * sizeof(T));
    }
};

}  // namespace

GRRTContext::~GRRTContext() {
    if (device_ready) {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        cudaFree(d_arena);
        cudaFree(d_queue);
        cudaFree(d_stats);
        cudaFree(d_out);
        cudaFree(d_freqs);
        cudaFree(d_spec_scratch);
        cudaFree(d_mixed_scratch);
        if (h_cancel) cudaFreeHost(h_cancel);
        if (h_stage) cudaFreeHost(h_stage);
        for (cudaEvent_t& e : ev_copy)
            if (e) cudaEventDestroy(e);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (cudaEvent_t& e : ev_phase)
            if (e) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
        if (cancel_stream) cudaStreamDestroy(cancel_stream);
        cudaSetDevice(prev);
    }
}

void GRRTContext::build(const GRRTParams& p) {
    params = p;
    // Defaults exactly as src/api.cpp:47-52.
    mass = p.mass > 0.0 ? p.mass : 1.0;
    observer_r = p.observer_r > 0.0 ? p.observer_r : 50.0;
    observer_theta = p.observer_theta > 0.0 ? p.observer_theta : 1.396;
    fov = p.fov > 0.0 ? p.fov : 1.047;
    max_steps = p.integrator_max_steps > 0 ? p.integrator_max_steps : 10000;
    tolerance = p.integrator_tolerance > 0.0 ? p.integrator_tolerance : 1e-8;
    // Kerr spin: only with GRRT_METRIC_KERR, and spin <= 0 selects 0.998 (api.cpp:55-59).
    spin_a = 0.0;
    if (p.metric_type == GRRT_METRIC_KERR) {
        const double s = p.spin > 0.0 ? p.spin : 0.998;
        spin_a = s * mass;
    }
    if (!(std::abs(spin_a) < mass)) throw std::invalid_argument("|a| must be below M (no horizon otherwise)");
    r_horizon = kerr_horizon(mass, spin_a);
    isco = kerr_isco(mass, spin_a);
    cam = build_camera(mass, spin_a, observer_r, observer_theta, p.observer_phi, fov, p.width, p.height);
    spectrum = build_spectrum_table();
    spp = p.samples_per_pixel > 0 ? p.samples_per_pixel : 1;

    has_disk = p.disk_enabled != 0;
    if (has_disk) {
        const double T = p.disk_temperature > 0.0 ? p.disk_temperature : 1e7;
        const double outer = p.disk_outer > 0.0 ? p.disk_outer : 20.0;
        const double inner = p.disk_inner > 0.0 ? p.disk_inner : isco;
        flux = build_flux_table(mass, spin_a, inner, outer, T);
        if (p.disk_volumetric) {
            double vT = p.disk_temperature > 0 ? p.disk_temperature : 1e7;
            if (p.mass_solar > 0.0 && p.eddington_fraction > 0.0 && p.disk_temperature <= 0.0) {
                vT = derived_peak_temperature(p.spin, p.mass_solar, p.eddington_fraction);
                std::printf("[GRRT] Derived T_peak = %.0f K from M=%.1f M_sun, f_Edd=%.3f\n", vT, p.mass_solar,
                            p.eddington_fraction);
            }
            VolumetricConfig vc;
            vc.alpha = p.disk_alpha;
            vc.turbulence = p.disk_turbulence;
            vc.seed = static_cast<uint32_t>(p.disk_seed);
            vc.noise_scale = p.disk_noise_scale;
            vc.noise_octaves = p.disk_noise_octaves;
            if (p.num_frequency_bins > 0 && p.frequency_bins_hz) {
                double lo = p.frequency_bins_hz[0], hi = p.frequency_bins_hz[0];
                for (int i = 1; i < p.num_frequency_bins; ++i) {
                    lo = std::min(lo, p.frequency_bins_hz[i]);
                    hi = std::max(hi, p.frequency_bins_hz[i]);
                }
                vc.opacity_nu_min = lo * 0.1;
                vc.opacity_nu_max = hi * 10.0;
            }
            // The disk takes the raw mass and spin parameters, as the reference does
            // (src/api.cpp:122-126).
            if (!(std::abs(p.spin) < p.mass)) throw std::invalid_argument("volumetric disk needs |spin| < mass");
            vol = std::make_unique<VolumetricTables>(build_volumetric_tables(
                p.mass, p.spin, p.disk_outer > 0 ? p.disk_outer : 30.0, vT, vc));
            ln_kabs.resize(vol->opacity.kappa_abs.size());
            for (size_t i = 0; i < ln_kabs.size(); ++i)
                ln_kabs[i] = std::log(std::max(vol->opacity.kappa_abs[i], 1e-100));
            std::printf("[GRRT] volumetric disk: r_isco=%.4f r_horizon=%.4f rho_scale=%.4e\n", vol->r_isco,
                        vol->r_horizon, vol->rho_scale);
            // half-thickness of the near-disk clamp slab, z_max + 6 H, at its
            // widest (the radial tables are linear between nodes and constant
            // beyond them)
            vol_reach_z = 0.0;
            for (size_t i = 0; i < vol->H.size() && i < vol->z_max.size(); ++i)
                vol_reach_z = std::max(vol_reach_z, vol->z_max[i] + 6.0 * vol->H[i]);
        }
    }
    has_stars = p.background_type == GRRT_BG_STARS;
    if (has_stars) stars = build_star_catalogue();
}

bool GRRTContext::fail_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return false;
    error = std::string(what) + ": " + cudaGetErrorString(e);
    cudaGetLastError();
    return true;
}

bool GRRTContext::ensure_device() {
    if (device_ready) {
        cudaSetDevice(device);
        return true;
    }
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        error = "no CUDA device available (libgrrt renders on the GPU only)";
        return false;
    }
    if (fail_cuda(cudaGetDevice(&device), "cudaGetDevice")) return false;
    cudaDeviceProp prop{};
    if (fail_cuda(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties")) return false;
    if (prop.major < 10) {
        error = "libgrrt is built for sm_100a (B200); the current device is sm_" + std::to_string(prop.major) +
                std::to_string(prop.minor);
        return false;
    }

    ArenaBuilder ab;
    size_t o_flux = 0, o_spec = ab.add(spectrum.color);
    if (has_disk) o_flux = ab.add(flux.flux);
    size_t o_st = 0, o_sp = 0, o_sb = 0, o_cs = 0, o_ci = 0;
    if (has_stars) {
        o_st = ab.add(stars.theta);
        o_sp = ab.add(stars.phi);
        o_sb = ab.add(stars.brightness);
        o_cs = ab.add(stars.cell_start);
        o_ci = ab.add(stars.cell_items);
    }
    size_t o_H = 0, o_zm = 0, o_rm = 0, o_rp = 0, o_tp = 0, o_perm = 0, o_lk = 0, o_kes = 0;
    if (vol) {
        o_H = ab.add(vol->H);
        o_zm = ab.add(vol->z_max);
        o_rm = ab.add(vol->rho_mid);
        o_rp = ab.add(vol->rho_profile);
        o_tp = ab.add(vol->T_profile);
        o_perm = ab.add(vol->perm.data(), vol->perm.size() * sizeof(int));
        o_lk = ab.add(ln_kabs);
        o_kes = ab.add(vol->opacity.kappa_es);
    }
    const size_t bytes = std::max<size_t>(ab.bytes.size(), 256);
    if (fail_cuda(cudaMalloc(&d_arena, bytes), "cudaMalloc(scene)")) return false;
    if (fail_cuda(cudaMemcpy(d_arena, ab.bytes.data(), ab.bytes.size(), cudaMemcpyHostToDevice), "upload scene"))
        return false;
    auto at = [&](size_t off) { return static_cast<unsigned char*>(d_arena) + off; };

    DevScene& S = dev;
    S.M = mass;
    S.a = spin_a;
    S.r_stop = r_horizon + 0.01;
    S.r_escape = 1000.0;
    S.tol = tolerance;
    S.dl0 = 0.01 * observer_r;
    S.observer_r = observer_r;
    S.max_steps = max_steps;
    for (int m = 0; m < 4; ++m) {
        S.cam_pos[m] = cam.pos[m];
        S.e0[m] = cam.e0[m];
        S.e1[m] = cam.e1[m];
        S.e2[m] = cam.e2[m];
        S.e3[m] = cam.e3[m];
        for (int k = 0; k < 4; ++k) S.g[4 * m + k] = cam.g[m][k];
    }
    S.fov = fov;
    S.width = cam.width;
    S.height = cam.height;
    S.grid = std::max(1, static_cast<int>(std::sqrt(static_cast<double>(spp))));
    S.cell = 1.0 / S.grid;
    S.inv_spp = 1.0 / (S.grid * S.grid);
    S.t_min = spectrum.t_min;
    S.t_max = spectrum.t_max;
    S.spec_n = spectrum.n;
    S.spec_color = reinterpret_cast<const double*>(at(o_spec));
    S.disk_on = (has_disk && !vol) ? 1 : 0;
    if (has_disk) {
        S.r_in = flux.r_inner;
        S.r_out = flux.r_outer;
        S.flux_max = flux.flux_max;
        S.peak_T = flux.peak_temperature;
        S.flux_n = static_cast<int>(flux.flux.size());
        S.flux = reinterpret_cast<const double*>(at(o_flux));
        S.u_t_obs = 1.0 / std::sqrt(1.0 - 2.0 * mass / observer_r);
    }
    S.stars_on = has_stars ? 1 : 0;
    if (has_stars) {
        S.stars.theta = reinterpret_cast<const double*>(at(o_st));
        S.stars.phi = reinterpret_cast<const double*>(at(o_sp));
        S.stars.brightness = reinterpret_cast<const double*>(at(o_sb));
        S.stars.cell_start = reinterpret_cast<const int*>(at(o_cs));
        S.stars.cell_items = reinterpret_cast<const int*>(at(o_ci));
        S.stars.tol2 = stars.angular_tolerance * stars.angular_tolerance;
    }
    S.vol_on = vol ? 1 : 0;
    if (vol) {
        DevVolume& V = S.vol;
        V.M = vol->M;
        V.a = vol->a;
        V.r_min = vol->r_min;
        V.r_outer = vol->r_outer;
        V.r_isco = vol->r_isco;
        V.r_horizon = vol->r_horizon;
        V.taper_width = vol->taper_width;
        V.E_isco = vol->E_isco;
        V.L_isco = vol->L_isco;
        V.rho_scale = vol->rho_scale;
        V.noise_scale = vol->noise_scale;
        V.turbulence = vol->cfg.turbulence;
        V.octaves = vol->cfg.noise_octaves;
        V.n_r = vol->n_r;
        V.n_z = vol->n_z;
        V.H = reinterpret_cast<const double*>(at(o_H));
        V.z_max = reinterpret_cast<const double*>(at(o_zm));
        V.rho_mid = reinterpret_cast<const double*>(at(o_rm));
        V.rho_prof = reinterpret_cast<const double*>(at(o_rp));
        V.T_prof = reinterpret_cast<const double*>(at(o_tp));
        V.perm = reinterpret_cast<const int*>(at(o_perm));
        const OpacityTables& op = vol->opacity;
        V.n_nu = op.n_nu;
        V.n_rho = op.n_rho;
        V.n_T = op.n_T;
        V.log_nu_min = op.log_nu_min;
        V.log_nu_max = op.log_nu_max;
        V.log_rho_min = op.log_rho_min;
        V.log_rho_max = op.log_rho_max;
        V.log_T_min = op.log_T_min;
        V.log_T_max = op.log_T_max;
        V.ln_kabs = reinterpret_cast<const double*>(at(o_lk));
        V.kes = reinterpret_cast<const double*>(at(o_kes));
        V.ut_obs = 1.0 / std::sqrt(1.0 - 2.0 / observer_r);
    }

    if (fail_cuda(cudaMalloc(&d_queue, 256), "cudaMalloc(queue)")) return false;
    if (fail_cuda(cudaMalloc(&d_stats, sizeof(DevStats)), "cudaMalloc(stats)")) return false;
    if (fail_cuda(cudaMemset(d_stats, 0, sizeof(DevStats)), "memset(stats)")) return false;
    if (fail_cuda(cudaHostAlloc(&h_cancel, 2 * sizeof(int), cudaHostAllocMapped), "cudaHostAlloc(cancel)"))
        return false;
    h_cancel[0] = 0;
    h_cancel[1] = 0x7f7f7f7f;  // beyond any work index; atomic adds after it cannot wrap
    if (fail_cuda(cudaStreamCreateWithFlags(&cancel_stream, cudaStreamNonBlocking), "cudaStreamCreate(cancel)"))
        return false;
    if (fail_cuda(cudaHostGetDevicePointer(reinterpret_cast<void**>(&d_cancel), h_cancel, 0), "map cancel flag"))
        return false;
    if (fail_cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate")) return false;
    if (fail_cuda(cudaEventCreate(&ev0), "cudaEventCreate")) return false;
    if (fail_cuda(cudaEventCreate(&ev1), "cudaEventCreate")) return false;
    for (cudaEvent_t& e : ev_phase)
        if (fail_cuda(cudaEventCreate(&e), "cudaEventCreate")) return false;
    device_ready = true;
    return true;
}

// Radius inside which the mixed forms' speculation treats a long sweep as a
// near-critical orbit: r_factor x r_horizon, and at least 1.25 x the outermost
// photon orbit (the retrograde equatorial one, 2M (1 + cos(2/3 acos(|a|/M))):
// 3M at a = 0, 4M at |a| = M), so that near-critical orbits of every spin lie
// inside it (3 r_horizon is only 3.19M at a = 0.998).
double GRRTContext::mixed_r_near() const {
    const double x = std::min(std::fabs(spin_a) / mass, 1.0);
    const double r_ph = 2.0 * mass * (1.0 + std::cos(2.0 / 3.0 * std::acos(x)));
    return std::max(mixed_r_factor * r_horizon, 1.25 * r_ph);
}

DevScene GRRTContext::scene_for_launch() const {
    DevScene S = dev;
    S.r_near_mixed = mixed_r_near();
    S.tol_fp32 = tol_fp32;
    S.mixed_margin = mixed_margin;
    return S;
}

// Raises the host-mapped flag (polled by the volumetric kernels, whose long
// rays must stop mid-trace) and pushes the running launch's work counters past
// every work index with a copy-engine write (the thin-disk and mixed kernels
// then take no new work and end once their lanes' current samples end). Safe
// to call from any thread while a render runs.
void GRRTContext::request_cancel() {
    if (!h_cancel) return;
    *reinterpret_cast<volatile int*>(h_cancel) = 1;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    for (unsigned* q : {cancel_q1.load(), cancel_q2.load()})
        if (q) cudaMemcpyAsync(q, h_cancel + 1, sizeof(unsigned), cudaMemcpyHostToDevice, cancel_stream);
    cudaGetLastError();
    cudaSetDevice(prev);
}

void* GRRTContext::scratch_output(size_t bytes) {
    if (bytes > d_out_bytes) {
        cudaFree(d_out);
        d_out = nullptr;
        d_out_bytes = 0;
        if (cudaMalloc(&d_out, bytes) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        d_out_bytes = bytes;
    }
    return d_out;
}

int GRRTContext::render_rgb_device(const DevTile& tile, float* d_rgba, double* d_rgb64, unsigned* d_fate,
                                   cudaStream_t s, bool reset_stats) {
    if (!ensure_device()) return -1;
    error.clear();
    // a cancel of an earlier render lands before this one starts
    cudaStreamSynchronize(cancel_stream);
    *reinterpret_cast<volatile int*>(h_cancel) = 0;
    if (reset_stats && fail_cuda(cudaMemsetAsync(d_stats, 0, sizeof(DevStats), s), "reset stats")) return -1;
    LaunchResources res;
    res.queue = d_queue;
    res.stats = d_stats;
    res.cancel = d_cancel;
    res.diag_hamiltonian = (diagnostics & GRRT_DIAG_HAMILTONIAN) != 0;
    ThinOutputs out;
    out.rgba = reinterpret_cast<float4*>(d_rgba);
    out.rgb64 = d_rgb64;
    out.fate = d_fate;
    const DevScene S = scene_for_launch();
    const bool mixed_thin = !vol && form == GRRT_FORM_MIXED;
    const bool mixed_vol = vol && form == GRRT_FORM_MIXED;
    // the thin-disk FP64 form traces by samples into the same per-sample
    // buffers (the Hamiltonian diagnostic keeps the per-pixel kernel)
    const bool fp64_thin = !vol && !mixed_thin && !res.diag_hamiltonian;
    size_t mixed_bytes = 0;
    if (mixed_thin || mixed_vol || fp64_thin) {
        mixed_bytes = mixed_scratch_bytes(tile, S.grid * S.grid);
        if (mixed_bytes > d_mixed_scratch_bytes) {
            cudaFree(d_mixed_scratch);
            d_mixed_scratch = nullptr;
            d_mixed_scratch_bytes = 0;
            if (fail_cuda(cudaMalloc(&d_mixed_scratch, mixed_bytes), "cudaMalloc(mixed scratch)")) return -1;
            d_mixed_scratch_bytes = mixed_bytes;
        }
    }
    n_phases = 0;
    progress_total = (mixed_thin || mixed_vol || fp64_thin)
                         ? static_cast<unsigned>(tile.w) * tile.h * (S.grid * S.grid)
                         : static_cast<unsigned>(tile.w) * tile.h;
    progress_header = (mixed_thin || mixed_vol) ? static_cast<const unsigned char*>(d_mixed_scratch) : nullptr;
    progress_done = vol != nullptr;
    cancel_q1 = d_queue;
    cancel_q2 = (mixed_thin || mixed_vol) ? reinterpret_cast<unsigned*>(static_cast<unsigned char*>(d_mixed_scratch) + 256)
                                          : nullptr;
    cudaEventRecord(ev0, s);
    cudaError_t e;
    if (mixed_vol)
        e = launch_volume_rgb_mixed(S, tile, out, res, d_mixed_scratch, d_mixed_scratch_bytes, vol_reach_z, ev_phase,
                                    s);
    else if (vol)
        e = launch_volume_rgb(S, tile, out, res, s);
    else if (mixed_thin)
        e = launch_thin_mixed(S, tile, out, res, d_mixed_scratch, d_mixed_scratch_bytes, mixed_margin,
                              mixed_r_near(), ev_phase, s);
    else if (fp64_thin)
        e = launch_thin_fp64(S, tile, out, res, d_mixed_scratch, d_mixed_scratch_bytes, ev_phase, s);
    else
        e = launch_thin(S, tile, out, res, s);
    cudaEventRecord(ev1, s);
    n_phases = (mixed_thin || mixed_vol) ? kMixedPhases : fp64_thin ? kFp64Phases : 0;
    if (fail_cuda(e, "render launch")) return -1;
    return 0;
}

int GRRTContext::wait_with_progress(cudaStream_t s, grrt_progress_fn cb, void* user) {
    if (cb) {
        // Poll the launch's work counters through a second stream while the
        // kernels run. Single-pass forms count pixels; the mixed forms count
        // samples in their speculation (the first half of the report) and
        // re-trace list entries against the list's length (the second half).
        cudaStream_t poll = nullptr;
        unsigned* h_q = nullptr;
        if (cudaStreamCreateWithFlags(&poll, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMallocHost(&h_q, 3 * sizeof(unsigned)) == cudaSuccess) {
            float last = -1.0f;
            while (cudaStreamQuery(s) == cudaErrorNotReady) {
                std::this_thread::sleep_for(std::chrono::milliseconds(5));
                h_q[0] = h_q[1] = h_q[2] = 0;
                // single pass: items finished (volumetric) or taken; mixed
                // forms: speculation items taken, then re-trace items
                const bool single_done = progress_done && !progress_header;
                if (cudaMemcpyAsync(h_q, d_queue + (single_done ? 1 : 0), sizeof(unsigned), cudaMemcpyDeviceToHost,
                                    poll) != cudaSuccess)
                    break;
                if (progress_header &&
                    (cudaMemcpyAsync(h_q + 1, progress_header + (progress_done ? 260 : 256), sizeof(unsigned),
                                     cudaMemcpyDeviceToHost, poll) != cudaSuccess ||
                     cudaMemcpyAsync(h_q + 2, progress_header + 512, sizeof(unsigned), cudaMemcpyDeviceToHost,
                                     poll) != cudaSuccess))
                    break;
                cudaStreamSynchronize(poll);
                float f = progress_total ? std::min(1.0f, static_cast<float>(h_q[0]) / progress_total) : 1.0f;
                if (progress_header) {
                    const float f2 = (f >= 1.0f && h_q[2] > 0)
                                         ? std::min(1.0f, static_cast<float>(h_q[1]) / static_cast<float>(h_q[2]))
                                         : 0.0f;
                    f = 0.5f * f + 0.5f * f2;
                }
                if (f > last && f < 1.0f) {
                    progress = f;
                    cb(f, user);
                    last = f;
                }
            }
        }
        cudaGetLastError();
        if (h_q) cudaFreeHost(h_q);
        if (poll) cudaStreamDestroy(poll);
    }
    if (fail_cuda(cudaStreamSynchronize(s), "render")) return -1;
    if (*reinterpret_cast<volatile int*>(h_cancel)) {
        error = "render cancelled";
        return -1;
    }
    progress = 1.0f;
    if (cb) cb(1.0f, user);
    return 0;
}

// Pinned host staging of at least `bytes`, kept across calls, and the
// chunk events of the pipelined copies. False when pinned memory cannot be
// had (the callers then copy without staging).
bool GRRTContext::stage_pinned(size_t bytes) {
    if (bytes > h_stage_bytes) {
        if (h_stage) cudaFreeHost(h_stage);
        h_stage = nullptr;
        h_stage_bytes = 0;
        if (cudaMallocHost(&h_stage, bytes) == cudaSuccess) {
            h_stage_bytes = bytes;
        } else {
            cudaGetLastError();
            h_stage = nullptr;
            return false;
        }
    }
    for (cudaEvent_t& e : ev_copy)
        if (!e && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            e = nullptr;
            return false;
        }
    return h_stage != nullptr;
}

// Device-to-host copy of a finished result into caller memory. Page-locked
// caller memory (cudaMallocHost, cudaHostRegister) takes one direct copy.
// Pageable memory, as a caller's framebuffer usually is, goes through a pinned
// staging buffer in kCopyChunks chunks, each chunk's copy into the caller's
// buffer spread over the host threads while the next chunks cross the bus;
// small results, or no pinned memory to be had, take one plain copy.
int GRRTContext::copy_to_host(void* host, const void* d, size_t bytes, cudaStream_t s) {
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, host) == cudaSuccess && attr.type == cudaMemoryTypeHost) {
        if (fail_cuda(cudaMemcpyAsync(host, d, bytes, cudaMemcpyDeviceToHost, s), "copy result") ||
            fail_cuda(cudaStreamSynchronize(s), "copy result"))
            return -1;
        return 0;
    }
    cudaGetLastError();
    constexpr size_t kMin = size_t(4) << 20;
    const bool events = bytes >= kMin && stage_pinned(bytes);
    if (!events) return fail_cuda(cudaMemcpy(host, d, bytes, cudaMemcpyDeviceToHost), "copy result") ? -1 : 0;
    const size_t chunk = (bytes + kCopyChunks - 1) / kCopyChunks;
    for (int k = 0; k < kCopyChunks; ++k) {
        const size_t off = chunk * k, len = std::min(chunk, bytes - std::min(bytes, off));
        if (len == 0) break;
        if (fail_cuda(cudaMemcpyAsync(static_cast<char*>(h_stage) + off, static_cast<const char*>(d) + off, len,
                                      cudaMemcpyDeviceToHost, s),
                      "copy result") ||
            fail_cuda(cudaEventRecord(ev_copy[k], s), "copy result"))
            return -1;
    }
    for (int k = 0; k < kCopyChunks; ++k) {
        const size_t off = chunk * k, len = std::min(chunk, bytes - std::min(bytes, off));
        if (len == 0) break;
        if (fail_cuda(cudaEventSynchronize(ev_copy[k]), "copy result")) return -1;
        const char* src = static_cast<const char*>(h_stage) + off;
        char* dst = static_cast<char*>(host) + off;
        constexpr size_t kPiece = size_t(256) << 10;
        const long long pieces = static_cast<long long>((len + kPiece - 1) / kPiece);
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < pieces; ++i) {
            const size_t o = static_cast<size_t>(i) * kPiece;
            std::memcpy(dst + o, src + o, std::min(kPiece, len - o));
        }
    }
    return 0;
}

int GRRTContext::render_rgb_to_host(const DevTile& tile, float* host, grrt_progress_fn cb, void* user) {
    if (!ensure_device()) return -1;
    progress = 0.0f;
    const size_t bytes = sizeof(float) * 4 * static_cast<size_t>(tile.w) * tile.h;
    auto* d = static_cast<float*>(scratch_output(bytes));
    if (!d) {
        error = "cudaMalloc(output) failed";
        return -1;
    }
    if (render_rgb_device(tile, d, nullptr, nullptr, stream, true) != 0) return -1;
    if (wait_with_progress(stream, cb, user) != 0) return -1;
    return copy_to_host(host, d, bytes, stream);
}

int GRRTContext::render_spectral_device(int width, int height, double* d_spec, unsigned* d_fate, cudaStream_t s,
                                        bool reset_stats) {
    DevTile tile;
    tile.w = width;
    tile.h = height;
    tile.out_pitch = width;
    return render_spectral_tile(tile, d_spec, d_fate, s, reset_stats);
}

int GRRTContext::render_spectral_tile(const DevTile& tile, double* d_spec, unsigned* d_fate, cudaStream_t s,
                                      bool reset_stats) {
    if (!ensure_device()) return -1;
    error.clear();
    // a cancel of an earlier render lands before this one starts
    cudaStreamSynchronize(cancel_stream);
    *reinterpret_cast<volatile int*>(h_cancel) = 0;
    const int width = tile.w, height = tile.h;
    const int nb = static_cast<int>(freq_bins.size());
    const size_t n = static_cast<size_t>(width) * height * nb;
    if (reset_stats && fail_cuda(cudaMemsetAsync(d_stats, 0, sizeof(DevStats), s), "reset stats")) return -1;
    if (!vol) {
        // No volumetric disk: the reference returns all-zero spectra
        // (src/geodesic_tracer.cpp:503-505).
        n_phases = 0;
        progress_total = 0;
        progress_header = nullptr;
        cudaEventRecord(ev0, s);
        cudaError_t e = cudaMemsetAsync(d_spec, 0, n * sizeof(double), s);
        if (d_fate && e == cudaSuccess) {
            // every sample reports "escaped" with no crossings
            const int grid = std::max(1, static_cast<int>(std::sqrt(static_cast<double>(spp))));
            const size_t ns = static_cast<size_t>(width) * height * grid * grid;
            e = cudaMemsetAsync(d_fate, 0, ns * sizeof(unsigned), s);
            if (e == cudaSuccess) {
                std::vector<unsigned> ones(ns, 1u);
                e = cudaMemcpyAsync(d_fate, ones.data(), ns * sizeof(unsigned), cudaMemcpyHostToDevice, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            }
        }
        cudaEventRecord(ev1, s);
        return fail_cuda(e, "zero spectra") ? -1 : 0;
    }
    if (d_freqs_n < freq_bins.size()) {
        cudaFree(d_freqs);
        d_freqs = nullptr;
        if (fail_cuda(cudaMalloc(&d_freqs, sizeof(double) * freq_bins.size()), "cudaMalloc(freqs)")) return -1;
        d_freqs_n = freq_bins.size();
    }
    if (fail_cuda(cudaMemcpyAsync(d_freqs, freq_bins.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s),
                  "upload frequencies"))
        return -1;
    const size_t need = volume_spectral_scratch_elems(nb);
    if (d_spec_scratch_n < need) {
        cudaFree(d_spec_scratch);
        d_spec_scratch = nullptr;
        d_spec_scratch_n = 0;
        if (fail_cuda(cudaMalloc(&d_spec_scratch, need * sizeof(double)), "cudaMalloc(spectral scratch)")) return -1;
        d_spec_scratch_n = need;
    }
    LaunchResources res;
    res.queue = d_queue;
    res.stats = d_stats;
    res.cancel = d_cancel;
    res.spectral_scratch = d_spec_scratch;
    res.spectral_scratch_elems = d_spec_scratch_n;
    SpectralOutputs out;
    out.spec = d_spec;
    out.fate = d_fate;
    const DevScene S = scene_for_launch();
    const bool mixed = form == GRRT_FORM_MIXED;
    if (mixed) {
        const size_t mb = volume_mixed_scratch_bytes(tile, S.grid * S.grid, nb);
        if (mb > d_mixed_scratch_bytes) {
            cudaFree(d_mixed_scratch);
            d_mixed_scratch = nullptr;
            d_mixed_scratch_bytes = 0;
            if (fail_cuda(cudaMalloc(&d_mixed_scratch, mb), "cudaMalloc(mixed scratch)")) return -1;
            d_mixed_scratch_bytes = mb;
        }
    }
    n_phases = 0;
    progress_total = mixed ? static_cast<unsigned>(width) * height * (S.grid * S.grid)
                           : static_cast<unsigned>(width) * height;
    progress_header = mixed ? static_cast<const unsigned char*>(d_mixed_scratch) : nullptr;
    progress_done = true;
    cancel_q1 = d_queue;
    cancel_q2 = mixed ? reinterpret_cast<unsigned*>(static_cast<unsigned char*>(d_mixed_scratch) + 256) : nullptr;
    cudaEventRecord(ev0, s);
    const cudaError_t e =
        mixed ? launch_volume_spectral_mixed(S, tile, d_freqs, nb, out, res, d_mixed_scratch, d_mixed_scratch_bytes,
                                             vol_reach_z, ev_phase, s)
              : launch_volume_spectral(S, tile, d_freqs, nb, out, res, s);
    cudaEventRecord(ev1, s);
    n_phases = mixed ? kVolMixedPhases : 0;
    return fail_cuda(e, "spectral launch") ? -1 : 0;
}

int GRRTContext::render_spectral_to_host(int width, int height, double* host, grrt_progress_fn cb, void* user) {
    if (!ensure_device()) return -1;
    progress = 0.0f;
    const size_t bytes = sizeof(double) * static_cast<size_t>(width) * height * freq_bins.size();
    auto* d = static_cast<double*>(scratch_output(bytes));
    if (!d) {
        error = "cudaMalloc(output) failed";
        return -1;
    }
    if (render_spectral_device(width, height, d, nullptr, stream, true) != 0) return -1;
    if (wait_with_progress(stream, cb, user) != 0) return -1;
    return copy_to_host(host, d, bytes, stream);
}

int GRRTContext::render_spectral_to_fits(const char* path, int width, int height, grrt_progress_fn cb, void* user) {
    if (!ensure_device()) return -1;
    progress = 0.0f;
    FitsMetadata meta;
    meta.spin = params.spin;
    meta.mass = params.mass > 0.0 ? params.mass : 1.0;
    meta.observer_r = params.observer_r > 0.0 ? params.observer_r : 50.0;
    meta.observer_theta = params.observer_theta > 0.0 ? params.observer_theta : 1.396;
    meta.fov = params.fov > 0.0 ? params.fov : 1.047;
    meta.samples_per_pixel = params.samples_per_pixel > 0 ? params.samples_per_pixel : 1;
    const int nb = static_cast<int>(freq_bins.size());
    const size_t cube = static_cast<size_t>(width) * height * nb;
    const size_t plane_bytes = sizeof(double) * static_cast<size_t>(width) * height;
    // The rendered cube and its big-endian FITS image side by side on the device.
    auto* d = static_cast<unsigned char*>(scratch_output(2 * sizeof(double) * cube));
    if (!d) {
        error = "cudaMalloc(cube) failed";
        return -1;
    }
    double* d_cube = reinterpret_cast<double*>(d);
    unsigned char* d_be = d + sizeof(double) * cube;
    try {
        FitsCubeWriter writer(path, width, height, nb, freq_bins, meta);
        if (render_spectral_device(width, height, d_cube, nullptr, stream, true) != 0) return -1;
        if (wait_with_progress(stream, cb, user) != 0) return -1;
        // The FITS data section is the planes back to back, so the packed cube
        // goes to the file as it is. Planes are packed and copied in groups on
        // the render stream; each group is written to the file while the next
        // groups are packed and cross the bus.
        const int groups = std::min(kCopyChunks, nb);
        const int per = (nb + groups - 1) / groups;
        if (stage_pinned(sizeof(double) * cube)) {
            auto* h = static_cast<unsigned char*>(h_stage);
            for (int g = 0; g < groups; ++g) {
                const int k0 = g * per, k1 = std::min(nb, k0 + per);
                if (k0 >= k1) break;
                const size_t off = plane_bytes * static_cast<size_t>(k0);
                if (fail_cuda(pack_fits_planes(d_cube, width, height, nb, k0, k1, d_be + off, stream), "pack planes") ||
                    fail_cuda(cudaMemcpyAsync(h + off, d_be + off, plane_bytes * static_cast<size_t>(k1 - k0),
                                              cudaMemcpyDeviceToHost, stream),
                              "copy planes") ||
                    fail_cuda(cudaEventRecord(ev_copy[g], stream), "copy planes"))
                    return -1;
            }
            for (int g = 0; g < groups; ++g) {
                const int k0 = g * per, k1 = std::min(nb, k0 + per);
                if (k0 >= k1) break;
                if (fail_cuda(cudaEventSynchronize(ev_copy[g]), "copy planes")) return -1;
                writer.write_planes(k0, k1, h + plane_bytes * static_cast<size_t>(k0));
            }
        } else {
            // no pinned memory: one plane at a time through pageable memory
            std::vector<unsigned char> host(plane_bytes);
            for (int k = 0; k < nb; ++k) {
                if (fail_cuda(pack_fits_planes(d_cube, width, height, nb, k, k + 1, d_be, stream), "pack plane") ||
                    fail_cuda(cudaMemcpyAsync(host.data(), d_be, plane_bytes, cudaMemcpyDeviceToHost, stream),
                              "copy plane") ||
                    fail_cuda(cudaStreamSynchronize(stream), "copy plane"))
                    return -1;
                writer.write_planes(k, k + 1, host.data());
            }
        }
        writer.finalize();
    } catch (const std::exception& e) {
        error = e.what();
        return -1;
    }
    return 0;
}

int GRRTContext::read_stats(GRRTStats* out) {
    std::memset(out, 0, sizeof(*out));
    if (!device_ready) return 0;
    cudaSetDevice(device);
    if (fail_cuda(cudaDeviceSynchronize(), "synchronize")) return -1;
    DevStats s{};
    if (fail_cuda(cudaMemcpy(&s, d_stats, sizeof(s), cudaMemcpyDeviceToHost), "read stats")) return -1;
    out->attempts = s.attempts;
    out->accepted = s.accepted;
    out->crossings = s.crossings;
    out->rays = s.rays;
    out->horizon = s.horizon;
    out->escaped = s.escaped;
    out->max_steps = s.max_steps;
    out->clamp_evals = s.clamp_evals;
    out->march_steps = s.march_steps;
    out->physics_steps = s.physics_steps;
    out->bin_updates = s.bin_updates;
    out->fp64_attempts = s.fp64_attempts;
    std::memcpy(&out->hamiltonian_max, &s.h_max_bits, sizeof(double));
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, ev0, ev1) == cudaSuccess) out->kernel_ms = ms;
    cudaGetLastError();
    return 0;
}

int GRRTContext::phase_ms(double* out, int cap) {
    if (!device_ready) return 0;
    cudaSetDevice(device);
    if (fail_cuda(cudaEventSynchronize(ev1), "synchronize")) return -1;
    const int n = n_phases > 0 ? n_phases : 1;
    for (int k = 0; k < n && k < cap; ++k) {
        float ms = 0.0f;
        const cudaError_t e = n_phases > 0 ? cudaEventElapsedTime(&ms, ev_phase[k], ev_phase[k + 1])
                                           : cudaEventElapsedTime(&ms, ev0, ev1);
        if (e != cudaSuccess) {
            cudaGetLastError();
            ms = 0.0f;
        }
        out[k] = ms;
    }
    return n;
}

bool GRRTContext::export_table(const std::string& name, std::vector<double>& v) const {
    auto from_ints = [&](const auto& src) { v.assign(src.begin(), src.end()); };
    if (name == "scalars") {
        v = {mass, spin_a, r_horizon, isco, observer_r, tolerance, static_cast<double>(max_steps),
             static_cast<double>(spp)};
        return true;
    }
    if (name == "camera") {
        v.clear();
        for (double x : cam.pos) v.push_back(x);
        for (const double* e : {cam.e0, cam.e1, cam.e2, cam.e3})
            for (int m = 0; m < 4; ++m) v.push_back(e[m]);
        for (int m = 0; m < 4; ++m)
            for (int k = 0; k < 4; ++k) v.push_back(cam.g[m][k]);
        v.push_back(cam.fov);
        v.push_back(cam.width);
        v.push_back(cam.height);
        return true;
    }
    if (name == "spectrum_color") { v = spectrum.color; return true; }
    if (name == "spectrum_lum") { v = spectrum.lum; return true; }
    if (has_disk) {
        if (name == "flux") { v = flux.flux; return true; }
        if (name == "flux_meta") { v = {flux.flux_max, flux.r_inner, flux.r_outer, flux.peak_temperature}; return true; }
    }
    if (has_stars) {
        if (name == "stars") {
            v.clear();
            for (size_t i = 0; i < stars.theta.size(); ++i) {
                v.push_back(stars.theta[i]);
                v.push_back(stars.phi[i]);
                v.push_back(stars.brightness[i]);
            }
            return true;
        }
        if (name == "star_cells") { from_ints(stars.cell_start); return true; }
        if (name == "star_items") { from_ints(stars.cell_items); return true; }
    }
    if (vol) {
        const VolumetricTables& t = *vol;
        if (name == "vol_H") { v = t.H; return true; }
        if (name == "vol_zmax") { v = t.z_max; return true; }
        if (name == "vol_rho_mid") { v = t.rho_mid; return true; }
        if (name == "vol_T_eff") { v = t.T_eff; return true; }
        if (name == "vol_rho_prof") { v = t.rho_profile; return true; }
        if (name == "vol_T_prof") { v = t.T_profile; return true; }
        if (name == "vol_perm") { from_ints(t.perm); return true; }
        if (name == "vol_scalars") {
            v = {t.r_min, t.r_outer, t.r_isco, t.r_horizon, t.rho_scale, t.E_isco, t.L_isco, t.taper_width,
                 t.noise_scale, t.peak_temperature, t.cfg.turbulence, t.M, t.a,
                 static_cast<double>(t.cfg.noise_octaves), static_cast<double>(t.n_r), static_cast<double>(t.n_z)};
            return true;
        }
        const OpacityTables& o = t.opacity;
        if (name == "op_kabs") { v = o.kappa_abs; return true; }
        if (name == "op_kes") { v = o.kappa_es; return true; }
        if (name == "op_kross") { v = o.kappa_ross; return true; }
        if (name == "op_mu") { v = o.mu; return true; }
        if (name == "op_scalars") {
            v = {static_cast<double>(o.n_nu), static_cast<double>(o.n_rho), static_cast<double>(o.n_T), o.log_nu_min,
                 o.log_nu_max, o.log_rho_min, o.log_rho_max, o.log_T_min, o.log_T_max};
            return true;
        }
    }
    return false;
}

int GRRTContext::debug_trace(double x, double y, GRRTDebugRecord* out, int capacity) {
    static_assert(sizeof(GRRTDebugRecord) == sizeof(DevDebugRecord), "debug record layout");
    static_assert(GRRT_DEBUG_START == kDebugStart && GRRT_DEBUG_STEP == kDebugStep &&
                      GRRT_DEBUG_THIN_HIT == kDebugThinHit && GRRT_DEBUG_MARCH_ENTRY == kDebugMarchEntry &&
                      GRRT_DEBUG_MARCH_EXIT == kDebugMarchExit && GRRT_DEBUG_END == kDebugEnd &&
                      GRRT_DEBUG_EVENT_CROSS == kDebugCross && GRRT_DEBUG_EVENT_INSIDE == kDebugInside &&
                      GRRT_DEBUG_EVENT_NEAR == kDebugNear,
                  "debug record codes");
    if (!ensure_device()) return -1;
    const int want = (out && capacity > 0) ? capacity : 1;
    const int cap = std::max(1, std::min(debug_trace_capacity(max_steps), want));
    void* d_buf = nullptr;
    const size_t rec_bytes = sizeof(DevDebugRecord) * static_cast<size_t>(cap);
    if (fail_cuda(cudaMalloc(&d_buf, rec_bytes + sizeof(int)), "cudaMalloc(debug trace)")) return -1;
    auto* d_rec = static_cast<DevDebugRecord*>(d_buf);
    int* d_count = reinterpret_cast<int*>(static_cast<char*>(d_buf) + rec_bytes);
    int n = -1;
    cudaError_t e = launch_debug_trace(scene_for_launch(), x, y, d_rec, cap, d_count, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess) e = cudaMemcpy(&n, d_count, sizeof n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && out && capacity > 0 && n > 0)
        e = cudaMemcpy(out, d_rec, sizeof(DevDebugRecord) * static_cast<size_t>(std::min(n, cap)),
                       cudaMemcpyDeviceToHost);
    cudaFree(d_buf);
    if (fail_cuda(e, "debug trace")) return -1;
    return n;
}

void GRRTContext::debug_pixel(int px, int py) {
    // The pixel centre's FP64 trace on the device, printed in the layout of
    // GeodesicTracer::trace_debug (src/geodesic_tracer.cpp:339-493).
    const int cap = debug_trace_capacity(max_steps);
    std::vector<GRRTDebugRecord> rec(static_cast<size_t>(cap));
    const int n = debug_trace(px + 0.5, py + 0.5, rec.data(), cap);
    std::printf("=== DEBUG PIXEL TRACE ===\n");
    if (n < 1) {
        std::printf("  (device trace failed: %s)\n", error.c_str());
        std::fflush(stdout);
        return;
    }
    const int shown = std::min(n, cap);
    const GRRTDebugRecord& s0 = rec[0];
    std::printf("  r0=%.4f theta0=%.6f phi0=%.4f\n", s0.v[0], s0.v[1], s0.v[2]);
    std::printf("  p0=(%+.4e %+.4e %+.4e %+.4e)\n", s0.v[3], s0.v[4], s0.v[5], s0.v[6]);
    if (vol) std::printf("  disk: r_in=%.3f r_out=%.3f r_isco=%.3f\n", vol->r_horizon, vol->r_outer, vol->r_isco);
    std::printf("%-6s %-10s %-10s %-10s %-12s %-8s %-8s %-6s\n", "step", "r", "theta", "z", "dlambda", "H", "zm",
                "event");
    std::printf("%s %s %s %s %s %s %s %s\n", "------", "----------", "----------", "----------", "------------",
                "--------", "--------", "------");
    static const char* events[] = {"  ", "CROSS", "INSIDE", "NEAR"};
    for (int k = 1; k < shown; ++k) {
        const GRRTDebugRecord& r = rec[k];
        switch (r.kind) {
            case GRRT_DEBUG_STEP:
                if (vol)
                    std::printf("%-6d %-10.4f %-10.6f %-10.4f %-12.4e %-8.4f %-8.4f %s\n", r.step, r.v[0], r.v[1],
                                r.v[2], r.v[3], r.v[4], r.v[5], events[r.event & 3]);
                else
                    std::printf("%-6d %-10.4f %-10.6f %-10.4f %-12.4e %-8s %-8s %s\n", r.step, r.v[0], r.v[1],
                                r.v[2], r.v[3], "-", "-", events[0]);
                break;
            case GRRT_DEBUG_THIN_HIT:
                std::printf("  -> THIN DISK HIT r_cross=%.4f emit=(%.4e %.4e %.4e)\n", r.v[0], r.v[1], r.v[2], r.v[3]);
                break;
            case GRRT_DEBUG_MARCH_ENTRY:
                std::printf("  -> RAYMARCH entry r=%.4f z=%.4f\n", r.v[0], r.v[1]);
                break;
            case GRRT_DEBUG_MARCH_EXIT:
                std::printf("  -> RAYMARCH exit  color=(%.4e %.4e %.4e)\n", r.v[0], r.v[1], r.v[2]);
                break;
            case GRRT_DEBUG_END:
                if (shown < n) std::printf("  ... %d record(s) not shown\n", n - shown);
                if (r.event == 0)
                    std::printf("%-6d %-10.4f  -> HORIZON\n", r.step, r.v[0]);
                else if (r.event == 1)
                    std::printf("%-6d %-10.4f  -> ESCAPED\n", r.step, r.v[0]);
                else
                    std::printf("  -> MAX STEPS  color=(%.4e %.4e %.4e)\n", r.v[3], r.v[4], r.v[5]);
                std::printf("  color=(%.4e %.4e %.4e) after %.0f attempts\n", r.v[3], r.v[4], r.v[5], r.v[6]);
                break;
            default:
                break;
        }
    }
    std::fflush(stdout);
}
