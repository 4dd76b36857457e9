// Test and baseline harness over the reference library compiled from its own
// sources (oracle/_ref/libgrrt_ref_{strict,fast}.so). It is test
// infrastructure: only tests, smoke() and bench.py's CPU-baseline leg load it.
//
// It builds the reference scene objects exactly the way grrt_create does
// (src/api.cpp:43-173) and exposes plain C entry points that
//   * dump every host-built table (flux LUT, spectrum LUT, star catalogue,
//     noise permutation, volumetric radial/vertical tables, opacity tables),
//   * trace individual camera samples through GeodesicTracer::trace /
//     trace_spectral and return double results,
//   * time the reference's OpenMP render loop on a subset of image rows
//     (the loop body of Renderer::render, src/renderer.cpp:42-79).
#include "grrt/types.h"
#include "grrt/camera/camera.h"
#include "grrt/render/fits_writer.h"
#include "grrt/color/spectrum.h"
#include "grrt/geodesic/geodesic_tracer.h"
#include "grrt/geodesic/rk4.h"
#include "grrt/scene/accretion_disk.h"
#include "grrt/scene/celestial_sphere.h"
#include "grrt/scene/volumetric_disk.h"
#include "grrt/spacetime/kerr.h"

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cstddef>
#include <string>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

namespace {

struct RefScene {
    GRRTParams params{};
    double mass = 1.0, spin_a = 0.0, observer_r = 50.0, tolerance = 1e-8;
    int max_steps = 10000, spp = 1;
    std::unique_ptr<grrt::Kerr> metric;
    std::unique_ptr<grrt::RK4> integrator;
    std::unique_ptr<grrt::Camera> camera;
    std::unique_ptr<grrt::SpectrumLUT> spectrum;
    std::unique_ptr<grrt::AccretionDisk> disk;
    std::unique_ptr<grrt::VolumetricDisk> vol;
    std::unique_ptr<grrt::GeodesicTracer> tracer;
    std::unique_ptr<grrt::CelestialSphere> sphere;
    std::vector<double> freq_bins;
};

// Same arithmetic as the reference's per-sample jitter (src/renderer.cpp:14-20),
// which is file-static there and so cannot be called from outside.
double jitter_hash(int i, int j, int s, int ch) {
    uint32_t h = static_cast<uint32_t>(i * 73856093u ^ j * 19349663u ^ s * 83492791u ^ ch * 45678917u);
    h ^= h >> 16;
    h *= 0x45d9f3bu;
    h ^= h >> 16;
    return (h & 0xFFFFu) / 65536.0;
}

}  // namespace

extern "C" {

void* rh_create(const GRRTParams* p) {
    auto* s = new RefScene{};
    s->params = *p;
    // Defaults exactly as src/api.cpp:47-52.
    s->mass = p->mass > 0.0 ? p->mass : 1.0;
    s->observer_r = p->observer_r > 0.0 ? p->observer_r : 50.0;
    const double observer_theta = p->observer_theta > 0.0 ? p->observer_theta : 1.396;
    const double fov = p->fov > 0.0 ? p->fov : 1.047;
    s->max_steps = p->integrator_max_steps > 0 ? p->integrator_max_steps : 10000;
    s->tolerance = p->integrator_tolerance > 0.0 ? p->integrator_tolerance : 1e-8;
    s->spin_a = 0.0;
    if (p->metric_type == GRRT_METRIC_KERR) {
        const double spin_param = p->spin > 0.0 ? p->spin : 0.998;
        s->spin_a = spin_param * s->mass;
    }
    s->metric = std::make_unique<grrt::Kerr>(s->mass, s->spin_a);
    s->integrator = std::make_unique<grrt::RK4>();
    s->camera = std::make_unique<grrt::Camera>(*s->metric, s->observer_r, observer_theta,
                                               p->observer_phi, fov, p->width, p->height);
    s->spectrum = std::make_unique<grrt::SpectrumLUT>();
    if (p->disk_enabled) {
        const double disk_temp = p->disk_temperature > 0.0 ? p->disk_temperature : 1e7;
        const double disk_outer = p->disk_outer > 0.0 ? p->disk_outer : 20.0;
        const double isco = s->metric->isco_radius();
        const double r_inner = p->disk_inner > 0.0 ? p->disk_inner : isco;
        s->disk = std::make_unique<grrt::AccretionDisk>(s->mass, s->spin_a, r_inner, disk_outer, disk_temp);
        if (p->disk_volumetric) {
            double vol_temp = p->disk_temperature > 0 ? p->disk_temperature : 1e7;
            if (p->mass_solar > 0.0 && p->eddington_fraction > 0.0 && p->disk_temperature <= 0.0) {
                const double a_star = std::abs(p->spin);
                const double Z1 = 1.0 + std::cbrt(1.0 - a_star * a_star)
                                       * (std::cbrt(1.0 + a_star) + std::cbrt(1.0 - a_star));
                const double Z2 = std::sqrt(3.0 * a_star * a_star + Z1 * Z1);
                const double r_isco_M = 3.0 + Z2 - std::sqrt((3.0 - Z1) * (3.0 + Z1 + 2.0 * Z2));
                const double v_isco = 1.0 / std::sqrt(r_isco_M);
                const double E_isco = (1.0 - 2.0 * v_isco * v_isco + a_star * v_isco * v_isco * v_isco)
                                    / std::sqrt(1.0 - 3.0 * v_isco * v_isco + 2.0 * a_star * v_isco * v_isco * v_isco);
                const double eta = 1.0 - E_isco;
                vol_temp = 5.0e7 * std::pow(eta, 0.25) * std::pow(p->mass_solar, -0.25)
                         * std::pow(p->eddington_fraction, 0.25);
            }
            grrt::VolumetricParams vp;
            vp.alpha = p->disk_alpha;
            vp.turbulence = p->disk_turbulence;
            vp.seed = static_cast<uint32_t>(p->disk_seed);
            vp.noise_scale = p->disk_noise_scale;
            vp.noise_octaves = p->disk_noise_octaves;
            if (p->num_frequency_bins > 0 && p->frequency_bins_hz) {
                double lo = p->frequency_bins_hz[0], hi = p->frequency_bins_hz[0];
                for (int i = 1; i < p->num_frequency_bins; ++i) {
                    lo = std::min(lo, p->frequency_bins_hz[i]);
                    hi = std::max(hi, p->frequency_bins_hz[i]);
                }
                vp.opacity_nu_min = lo * 0.1;
                vp.opacity_nu_max = hi * 10.0;
            }
            s->vol = std::make_unique<grrt::VolumetricDisk>(
                p->mass, p->spin, p->disk_outer > 0 ? p->disk_outer : 30.0, vol_temp, vp);
        }
    }
    s->tracer = std::make_unique<grrt::GeodesicTracer>(*s->metric, *s->integrator, s->observer_r,
                                                       s->max_steps, 1000.0, s->tolerance, s->vol.get());
    if (p->background_type == GRRT_BG_STARS) s->sphere = std::make_unique<grrt::CelestialSphere>();
    s->spp = p->samples_per_pixel > 0 ? p->samples_per_pixel : 1;
    return s;
}

void rh_destroy(void* h) { delete static_cast<RefScene*>(h); }

void rh_set_frequency_bins(void* h, const double* f, int n) {
    auto* s = static_cast<RefScene*>(h);
    s->freq_bins.assign(f, f + n);
}

double rh_horizon(void* h) { return static_cast<RefScene*>(h)->metric->horizon_radius(); }
double rh_isco(void* h) { return static_cast<RefScene*>(h)->metric->isco_radius(); }

// Flux LUT: out[n], meta = {flux_max, r_min, r_max, n}.
int rh_flux_lut(void* h, double* out, double* meta) {
    auto* s = static_cast<RefScene*>(h);
    if (!s->disk) return 0;
    const auto& v = s->disk->flux_lut_data();
    if (out) std::memcpy(out, v.data(), v.size() * sizeof(double));
    if (meta) {
        meta[0] = s->disk->flux_max();
        meta[1] = s->disk->flux_r_min();
        meta[2] = s->disk->flux_r_max();
        meta[3] = static_cast<double>(v.size());
    }
    return static_cast<int>(v.size());
}

// Spectrum LUT: color[3*n], lum[n].
int rh_spectrum_lut(void* h, double* color, double* lum) {
    auto* s = static_cast<RefScene*>(h);
    const auto& c = s->spectrum->color_lut_data();
    const auto& l = s->spectrum->luminosity_lut_data();
    for (size_t i = 0; i < c.size(); ++i)
        for (int k = 0; k < 3; ++k) color[3 * i + k] = c[i][k];
    std::memcpy(lum, l.data(), l.size() * sizeof(double));
    return static_cast<int>(c.size());
}

// Star catalogue: out[3*n] = (theta, phi, brightness).
int rh_stars(void* h, double* out) {
    auto* s = static_cast<RefScene*>(h);
    if (!s->sphere) return 0;
    const auto& st = s->sphere->star_data();
    for (size_t i = 0; i < st.size(); ++i) {
        out[3 * i + 0] = st[i].theta;
        out[3 * i + 1] = st[i].phi;
        out[3 * i + 2] = st[i].brightness;
    }
    return static_cast<int>(st.size());
}

// Volumetric tables. sizes = {n_r, n_z, n_nu, n_rho, n_T}.
int rh_vol_sizes(void* h, int* sizes) {
    auto* s = static_cast<RefScene*>(h);
    if (!s->vol) return 0;
    const auto& o = s->vol->opacity_luts();
    sizes[0] = s->vol->radial_bins();
    sizes[1] = s->vol->vertical_bins();
    sizes[2] = o.n_nu;
    sizes[3] = o.n_rho;
    sizes[4] = o.n_T;
    return 1;
}

// scal = {r_min, r_max, r_isco, r_horizon, rho_scale, E_isco, L_isco, taper_width,
//         noise_scale, peak_temperature, turbulence,
//         log_nu_min, log_nu_max, log_rho_min, log_rho_max, log_T_min, log_T_max}
int rh_vol_tables(void* h, double* H, double* rho_mid, double* rho_prof, double* T_prof,
                  double* zmax, double* kabs, double* kes, double* kross, double* mu,
                  int* perm, double* scal) {
    auto* s = static_cast<RefScene*>(h);
    if (!s->vol) return 0;
    const auto& v = *s->vol;
    auto cp = [](double* dst, const std::vector<double>& src) {
        if (dst) std::memcpy(dst, src.data(), src.size() * sizeof(double));
    };
    cp(H, v.scale_height_lut());
    cp(rho_mid, v.rho_mid_lut());
    cp(rho_prof, v.density_profile_lut());
    cp(T_prof, v.temperature_profile_lut());
    cp(zmax, v.z_max_lut());
    const auto& o = v.opacity_luts();
    cp(kabs, o.kappa_abs_lut);
    cp(kes, o.kappa_es_lut);
    cp(kross, o.kappa_ross_lut);
    cp(mu, o.mu_lut);
    if (perm) {
        const auto& p = v.noise().permutation_table();
        for (int i = 0; i < 512; ++i) perm[i] = p[i];
    }
    if (scal) {
        const double vals[] = {v.r_min(), v.r_max(), v.r_isco(), v.r_horizon(), v.rho_scale(),
                               v.E_isco(), v.L_isco(), v.taper_width(), v.noise_scale(),
                               v.peak_temperature(), v.turbulence(),
                               o.log_nu_min, o.log_nu_max, o.log_rho_min, o.log_rho_max,
                               o.log_T_min, o.log_T_max};
        std::memcpy(scal, vals, sizeof(vals));
    }
    return 1;
}

// Initial state of camera samples at fractional pixel coordinates: out[8*n].
void rh_camera_rays(void* h, int n, const double* px, const double* py, double* out) {
    auto* s = static_cast<RefScene*>(h);
    for (int k = 0; k < n; ++k) {
        grrt::GeodesicState st = s->camera->ray_for_pixel(px[k], py[k]);
        for (int m = 0; m < 4; ++m) {
            out[8 * k + m] = st.position[m];
            out[8 * k + 4 + m] = st.momentum[m];
        }
    }
}

// Per-sample RGB traces: rgb[3n] = disk emission (+ star if escaped and stars on),
// term[n] (0 horizon, 1 escaped, 2 max steps), fin[8n] = final x^mu, p_mu.
void rh_trace_rgb(void* h, int n, const double* px, const double* py, double* rgb, int* term,
                  double* fin) {
    auto* s = static_cast<RefScene*>(h);
#pragma omp parallel for schedule(dynamic, 16)
    for (int k = 0; k < n; ++k) {
        grrt::GeodesicState st = s->camera->ray_for_pixel(px[k], py[k]);
        grrt::TraceResult r = s->tracer->trace(st, s->disk.get(), s->spectrum.get());
        grrt::Vec3 c = r.accumulated_color;
        if (r.termination == grrt::RayTermination::Escaped && s->sphere) c += s->sphere->sample(r.final_position);
        for (int m = 0; m < 3; ++m) rgb[3 * k + m] = c[m];
        term[k] = static_cast<int>(r.termination);
        if (fin)
            for (int m = 0; m < 4; ++m) {
                fin[8 * k + m] = r.final_position[m];
                fin[8 * k + 4 + m] = r.final_momentum[m];
            }
    }
}

// Per-sample spectral traces: spec[n*nb], term[n].
void rh_trace_spectral(void* h, int n, const double* px, const double* py, double* spec, int* term) {
    auto* s = static_cast<RefScene*>(h);
    const int nb = static_cast<int>(s->freq_bins.size());
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < n; ++k) {
        grrt::GeodesicState st = s->camera->ray_for_pixel(px[k], py[k]);
        grrt::SpectralTraceResult r = s->tracer->trace_spectral(st, s->freq_bins);
        for (int b = 0; b < nb; ++b) spec[static_cast<size_t>(k) * nb + b] = r.spectral_intensity[b];
        term[k] = static_cast<int>(r.termination);
    }
}

// The reference render loop (Renderer::render body) over rows row0, row0+stride, ...
// of the full image, with the same jitter and spp averaging, into fb (W*H*4, only the
// selected rows written). Returns wall seconds; *threads_used = OpenMP team size.
double rh_render_rows(void* h, int row0, int stride, float* fb, int* threads_used) {
    auto* s = static_cast<RefScene*>(h);
    const int W = s->params.width, H = s->params.height;
    const int grid = std::max(1, static_cast<int>(std::sqrt(static_cast<double>(s->spp))));
    const double inv_spp = 1.0 / (grid * grid);
    const double cell = 1.0 / grid;
    std::vector<int> rows;
    for (int j = row0; j < H; j += stride) rows.push_back(j);
    const int npix = static_cast<int>(rows.size()) * W;
    int team = 1;
    const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel
    {
#pragma omp single
        team = omp_get_num_threads();
#pragma omp for schedule(guided)
        for (int q = 0; q < npix; ++q) {
            const int j = rows[q / W], i = q % W;
            grrt::Vec3 acc;
            for (int sy = 0; sy < grid; ++sy)
                for (int sx = 0; sx < grid; ++sx) {
                    const int smp = sy * grid + sx;
                    const double x = i + (sx + jitter_hash(i, j, smp, 0)) * cell;
                    const double y = j + (sy + jitter_hash(i, j, smp, 1)) * cell;
                    grrt::GeodesicState st = s->camera->ray_for_pixel(x, y);
                    grrt::TraceResult r = s->tracer->trace(st, s->disk.get(), s->spectrum.get());
                    grrt::Vec3 c = r.accumulated_color;
                    if (r.termination == grrt::RayTermination::Escaped && s->sphere)
                        c += s->sphere->sample(r.final_position);
                    acc = acc + c;
                }
            float* o = fb + 4 * (static_cast<size_t>(j) * W + i);
            o[0] = static_cast<float>(acc[0] * inv_spp);
            o[1] = static_cast<float>(acc[1] * inv_spp);
            o[2] = static_cast<float>(acc[2] * inv_spp);
            o[3] = 1.0f;
        }
    }
    const auto t1 = std::chrono::steady_clock::now();
    if (threads_used) *threads_used = team;
    return std::chrono::duration<double>(t1 - t0).count();
}

// Spectral render loop (Renderer::render_spectral body) over selected rows.
double rh_render_spectral_rows(void* h, int row0, int stride, double* out, int* threads_used) {
    auto* s = static_cast<RefScene*>(h);
    const int W = s->params.width, H = s->params.height;
    const int nb = static_cast<int>(s->freq_bins.size());
    const int grid = std::max(1, static_cast<int>(std::sqrt(static_cast<double>(s->spp))));
    const double inv_spp = 1.0 / (grid * grid);
    const double cell = 1.0 / grid;
    std::vector<int> rows;
    for (int j = row0; j < H; j += stride) rows.push_back(j);
    const int npix = static_cast<int>(rows.size()) * W;
    int team = 1;
    const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel
    {
#pragma omp single
        team = omp_get_num_threads();
        std::vector<double> acc(nb);
#pragma omp for schedule(guided)
        for (int q = 0; q < npix; ++q) {
            const int j = rows[q / W], i = q % W;
            std::fill(acc.begin(), acc.end(), 0.0);
            for (int sy = 0; sy < grid; ++sy)
                for (int sx = 0; sx < grid; ++sx) {
                    const int smp = sy * grid + sx;
                    const double x = i + (sx + jitter_hash(i, j, smp, 0)) * cell;
                    const double y = j + (sy + jitter_hash(i, j, smp, 1)) * cell;
                    grrt::GeodesicState st = s->camera->ray_for_pixel(x, y);
                    grrt::SpectralTraceResult r = s->tracer->trace_spectral(st, s->freq_bins);
                    for (int b = 0; b < nb; ++b) acc[b] += r.spectral_intensity[b];
                }
            double* o = out + (static_cast<size_t>(j) * W + i) * nb;
            for (int b = 0; b < nb; ++b) o[b] = acc[b] * inv_spp;
        }
    }
    const auto t1 = std::chrono::steady_clock::now();
    if (threads_used) *threads_used = team;
    return std::chrono::duration<double>(t1 - t0).count();
}

// Writes a cube through the reference's own FITS writer (src/fits_writer.cpp:242-300).
int rh_write_fits(const char* path, const double* data, int W, int H, int nb, const double* freqs,
                  double spin, double mass, double r_obs, double theta_obs, double fov, int spp) {
    grrt::FITSMetadata m;
    m.spin = spin;
    m.mass = mass;
    m.observer_r = r_obs;
    m.observer_theta = theta_obs;
    m.fov = fov;
    m.samples_per_pixel = spp;
    try {
        grrt::write_fits(path, data, W, H, nb, std::vector<double>(freqs, freqs + nb), m);
    } catch (...) {
        return -1;
    }
    return 0;
}

// sizeof(GRRTParams) and offsetof every member, in declaration order, from the
// reference header (include/grrt/types.h). Returns the number of members.
int rh_params_layout(long* out) {
    int k = 0;
    out[k++] = static_cast<long>(sizeof(GRRTParams));
#define OFF(m) out[k++] = static_cast<long>(offsetof(GRRTParams, m))
    OFF(width); OFF(height); OFF(metric_type); OFF(mass); OFF(spin); OFF(observer_r);
    OFF(observer_theta); OFF(observer_phi); OFF(fov); OFF(cam_yaw); OFF(cam_pitch); OFF(cam_roll);
    OFF(disk_enabled); OFF(disk_inner); OFF(disk_outer); OFF(disk_temperature); OFF(disk_volumetric);
    OFF(disk_alpha); OFF(disk_turbulence); OFF(disk_seed); OFF(disk_noise_scale); OFF(disk_noise_octaves);
    OFF(mass_solar); OFF(eddington_fraction); OFF(background_type); OFF(background_texture_path);
    OFF(integrator_tolerance); OFF(integrator_max_steps); OFF(samples_per_pixel); OFF(thread_count);
    OFF(backend); OFF(num_frequency_bins); OFF(frequency_bins_hz);
#undef OFF
    return k - 1;
}

}  // extern "C"
