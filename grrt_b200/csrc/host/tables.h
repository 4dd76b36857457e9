// Host-side construction of every table the per-pixel path reads.
//
// Each builder restates the reference's construction with the same floating
// point operations in the same order (compiled with -ffp-contract=off), so the
// tables are bit-identical to the reference's when both use the same libm.
// The tests compare them bitwise against the reference compiled from source.
#pragma once

#include <array>
#include <cstdint>
#include <vector>

namespace grrt_b200 {

// Outer event horizon r+ = M + sqrt(M^2 - a^2)   (src/kerr.cpp:46-50)
double kerr_horizon(double M, double a);
// Prograde ISCO, Bardeen-Press-Teukolsky 1972   (src/kerr.cpp:52-63)
double kerr_isco(double M, double a);

// Static-observer orthonormal tetrad at the camera   (src/camera.cpp:29-63).
struct CameraFrame {
    double pos[4];       // (t, r, theta, phi)
    double e0[4], e1[4], e2[4], e3[4];
    double g[4][4];      // covariant Boyer-Lindquist metric at pos
    double fov;
    int width, height;
};
CameraFrame build_camera(double M, double a, double r_obs, double theta_obs, double phi_obs,
                         double fov, int width, int height);
// Covariant null momentum for a fractional pixel coordinate   (src/camera.cpp:69-96).
void camera_ray(const CameraFrame& cam, double x, double y, double pos[4], double p_cov[4]);
// Covariant metric g_mu_nu in Boyer-Lindquist coordinates   (src/kerr.cpp:19-40).
void kerr_g_lower(double M, double a, const double x[4], double g[4][4]);

// Novikov-Thorne flux table of the thin disk   (src/accretion_disk.cpp:45-94).
struct FluxTable {
    std::vector<double> flux;  // n entries over [r_inner, r_outer]
    double flux_max = 0.0;
    double r_inner = 0.0, r_outer = 0.0;
    double peak_temperature = 0.0;
    double M = 1.0, a = 0.0;
};
FluxTable build_flux_table(double M, double a, double r_inner, double r_outer,
                           double peak_temperature, int n = 500);

// Normalised blackbody chromaticity, CIE 1931 -> linear sRGB   (src/spectrum.cpp:49-96).
struct SpectrumTable {
    std::vector<double> color;  // 3*n, rgb per entry
    std::vector<double> lum;    // n
    double t_min = 1000.0, t_max = 100000.0;
    int n = 1000;
};
SpectrumTable build_spectrum_table(double t_min = 1000.0, double t_max = 100000.0, int n = 1000);

// Power-law star field with a 180x360 bucket grid   (src/celestial_sphere.cpp:9-30).
struct StarCatalogue {
    static constexpr int kGridTheta = 180;
    static constexpr int kGridPhi = 360;
    std::vector<double> theta, phi, brightness;
    std::vector<int> cell_start;  // kGridTheta*kGridPhi + 1 offsets into cell_items
    std::vector<int> cell_items;  // star indices, insertion order within each cell
    double angular_tolerance = 0.003;
};
StarCatalogue build_star_catalogue(int num_stars = 5000, unsigned int seed = 42);

// 512-entry simplex-noise permutation   (src/noise.cpp:23-36).
std::array<int, 512> build_noise_permutation(uint32_t seed);

// Multi-element Saha ionisation and opacity tables   (src/opacity.cpp:16-303).
struct OpacityTables {
    int n_nu = 0, n_rho = 100, n_T = 100;
    double log_nu_min = 0, log_nu_max = 0, log_rho_min = 0, log_rho_max = 0,
           log_T_min = 0, log_T_max = 0;
    std::vector<double> kappa_abs;   // [n_nu][n_rho][n_T]
    std::vector<double> kappa_es;    // [n_rho][n_T]
    std::vector<double> kappa_ross;  // [n_rho][n_T]
    std::vector<double> mu;          // [n_rho][n_T]
    double lookup_kappa_es(double rho, double T) const;
    double lookup_kappa_ross(double rho, double T) const;
    double lookup_mu(double rho, double T) const;
};
OpacityTables build_opacity_tables(double rho_min, double rho_max, double T_min, double T_max,
                                   double nu_min, double nu_max);

// Volumetric Shakura-Sunyaev disk   (src/volumetric_disk.cpp:33-849).
struct VolumetricConfig {
    double alpha = 0.1, turbulence = 0.4, tau_mid = 100.0, noise_scale = 0.0;
    uint32_t seed = 42;
    int noise_octaves = 2;
    double opacity_nu_min = 1e14, opacity_nu_max = 1e16;
};
struct VolumetricTables {
    double M = 1, a = 0, r_outer = 30, peak_temperature = 1e7;
    double r_isco = 0, r_horizon = 0, r_min = 0, taper_width = 0;
    double E_isco = 0, L_isco = 0, rho_scale = 1.0, noise_scale = 1.0;
    int n_r = 500, n_z = 128;
    VolumetricConfig cfg;
    std::vector<double> H, rho_mid, T_eff;       // n_r
    std::vector<double> rho_profile, T_profile;  // n_r * n_z
    std::vector<double> z_max;                   // n_r
    std::array<int, 512> perm{};
    OpacityTables opacity;
};
VolumetricTables build_volumetric_tables(double M, double a, double r_outer,
                                         double peak_temperature, const VolumetricConfig& cfg);

// Peak temperature from mass and Eddington fraction   (src/api.cpp:82-102).
double derived_peak_temperature(double spin, double mass_solar, double eddington_fraction);

}  // namespace grrt_b200
