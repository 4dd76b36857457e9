// Thin-disk scene tables: Kerr radii, camera tetrad, Novikov-Thorne flux,
// blackbody chromaticity, star catalogue and the noise permutation.
//
// Operation order follows the reference expressions term by term so that,
// compiled without FMA contraction, every table is bit-identical to the one
// the reference builds (the tests check this against the reference library).
#include "tables.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <utility>

namespace grrt_b200 {
namespace {

constexpr double kPi = 3.141592653589793;  // the double nearest pi (std::numbers::pi)

// The standard library's min/max/clamp semantics, spelled out so NaN inputs
// propagate the same way they do in the reference.
inline double max_of(double a, double b) { return (a < b) ? b : a; }
inline double min_of(double a, double b) { return (b < a) ? b : a; }

double metric_inner(const double g[4][4], const double u[4], const double v[4]) {
    double sum = 0.0;
    for (int m = 0; m < 4; ++m)
        for (int n = 0; n < 4; ++n) sum += g[m][n] * u[m] * v[n];
    return sum;
}

void normalise(const double g[4][4], const double v[4], double out[4]) {
    const double n2 = metric_inner(g, v, v);
    const double inv = 1.0 / std::sqrt(std::abs(n2));
    for (int m = 0; m < 4; ++m) out[m] = v[m] * inv;
}

// v - e <v,e>/<e,e>
void remove_component(const double g[4][4], const double v[4], const double e[4], double out[4]) {
    const double ve = metric_inner(g, v, e);
    const double ee = metric_inner(g, e, e);
    const double c = ve / ee;
    for (int m = 0; m < 4; ++m) out[m] = v[m] - e[m] * c;
}

}  // namespace

double kerr_horizon(double M, double a) { return M + std::sqrt(M * M - a * a); }

double kerr_isco(double M, double a) {
    const double s = a / M;
    const double z1 = 1.0 + std::cbrt(1.0 - s * s) * (std::cbrt(1.0 + s) + std::cbrt(1.0 - s));
    const double z2 = std::sqrt(3.0 * s * s + z1 * z1);
    return M * (3.0 + z2 - std::sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2)));
}

void kerr_g_lower(double M, double a, const double x[4], double g[4][4]) {
    const double r = x[1];
    const double th = x[2];
    const double s = std::sin(th);
    const double s2 = max_of(s * s, 1e-20);
    const double c = std::cos(th);
    const double sig = max_of(r * r + a * a * c * c, 1e-20);
    const double del = r * r - 2.0 * M * r + a * a;
    for (int m = 0; m < 4; ++m)
        for (int n = 0; n < 4; ++n) g[m][n] = 0.0;
    g[0][0] = -(1.0 - 2.0 * M * r / sig);
    g[0][3] = -2.0 * M * a * r * s2 / sig;
    g[3][0] = g[0][3];
    g[1][1] = sig / del;
    g[2][2] = sig;
    g[3][3] = (r * r + a * a + 2.0 * M * a * a * r * s2 / sig) * s2;
}

CameraFrame build_camera(double M, double a, double r_obs, double theta_obs, double phi_obs,
                         double fov, int width, int height) {
    CameraFrame cam{};
    cam.pos[0] = 0.0;
    cam.pos[1] = r_obs;
    cam.pos[2] = theta_obs;
    cam.pos[3] = phi_obs;
    cam.fov = fov;
    cam.width = width;
    cam.height = height;
    kerr_g_lower(M, a, cam.pos, cam.g);
    const auto& g = cam.g;

    // Static observer: u = (1/sqrt(-g_tt), 0, 0, 0).
    cam.e0[0] = 1.0 / std::sqrt(-g[0][0]);
    cam.e0[1] = cam.e0[2] = cam.e0[3] = 0.0;

    // Forward: radially inward; up: towards the pole (-theta); right: +phi.
    const double inward[4] = {0.0, -1.0, 0.0, 0.0};
    const double upward[4] = {0.0, 0.0, -1.0, 0.0};
    const double rightward[4] = {0.0, 0.0, 0.0, 1.0};
    double t1[4], t2[4], t3[4];

    remove_component(g, inward, cam.e0, t1);
    normalise(g, t1, cam.e3);

    remove_component(g, upward, cam.e0, t1);
    remove_component(g, t1, cam.e3, t2);
    normalise(g, t2, cam.e2);

    remove_component(g, rightward, cam.e0, t1);
    remove_component(g, t1, cam.e3, t2);
    remove_component(g, t2, cam.e2, t3);
    normalise(g, t3, cam.e1);
    return cam;
}

void camera_ray(const CameraFrame& cam, double x, double y, double pos[4], double p_cov[4]) {
    const double alpha = (x - cam.width / 2.0) * cam.fov / cam.width;
    const double beta = (y - cam.height / 2.0) * cam.fov / cam.width;  // both over width
    const double ca = std::cos(beta) * std::sin(alpha);
    const double cb = std::sin(beta);
    const double cc = std::cos(beta) * std::cos(alpha);
    double p_up[4];
    for (int m = 0; m < 4; ++m) {
        const double d = -ca * cam.e1[m] - cb * cam.e2[m] + cc * cam.e3[m];
        p_up[m] = -cam.e0[m] + d;
    }
    for (int m = 0; m < 4; ++m) {
        double sum = 0.0;
        for (int n = 0; n < 4; ++n) sum += cam.g[m][n] * p_up[n];
        p_cov[m] = sum;
        pos[m] = cam.pos[m];
    }
}

// ---------------------------------------------------------------------------
// Novikov-Thorne flux
// ---------------------------------------------------------------------------
namespace {
struct CircularOrbit {
    double M, a;
    double kepler(double r) const { return std::sqrt(M / (r * r * r)); }
    double omega(double r) const {
        const double w = kepler(r);
        return w / (1.0 + a * w);
    }
    double energy(double r) const {
        const double aw = a * kepler(r);
        return (1.0 - 2.0 * M / r + aw) / std::sqrt(1.0 - 3.0 * M / r + 2.0 * aw);
    }
    double ang_mom(double r) const {
        const double aw = a * kepler(r);
        return std::sqrt(M * r) * (1.0 - 2.0 * aw + a * a / (r * r))
               / std::sqrt(1.0 - 3.0 * M / r + 2.0 * aw);
    }
};
}  // namespace

FluxTable build_flux_table(double M, double a, double r_inner, double r_outer,
                           double peak_temperature, int n) {
    FluxTable t;
    t.M = M;
    t.a = a;
    t.r_inner = r_inner;
    t.r_outer = r_outer;
    t.peak_temperature = peak_temperature;
    t.flux.assign(n, 0.0);
    const CircularOrbit orb{M, a};
    const double e_in = orb.energy(r_inner);
    const double l_in = orb.ang_mom(r_inner);
    constexpr double h = 1e-6;  // central-difference step
    double integral = 0.0;
    double last = 0.0;
    t.flux_max = 0.0;
    for (int i = 1; i < n; ++i) {
        const double r = r_inner + (r_outer - r_inner) * i / (n - 1);
        const double de = (orb.energy(r + h) - orb.energy(r - h)) / (2.0 * h);
        const double dl = (orb.ang_mom(r + h) - orb.ang_mom(r - h)) / (2.0 * h);
        const double f = (orb.energy(r) - e_in) * dl - (orb.ang_mom(r) - l_in) * de;
        const double dr = (r_outer - r_inner) / (n - 1);
        integral += 0.5 * (last + f) * dr;
        last = f;
        const double om = orb.omega(r);
        const double e_r = orb.energy(r);
        const double l_r = orb.ang_mom(r);
        const double dom = (orb.omega(r + h) - orb.omega(r - h)) / (2.0 * h);
        const double den = e_r - om * l_r;
        if (std::abs(den) < 1e-20) {
            t.flux[i] = 0.0;
            continue;
        }
        const double F = (3.0 * M / (8.0 * kPi * r * r * r)) * (1.0 / den) * (-dom) * integral;
        t.flux[i] = max_of(F, 0.0);
        if (t.flux[i] > t.flux_max) t.flux_max = t.flux[i];
    }
    return t;
}

// ---------------------------------------------------------------------------
// Blackbody chromaticity
// ---------------------------------------------------------------------------
namespace {
// CIE 1931 2-degree colour matching functions, 380-780 nm at 5 nm, rounded to
// four decimals (the same tabulation the reference integrates against).
constexpr double kCieX[81] = {
    0.0014, 0.0022, 0.0042, 0.0076, 0.0143, 0.0232, 0.0435, 0.0776, 0.1344, 0.2148,
    0.2839, 0.3285, 0.3483, 0.3481, 0.3362, 0.3187, 0.2908, 0.2511, 0.1954, 0.1421,
    0.0956, 0.0580, 0.0320, 0.0147, 0.0049, 0.0024, 0.0093, 0.0291, 0.0633, 0.1096,
    0.1655, 0.2257, 0.2904, 0.3597, 0.4334, 0.5121, 0.5945, 0.6784, 0.7621, 0.8425,
    0.9163, 0.9786, 1.0263, 1.0567, 1.0622, 1.0456, 1.0026, 0.9384, 0.8544, 0.7514,
    0.6424, 0.5419, 0.4479, 0.3608, 0.2835, 0.2187, 0.1649, 0.1212, 0.0874, 0.0636,
    0.0468, 0.0329, 0.0227, 0.0158, 0.0114, 0.0081, 0.0058, 0.0041, 0.0029, 0.0020,
    0.0014, 0.0010, 0.0007, 0.0005, 0.0003, 0.0002, 0.0002, 0.0001, 0.0001, 0.0001,
    0.0000};
constexpr double kCieY[81] = {
    0.0000, 0.0001, 0.0001, 0.0002, 0.0004, 0.0006, 0.0012, 0.0022, 0.0040, 0.0073,
    0.0116, 0.0168, 0.0230, 0.0298, 0.0380, 0.0480, 0.0600, 0.0739, 0.0910, 0.1126,
    0.1390, 0.1693, 0.2080, 0.2586, 0.3230, 0.4073, 0.5030, 0.6082, 0.7100, 0.7932,
    0.8620, 0.9149, 0.9540, 0.9803, 0.9950, 1.0002, 0.9950, 0.9786, 0.9520, 0.9154,
    0.8700, 0.8163, 0.7570, 0.6949, 0.6310, 0.5668, 0.5030, 0.4412, 0.3810, 0.3210,
    0.2650, 0.2170, 0.1750, 0.1382, 0.1070, 0.0816, 0.0610, 0.0446, 0.0320, 0.0232,
    0.0170, 0.0119, 0.0082, 0.0057, 0.0041, 0.0029, 0.0021, 0.0015, 0.0010, 0.0007,
    0.0005, 0.0004, 0.0002, 0.0002, 0.0001, 0.0001, 0.0001, 0.0000, 0.0000, 0.0000,
    0.0000};
constexpr double kCieZ[81] = {
    0.0065, 0.0105, 0.0201, 0.0362, 0.0679, 0.1102, 0.2074, 0.3713, 0.6456, 1.0391,
    1.3856, 1.6230, 1.7471, 1.7826, 1.7721, 1.7441, 1.6692, 1.5281, 1.2876, 1.0419,
    0.8130, 0.6162, 0.4652, 0.3533, 0.2720, 0.2123, 0.1582, 0.1117, 0.0782, 0.0573,
    0.0422, 0.0298, 0.0203, 0.0134, 0.0087, 0.0057, 0.0039, 0.0027, 0.0021, 0.0018,
    0.0017, 0.0014, 0.0011, 0.0010, 0.0008, 0.0006, 0.0003, 0.0002, 0.0002, 0.0001,
    0.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000,
    0.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000,
    0.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000, 0.0000,
    0.0000};

// SI constants of the visible-band Planck law.
constexpr double kH = 6.62607015e-34;
constexpr double kC = 2.99792458e8;
constexpr double kK = 1.380649e-23;
constexpr double kSigma = 5.670374419e-8;

double planck_lambda(double lam, double T) {
    const double x = kH * kC / (lam * kK * T);
    if (x > 500.0) return 0.0;
    return (2.0 * kH * kC * kC) / (lam * lam * lam * lam * lam * (std::exp(x) - 1.0));
}
}  // namespace

SpectrumTable build_spectrum_table(double t_min, double t_max, int n) {
    SpectrumTable s;
    s.t_min = t_min;
    s.t_max = t_max;
    s.n = n;
    s.color.assign(3 * static_cast<size_t>(n), 0.0);
    s.lum.assign(n, 0.0);
    const double lum_top = kSigma * t_max * t_max * t_max * t_max;
    for (int i = 0; i < n; ++i) {
        const double T = t_min + (t_max - t_min) * i / (n - 1);
        double X = 0.0, Y = 0.0, Z = 0.0;
        for (int k = 0; k < 81; ++k) {
            const double lam = 380e-9 + k * 5e-9;
            const double B = planck_lambda(lam, T);
            X += B * kCieX[k] * 5e-9;
            Y += B * kCieY[k] * 5e-9;
            Z += B * kCieZ[k] * 5e-9;
        }
        double rgb[3] = {3.2406 * X - 1.5372 * Y - 0.4986 * Z,
                         -0.9689 * X + 1.8758 * Y + 0.0415 * Z,
                         0.0557 * X - 0.2040 * Y + 1.0570 * Z};
        for (double& v : rgb) v = max_of(v, 0.0);
        const double top = std::fmax(rgb[0], std::fmax(rgb[1], rgb[2]));
        if (top > 0.0) {
            const double inv = 1.0 / top;
            for (double& v : rgb) v = v * inv;
        }
        for (int k = 0; k < 3; ++k) s.color[3 * static_cast<size_t>(i) + k] = rgb[k];
        s.lum[i] = (kSigma * T * T * T * T) / lum_top;
    }
    return s;
}

// ---------------------------------------------------------------------------
// Stars
// ---------------------------------------------------------------------------
StarCatalogue build_star_catalogue(int num_stars, unsigned int seed) {
    StarCatalogue c;
    std::mt19937 gen(seed);
    std::uniform_real_distribution<double> unit(0.0, 1.0);
    c.theta.resize(num_stars);
    c.phi.resize(num_stars);
    c.brightness.resize(num_stars);
    for (int i = 0; i < num_stars; ++i) {
        // Three draws per star, in this order: polar angle, azimuth, brightness.
        const double u_theta = unit(gen);
        c.theta[i] = std::acos(1.0 - 2.0 * u_theta);
        const double u_phi = unit(gen);
        c.phi[i] = 2.0 * kPi * u_phi - kPi;
        const double u_b = unit(gen);
        const double b = 0.1 * std::pow(max_of(u_b, 0.001), -2.5);
        c.brightness[i] = min_of(b, 50.0);
    }
    constexpr int nt = StarCatalogue::kGridTheta, np = StarCatalogue::kGridPhi;
    std::vector<int> cell_of(num_stars);
    std::vector<int> count(nt * np, 0);
    for (int i = 0; i < num_stars; ++i) {
        int tb = static_cast<int>(c.theta[i] * nt / kPi);
        int pb = static_cast<int>((c.phi[i] + kPi) * np / (2.0 * kPi));
        tb = std::clamp(tb, 0, nt - 1);
        pb = std::clamp(pb, 0, np - 1);
        cell_of[i] = tb * np + pb;
        ++count[cell_of[i]];
    }
    c.cell_start.assign(nt * np + 1, 0);
    for (int k = 0; k < nt * np; ++k) c.cell_start[k + 1] = c.cell_start[k] + count[k];
    c.cell_items.assign(num_stars, 0);
    std::vector<int> fill(c.cell_start.begin(), c.cell_start.end() - 1);
    for (int i = 0; i < num_stars; ++i) c.cell_items[fill[cell_of[i]]++] = i;
    return c;
}

// ---------------------------------------------------------------------------
// Noise permutation: Fisher-Yates over 0..255 driven by mt19937(seed).
// ---------------------------------------------------------------------------
std::array<int, 512> build_noise_permutation(uint32_t seed) {
    std::array<int, 256> p{};
    std::iota(p.begin(), p.end(), 0);
    std::mt19937 gen(seed);
    for (int i = 255; i > 0; --i) {
        std::uniform_int_distribution<int> pick(0, i);
        const int j = pick(gen);
        std::swap(p[i], p[j]);
    }
    std::array<int, 512> out{};
    for (int i = 0; i < 256; ++i) out[i] = out[i + 256] = p[i];
    return out;
}

double derived_peak_temperature(double spin, double mass_solar, double eddington_fraction) {
    const double s = std::abs(spin);
    const double z1 = 1.0 + std::cbrt(1.0 - s * s) * (std::cbrt(1.0 + s) + std::cbrt(1.0 - s));
    const double z2 = std::sqrt(3.0 * s * s + z1 * z1);
    const double r_isco = 3.0 + z2 - std::sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2));
    const double v = 1.0 / std::sqrt(r_isco);
    const double e_isco = (1.0 - 2.0 * v * v + s * v * v * v)
                          / std::sqrt(1.0 - 3.0 * v * v + 2.0 * s * v * v * v);
    const double eta = 1.0 - e_isco;
    return 5.0e7 * std::pow(eta, 0.25) * std::pow(mass_solar, -0.25)
           * std::pow(eddington_fraction, 0.25);
}

}  // namespace grrt_b200
