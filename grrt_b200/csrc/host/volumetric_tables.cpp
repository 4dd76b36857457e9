// Volumetric disk tables: multi-element Saha ionisation, frequency-dependent
// opacity tables, the Shakura-Sunyaev radial structure, the flux-limited
// hydrostatic vertical profiles and the density normalisation.
//
// Restates src/opacity.cpp:12-363, include/grrt/color/atomic_data.h and
// src/volumetric_disk.cpp:16-849 with identical floating-point operation order,
// so every table is bit-identical to the reference's. Independent table cells
// (each (rho, T) node, each radius) are built in parallel with OpenMP; a cell's
// arithmetic does not depend on the schedule.
#include "tables.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

namespace grrt_b200 {
namespace {

constexpr double kPi = 3.141592653589793;

// CGS constants (include/grrt/math/constants.h values).
constexpr double kB = 1.380649e-16;
constexpr double kSigmaSB = 5.670374e-5;
constexpr double kMp = 1.672622e-24;
constexpr double kMe = 9.10938e-28;
constexpr double kC = 2.997924e10;
constexpr double kHp = 6.626070e-27;
constexpr double kSigmaT = 6.652e-25;
constexpr double kEv = 1.602e-12;
constexpr double kGammaE = 1.7811;
constexpr double kCff = 3.69e8;
constexpr double kArad = 4.0 * kSigmaSB / kC;
constexpr double kXH = 0.70;

inline double max_of(double a, double b) { return (a < b) ? b : a; }
inline double min_of(double a, double b) { return (b < a) ? b : a; }
inline double clamp_of(double v, double lo, double hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

// Five tracked elements, up to five ionisation stages each: mass fraction,
// atomic mass (m_p), stage count, ionisation potentials (eV), ground-state
// statistical weights, Kramers effective charge, outer-shell quantum number.
constexpr int kStages = 5;
constexpr int kElements = 5;
struct Species {
    double mass_fraction, atomic_mass;
    int stages;
    double chi_eV[kStages], g0[kStages], z_eff[kStages];
    int n_outer[kStages];
};
constexpr Species kSpecies[kElements] = {
    {0.70, 1.0, 2, {13.60, 0, 0, 0, 0}, {2.0, 1.0, 0, 0, 0}, {1.0, 0, 0, 0, 0}, {1, 0, 0, 0, 0}},
    {0.28, 4.0, 3, {24.59, 54.42, 0, 0, 0}, {1.0, 2.0, 1.0, 0, 0}, {1.0, 2.0, 0, 0, 0}, {1, 1, 0, 0, 0}},
    {3.0e-3, 12.0, 5, {11.26, 24.38, 47.89, 64.49, 0}, {9.0, 6.0, 1.0, 6.0, 9.0},
     {1.0, 1.5, 2.0, 2.5, 0}, {2, 2, 2, 2, 0}},
    {6.6e-3, 16.0, 5, {13.62, 35.12, 54.93, 77.41, 0}, {9.0, 4.0, 9.0, 4.0, 1.0},
     {1.0, 1.5, 2.0, 2.5, 0}, {2, 2, 2, 2, 0}},
    {1.2e-3, 56.0, 5, {7.90, 16.19, 30.65, 54.80, 0}, {25.0, 30.0, 25.0, 28.0, 25.0},
     {1.0, 1.5, 2.0, 2.5, 0}, {4, 4, 3, 3, 0}},
};
constexpr double kChiHminus = 0.754 * 1.602e-12;  // H- electron affinity, erg

// H- bound-free cross-section (Wishart 1979): wavelength nm -> cm^2.
constexpr int kBfN = 16;
constexpr double kBfLambda[kBfN] = {200, 300, 400, 450, 500, 550, 600, 650,
                                    700, 750, 800, 850, 900, 1000, 1200, 1642};
constexpr double kBfSigma[kBfN] = {0.36e-17, 1.06e-17, 1.63e-17, 2.33e-17, 3.02e-17, 3.58e-17,
                                   3.96e-17, 4.14e-17, 4.09e-17, 3.98e-17, 3.93e-17, 3.98e-17,
                                   3.85e-17, 3.40e-17, 2.23e-17, 0.0};
// H- free-free cross-section (Bell & Berrington 1987): [T][lambda], cm^5.
constexpr int kFfT = 8, kFfL = 7;
constexpr double kFfTemps[kFfT] = {2000, 3000, 4000, 5000, 6000, 7000, 8000, 10000};
constexpr double kFfLambda[kFfL] = {400, 500, 600, 700, 800, 900, 1000};
constexpr double kFfSigma[kFfT * kFfL] = {
    2.21e-39, 3.44e-39, 4.91e-39, 6.61e-39, 8.55e-39, 1.07e-38, 1.31e-38,
    3.30e-39, 5.15e-39, 7.35e-39, 9.90e-39, 1.28e-38, 1.60e-38, 1.96e-38,
    4.39e-39, 6.86e-39, 9.79e-39, 1.32e-38, 1.70e-38, 2.13e-38, 2.61e-38,
    5.48e-39, 8.56e-39, 1.22e-38, 1.65e-38, 2.13e-38, 2.67e-38, 3.27e-38,
    6.57e-39, 1.03e-38, 1.47e-38, 1.98e-38, 2.56e-38, 3.20e-38, 3.92e-38,
    7.66e-39, 1.20e-38, 1.71e-38, 2.30e-38, 2.98e-38, 3.73e-38, 4.57e-38,
    8.76e-39, 1.37e-38, 1.95e-38, 2.63e-38, 3.41e-38, 4.27e-38, 5.22e-38,
    1.09e-38, 1.71e-38, 2.44e-38, 3.29e-38, 4.26e-38, 5.33e-38, 6.53e-38,
};

struct Ionisation {
    double n_e = 0, mu = 0, n_ion_eff = 0, n_HI = 0, n_Hminus = 0;
    double pop[kElements][kStages] = {};
};

Ionisation saha(double rho, double T) {
    Ionisation out;
    if (T < 100.0 || rho <= 0.0) {
        out.mu = 1.3;
        for (int s = 0; s < kElements; ++s) {
            const double n = rho * kSpecies[s].mass_fraction / (kSpecies[s].atomic_mass * kMp);
            out.pop[s][0] = n;
            if (s == 0) out.n_HI = n;
        }
        return out;
    }
    const double ldb = kHp / std::sqrt(2.0 * kPi * kMe * kB * T);
    const double ldb3 = ldb * ldb * ldb;
    const double pref = 2.0 / ldb3;
    double n_tot[kElements];
    for (int s = 0; s < kElements; ++s)
        n_tot[s] = rho * kSpecies[s].mass_fraction / (kSpecies[s].atomic_mass * kMp);
    double n_e = rho * (1.0 + kXH) / (2.0 * kMp);
    for (int it = 0; it < 50; ++it) {
        double n_e_next = 0.0;
        for (int s = 0; s < kElements; ++s) {
            const Species& sp = kSpecies[s];
            double ratio[kStages] = {};
            for (int i = 0; i < sp.stages - 1; ++i) {
                const double chi = sp.chi_eV[i] * kEv;
                ratio[i] = (pref / n_e) * (sp.g0[i + 1] / sp.g0[i]) * std::exp(-chi / (kB * T));
            }
            double denom = 1.0, prod = 1.0;
            for (int i = 0; i < sp.stages - 1; ++i) {
                prod *= ratio[i];
                denom += prod;
            }
            const double f0 = 1.0 / denom;
            out.pop[s][0] = f0 * n_tot[s];
            prod = f0;
            for (int i = 0; i < sp.stages - 1; ++i) {
                prod *= ratio[i];
                out.pop[s][i + 1] = prod * n_tot[s];
            }
            for (int i = 1; i < sp.stages; ++i) n_e_next += i * out.pop[s][i];
        }
        const double change = std::abs(n_e_next - n_e) / max_of(n_e, 1e-30);
        n_e = n_e_next;
        if (change < 1e-6) break;
    }
    out.n_e = n_e;
    out.n_HI = out.pop[0][0];
    out.n_ion_eff = 0.0;
    for (int s = 0; s < kElements; ++s)
        for (int i = 1; i < kSpecies[s].stages; ++i)
            out.n_ion_eff += static_cast<double>(i * i) * out.pop[s][i];
    double n_part = n_e;
    for (int s = 0; s < kElements; ++s)
        for (int i = 0; i < kSpecies[s].stages; ++i) n_part += out.pop[s][i];
    out.mu = rho / (n_part * kMp);
    const double hm = n_e * ldb3 * 0.25 * std::exp(kChiHminus / (kB * T));
    out.n_Hminus = out.n_HI * hm;
    return out;
}

double gaunt_ff(double nu, double T) {
    const double arg = 4.0 * kB * T / (kGammaE * kHp * nu);
    const double g = (std::sqrt(3.0) / kPi) * std::log(max_of(arg, 1.0));
    return max_of(g, 1.0);
}

double alpha_ff(double nu, double T, const Ionisation& ion) {
    if (ion.n_e <= 0.0 || ion.n_ion_eff <= 0.0 || nu <= 0.0 || T <= 0.0) return 0.0;
    const double g = gaunt_ff(nu, T);
    const double stim = 1.0 - std::exp(-kHp * nu / (kB * T));
    return kCff * (ion.n_e * ion.n_ion_eff / (nu * nu * nu)) * g * std::pow(T, -0.5) * stim;
}

double hminus_bf_sigma(double lambda_cm) {
    const double nm = lambda_cm * 1e7;
    if (nm >= kBfLambda[kBfN - 1] || nm <= 0.0) return 0.0;
    if (nm <= kBfLambda[0]) return kBfSigma[0];
    for (int i = 0; i < kBfN - 1; ++i) {
        if (nm >= kBfLambda[i] && nm <= kBfLambda[i + 1]) {
            const double f = (nm - kBfLambda[i]) / (kBfLambda[i + 1] - kBfLambda[i]);
            return kBfSigma[i] + f * (kBfSigma[i + 1] - kBfSigma[i]);
        }
    }
    return 0.0;
}

double hminus_ff_sigma(double lambda_cm, double T) {
    const double nm = lambda_cm * 1e7;
    const double lc = clamp_of(nm, kFfLambda[0], kFfLambda[kFfL - 1]);
    const double tc = clamp_of(T, kFfTemps[0], kFfTemps[kFfT - 1]);
    int il = 0;
    for (int i = 0; i < kFfL - 1; ++i)
        if (lc >= kFfLambda[i]) il = i;
    const int il1 = std::min(il + 1, kFfL - 1);
    const double fl = (il == il1) ? 0.0 : (lc - kFfLambda[il]) / (kFfLambda[il1] - kFfLambda[il]);
    int it = 0;
    for (int i = 0; i < kFfT - 1; ++i)
        if (tc >= kFfTemps[i]) it = i;
    const int it1 = std::min(it + 1, kFfT - 1);
    const double ft = (it == it1) ? 0.0 : (tc - kFfTemps[it]) / (kFfTemps[it1] - kFfTemps[it]);
    const double s00 = kFfSigma[it * kFfL + il], s01 = kFfSigma[it * kFfL + il1];
    const double s10 = kFfSigma[it1 * kFfL + il], s11 = kFfSigma[it1 * kFfL + il1];
    return s00 * (1 - fl) * (1 - ft) + s01 * fl * (1 - ft) + s10 * (1 - fl) * ft + s11 * fl * ft;
}

double alpha_hminus(double nu, double T, const Ionisation& ion) {
    if (T < 1500.0 || ion.n_HI <= 0.0) return 0.0;
    const double lam = kC / nu;
    const double stim = 1.0 - std::exp(-kHp * nu / (kB * T));
    const double bf = ion.n_Hminus * hminus_bf_sigma(lam) * stim;
    const double ff = ion.n_HI * ion.n_e * hminus_ff_sigma(lam, T);
    return bf + ff;
}

double alpha_bf_ions(double nu, double T, const Ionisation& ion) {
    const double stim = 1.0 - std::exp(-kHp * nu / (kB * T));
    double total = 0.0;
    for (int s = 0; s < kElements; ++s) {
        const Species& sp = kSpecies[s];
        for (int i = 0; i < sp.stages - 1; ++i) {
            if (sp.z_eff[i] <= 0.0 || sp.n_outer[i] <= 0) continue;
            const double chi = sp.chi_eV[i] * kEv;
            const double nu_th = chi / kHp;
            if (nu < nu_th) continue;
            const double n = static_cast<double>(sp.n_outer[i]);
            const double z = sp.z_eff[i];
            const double s0 = 7.91e-18 * n / (z * z);
            const double sigma = s0 * std::pow(nu_th / nu, 3.0);
            total += ion.pop[s][i] * sigma * stim;
        }
    }
    return total;
}

double kappa_es_of(double rho, const Ionisation& ion) {
    if (rho <= 0.0) return 0.0;
    return kSigmaT * ion.n_e / rho;
}

double kappa_abs_of(double nu, double rho, double T, const Ionisation& ion) {
    const double a = alpha_ff(nu, T, ion) + alpha_hminus(nu, T, ion) + alpha_bf_ions(nu, T, ion);
    if (rho <= 0.0) return 0.0;
    return a / rho;
}

double dplanck_dT(double nu, double T) {
    const double x = kHp * nu / (kB * T);
    if (x > 500.0) return 0.0;
    const double ex = std::exp(x);
    const double den = (ex - 1.0) * (ex - 1.0);
    return (2.0 * kHp * kHp * nu * nu * nu * nu / (kC * kC * kB * T * T)) * ex / den;
}

void grid_locate(double v, double lo, double hi, int n, int& idx, double& frac) {
    double t = (v - lo) / (hi - lo) * (n - 1);
    t = clamp_of(t, 0.0, static_cast<double>(n - 2));
    idx = static_cast<int>(t);
    frac = t - idx;
}

double bilinear(const std::vector<double>& lut, const OpacityTables& o, double rho, double T) {
    int ir, iT;
    double fr, fT;
    grid_locate(std::log10(rho), o.log_rho_min, o.log_rho_max, o.n_rho, ir, fr);
    grid_locate(std::log10(T), o.log_T_min, o.log_T_max, o.n_T, iT, fT);
    const double v00 = lut[ir * o.n_T + iT], v01 = lut[ir * o.n_T + iT + 1];
    const double v10 = lut[(ir + 1) * o.n_T + iT], v11 = lut[(ir + 1) * o.n_T + iT + 1];
    return v00 * (1 - fr) * (1 - fT) + v01 * (1 - fr) * fT + v10 * fr * (1 - fT) + v11 * fr * fT;
}

}  // namespace

double OpacityTables::lookup_kappa_es(double rho, double T) const { return bilinear(kappa_es, *this, rho, T); }
double OpacityTables::lookup_kappa_ross(double rho, double T) const { return bilinear(kappa_ross, *this, rho, T); }
double OpacityTables::lookup_mu(double rho, double T) const { return bilinear(mu, *this, rho, T); }

OpacityTables build_opacity_tables(double rho_min, double rho_max, double T_min, double T_max,
                                   double nu_min, double nu_max) {
    OpacityTables o;
    const double decades = std::log10(nu_max) - std::log10(nu_min);
    o.n_nu = std::max(20, static_cast<int>(decades * 10));
    o.n_rho = 100;
    o.n_T = 100;
    o.log_nu_min = std::log10(nu_min);
    o.log_nu_max = std::log10(nu_max);
    o.log_rho_min = std::log10(rho_min);
    o.log_rho_max = std::log10(rho_max);
    o.log_T_min = std::log10(T_min);
    o.log_T_max = std::log10(T_max);
    const size_t n2 = static_cast<size_t>(o.n_rho) * o.n_T;
    o.kappa_abs.assign(n2 * o.n_nu, 0.0);
    o.kappa_es.assign(n2, 0.0);
    o.kappa_ross.assign(n2, 0.0);
    o.mu.assign(n2, 0.0);

    constexpr int n_ross = 50;
    const double lr_min = std::log10(1e13);
    const double lr_max = std::log10(1e16);

#pragma omp parallel for schedule(dynamic, 4) collapse(2)
    for (int j = 0; j < o.n_rho; ++j) {
        for (int k = 0; k < o.n_T; ++k) {
            const double log_rho = o.log_rho_min + j * (o.log_rho_max - o.log_rho_min) / (o.n_rho - 1);
            const double rho = std::pow(10.0, log_rho);
            const double log_T = o.log_T_min + k * (o.log_T_max - o.log_T_min) / (o.n_T - 1);
            const double T = std::pow(10.0, log_T);
            const Ionisation ion = saha(rho, T);
            const size_t c2 = static_cast<size_t>(j) * o.n_T + k;
            o.kappa_es[c2] = kappa_es_of(rho, ion);
            o.mu[c2] = ion.mu;
            for (int i = 0; i < o.n_nu; ++i) {
                const double log_nu = o.log_nu_min + i * (o.log_nu_max - o.log_nu_min) / (o.n_nu - 1);
                const double nu = std::pow(10.0, log_nu);
                o.kappa_abs[static_cast<size_t>(i) * n2 + c2] = kappa_abs_of(nu, rho, T, ion);
            }
            double num = 0.0, den = 0.0;
            for (int i = 0; i < n_ross; ++i) {
                const double log_nu = lr_min + i * (lr_max - lr_min) / (n_ross - 1);
                const double nu = std::pow(10.0, log_nu);
                const double dnu = nu * (lr_max - lr_min) / (n_ross - 1) * std::log(10.0);
                const double dB = dplanck_dT(nu, T);
                const double ka = kappa_abs_of(nu, rho, T, ion);
                if (ka > 1e-30 && dB > 0.0) num += (1.0 / ka) * dB * dnu;
                den += dB * dnu;
            }
            o.kappa_ross[c2] = (num > 0.0 && den > 0.0) ? den / num : 0.0;
        }
    }
    return o;
}

// ---------------------------------------------------------------------------
// Volumetric disk
// ---------------------------------------------------------------------------
namespace {

struct KerrOrbit {
    double M, a;
    // Prograde orbital frequency sqrt(M)/(r^1.5 + a sqrt(M))   (volumetric_disk.cpp:79-82)
    double omega(double r) const { return std::sqrt(M) / (r * std::sqrt(r) + a * std::sqrt(M)); }
    // Vertical epicyclic frequency squared   (volumetric_disk.cpp:84-91)
    double omega_z_sq(double r) const {
        const double w = omega(r);
        const double sm = std::sqrt(M);
        const double r3 = r * r * r;
        return w * w * (1.0 - 4.0 * a * sm / std::sqrt(r3) + 3.0 * a * a / (r * r));
    }
};

double radial_node(const VolumetricTables& v, int i) {
    return v.r_min + (v.r_outer - v.r_min) * i / (v.n_r - 1);
}

// Levermore-Pomraning Eddington factor f(R) = lambda + lambda^2 R^2.
double lp_factor(double R) {
    const double lam = (2.0 + R) / (6.0 + 3.0 * R + R * R);
    return lam + lam * lam * R * R;
}

void radial_structure(VolumetricTables& v) {
    const KerrOrbit orb{v.M, v.a};
    const FluxTable ft = build_flux_table(v.M, v.a, v.r_isco, v.r_outer, 0.0, v.n_r);
    const std::vector<double>& fl = ft.flux;
    const double fmax = ft.flux_max;
    const int nf = static_cast<int>(fl.size());
    auto flux_at = [&](double r) -> double {
        if (r <= v.r_isco || r >= v.r_outer || fmax <= 0.0) return 0.0;
        const double frac = (r - v.r_isco) / (v.r_outer - v.r_isco) * (nf - 1);
        const int idx = static_cast<int>(frac);
        const double t = frac - idx;
        if (idx >= nf - 1) return fl[nf - 1];
        return fl[idx] * (1.0 - t) + fl[idx + 1] * t;
    };
    v.H.assign(v.n_r, 0.0);
    v.rho_mid.assign(v.n_r, 0.0);
    v.T_eff.assign(v.n_r, 0.0);
    const double T_plunge =
        (fmax > 0.0) ? v.peak_temperature * std::pow(flux_at(v.r_isco + 0.01) / fmax, 0.25) : 0.0;
    double H_isco = 0.0;
    int isco_idx = -1;
    for (int i = 0; i < v.n_r; ++i) {
        const double r = radial_node(v, i);
        double T_eff = 0.0;
        if (r >= v.r_isco) {
            const double F = flux_at(r);
            if (F > 0.0 && fmax > 0.0) T_eff = v.peak_temperature * std::pow(F / fmax, 0.25);
        } else {
            T_eff = T_plunge;
        }
        v.T_eff[i] = T_eff;
        if (r >= v.r_isco && isco_idx < 0) isco_idx = i;
        if (T_eff <= 0.0) {
            v.H[i] = (H_isco > 0.0) ? H_isco : 0.01 * v.M;
            v.rho_mid[i] = 0.0;
            continue;
        }
        const double Omz2 = orb.omega_z_sq(r);
        if (r < v.r_isco || Omz2 <= 0.0) {
            v.H[i] = (H_isco > 0.0) ? H_isco : 0.01 * v.M;
            const int src = isco_idx >= 0 ? isco_idx : i - 1;
            if (i > 0 && v.rho_mid[src] > 0.0)
                v.rho_mid[i] = v.rho_mid[src];
            else
                v.rho_mid[i] = 1.0;
            continue;
        }
        const double Omz = std::sqrt(Omz2);
        double mu = v.opacity.lookup_mu(clamp_of(1e-10, 1e-18, 1e-6), clamp_of(T_eff, 3000.0, 1e8));
        if (mu <= 0.0 || !std::isfinite(mu)) mu = 0.6;
        const double cg2 = kB * T_eff / (mu * kMp * kC * kC);
        double H = std::sqrt(cg2) / Omz;
        const double sm = std::sqrt(v.M);
        const double ds = r * std::sqrt(r) + v.a * sm;
        const double dOm = -1.5 * sm * std::sqrt(r) / (ds * ds);
        const double shear2 = r * r * dOm * dOm;
        const double cs = std::sqrt(cg2) * kC;
        const double visc = v.cfg.alpha * cs * H;
        const double F = (r >= v.r_isco) ? flux_at(r) : flux_at(v.r_isco + 0.01);
        double rho_mid = 1.0;
        if (shear2 > 0.0 && visc > 0.0 && H > 0.0 && F > 0.0) {
            const double surf = F / (visc * shear2);
            rho_mid = surf / (std::sqrt(2.0 * kPi) * H);
        }
        H = clamp_of(H, 0.001 * v.M, 5.0 * v.M);
        v.H[i] = H;
        v.rho_mid[i] = rho_mid;
        if (r >= v.r_isco && (H_isco <= 0.0 || (isco_idx >= 0 && i == isco_idx))) H_isco = H;
    }
    if (H_isco > 0.0)
        for (int i = 0; i < v.n_r; ++i)
            if (radial_node(v, i) < v.r_isco) v.H[i] = H_isco;
}

// One radius of the iterated hydrostatic / Eddington T(tau) solve.
void vertical_column(VolumetricTables& v, int ri) {
    const OpacityTables& op = v.opacity;
    const int nz = v.n_z;
    const double r = radial_node(v, ri);
    const double H = v.H[ri];
    const double T_eff = v.T_eff[ri];
    const double rho_mid_val = v.rho_mid[ri];
    double* rho_out = &v.rho_profile[static_cast<size_t>(ri) * nz];
    double* T_out = &v.T_profile[static_cast<size_t>(ri) * nz];
    if (H <= 0.0 || T_eff <= 0.0 || rho_mid_val <= 0.0) {
        v.z_max[ri] = 3.0 * H;
        rho_out[0] = 1.0;
        T_out[0] = T_eff;
        for (int z = 1; z < nz; ++z) {
            rho_out[z] = 0.0;
            T_out[z] = T_eff;
        }
        return;
    }
    const KerrOrbit orb{v.M, v.a};
    double Omz2 = orb.omega_z_sq(r);
    if (r < v.r_isco || Omz2 <= 0.0) {
        Omz2 = orb.omega_z_sq(v.r_isco);
        if (Omz2 <= 0.0) Omz2 = orb.omega(v.r_isco) * orb.omega(v.r_isco);
    }
    auto rc = [](double x) { return clamp_of(x, 1e-18, 1e-6); };
    auto tc = [](double x) { return clamp_of(x, 3000.0, 1e8); };
    const double kR_ref = op.lookup_kappa_ross(1e-10, tc(T_eff));
    const double kE_ref = op.lookup_kappa_es(1e-10, tc(T_eff));
    const double k_ref = max_of(kR_ref + kE_ref, 1.0);
    const double rho_ref = clamp_of(v.cfg.tau_mid / (k_ref * 3.0 * H), 1e-18, 1e-6);
    const double Tm4 = 0.75 * T_eff * T_eff * T_eff * T_eff * (v.cfg.tau_mid + 2.0 / 3.0);
    const double T_mid = std::pow(Tm4, 0.25);
    double z_max = 3.0 * H;
    constexpr double kCap = 20.0;
    constexpr double kFloor = 1e-15;

    std::vector<double> rho_z(nz), T_z(nz), tau_z(nz), E_z(nz), f_z(nz), mu_z(nz);
    std::vector<double> dcs2(nz), dfE(nz), prev(nz, 1.0);
    for (int iter = 0; iter < 8; ++iter) {
        const double dz = z_max / (nz - 1);
        std::fill(rho_z.begin(), rho_z.end(), 1.0);
        std::fill(T_z.begin(), T_z.end(), T_mid);
        rho_z[0] = 1.0;
        T_z[0] = T_mid;
        std::fill(tau_z.begin(), tau_z.end(), 0.0);
        for (int z = nz - 2; z >= 0; --z) {
            const double rh = rho_z[z] * rho_ref;
            const double rn = rho_z[z + 1] * rho_ref;
            const double kRh = op.lookup_kappa_ross(rc(rh), tc(T_z[z]));
            const double kEh = op.lookup_kappa_es(rc(rh), tc(T_z[z]));
            const double kRn = op.lookup_kappa_ross(rc(rn), tc(T_z[z + 1]));
            const double kEn = op.lookup_kappa_es(rc(rn), tc(T_z[z + 1]));
            const double dtau = 0.5 * ((kRh + kEh) * rh + (kRn + kEn) * rn) * dz;
            tau_z[z] = tau_z[z + 1] + dtau;
        }
        for (int z = 0; z < nz; ++z) {
            const double T4 = 0.75 * T_eff * T_eff * T_eff * T_eff * (tau_z[z] + 2.0 / 3.0);
            T_z[z] = std::pow(max_of(T4, 0.0), 0.25);
        }
        for (int z = 0; z < nz; ++z) {
            E_z[z] = kArad * T_z[z] * T_z[z] * T_z[z] * T_z[z];
            const double rho_cgs = rho_z[z] * rho_ref;
            mu_z[z] = op.lookup_mu(rc(rho_cgs), tc(T_z[z]));
            if (mu_z[z] <= 0.0 || !std::isfinite(mu_z[z])) mu_z[z] = 0.6;
        }
        for (int z = 0; z < nz; ++z) {
            double dE = 0.0;
            if (z == 0)
                dE = 0.0;
            else if (z == nz - 1)
                dE = (E_z[z] - E_z[z - 1]) / dz;
            else
                dE = (E_z[z + 1] - E_z[z - 1]) / (2.0 * dz);
            const double rho_cgs = rho_z[z] * rho_ref;
            const double kR = op.lookup_kappa_ross(rc(rho_cgs), tc(T_z[z]));
            const double den = kR * rho_cgs * E_z[z];
            const double R = (den < 1e-30) ? 1e30 : std::abs(dE) / den;
            f_z[z] = lp_factor(R);
        }
        for (int z = 0; z < nz; ++z) {
            if (z == 0) {
                dcs2[z] = 0.0;
            } else if (z == nz - 1) {
                const double here = kB * T_z[z] / (mu_z[z] * kMp);
                const double before = kB * T_z[z - 1] / (mu_z[z - 1] * kMp);
                dcs2[z] = (here - before) / dz;
            } else {
                const double after = kB * T_z[z + 1] / (mu_z[z + 1] * kMp);
                const double before = kB * T_z[z - 1] / (mu_z[z - 1] * kMp);
                dcs2[z] = (after - before) / (2.0 * dz);
            }
            if (z == 0)
                dfE[z] = 0.0;
            else if (z == nz - 1)
                dfE[z] = (f_z[z] * E_z[z] - f_z[z - 1] * E_z[z - 1]) / dz;
            else
                dfE[z] = (f_z[z + 1] * E_z[z + 1] - f_z[z - 1] * E_z[z - 1]) / (2.0 * dz);
        }
        auto rhs = [&](double ze, double re) -> double {
            const double zf = ze / dz;
            const int idx = std::clamp(static_cast<int>(zf), 0, nz - 2);
            const double t = zf - idx;
            const double cs2 = kB * ((1.0 - t) * T_z[idx] + t * T_z[idx + 1])
                               / (((1.0 - t) * mu_z[idx] + t * mu_z[idx + 1]) * kMp);
            const double d_cs2 = (1.0 - t) * dcs2[idx] + t * dcs2[idx + 1];
            const double d_fE = (1.0 - t) * dfE[idx] + t * dfE[idx + 1];
            const double grav = Omz2 * ze;
            if (cs2 < 1e-30) return 0.0;
            const double cs2g = cs2 / (kC * kC);
            const double dcs2g = d_cs2 / (kC * kC);
            const double dfEg = d_fE / (rho_ref * kC * kC);
            return (-re * grav - re * dcs2g - dfEg) / max_of(cs2g, 1e-30);
        };
        rho_z[0] = 1.0;
        for (int z = 0; z < nz - 1; ++z) {
            const double z0 = z * dz;
            const double y = rho_z[z];
            const double k1 = dz * rhs(z0, y);
            const double k2 = dz * rhs(z0 + 0.5 * dz, max_of(y + 0.5 * k1, kFloor));
            const double k3 = dz * rhs(z0 + 0.5 * dz, max_of(y + 0.5 * k2, kFloor));
            const double k4 = dz * rhs(z0 + dz, max_of(y + k3, kFloor));
            rho_z[z + 1] = max_of(y + (k1 + 2.0 * k2 + 2.0 * k3 + k4) / 6.0, kFloor);
        }
        if (rho_z[nz - 1] > 1e-10 && z_max < kCap * H) {
            z_max = min_of(z_max + H, kCap * H);
            prev = rho_z;
            continue;
        }
        double worst = 0.0;
        for (int z = 0; z < nz; ++z)
            if (prev[z] > kFloor * 10.0) worst = max_of(worst, std::abs(rho_z[z] - prev[z]) / prev[z]);
        prev = rho_z;
        if (iter > 0 && worst < 0.001) break;
    }
    v.z_max[ri] = z_max;
    for (int z = 0; z < nz; ++z) {
        rho_out[z] = rho_z[z];
        T_out[z] = T_z[z];
    }
}

void normalise_density(VolumetricTables& v) {
    int peak = 0;
    double peak_rho = 0.0;
    for (int i = 0; i < v.n_r; ++i)
        if (radial_node(v, i) >= v.r_isco && v.rho_mid[i] > peak_rho) {
            peak_rho = v.rho_mid[i];
            peak = i;
        }
    if (peak_rho <= 0.0) {
        v.rho_scale = 1.0;
        return;
    }
    v.noise_scale = (v.cfg.noise_scale > 0.0) ? v.cfg.noise_scale : 2.0 * v.H[peak];
    if (v.noise_scale < 0.01) v.noise_scale = 0.01;
    const double zm = v.z_max[peak];
    const double dz = zm / (v.n_z - 1);
    double column = 0.0;
    for (int z = 0; z < v.n_z - 1; ++z)
        column += 0.5 * (v.rho_profile[static_cast<size_t>(peak) * v.n_z + z]
                         + v.rho_profile[static_cast<size_t>(peak) * v.n_z + z + 1]) * dz;
    column *= 2.0;
    const double T_peak = v.T_eff[peak];
    double guess = 1e-10;
    for (int it = 0; it < 3; ++it) {
        const double kR = v.opacity.lookup_kappa_ross(clamp_of(guess, 1e-18, 1e-6), clamp_of(T_peak, 3000.0, 1e8));
        const double kE = v.opacity.lookup_kappa_es(clamp_of(guess, 1e-18, 1e-6), clamp_of(T_peak, 3000.0, 1e8));
        const double k = kR + kE;
        if (k <= 0.0 || column <= 0.0) {
            v.rho_scale = 1.0;
            return;
        }
        v.rho_scale = v.cfg.tau_mid / (k * peak_rho * column);
        guess = clamp_of(v.rho_scale * peak_rho, 1e-18, 1e-6);
    }
}

}  // namespace

VolumetricTables build_volumetric_tables(double M, double a, double r_outer,
                                         double peak_temperature, const VolumetricConfig& cfg) {
    VolumetricTables v;
    v.M = M;
    v.a = a;
    v.r_outer = r_outer;
    v.peak_temperature = peak_temperature;
    v.cfg = cfg;
    v.perm = build_noise_permutation(cfg.seed);
    v.r_isco = kerr_isco(M, a);
    v.r_horizon = kerr_horizon(M, a);
    v.r_min = v.r_horizon + 0.01 * M;
    v.taper_width = (v.r_isco - v.r_horizon) / 3.0;
    {
        const double u = std::sqrt(M / v.r_isco);
        const double s = a / M;
        const double u3 = u * u * u;
        const double den = std::sqrt(1.0 - 3.0 * u * u + 2.0 * s * u3);
        v.E_isco = (1.0 - 2.0 * u * u + s * u3) / den;
        v.L_isco = std::sqrt(M * v.r_isco) * (1.0 - 2.0 * s * u3 + s * s * u * u * u * u) / den;
    }
    v.opacity = build_opacity_tables(1e-18, 1e-6, 3000.0, 1e8, cfg.opacity_nu_min, cfg.opacity_nu_max);
    radial_structure(v);
    v.z_max.assign(v.n_r, 0.0);
    v.rho_profile.assign(static_cast<size_t>(v.n_r) * v.n_z, 0.0);
    v.T_profile.assign(static_cast<size_t>(v.n_r) * v.n_z, 0.0);
#pragma omp parallel for schedule(dynamic, 4)
    for (int ri = 0; ri < v.n_r; ++ri) vertical_column(v, ri);
    normalise_density(v);
    return v;
}

}  // namespace grrt_b200
