// Volumetric Shakura-Sunyaev disk queries on the device: radial and
// per-column z-normalised profile interpolation, soft photosphere edge, ISCO
// taper, simplex-noise fBm turbulence, emitter four-velocities, and the
// opacity / Planck lookups of the radiative transfer.
//
// Restates src/volumetric_disk.cpp:97-273, src/noise.cpp:38-115 and
// src/opacity.cpp:209-345 with the same operation order. The one planned
// difference is the absorption table, stored as ln(max(kappa, 1e-100)) at
// scene build (the values the reference takes the log of at every lookup), so
// each lookup needs one exp instead of eight logs and an exp.
#pragma once

#include "scene.h"

namespace grrt_b200 {

__device__ __forceinline__ double vmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double vmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double vclamp(double v, double lo, double hi) {
    return (v < lo) ? lo : (hi < v) ? hi : v;
}
__device__ __forceinline__ int iclamp(int v, int lo, int hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

// Integer part of a table coordinate, safe for NaN and huge values.
__device__ __forceinline__ int table_index(double t, int lo, int hi) {
    if (!(t >= static_cast<double>(lo))) return lo;
    if (t >= static_cast<double>(hi)) return hi;
    return static_cast<int>(t);
}

__device__ __forceinline__ double v_radial(const DevVolume& V, const double* lut, double r) {
    if (r <= V.r_min) return __ldg(lut);
    if (r >= V.r_outer) return __ldg(lut + V.n_r - 1);
    const double frac = (r - V.r_min) / (V.r_outer - V.r_min) * (V.n_r - 1);
    const int idx = table_index(frac, 0, V.n_r - 2);
    const double t = frac - idx;
    return __ldg(lut + idx) * (1.0 - t) + __ldg(lut + idx + 1) * t;
}

__device__ __forceinline__ double v_scale_height(const DevVolume& V, double r) { return v_radial(V, V.H, r); }
__device__ __forceinline__ double v_zmax(const DevVolume& V, double r) { return v_radial(V, V.z_max, r); }

__device__ __forceinline__ double v_column(const DevVolume& V, const double* lut, int ri, double zm, double z_abs) {
    const double zf = vclamp(z_abs / zm * (V.n_z - 1), 0.0, static_cast<double>(V.n_z - 1));
    const int zi = min(table_index(zf, 0, V.n_z - 1), V.n_z - 2);
    const double tz = zf - zi;
    return (1.0 - tz) * __ldg(lut + ri * V.n_z + zi) + tz * __ldg(lut + ri * V.n_z + zi + 1);
}

__device__ __forceinline__ double v_interp_2d(const DevVolume& V, const double* lut, double r, double z_abs) {
    const double rf = vclamp((r - V.r_min) / (V.r_outer - V.r_min) * (V.n_r - 1), 0.0,
                             static_cast<double>(V.n_r - 1));
    const int ri = min(table_index(rf, 0, V.n_r - 1), V.n_r - 2);
    const double tr = rf - ri;
    const double zm_lo = __ldg(V.z_max + ri);
    const int ri1 = min(ri + 1, V.n_r - 1);
    const double zm_hi = __ldg(V.z_max + ri1);
    if ((zm_lo <= 0.0 || z_abs >= zm_lo) && (zm_hi <= 0.0 || z_abs >= zm_hi)) return 0.0;
    double lo = 0.0, hi = 0.0;
    if (zm_lo > 0.0 && z_abs < zm_lo) lo = v_column(V, lut, ri, zm_lo, z_abs);
    if (zm_hi > 0.0 && z_abs < zm_hi) hi = v_column(V, lut, ri1, zm_hi, z_abs);
    return (1.0 - tr) * lo + tr * hi;
}

__device__ __forceinline__ bool v_inside(const DevVolume& V, double r, double z) {
    if (r <= V.r_horizon || r > V.r_outer) return false;
    return fabs(z) < v_zmax(V, r) + 1.5 * v_scale_height(V, r);
}

// 3D simplex noise (src/noise.cpp:38-96): skewed cell, corner ranking, 12 edge
// gradients, (0.6 - r^2)^4 kernel, scaled by 32.
__device__ __forceinline__ double simplex_corner(double x, double y, double z, int gi) {
    double t0 = 0.6 - x * x - y * y - z * z;
    if (t0 < 0.0) return 0.0;
    t0 *= t0;
    // gradients to the midpoints of the 12 cube edges
    const int g = gi % 12;
    const double gx = (g < 8) ? ((g & 1) ? -1.0 : 1.0) : 0.0;
    const double gy = (g < 4) ? ((g & 2) ? -1.0 : 1.0) : (g < 8) ? 0.0 : ((g & 1) ? -1.0 : 1.0);
    const double gz = (g < 4) ? 0.0 : (g < 8) ? ((g & 2) ? -1.0 : 1.0) : ((g & 2) ? -1.0 : 1.0);
    return t0 * t0 * (gx * x + gy * y + gz * z);
}

__device__ __forceinline__ double simplex3(const int* __restrict__ P, double x, double y, double z) {
    constexpr double F3 = 1.0 / 3.0, G3 = 1.0 / 6.0;
    const double s = (x + y + z) * F3;
    const int i = static_cast<int>(floor(x + s)), j = static_cast<int>(floor(y + s)), k = static_cast<int>(floor(z + s));
    const double t = (i + j + k) * G3;
    const double x0 = x - (i - t), y0 = y - (j - t), z0 = z - (k - t);
    int i1, j1, k1, i2, j2, k2;
    if (x0 >= y0) {
        if (y0 >= z0) { i1 = 1; j1 = 0; k1 = 0; i2 = 1; j2 = 1; k2 = 0; }
        else if (x0 >= z0) { i1 = 1; j1 = 0; k1 = 0; i2 = 1; j2 = 0; k2 = 1; }
        else { i1 = 0; j1 = 0; k1 = 1; i2 = 1; j2 = 0; k2 = 1; }
    } else {
        if (y0 < z0) { i1 = 0; j1 = 0; k1 = 1; i2 = 0; j2 = 1; k2 = 1; }
        else if (x0 < z0) { i1 = 0; j1 = 1; k1 = 0; i2 = 0; j2 = 1; k2 = 1; }
        else { i1 = 0; j1 = 1; k1 = 0; i2 = 1; j2 = 1; k2 = 0; }
    }
    const double x1 = x0 - i1 + G3, y1 = y0 - j1 + G3, z1 = z0 - k1 + G3;
    const double x2 = x0 - i2 + 2 * G3, y2 = y0 - j2 + 2 * G3, z2 = z0 - k2 + 2 * G3;
    const double x3 = x0 - 1 + 3 * G3, y3 = y0 - 1 + 3 * G3, z3 = z0 - 1 + 3 * G3;
    const int ii = i & 255, jj = j & 255, kk = k & 255;
    const double n0 = simplex_corner(x0, y0, z0, P[ii + P[jj + P[kk]]]);
    const double n1 = simplex_corner(x1, y1, z1, P[ii + i1 + P[jj + j1 + P[kk + k1]]]);
    const double n2 = simplex_corner(x2, y2, z2, P[ii + i2 + P[jj + j2 + P[kk + k2]]]);
    const double n3 = simplex_corner(x3, y3, z3, P[ii + 1 + P[jj + 1 + P[kk + 1]]]);
    return 32.0 * (n0 + n1 + n2 + n3);
}

// Density with the soft photosphere edge, ISCO taper and fBm turbulence
// (src/volumetric_disk.cpp:228-257). P is the 512-entry permutation.
__device__ __forceinline__ double v_density(const DevVolume& V, const int* __restrict__ P, double r, double z,
                                            double phi) {
    if (r <= V.r_horizon || r > V.r_outer) return 0.0;
    const double z_abs = fabs(z);
    const double zm = v_zmax(V, r);
    const double H = v_scale_height(V, r);
    double edge = 1.0, z_look = z_abs;
    if (z_abs >= zm) {
        const double dz = z_abs - zm;
        if (dz >= 1.5 * H) return 0.0;
        edge = exp(-2.0 * (dz / H) * (dz / H));
        z_look = zm * 0.9999;
    }
    const double rho_mid = v_radial(V, V.rho_mid, r);
    const double rho_norm = v_interp_2d(V, V.rho_prof, r, z_look);
    double taper = 1.0;
    if (r < V.r_isco) {
        const double dr = V.r_isco - r;
        taper = exp(-(dr * dr) / (V.taper_width * V.taper_width));
    }
    const double base = rho_mid * rho_norm * V.rho_scale * taper * edge;
    double sp, cp;
    sincos(phi, &sp, &cp);
    const double nx = r * cp / V.noise_scale;
    const double ny = r * sp / V.noise_scale;
    const double nz = z / V.noise_scale;
    double n = 0.0, amp = 1.0, freq = 1.0;
    for (int o = 0; o < V.octaves; ++o) {
        n += amp * simplex3(P, nx * freq, ny * freq, nz * freq);
        amp *= 0.5;
        freq *= 2.0;
    }
    return vmax(0.0, base * (1.0 + V.turbulence * n));
}

// Temperature from the vertical profile, surface value in the soft edge
// (src/volumetric_disk.cpp:264-273).
__device__ __forceinline__ double v_temperature(const DevVolume& V, double r, double z) {
    if (r <= V.r_horizon || r > V.r_outer) return 0.0;
    const double z_abs = fabs(z);
    const double zm = v_zmax(V, r);
    const double H = v_scale_height(V, r);
    if (z_abs >= zm + 1.5 * H) return 0.0;
    return v_interp_2d(V, V.T_prof, r, vmin(z_abs, zm * 0.9999));
}

// Emitter four-velocity (circular orbit outside the ISCO, plunging geodesic
// with ISCO constants inside; src/volumetric_disk.cpp:97-137) and the redshift
// g = (p.u)_emit / (p.u)_obs (src/geodesic_tracer.cpp:279-292).
__device__ __forceinline__ void v_redshift(const DevVolume& V, double pt, double pr, double pph, double r,
                                           double theta, double& g, double& pue) {
    const double M = V.M, a = V.a;
    double ut, ur = 0.0, uphi;
    if (r >= V.r_isco) {
        const double sM = sqrt(M);
        const double Omg = sM / (r * sqrt(r) + a * sM);
        const double g_tt = -(1.0 - 2.0 * M / r);
        const double g_tphi = -2.0 * M * a / r;
        const double g_phph = r * r + a * a + 2.0 * M * a * a / r;
        const double den = -(g_tt + 2.0 * g_tphi * Omg + g_phph * Omg * Omg);
        ut = 1.0 / sqrt(vmax(den, 1e-30));
        uphi = Omg * ut;
    } else {
        const double E = V.E_isco, L = V.L_isco;
        const double Delta = r * r - 2.0 * M * r + a * a;
        const double c = cos(theta);
        const double Sigma = r * r + a * a * c * c;
        ut = (E * (r * r + a * a + 2.0 * M * a * a / r) - 2.0 * M * a * L / r) / Delta;
        uphi = (L * (1.0 - 2.0 * M / r) + 2.0 * M * a * E / r) / Delta;
        const double EaL = E * (r * r + a * a) - a * L;
        const double LaE = L - a * E;
        const double R = EaL * EaL - Delta * (r * r + LaE * LaE);
        ur = -sqrt(vmax(0.0, R)) / Sigma;
    }
    pue = pt * ut + pr * ur + pph * uphi;
    g = pue / (pt * V.ut_obs);
}

// Table coordinate of a log-spaced axis (src/opacity.cpp:218-224).
__device__ __forceinline__ void log_locate(double lv, double lo, double hi, int n, int& idx, double& frac) {
    double t = (lv - lo) / (hi - lo) * (n - 1);
    t = vclamp(t, 0.0, static_cast<double>(n - 2));
    idx = table_index(t, 0, n - 2);
    frac = t - idx;
}

// Electron-scattering opacity, bilinear in the (rho, T) cell.
__device__ __forceinline__ double v_kappa_es(const DevVolume& V, int ir, double fr, int iT, double fT) {
    const double* L = V.kes;
    const int nt = V.n_T;
    const double v00 = __ldg(L + ir * nt + iT), v01 = __ldg(L + ir * nt + iT + 1);
    const double v10 = __ldg(L + (ir + 1) * nt + iT), v11 = __ldg(L + (ir + 1) * nt + iT + 1);
    return v00 * (1 - fr) * (1 - fT) + v01 * (1 - fr) * fT + v10 * fr * (1 - fT) + v11 * fr * fT;
}

// Absorption opacity: trilinear in ln kappa over (nu, rho, T), then exp.
__device__ __forceinline__ double v_kappa_abs(const DevVolume& V, double nu, int ir, double fr, int iT, double fT) {
    int inu;
    double fnu;
    log_locate(log10(nu), V.log_nu_min, V.log_nu_max, V.n_nu, inu, fnu);
    const size_t s0 = static_cast<size_t>(V.n_rho) * V.n_T;
    const double* L0 = V.ln_kabs + inu * s0 + ir * V.n_T + iT;
    const double* L1 = L0 + s0;
    const int nt = V.n_T;
    const double l00 = __ldg(L0) * (1 - fT) + __ldg(L0 + 1) * fT;
    const double l01 = __ldg(L0 + nt) * (1 - fT) + __ldg(L0 + nt + 1) * fT;
    const double l10 = __ldg(L1) * (1 - fT) + __ldg(L1 + 1) * fT;
    const double l11 = __ldg(L1 + nt) * (1 - fT) + __ldg(L1 + nt + 1) * fT;
    const double l0 = l00 * (1 - fr) + l01 * fr;
    const double l1 = l10 * (1 - fr) + l11 * fr;
    return exp(l0 * (1 - fnu) + l1 * fnu);
}

// Planck B_nu in CGS (src/opacity.cpp:209-214).
__device__ __forceinline__ double planck_nu(double nu, double T) {
    constexpr double h = 6.626070e-27, k = 1.380649e-16, c = 2.997924e10;
    if (nu <= 0.0 || T <= 0.0) return 0.0;
    const double x = h * nu / (k * T);
    if (x > 500.0) return 0.0;
    return (2.0 * h * nu * nu * nu / (c * c)) / (exp(x) - 1.0);
}

}  // namespace grrt_b200
