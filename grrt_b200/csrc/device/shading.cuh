// Per-sample shading on the device: camera rays, the reference jitter hash,
// thin-disk emission and the star lookup.
#pragma once

#include <cstdint>

#include "kerr.cuh"
#include "scene.h"

namespace grrt_b200 {

constexpr double kPiD = 3.141592653589793;
constexpr double kHalfPi = kPiD / 2.0;

// Stratified jitter hash (src/renderer.cpp:14-20): exact 32-bit integer mixing.
__device__ __forceinline__ double pixel_hash(int i, int j, int s, int ch) {
    uint32_t h = (static_cast<uint32_t>(i) * 73856093u) ^ (static_cast<uint32_t>(j) * 19349663u)
                 ^ (static_cast<uint32_t>(s) * 83492791u) ^ (static_cast<uint32_t>(ch) * 45678917u);
    h ^= h >> 16;
    h *= 0x45d9f3bu;
    h ^= h >> 16;
    return (h & 0xFFFFu) / 65536.0;
}

// Covariant null momentum of a camera sample (src/camera.cpp:69-96):
// screen angles both scaled by the width, local direction in the static
// observer's tetrad, p^mu = -e0 + d, lowered with the camera's g_mu_nu.
__device__ __forceinline__ void camera_momentum(const DevScene& S, double x, double y, double p[4]) {
    const double alpha = (x - S.width / 2.0) * S.fov / S.width;
    const double beta = (y - S.height / 2.0) * S.fov / S.width;
    double sa, ca_, sb, cb_;
    sincos(alpha, &sa, &ca_);
    sincos(beta, &sb, &cb_);
    const double ca = cb_ * sa;
    const double cb = sb;
    const double cc = cb_ * ca_;
    double pu[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) pu[m] = -S.e0[m] + (-ca * S.e1[m] - cb * S.e2[m] + cc * S.e3[m]);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        double sum = 0.0;
#pragma unroll
        for (int n = 0; n < 4; ++n) sum += S.g[4 * m + n] * pu[n];
        p[m] = sum;
    }
}

// Thin-disk emission at a crossing radius (src/accretion_disk.cpp:96-147 and
// src/spectrum.cpp:115-131): Novikov-Thorne temperature from the flux table,
// redshift g between the circular-orbit emitter and the static observer,
// chromaticity of g*T times (T/t_max)^4 * g^4.
static __device__ __noinline__ void disk_emission(const DevScene& S, double r, double pt, double pph,
                                           double& c0, double& c1, double& c2) {
    c0 = c1 = c2 = 0.0;
    if (r <= S.r_in || r >= S.r_out || S.flux_max <= 0.0) return;
    const int n = S.flux_n;
    const double frac = (r - S.r_in) / (S.r_out - S.r_in) * (n - 1);
    const int idx = static_cast<int>(frac);
    const double t = frac - idx;
    const double F = (idx >= n - 1) ? __ldg(S.flux + n - 1)
                                    : __ldg(S.flux + idx) * (1.0 - t) + __ldg(S.flux + idx + 1) * t;
    if (F <= 0.0) return;
    const double T = S.peak_T * pow(F / S.flux_max, 0.25);
    if (T <= 0.0) return;
    const double M = S.M, a = S.a;
    const double pu_obs = pt * S.u_t_obs;
    const double w = sqrt(M / (r * r * r));
    const double aw = a * w;
    const double u_t = 1.0 / sqrt(1.0 - 3.0 * M / r + 2.0 * aw);
    const double u_phi = (w / (1.0 + aw)) * u_t;
    const double pu_emit = pt * u_t + pph * u_phi;
    const double g = (fabs(pu_obs) < 1e-30) ? 1.0 : pu_emit / pu_obs;
    const double T_obs = g * T;
    if (T_obs < 100.0) return;
    const double Tc = (T_obs < S.t_min) ? S.t_min : (S.t_max < T_obs) ? S.t_max : T_obs;
    const double f = (Tc - S.t_min) / (S.t_max - S.t_min) * (S.spec_n - 1);
    const int k = static_cast<int>(f);
    const double u = f - k;
    double ch[3];
    if (k >= S.spec_n - 1) {
#pragma unroll
        for (int q = 0; q < 3; ++q) ch[q] = __ldg(S.spec_color + 3 * (S.spec_n - 1) + q);
    } else {
#pragma unroll
        for (int q = 0; q < 3; ++q)
            ch[q] = __ldg(S.spec_color + 3 * k + q) * (1.0 - u) + __ldg(S.spec_color + 3 * (k + 1) + q) * u;
    }
    const double ratio = T / S.t_max;
    const double lum = ratio * ratio * ratio * ratio;
    const double g4 = g * g * g * g;
    const double wgt = lum * g4;
    c0 = ch[0] * wgt;
    c1 = ch[1] * wgt;
    c2 = ch[2] * wgt;
}

// First star within the angular tolerance in the 3x3 cells around the escape
// direction, scanned in the reference order (src/celestial_sphere.cpp:48-90).
static __device__ __noinline__ double star_brightness(const DevStars& st, double theta, double phi) {
    theta = fmod(theta, 2.0 * kPiD);
    if (theta < 0.0) theta += 2.0 * kPiD;
    if (theta > kPiD) {
        theta = 2.0 * kPiD - theta;
        phi += kPiD;
    }
    phi = fmod(phi, 2.0 * kPiD);
    if (phi > kPiD) phi -= 2.0 * kPiD;
    if (phi < -kPiD) phi += 2.0 * kPiD;
    constexpr int nt = 180, np = 360;
    const int tb = static_cast<int>(theta * nt / kPiD);
    const int pb = static_cast<int>((phi + kPiD) * np / (2.0 * kPiD));
    const double s = sin(theta);
    for (int dt = -1; dt <= 1; ++dt) {
        int t = tb + dt;
        t = (t < 0) ? 0 : (t > nt - 1) ? nt - 1 : t;
        for (int dp = -1; dp <= 1; ++dp) {
            const int p = (((pb + dp) % np) + np) % np;
            const int cell = t * np + p;
            const int q1 = __ldg(st.cell_start + cell + 1);
            for (int q = __ldg(st.cell_start + cell); q < q1; ++q) {
                const int si = __ldg(st.cell_items + q);
                const double dth = theta - __ldg(st.theta + si);
                double dph = phi - __ldg(st.phi + si);
                if (dph > kPiD) dph -= 2.0 * kPiD;
                if (dph < -kPiD) dph += 2.0 * kPiD;
                if (dth * dth + dph * dph * s * s < st.tol2) return __ldg(st.brightness + si);
            }
        }
    }
    return 0.0;
}

}  // namespace grrt_b200
