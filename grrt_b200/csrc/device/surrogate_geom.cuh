// Closed-form ray geometry for the learned surrogate, host and device.
//
// A Kerr null geodesic has three constants: E = -p_t, L = p_phi and the Carter
// constant Q = p_theta^2 + cos^2(theta) (L^2 / sin^2(theta) - a^2 E^2). With
//   R(r)  = ((r^2 + a^2) E - a L)^2 - Delta(r) (Q + (L - a E)^2)
//   Th(mu) = Q - mu^2 (Q + L^2 - a^2 E^2) - a^2 E^2 mu^4,   mu = cos(theta),
// the ray moves where R >= 0 and Th >= 0. From them, without integrating:
//   - capture: an ingoing ray from the camera falls in iff R > 0 on
//     (r_+, r_camera]; near the critical curve R has a near-double root, so
//     the minimum of R / (E^2 r^4) (R's leading term) is the distance to the
//     curve used for the fallback band. (R / (E^2 r^4) stays finite near the
//     horizon, where P and Delta both vanish for the near-extremal prograde
//     orbits.)
//   - theta range: mu^2 oscillates up to mu_+^2 (Q >= 0: across the equator),
//     or between mu_-^2 and mu_+^2 (Q < 0: one hemisphere, never crossing).
//     A ray that turns close to the equator grazes the disk plane; the
//     surrogate sends those to the exact integrator.
#pragma once

#include "kerr.cuh"

namespace grrt_b200 {
namespace surr {

struct RayConstants {
    double E, L, Q;
};

GRRT_HD RayConstants constants(double a, double theta, const double p[4]) {
    RayConstants k;
    k.E = -p[0];
    k.L = p[3];
    const double s = sin(theta), c = cos(theta);
    const double s2 = (s * s < 1e-20) ? 1e-20 : s * s;
    k.Q = p[2] * p[2] + c * c * (k.L * k.L / s2 - a * a * k.E * k.E);
    return k;
}

GRRT_HD double radial_potential(double M, double a, const RayConstants& k, double r) {
    const double P = (r * r + a * a) * k.E - a * k.L;
    const double D = r * r - 2.0 * M * r + a * a;
    const double lae = k.L - a * k.E;
    return P * P - D * (k.Q + lae * lae);
}

// R / (E^2 r^4): 1 at large r for any ray, 0 at a turning point.
GRRT_HD double scaled_potential(double M, double a, const RayConstants& k, double r) {
    const double r2 = r * r;
    return radial_potential(M, a, k, r) / (k.E * k.E * r2 * r2);
}

// Capture test of a ray that starts at r_cam moving inward (p_r < 0).
// Returns the minimum of the scaled potential over [r_h, r_cam]: > 0
// captured, < 0 a turning point (escapes); |value| small = close to the
// critical curve. Sampled on a geometric grid, the minimum refined by golden
// section (R has at most two local extrema outside the horizon).
GRRT_HD double capture_margin(double M, double a, const RayConstants& k, double r_h, double r_cam) {
    constexpr int kN = 96;
    const double lo = r_h * (1.0 + 1e-9), hi = r_cam;
    const double q = pow(hi / lo, 1.0 / (kN - 1));
    double best = 1e300, r_best = lo, r = lo;
    int i_best = 0;
    for (int i = 0; i < kN; ++i) {
        const double v = scaled_potential(M, a, k, r);
        if (v < best) {
            best = v;
            r_best = r;
            i_best = i;
        }
        r *= q;
    }
    // refine in the bracket around the best grid point
    double x0 = (i_best > 0) ? r_best / q : lo, x1 = (i_best < kN - 1) ? r_best * q : hi;
    constexpr double g = 0.6180339887498949;
    double xa = x1 - g * (x1 - x0), xb = x0 + g * (x1 - x0);
    double fa = scaled_potential(M, a, k, xa), fb = scaled_potential(M, a, k, xb);
    for (int it = 0; it < 40; ++it) {
        if (fa < fb) {
            x1 = xb;
            xb = xa;
            fb = fa;
            xa = x1 - g * (x1 - x0);
            fa = scaled_potential(M, a, k, xa);
        } else {
            x0 = xa;
            xa = xb;
            fa = fb;
            xb = x0 + g * (x1 - x0);
            fb = scaled_potential(M, a, k, xb);
        }
    }
    const double v = fa < fb ? fa : fb;
    return v < best ? v : best;
}

// Smallest radius of a ray that starts at r_cam moving inward: its outermost
// radial turning point (largest root of R below r_cam), or r_h when it falls
// in. R / (E^2 r^4) is scanned on a geometric grid from r_cam inward and the
// first sign change is bisected; the result is taken on the forbidden side,
// so it never exceeds the root. A forbidden interval narrower than the grid
// spacing is missed and the ray counts as falling in (a smaller radius).
GRRT_HD double turning_radius(double M, double a, const RayConstants& k, double r_h, double r_cam) {
    constexpr int kN = 96;
    const double lo = r_h * (1.0 + 1e-9);
    const double q = pow(r_cam / lo, 1.0 / (kN - 1));
    double r_prev = r_cam;
    for (int i = 1; i < kN; ++i) {
        const double r = (i == kN - 1) ? lo : r_prev / q;
        if (scaled_potential(M, a, k, r) < 0.0) {
            double x0 = r, x1 = r_prev;
            for (int it = 0; it < 60; ++it) {
                const double xm = 0.5 * (x0 + x1);
                if (scaled_potential(M, a, k, xm) < 0.0)
                    x0 = xm;
                else
                    x1 = xm;
            }
            return x0;
        }
        r_prev = r;
    }
    return r_h;
}

// Smallest radius a camera ray (covariant momentum p at the camera, r_cam,
// theta_cam) ever reaches: r_cam for an outgoing ray (it only moves out:
// every photon orbit lies far inside the camera radius), else turning_radius.
GRRT_HD double camera_ray_min_radius(double M, double a, double r_h, double r_cam, double theta_cam,
                                     const double p[4]) {
    if (p[1] >= 0.0) return r_cam;
    return turning_radius(M, a, constants(a, theta_cam, p), r_h, r_cam);
}

// Whether a camera ray's smallest radius exceeds r_gate (< r_cam): the same
// answer as camera_ray_min_radius(...) > r_gate, from the same inward scan,
// but the scan stops at r_gate and the bracket that holds r_gate is settled by
// the sign of R at r_gate (the turning point lies above r_gate exactly when
// r_gate is in the forbidden region) instead of by bisection.
// Only signs of R are taken (R and R / (E^2 r^4) have the same sign), so no
// division is made.
GRRT_HD bool camera_ray_clears(double M, double a, double r_h, double r_cam, double theta_cam, const double p[4],
                               double r_gate) {
    if (p[1] >= 0.0) return r_cam > r_gate;
    const RayConstants k = constants(a, theta_cam, p);
    constexpr int kN = 96;
    const double lo = r_h * (1.0 + 1e-9);
    const double q = pow(r_cam / lo, 1.0 / (kN - 1));
    double r_prev = r_cam;
    for (int i = 1; i < kN; ++i) {
        const double r = (i == kN - 1) ? lo : r_prev / q;
        if (r <= r_gate) {
            // R >= 0 at r: any turning point lies below r <= r_gate
            if (!(radial_potential(M, a, k, r) < 0.0)) return false;
            return radial_potential(M, a, k, r_gate) < 0.0;
        }
        if (radial_potential(M, a, k, r) < 0.0) return true;  // turning point in (r, r_prev), above r_gate
        r_prev = r;
    }
    return false;
}

// Distance (in mu = cos theta) of the ray's theta turning point from the
// equator: mu_+ when Q >= 0 (the ray crosses the plane and turns at +-mu_+),
// mu_- when Q < 0 (it stays in one hemisphere between mu_- and mu_+).
GRRT_HD double graze_margin(double a, const RayConstants& k) {
    const double A = a * a * k.E * k.E;
    const double B = k.Q + k.L * k.L - A;
    double xp, xm;  // roots in mu^2 of A x^2 + B x - Q = 0
    if (A < 1e-14 * (fabs(B) + 1e-300)) {
        xp = (B != 0.0) ? k.Q / B : 0.0;
        xm = xp;
    } else {
        const double disc = sqrt(fmax(B * B + 4.0 * A * k.Q, 0.0));
        xp = (-B + disc) / (2.0 * A);
        xm = (-B - disc) / (2.0 * A);
    }
    if (k.Q >= 0.0) return sqrt(fmax(xp, 0.0));
    return sqrt(fmax(fmin(xp, xm), 0.0));
}

// Network input encoding: image-plane angles over the 90 degree field,
// spin in [0, 1), inclination in [5, 90] degrees, each mapped to [-1, 1].
GRRT_HD void encode_inputs(double alpha, double beta, double spin, double incl, float out[4]) {
    constexpr double kQuarterPi = 0.78539816339744831;
    constexpr double kDeg = 0.017453292519943295;
    out[0] = static_cast<float>(alpha / kQuarterPi);
    out[1] = static_cast<float>(beta / kQuarterPi);
    out[2] = static_cast<float>(2.0 * spin - 1.0);
    out[3] = static_cast<float>((incl - 47.5 * kDeg) / (42.5 * kDeg));
}

// Output slots of the network (9 used of the 16 the last GEMM computes): the
// six quantities, then log sigma of the network's own error on u1, u2 and on
// the sky direction (outputs 2-4).
enum : int {
    kOutU1 = 0, kOutU2 = 1, kOutCosTh = 2, kOutSinPh = 3, kOutCosPh = 4, kOutCTh = 5,
    kOutLogSig1 = 6, kOutLogSig2 = 7, kOutLogSigDir = 8, kOutputs = 9
};
constexpr double kCThScale = 1.0 / 32.0;  // c_theta = r^2 dtheta/dr is O(b) ~ tens of M

}  // namespace surr
}  // namespace grrt_b200
