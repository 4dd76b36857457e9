// Decisions of the speculative (FP32) pass of the mixed-precision thin-disk
// form, shared by the kernels and the host-side tests.
//
// A thin-disk sample's colour is exactly 0 (horizon, or escape with no star),
// exactly a star's brightness, or emission summed at disk crossings whose
// radius is interpolated between two accepted steps
// (src/geodesic_tracer.cpp:156-176). Only the last two depend on where the
// FP64 steps land. The speculative pass integrates every sample with FP32
// right-hand sides and marks for the FP64 re-trace each sample whose colour
// the FP64 step sequence could make non-zero or move:
//   - an equatorial crossing with interpolated radius in [r_in - m, r_out + m]
//     widened by kCrossStepFrac of the step's radial extent (the interpolated
//     radius moves with the step placement: chord error), or, when the step
//     holds a radial turning point, any overlap of the step's radii with that
//     band;
//   - an accepted step over those radii closer than kGrazeAbs to the plane, or
//     a theta turning point there closer than kGrazeTurn (a graze, which the
//     FP64 steps may turn into a crossing or step over);
//   - more than kSweptMax radians swept inside r_near (near-critical orbits:
//     trajectory differences grow about e-fold per radian there; r_near covers
//     every photon orbit);
//   - a step ending within kPoleSin (|sin theta|) of a pole or stepping across
//     one, where the FP32 right-hand side is not accurate enough;
//   - the step budget;
//   - an escape whose star lookup could find a star (see EscapeArc).
#pragma once

#include "integrate.cuh"
#include "scene.h"

#ifdef __CUDA_ARCH__
#define GRRT_LDG(p) __ldg(p)
#else
#define GRRT_LDG(p) (*(p))
#endif

namespace grrt_b200 {
namespace mixed {

constexpr double kCrossStepFrac = 0.2;
constexpr double kGrazeAbs = 2e-3;
constexpr double kGrazeTurn = 0.1;
constexpr double kSweptMax = 3.0;
constexpr float kPoleSin = 0.02f;
constexpr double kPi = 3.14159265358979323846;

// sample_fate value of an escape whose star test is still to run.
constexpr unsigned kFateStarPending = 0xffffffffu;

// Early end of a speculative trace on a black sky: an outgoing ray (p_r > 0)
// beyond r_min can no longer come back (a null geodesic turns back outward of
// the photon orbits only at a radius below its outermost turning point, which
// an outgoing ray has passed), so it escapes with no further disk crossing or
// near-hole sweep, and with no star to look up its colour is already final.
// r_min must lie outside the region the pass tests (disk radii plus margins,
// r_near) and outside every photon orbit (kEscapeRMin >= 4 M for |a| <= M).
// steps: the FP32 pass's accepted steps so far; the FP64 trace, which takes
// more steps, must still be far from the step budget on its way out.
constexpr double kEscapeRMin = 5.0;
GRRT_HD bool certain_escape(const Vec5<double>& y, double r_min, int steps, int max_steps) {
    return y.pr > 0.0 && y.r > r_min && 3 * steps + 1000 < max_steps;
}

struct Tracker {
    double lo = 0.0, hi = 0.0, r_near = 0.0;
    bool disk = false;
    double swept = 0.0;
    double a2e2 = 0.0, l2 = 0.0;  // a^2 p_t^2 and p_phi^2 of the ray
    float sin_th = 0.0f;          // FP32 sin(theta) of the current state

    // th0: the ray's initial theta.
    GRRT_HD void reset(bool disk_on, double r_in, double r_out, double margin, double r_near_, double a, double pt,
                       double pph, double th0) {
        disk = disk_on;
        lo = r_in - margin;
        hi = r_out + margin;
        r_near = r_near_;
        swept = 0.0;
        a2e2 = a * a * pt * pt;
        l2 = pph * pph;
        float c0;
        rhs_sincos(static_cast<float>(th0), sin_th, c0);
    }

    // cos^2 of the colatitude where the theta motion turns, from the Carter
    // constant Q = p_theta^2 + cos^2(theta) (p_phi^2 / sin^2(theta) - a^2 p_t^2)
    // at a state with sin, cos of theta (s, c): the root u in [0, 1] of
    // a^2 p_t^2 u^2 + (Q + p_phi^2 - a^2 p_t^2) u - Q = 0.
    GRRT_HD double turning_cos2(double pth, double s, double c) const {
        const double s2 = fmax(s * s, 1e-30), c2 = c * c;
        const double Q = fmax(pth * pth + c2 * (l2 / s2 - a2e2), 0.0);
        const double B = Q + l2 - a2e2;
        if (a2e2 <= 0.0) return (Q + l2 > 0.0) ? Q / (Q + l2) : 0.0;
        const double disc = sqrt(B * B + 4.0 * a2e2 * Q);
        return (B >= 0.0) ? 2.0 * Q / (B + disc) : (disc - B) / (2.0 * a2e2);
    }

    // One accepted step y -> y5 of affine length h; true when the sample
    // needs the FP64 re-trace.
    GRRT_HD bool step(const Vec5<double>& y, const Vec5<double>& y5, double h) {
        bool hit = false;
        if (disk) {
            const double d_prev = y.th - 0.5 * kPi, d_new = y5.th - 0.5 * kPi;
            if (d_prev * d_new < 0.0 && fabs(d_prev - d_new) > 1e-12) {
                const double rc = y.r + (-d_prev / (d_new - d_prev)) * (y5.r - y.r);
                const double w = kCrossStepFrac * fabs(y5.r - y.r);
                hit = rc >= lo - w && rc <= hi + w;
                // A radial turning point inside the step (p_r changes sign):
                // r is then far from linear in theta and the chord can miss
                // the crossing radius by most of the step's radial extent. The
                // radii along the step lie in [min r - dip, max r], with
                // dip <= h min|p_r| / 2 for a quadratic r(lambda) with
                // dr/dlambda = (Delta / Sigma) p_r and Delta / Sigma <= 1
                // (taken twice for the higher terms); an overlap with the band
                // counts.
                if (!hit && y.pr * y5.pr <= 0.0) {
                    const double dip = fabs(h) * fmin(fabs(y.pr), fabs(y5.pr));
                    hit = fmin(y.r, y5.r) - dip <= hi + w && fmax(y.r, y5.r) >= lo - w;
                }
            } else if (y5.r >= lo && y5.r <= hi) {
                const double m = fmin(fabs(d_prev), fabs(d_new));
                hit = m < kGrazeAbs || (y.pth * y5.pth <= 0.0 && m < kGrazeTurn);
            }
        }
        // Near a pole the right-hand side's 1/sin(theta) terms amplify the
        // FP32 sine's absolute error (about 1e-7) into the trajectory; a ray
        // that ends a step within kPoleSin of the axis, steps across it
        // (sin(theta) changes sign), or turns in theta inside a step closer to
        // it than kPoleSin (the turning colatitude from the Carter constant:
        // a long step can pass the pole between its ends) is re-traced.
        const float s0 = sin_th;  // sin(theta) at y, from the previous step
        float s5, c5;
        rhs_sincos(static_cast<float>(y5.th), s5, c5);
        sin_th = s5;
        if (fabsf(s5) < kPoleSin || s0 * s5 <= 0.0f) hit = true;
        if (!hit && y.pth * y5.pth <= 0.0 &&
            1.0 - turning_cos2(y5.pth, s5, c5) < static_cast<double>(kPoleSin) * kPoleSin)
            hit = true;
        if (y.r < r_near) {
            swept += fabs(y5.th - y.th) + fabs(y5.ph - y.ph) * static_cast<double>(fabsf(s0));
            if (swept > kSweptMax) hit = true;
        }
        return hit;
    }
};

// The arc of sky an escaping ray's star lookup can land on. The reference looks
// the star up at the first accepted step past r_escape, whose radius depends on
// the step sequence; a step is capped at 5 max(r, 1) in the affine parameter,
// so it lands below 6 r_escape. In the far field
// angle(r) = angle_f + c (1/r_f - 1/r) with c = r^2 d(angle)/dr, a straight
// segment in (theta, phi) from r = r_escape (th0, ph0) to r = 7 r_escape
// (th0 + dth, ph0 + dph), unfolded (no pole or 2 pi wrap applied).
struct EscapeArc {
    double th0, ph0;
    float dth, dph;
};

// k = right-hand side at the escape state y (dr, dtheta, dphi used).
GRRT_HD EscapeArc escape_arc(double r_escape, const Vec5<double>& y, const Vec5<float>& k) {
    EscapeArc e;
    const double r_f = y.r;
    const double dr = static_cast<double>(k.r);
    const double c_th = dr > 0.0 ? r_f * r_f * static_cast<double>(k.th) / dr : 0.0;
    const double c_ph = dr > 0.0 ? r_f * r_f * static_cast<double>(k.ph) / dr : 0.0;
    const double u0 = 1.0 / r_f - 1.0 / r_escape;
    const double du = (1.0 / r_escape - 1.0 / (7.0 * r_escape));
    e.th0 = y.th + c_th * u0;
    e.ph0 = y.ph + c_ph * u0;
    // a non-outgoing ray (dr <= 0 cannot escape past r_escape in the far field)
    // gets an arc long enough to be sent to the re-trace
    e.dth = dr > 0.0 ? static_cast<float>(c_th * du) : 1.0f;
    e.dph = dr > 0.0 ? static_cast<float>(c_ph * du) : 1.0f;
    return e;
}

// Folds (theta, phi) the way the star lookup does (src/celestial_sphere.cpp:48-90):
// theta into [0, pi] (phi + pi when it passes a pole), phi into [-pi, pi].
// Returns whether theta was reflected.
GRRT_HD bool fold_sky(double& theta, double& phi) {
    theta = fmod(theta, 2.0 * kPi);
    if (theta < 0.0) theta += 2.0 * kPi;
    bool flip = false;
    if (theta > kPi) {
        theta = 2.0 * kPi - theta;
        phi += kPi;
        flip = true;
    }
    phi = fmod(phi, 2.0 * kPi);
    if (phi > kPi) phi -= 2.0 * kPi;
    if (phi < -kPi) phi += 2.0 * kPi;
    return flip;
}

GRRT_HD int imax(int a, int b) { return a > b ? a : b; }
GRRT_HD int imin(int a, int b) { return a < b ? a : b; }

// True when the star lookup at any point of the arc could find a star: one
// scan of the cells every lookup along it can reach (the arc's cell span plus
// the lookup's one-cell border), with a point-to-segment distance per star
// against the lookup tolerance plus `slack` rad (default 1e-4: far-field
// model and FP32 trajectory). Arcs near a pole, where the picture and the cell scan
// break down, count as in reach.
GRRT_HD bool star_in_reach(const DevStars& st, const mixed::EscapeArc& e, double slack = 1e-4) {
    double th0 = e.th0, ph0 = e.ph0;
    double th1 = e.th0 + e.dth, ph1 = e.ph0 + e.dph;
    const bool f0 = mixed::fold_sky(th0, ph0), f1 = mixed::fold_sky(th1, ph1);
    constexpr double kCell = kPi / 180.0;  // star grid cells are 1 degree
    if (f0 != f1 || fmin(th0, th1) < 3.0 * kCell || fmax(th0, th1) > kPi - 3.0 * kCell) return true;
    double dph = ph1 - ph0;
    if (dph > kPi) dph -= 2.0 * kPi;
    if (dph < -kPi) dph += 2.0 * kPi;
    if (fabs(dph) > 10.0 * kCell || fabs(th1 - th0) > 10.0 * kCell) return true;
    // the lookup's distance metric weighs phi by sin(theta): take its smallest
    // value along the segment (sin is concave on [0, pi])
    const double s = fmin(sin(th0), sin(th1));
    const double tol = sqrt(st.tol2) + slack;
    const double ex = th1 - th0, ey = dph * s;
    const double e2 = ex * ex + ey * ey;
    constexpr int nt = 180, np = 360;
    const int t_lo = imax(static_cast<int>(fmin(th0, th1) * nt / kPi) - 1, 0);
    const int t_hi = imin(static_cast<int>(fmax(th0, th1) * nt / kPi) + 1, nt - 1);
    const double pa = fmin(ph0, ph0 + dph), pb = fmax(ph0, ph0 + dph);
    const int p_lo = static_cast<int>(floor((pa + kPi) * np / (2.0 * kPi))) - 1;
    const int p_hi = static_cast<int>(floor((pb + kPi) * np / (2.0 * kPi))) + 1;
    for (int t = t_lo; t <= t_hi; ++t) {
        for (int pc = p_lo; pc <= p_hi; ++pc) {
            const int cell = t * np + ((pc % np) + np) % np;
            const int q1 = GRRT_LDG(st.cell_start + cell + 1);
            for (int q = GRRT_LDG(st.cell_start + cell); q < q1; ++q) {
                const int si = GRRT_LDG(st.cell_items + q);
                const double qx = GRRT_LDG(st.theta + si) - th0;
                double qp = GRRT_LDG(st.phi + si) - ph0;
                if (qp > kPi) qp -= 2.0 * kPi;
                if (qp < -kPi) qp += 2.0 * kPi;
                const double qy = qp * s;
                double t_seg = e2 > 0.0 ? (qx * ex + qy * ey) / e2 : 0.0;
                t_seg = fmin(fmax(t_seg, 0.0), 1.0);
                const double dx = qx - t_seg * ex, dy = qy - t_seg * ey;
                if (dx * dx + dy * dy < tol * tol) return true;
            }
        }
    }
    return false;
}

}  // namespace mixed
}  // namespace grrt_b200
