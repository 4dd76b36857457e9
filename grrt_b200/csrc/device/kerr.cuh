// Kerr null-geodesic right-hand side in Boyer-Lindquist coordinates, for the
// Hamiltonian form H = 1/2 g^{mu nu} p_mu p_nu with covariant momenta.
//
// Follows Kerr::compute_derivatives_inline (include/grrt/spacetime/kerr.h:31-109):
// same metric, same analytic derivatives, same pole clamp and the same
// Cody-Waite/Cephes sin-cos (include/grrt/math/fast_trig.h:21-82). The algebra
// is rearranged for the GPU: the (t,phi) block inverse and the r/theta terms
// share 1/Sigma and 1/det, and 1/Delta cancels against dx^r = Delta p_r / Sigma,
// so one evaluation needs two divisions instead of seventeen. The result equals
// the reference expression up to rounding (a few ulp per evaluation).
//
// State layout: r, theta, phi, p_r, p_theta; p_t and p_phi are constants of
// motion (dp_t = dp_phi = 0) and t does not feed back, so neither is integrated.
#pragma once

#include <cuda_runtime.h>

namespace grrt_b200 {

template <typename T>
struct Vec5 {
    T r, th, ph, pr, pth;
};

// Cody-Waite reduction to [-pi/4, pi/4], then the degree-11/10 Cephes
// polynomials (public-domain coefficients, S. Moshier), as fast_trig.h:21-82.
__device__ __forceinline__ void fast_sincos(double x, double& s, double& c) {
    constexpr double DP1 = 7.85398125648498535156e-1, DP2 = 3.77489470793079817668e-8,
                     DP3 = 2.69515142907905952645e-15, FOPI = 1.27323954473516268615;
    constexpr double S0 = -1.66666666666666324348e-01, S1 = 8.33333333332248946124e-03,
                     S2 = -1.98412698298579493134e-04, S3 = 2.75573137070700676789e-06,
                     S4 = -2.50507602534068634195e-08, S5 = 1.58969099521155010221e-10;
    constexpr double C0 = 4.16666666666666019037e-02, C1 = -1.38888888888741095749e-03,
                     C2 = 2.48015872894767294178e-05, C3 = -2.75573143513906633035e-07,
                     C4 = 2.08757232129817482790e-09, C5 = -1.13596475577881948265e-11;
    double ax = fabs(x);
    const bool neg = x < 0.0;
    int j = static_cast<int>(ax * FOPI);
    j = (j + 1) & ~1;
    const double y = static_cast<double>(j);
    ax = ((ax - y * DP1) - y * DP2) - y * DP3;
    int oct = j & 7;
    bool flip_s = neg, flip_c = false;
    if (oct > 3) { flip_s = !flip_s; flip_c = !flip_c; oct -= 4; }
    if (oct > 1) flip_c = !flip_c;
    const double z = ax * ax;
    const double ps = ((((S5 * z + S4) * z + S3) * z + S2) * z + S1) * z + S0;
    const double pc = (((((C5 * z + C4) * z + C3) * z + C2) * z + C1) * z + C0);
    const double sr = ax + ax * z * ps;
    const double cr = 1.0 - 0.5 * z + z * z * pc;
    const bool swap = (oct == 1 || oct == 2);
    const double sv = swap ? cr : sr;
    const double cv = swap ? sr : cr;
    s = flip_s ? -sv : sv;
    c = flip_c ? -cv : cv;
}

// FP32 counterpart for the mixed form: CUDA's single-precision sincosf
// (full range reduction, a few ulp).
__device__ __forceinline__ void fast_sincos(float x, float& s, float& c) { sincosf(x, &s, &c); }

// Returns dx/dlambda and dp/dlambda for (r, theta, phi, p_r, p_theta) given the
// constants p_t, p_phi.
template <typename T>
__device__ __forceinline__ Vec5<T> kerr_rhs(T M, T a, T pt, T pph, const Vec5<T>& y) {
    const T r = y.r;
    T s, c;
    fast_sincos(y.th, s, c);
    if (fabs(s) < T(1e-10)) s = (s >= T(0)) ? T(1e-10) : T(-1e-10);
    const T r2 = r * r, a2 = a * a;
    const T s2 = s * s, c2 = c * c;
    const T s2t = T(2) * s * c;
    const T Mr = M * r;
    const T Sigma = r2 + a2 * c2;
    const T Delta = r2 - T(2) * Mr + a2;
    const T iS = T(1) / Sigma;
    const T iS2 = iS * iS;
    // covariant (t, phi) block
    const T two_Mr_iS = T(2) * Mr * iS;
    const T g_tt = two_Mr_iS - T(1);
    const T g_tphi = -two_Mr_iS * a * s2;
    const T g_phph = (r2 + a2 + two_Mr_iS * a2 * s2) * s2;
    const T idet = T(1) / (g_tt * g_phph - g_tphi * g_tphi);
    // dx^mu = g^{mu nu} p_nu
    const T dt = (g_phph * pt - g_tphi * pph) * idet;
    const T dph = (g_tt * pph - g_tphi * pt) * idet;
    const T dr = Delta * iS * y.pr;
    const T dth = iS * y.pth;
    // -dH/dr
    const T Sm = Sigma - T(2) * r2;
    const T dgtt_r = T(2) * M * Sm * iS2;
    const T dgtp_r = -a * s2 * dgtt_r;
    const T dgpp_r = T(2) * r * s2 + a2 * s2 * s2 * dgtt_r;
    const T grr_r_pr2 = (T(2) * r * Delta - T(2) * Sigma * (r - M)) * iS2 * y.pr * y.pr;
    const T dp_r = T(0.5) * (dgtt_r * dt * dt + T(2) * dgtp_r * dt * dph + grr_r_pr2
                             + T(2) * r * dth * dth + dgpp_r * dph * dph);
    // -dH/dtheta
    const T k = T(2) * Mr * a2 * s2t * iS2;  // d g_tt / d theta
    const T dgtp_th = -T(2) * Mr * a * s2t * (Sigma + a2 * s2) * iS2;
    const T grr_th_pr2 = -a2 * s2t * Delta * iS2 * y.pr * y.pr;
    const T dgpp_th = (r2 + a2) * s2t + k * s2 * (T(2) * Sigma + a2 * s2);
    const T dp_th = T(0.5) * (k * dt * dt + T(2) * dgtp_th * dt * dph + grr_th_pr2
                              - a2 * s2t * dth * dth + dgpp_th * dph * dph);
    return Vec5<T>{dr, dth, dph, dp_r, dp_th};
}

}  // namespace grrt_b200
