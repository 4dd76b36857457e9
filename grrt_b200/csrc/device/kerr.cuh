// Kerr null-geodesic right-hand side in Boyer-Lindquist coordinates, for the
// Hamiltonian H = 1/2 g^{mu nu} p_mu p_nu with covariant momenta: the same
// equations as Kerr::compute_derivatives_inline
// (include/grrt/spacetime/kerr.h:31-109), with the same pole clamp of sin(theta)
// and the same Cody-Waite/Cephes sin-cos (include/grrt/math/fast_trig.h:21-82).
//
// The Kerr inverse metric separates (Carter): with
//     P(r) = (r^2 + a^2) p_t + a p_phi,   Q(theta) = a sin(theta) p_t + p_phi / sin(theta),
//     2 Sigma H = F(r) + G(theta),  F = Delta p_r^2 - P^2 / Delta,  G = p_theta^2 + Q^2,
// so dx/dlambda = dH/dp and dp/dlambda = -dH/dx follow from F, G and their
// derivatives with one division (1/(Sigma Delta sin)) instead of the
// reference's seventeen. The value is the reference's function; the rounding
// differs by a few ulp per evaluation. The identity is checked against the
// reference form on the CPU (tests/test_device_math.py).
//
// State layout: r, theta, phi, p_r, p_theta; p_t and p_phi are constants of
// motion (dp_t = dp_phi = 0) and t does not feed back, so neither is integrated.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

#define GRRT_HD __host__ __device__ __forceinline__
// The right-hand side is inlined at its call sites (seven per attempt) unless
// the translation unit sets GRRT_RHS_CALL_F64, which makes the FP64 one a
// call to one shared body (less code to fetch, a call per evaluation). The
// FP32 one stays inlined: its kernels are issue-bound and lose to the calls.

namespace grrt_b200 {

template <typename T>
struct Vec5 {
    T r, th, ph, pr, pth;
};

// Cody-Waite reduction to [-pi/4, pi/4], then the degree-11/10 Cephes
// polynomials (public-domain coefficients, S. Moshier), as fast_trig.h:21-82.
GRRT_HD void fast_sincos(double x, double& s, double& c) {
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

// FP32 counterpart for the mixed form: the same octant reduction with a
// three-part float pi/4 and the Cephes single-precision polynomials
// (public-domain coefficients, S. Moshier), accurate to a few float ulp for the
// |theta| < 1e4 the integrator can reach.
GRRT_HD void fast_sincos(float x, float& s, float& c) {
    constexpr float DP1 = 0.78515625f, DP2 = 2.4187564849853515625e-4f, DP3 = 3.77489497744594108e-8f;
    constexpr float FOPI = 1.27323954473516f;
    float ax = fabsf(x);
    const bool neg = x < 0.0f;
    int j = static_cast<int>(ax * FOPI);
    j = (j + 1) & ~1;
    const float y = static_cast<float>(j);
    ax = ((ax - y * DP1) - y * DP2) - y * DP3;
    int oct = j & 7;
    bool flip_s = neg, flip_c = false;
    if (oct > 3) { flip_s = !flip_s; flip_c = !flip_c; oct -= 4; }
    if (oct > 1) flip_c = !flip_c;
    const float z = ax * ax;
    const float sr = ((-1.9515295891e-4f * z + 8.3321608736e-3f) * z - 1.6666654611e-1f) * z * ax + ax;
    const float cr = ((2.443315711809948e-5f * z - 1.388731625493765e-3f) * z + 4.166664568298827e-2f) * z * z
                     - 0.5f * z + 1.0f;
    const bool swap = (oct == 1 || oct == 2);
    const float sv = swap ? cr : sr;
    const float cv = swap ? sr : cr;
    s = flip_s ? -sv : sv;
    c = flip_c ? -cv : cv;
}

// sin and cos for the right-hand side: the reference's polynomial in FP64; in
// FP32 on the device the hardware approximations (__sincosf, two
// special-function ops instead of the ~25 instructions of the polynomial; the
// FP32 form's error budget absorbs their few-ulp error), the FP32 polynomial
// on the host.
GRRT_HD void rhs_sincos(double x, double& s, double& c) { fast_sincos(x, s, c); }
GRRT_HD void rhs_sincos(float x, float& s, float& c) {
#ifdef __CUDA_ARCH__
    __sincosf(x, &s, &c);
#else
    fast_sincos(x, s, c);
#endif
}

// 1/x: IEEE division in FP64; in FP32 the hardware reciprocal approximation
// (about 1 ulp), which the FP32 form's error budget absorbs.
GRRT_HD double recip(double x) { return 1.0 / x; }
GRRT_HD float recip(float x) {
#ifdef __CUDA_ARCH__
    return __fdividef(1.0f, x);
#else
    return 1.0f / x;
#endif
}

// Returns dx/dlambda and dp/dlambda for (r, theta, phi, p_r, p_theta) given the
// constants p_t, p_phi.
template <typename T>
GRRT_HD Vec5<T> kerr_rhs_body(T M, T a, T pt, T pph, const Vec5<T>& y) {
    using std::fabs;
    const T r = y.r, pr = y.pr, pth = y.pth;
    T s, c;
    rhs_sincos(y.th, s, c);
    if (fabs(s) < T(1e-10)) s = (s >= T(0)) ? T(1e-10) : T(-1e-10);
    const T r2 = r * r, a2 = a * a;
    const T Sigma = r2 + a2 * c * c;
    const T Delta = r2 - T(2) * M * r + a2;
    const T SD = Sigma * Delta;
    const T inv = recip(SD * s);
    const T iS = Delta * s * inv;  // 1/Sigma
    const T iD = Sigma * s * inv;  // 1/Delta
    const T is = SD * inv;         // 1/sin(theta)
    const T P = (r2 + a2) * pt + a * pph;
    const T Q = a * s * pt + pph * is;
    const T PiD = P * iD;
    const T hiS = T(0.5) * iS;
    const T H = (Delta * pr * pr - P * PiD + pth * pth + Q * Q) * hiS;  // 0 on the light cone
    // dx/dlambda = dH/dp
    const T dr = Delta * pr * iS;
    const T dth = pth * iS;
    const T dph = (Q * is - a * PiD) * iS;
    // dF/dr at fixed momenta and dG/dtheta
    const T dF = T(2) * (r - M) * (pr * pr + PiD * PiD) - T(4) * r * pt * PiD;
    const T dG = T(2) * Q * c * (a * pt - pph * is * is);
    // dp/dlambda = -dH/dx, with dSigma/dr = 2r and dSigma/dtheta = -2 a^2 sin cos
    const T dpr = H * T(2) * r * iS - dF * hiS;
    const T dpth = -(dG * hiS + H * T(2) * a2 * s * c * iS);
    return Vec5<T>{dr, dth, dph, dpr, dpth};
}

// H = 1/2 g^{mu nu} p_mu p_nu at the state, in the separable form the
// right-hand side uses (2 Sigma H = Delta p_r^2 - P^2/Delta + p_theta^2 + Q^2):
// 0 on the light cone, so |H| / p_t^2 measures how far the integrated momenta
// have drifted off the null cone (the constraint the reference monitors,
// README "Physics Notes"; its CUDA tests hold |H| < 1e-7 along a geodesic).
template <typename T>
GRRT_HD T kerr_hamiltonian(T M, T a, T pt, T pph, const Vec5<T>& y) {
    using std::fabs;
    T s, c;
    rhs_sincos(y.th, s, c);
    if (fabs(s) < T(1e-10)) s = (s >= T(0)) ? T(1e-10) : T(-1e-10);
    const T r2 = y.r * y.r, a2 = a * a;
    const T Sigma = r2 + a2 * c * c;
    const T Delta = r2 - T(2) * M * y.r + a2;
    const T P = (r2 + a2) * pt + a * pph;
    const T Q = a * s * pt + pph / s;
    return (Delta * y.pr * y.pr - P * P / Delta + y.pth * y.pth + Q * Q) / (T(2) * Sigma);
}

#ifdef GRRT_RHS_CALL_F64
// The state is passed by value, so the call passes it in registers.
static __host__ __device__ __noinline__ Vec5<double> kerr_rhs_f64_call(double M, double a, double pt, double pph,
                                                                       Vec5<double> y) {
    return kerr_rhs_body<double>(M, a, pt, pph, y);
}
#endif

template <typename T>
GRRT_HD Vec5<T> kerr_rhs(T M, T a, T pt, T pph, const Vec5<T>& y) {
#ifdef GRRT_RHS_CALL_F64
    if constexpr (sizeof(T) == sizeof(double)) return kerr_rhs_f64_call(M, a, pt, pph, y);
    else
#endif
        return kerr_rhs_body<T>(M, a, pt, pph, y);
}

}  // namespace grrt_b200
