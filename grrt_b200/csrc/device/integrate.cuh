// Dormand-Prince 5(4) attempt and the PI step controller, one attempt per
// call, so a warp advances all its rays in lock-step at attempt granularity.
//
// Method and constants follow RK4::step_kerr_rkdp45
// (include/grrt/geodesic/rk4.h:73-177) and RK4::adaptive_step_kerr_dp45
// (src/rk4.cpp:87-136): Butcher tableau of Dormand & Prince (1980), the
// 5th-order solution is kept, the error is y5 - y4 evaluated with k7 = f(y5),
// the norm is the max over r, theta, phi, p_r, p_theta of |e|/(|y5|+1e-10)
// (the p_t and p_phi terms of the reference norm are identically zero).
#pragma once

#include "kerr.cuh"

namespace grrt_b200 {

// Dormand-Prince (1980) tableau.
namespace dp {
constexpr double a21 = 1.0 / 5.0;
constexpr double a31 = 3.0 / 40.0, a32 = 9.0 / 40.0;
constexpr double a41 = 44.0 / 45.0, a42 = -56.0 / 15.0, a43 = 32.0 / 9.0;
constexpr double a51 = 19372.0 / 6561.0, a52 = -25360.0 / 2187.0, a53 = 64448.0 / 6561.0,
                 a54 = -212.0 / 729.0;
constexpr double a61 = 9017.0 / 3168.0, a62 = -355.0 / 33.0, a63 = 46732.0 / 5247.0,
                 a64 = 49.0 / 176.0, a65 = -5103.0 / 18656.0;
constexpr double b1 = 35.0 / 384.0, b3 = 500.0 / 1113.0, b4 = 125.0 / 192.0,
                 b5 = -2187.0 / 6784.0, b6 = 11.0 / 84.0;
constexpr double e1 = 71.0 / 57600.0, e3 = -71.0 / 16695.0, e4 = 71.0 / 1920.0,
                 e5 = -17253.0 / 339200.0, e6 = 22.0 / 525.0, e7 = -1.0 / 40.0;
}  // namespace dp

template <typename T>
GRRT_HD Vec5<T> axpy(const Vec5<T>& y, T h, const Vec5<T>& k) {
    return Vec5<T>{y.r + h * k.r, y.th + h * k.th, y.ph + h * k.ph, y.pr + h * k.pr, y.pth + h * k.pth};
}

// Classic RK4 step (include/grrt/geodesic/rk4.h:34-52).
template <typename T>
GRRT_HD Vec5<T> rk4_step(T M, T a, T pt, T pph, const Vec5<T>& y, T h) {
    const Vec5<T> k1 = kerr_rhs<T>(M, a, pt, pph, y);
    const Vec5<T> k2 = kerr_rhs<T>(M, a, pt, pph, axpy(y, h * T(0.5), k1));
    const Vec5<T> k3 = kerr_rhs<T>(M, a, pt, pph, axpy(y, h * T(0.5), k2));
    const Vec5<T> k4 = kerr_rhs<T>(M, a, pt, pph, axpy(y, h, k3));
    const T w = h / T(6);
#define GRRT_RK4C(f) y.f + (k1.f + T(2) * k2.f + T(2) * k3.f + k4.f) * w
    return Vec5<T>{GRRT_RK4C(r), GRRT_RK4C(th), GRRT_RK4C(ph), GRRT_RK4C(pr), GRRT_RK4C(pth)};
#undef GRRT_RK4C
}

// One DP45 attempt with k1 = f(y) given by the caller: returns the error
// norm, the 5th-order state in y5 and k7 = f(y5). The reference evaluates
// f(y) afresh at every attempt; mathematically it is the previous accepted
// attempt's k7 (same state, same constants) or the rejected attempt's k1
// (same state), so a caller that keeps it evaluates six right-hand sides per
// attempt instead of seven. Without FMA contraction the kept value is
// bit-identical to a fresh one; the device compiler may contract each inlined
// copy of the right-hand side differently, so on the GPU the two can differ
// in the last bits (the method and its step decisions are unchanged).
template <typename T>
GRRT_HD T dp45_attempt_k1(T M, T a, T pt, T pph, const Vec5<T>& y, T h, const Vec5<T>& k1, Vec5<T>& y5,
                          Vec5<T>& k7_out) {
    using namespace dp;
#define GRRT_S2(f) y.f + h * (T(a21) * k1.f)
    const Vec5<T> k2 = kerr_rhs<T>(M, a, pt, pph, Vec5<T>{GRRT_S2(r), GRRT_S2(th), GRRT_S2(ph), GRRT_S2(pr), GRRT_S2(pth)});
#define GRRT_S3(f) y.f + h * (T(a31) * k1.f + T(a32) * k2.f)
    const Vec5<T> k3 = kerr_rhs<T>(M, a, pt, pph, Vec5<T>{GRRT_S3(r), GRRT_S3(th), GRRT_S3(ph), GRRT_S3(pr), GRRT_S3(pth)});
#define GRRT_S4(f) y.f + h * (T(a41) * k1.f + T(a42) * k2.f + T(a43) * k3.f)
    const Vec5<T> k4 = kerr_rhs<T>(M, a, pt, pph, Vec5<T>{GRRT_S4(r), GRRT_S4(th), GRRT_S4(ph), GRRT_S4(pr), GRRT_S4(pth)});
#define GRRT_S5(f) y.f + h * (T(a51) * k1.f + T(a52) * k2.f + T(a53) * k3.f + T(a54) * k4.f)
    const Vec5<T> k5 = kerr_rhs<T>(M, a, pt, pph, Vec5<T>{GRRT_S5(r), GRRT_S5(th), GRRT_S5(ph), GRRT_S5(pr), GRRT_S5(pth)});
#define GRRT_S6(f) y.f + h * (T(a61) * k1.f + T(a62) * k2.f + T(a63) * k3.f + T(a64) * k4.f + T(a65) * k5.f)
    const Vec5<T> k6 = kerr_rhs<T>(M, a, pt, pph, Vec5<T>{GRRT_S6(r), GRRT_S6(th), GRRT_S6(ph), GRRT_S6(pr), GRRT_S6(pth)});
#define GRRT_Y5(f) y.f + h * (T(b1) * k1.f + T(b3) * k3.f + T(b4) * k4.f + T(b5) * k5.f + T(b6) * k6.f)
    y5 = Vec5<T>{GRRT_Y5(r), GRRT_Y5(th), GRRT_Y5(ph), GRRT_Y5(pr), GRRT_Y5(pth)};
#define GRRT_E6(f) (T(e1) * k1.f + T(e3) * k3.f + T(e4) * k4.f + T(e5) * k5.f + T(e6) * k6.f)
    Vec5<T> e = Vec5<T>{GRRT_E6(r), GRRT_E6(th), GRRT_E6(ph), GRRT_E6(pr), GRRT_E6(pth)};
#undef GRRT_S2
#undef GRRT_S3
#undef GRRT_S4
#undef GRRT_S5
#undef GRRT_S6
#undef GRRT_Y5
#undef GRRT_E6
    const Vec5<T> k7 = kerr_rhs<T>(M, a, pt, pph, y5);
    k7_out = k7;
    // err = max |h (sum e_i k_i)| / (|y5| + 1e-10); max written as the
    // standard library's (a < b) ? b : a so a NaN term is skipped as there.
    // The largest quotient is picked by cross-multiplied comparisons
    // (numerators >= 0, denominators > 0) and divided once: the same value as
    // dividing each and taking the maximum, but for quotients within a rounding
    // of each other, where either may be taken. A NaN term fails every
    // comparison and is skipped.
    T num = T(0), den = T(1);
#define GRRT_ERR(f)                                            \
    {                                                          \
        const T n_ = fabs(h * (e.f + T(e7) * k7.f));           \
        const T d_ = fabs(y5.f) + T(1e-10);                    \
        if (num * d_ < n_ * den) {                             \
            num = n_;                                          \
            den = d_;                                          \
        }                                                      \
    }
    GRRT_ERR(r) GRRT_ERR(th) GRRT_ERR(ph) GRRT_ERR(pr) GRRT_ERR(pth)
#undef GRRT_ERR
    return num / den;
}

// One DP45 attempt from scratch: returns the 5th-order state in y5 and the error norm.
template <typename T>
GRRT_HD T dp45_attempt(T M, T a, T pt, T pph, const Vec5<T>& y, T h, Vec5<T>& y5) {
    const Vec5<T> k1 = kerr_rhs<T>(M, a, pt, pph, y);
    Vec5<T> k7;
    return dp45_attempt_k1<T>(M, a, pt, pph, y, h, k1, y5, k7);
}

// f(y) in FP32 as the mixed-precision attempt forms it (state rounded to FP32).
GRRT_HD Vec5<float> mixed_k1(float M, float a, float pt, float pph, const Vec5<double>& y) {
    const Vec5<float> yf{static_cast<float>(y.r), static_cast<float>(y.th), static_cast<float>(y.ph),
                         static_cast<float>(y.pr), static_cast<float>(y.pth)};
    return kerr_rhs<float>(M, a, pt, pph, yf);
}

// Packed FP32 pairs: sm_100's two-wide FP32 fused multiply-add and multiply,
// one instruction for two lanes, each lane rounded as fmaf / the float
// product (elsewhere the lanes are computed one by one, with the same results).
GRRT_HD float2 pk(float x, float y) { return make_float2(x, y); }
GRRT_HD float2 pk_fma(float2 a, float2 b, float2 c) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    return __ffma2_rn(a, b, c);
#else
    return make_float2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y));
#endif
}
GRRT_HD float2 pk_mul(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    return __fmul2_rn(a, b);
#else
    return make_float2(a.x * b.x, a.y * b.y);
#endif
}

// A 5-vector as two packed pairs (r, theta), (phi, p_r) and p_theta alone.
struct Pk5 {
    float2 a, b;
    float c;
};
GRRT_HD Pk5 pack5(const Vec5<float>& v) { return Pk5{pk(v.r, v.th), pk(v.ph, v.pr), v.pth}; }
GRRT_HD Vec5<float> unpack5(const Pk5& v) { return Vec5<float>{v.a.x, v.a.y, v.b.x, v.b.y, v.c}; }
// c * v, and c * v + w, per component
GRRT_HD Pk5 pk5_mul(float c, const Pk5& v) {
    const float2 cc = pk(c, c);
    return Pk5{pk_mul(cc, v.a), pk_mul(cc, v.b), c * v.c};
}
GRRT_HD Pk5 pk5_fma(float c, const Pk5& v, const Pk5& w) {
    const float2 cc = pk(c, c);
    return Pk5{pk_fma(cc, v.a, w.a), pk_fma(cc, v.b, w.b), fmaf(c, v.c, w.c)};
}

// Mixed-precision attempt: the seven right-hand sides and the stage sums in
// FP32, the state and its update in FP64 (y5 = y + double(h * sum b_i k_i)),
// so round-off does not accumulate along the ray. The error norm is formed in
// FP32; its noise floor (about 1e-7 of |h k|/|y|) is why FP32 steps are
// controlled against their own tolerance (DevScene::tol_fp32). The stage sums
// run on packed pairs (three lanes of work for five components): each stage
// state is y + h * (sum_j a_sj k_j), the sum accumulated in the tableau's
// order with fused multiply-adds.
// k1 = mixed_k1(y) is given by the caller (the previous accepted attempt's
// k7, which is f at float(y5) = float(new y), or the rejected attempt's k1).
GRRT_HD double mixed_attempt_k1(float M, float a, float pt, float pph, const Vec5<double>& y, double dl,
                                const Vec5<float>& k1v, Vec5<double>& y5, Vec5<float>& k7_out) {
    using namespace dp;
    const Pk5 Y = pack5(Vec5<float>{static_cast<float>(y.r), static_cast<float>(y.th), static_cast<float>(y.ph),
                                    static_cast<float>(y.pr), static_cast<float>(y.pth)});
    const float h = static_cast<float>(dl);
    // y + h * s
    auto stage = [&](const Pk5& sum) { return unpack5(pk5_fma(h, sum, Y)); };
    const Pk5 K1 = pack5(k1v);
    const Pk5 K2 = pack5(kerr_rhs<float>(M, a, pt, pph, stage(pk5_mul(float(a21), K1))));
    const Pk5 K3 = pack5(kerr_rhs<float>(M, a, pt, pph, stage(pk5_fma(float(a32), K2, pk5_mul(float(a31), K1)))));
    const Pk5 K4 = pack5(kerr_rhs<float>(
        M, a, pt, pph, stage(pk5_fma(float(a43), K3, pk5_fma(float(a42), K2, pk5_mul(float(a41), K1))))));
    const Pk5 K5 = pack5(kerr_rhs<float>(
        M, a, pt, pph,
        stage(pk5_fma(float(a54), K4, pk5_fma(float(a53), K3, pk5_fma(float(a52), K2, pk5_mul(float(a51), K1)))))));
    const Pk5 K6 = pack5(kerr_rhs<float>(
        M, a, pt, pph,
        stage(pk5_fma(float(a65), K5,
                      pk5_fma(float(a64), K4,
                              pk5_fma(float(a63), K3, pk5_fma(float(a62), K2, pk5_mul(float(a61), K1))))))));
    const Pk5 B = pk5_fma(float(b6), K6,
                          pk5_fma(float(b5), K5, pk5_fma(float(b4), K4, pk5_fma(float(b3), K3, pk5_mul(float(b1), K1)))));
    const Pk5 I = Pk5{pk_mul(pk(h, h), B.a), pk_mul(pk(h, h), B.b), h * B.c};
    y5 = Vec5<double>{y.r + double(I.a.x), y.th + double(I.a.y), y.ph + double(I.b.x), y.pr + double(I.b.y),
                      y.pth + double(I.c)};
    const Pk5 E = pk5_fma(float(e6), K6,
                          pk5_fma(float(e5), K5, pk5_fma(float(e4), K4, pk5_fma(float(e3), K3, pk5_mul(float(e1), K1)))));
    const Vec5<float> y5f{static_cast<float>(y5.r), static_cast<float>(y5.th), static_cast<float>(y5.ph),
                          static_cast<float>(y5.pr), static_cast<float>(y5.pth)};
    const Vec5<float> k7 = kerr_rhs<float>(M, a, pt, pph, y5f);
    k7_out = k7;
    const Vec5<float> ev = unpack5(pk5_fma(float(e7), pack5(k7), E));
    float err = 0.0f;
#define GRRT_ERRF(f)                                                       \
    {                                                                      \
        const float v = fabsf(h * ev.f) * recip(fabsf(y5f.f) + 1e-10f);    \
        err = (err < v) ? v : err;                                         \
    }
    GRRT_ERRF(r) GRRT_ERRF(th) GRRT_ERRF(ph) GRRT_ERRF(pr) GRRT_ERRF(pth)
#undef GRRT_ERRF
    return static_cast<double>(err);
}

GRRT_HD double mixed_attempt_impl(float M, float a, float pt, float pph, const Vec5<double>& y, double dl,
                                  Vec5<double>& y5, Vec5<float>& k7_out) {
    return mixed_attempt_k1(M, a, pt, pph, y, dl, mixed_k1(M, a, pt, pph, y), y5, k7_out);
}

// Outcome of the controller after one attempt (src/rk4.cpp:87-136).
struct StepDecision {
    bool accept;    // take y5 and start a new outer step
    double next;    // accepted: step size for the next outer step; rejected: the new trial size
};

// (tol/err)^0.2 for the step-size factor. The factor only sets the next trial
// step, on which the solution depends through the truncation error (a relative
// change d in the step moves the result by about 5 d times the local error), so
// single precision (2^-22 relative) is ample and avoids an FP64 pow per attempt.
GRRT_HD double step_factor_pow(double x) {
#ifdef __CUDA_ARCH__
    return static_cast<double>(__powf(static_cast<float>(x), 0.2f));
#else
    return static_cast<double>(powf(static_cast<float>(x), 0.2f));
#endif
}

// retry = number of rejected attempts so far in this outer step (0..20). The
// 21st attempt (retry == 20) is taken unconditionally with next = dl, as the
// reference's "exhausted retries" path.
GRRT_HD StepDecision pi_control(double err, double tol, double dl, int retry,
                                                   double r5) {
    constexpr double safety = 0.9, grow_max = 5.0, shrink_max = 0.2, dl_min = 1e-6;
    StepDecision d;
    const double ar = fabs(r5);
    const double cap = 5.0 * ((ar < 1.0) ? 1.0 : ar);
    if (retry >= 20) {
        d.accept = true;
        d.next = dl;
        return d;
    }
    if (err <= tol) {
        double f = (err > 1e-30) ? safety * step_factor_pow(tol / err) : grow_max;
        f = (f < 1.0) ? 1.0 : (grow_max < f) ? grow_max : f;
        const double nx = dl * f;
        d.accept = true;
        d.next = (cap < nx) ? cap : nx;
        return d;
    }
    double f = safety * step_factor_pow(tol / err);
    f = (f < shrink_max) ? shrink_max : (1.0 < f) ? 1.0 : f;
    const double ndl = dl * f;
    if (ndl < dl_min) {
        d.accept = true;
        d.next = (cap < dl_min) ? cap : dl_min;
        return d;
    }
    d.accept = false;
    d.next = ndl;
    return d;
}

// The FP32 pass's controller: pi_control with (tol/err)^0.2 formed from a
// single-precision quotient (the FP32 error norm carries no more digits).
GRRT_HD double step_factor_ratio(double tol, double err) {
#ifdef __CUDA_ARCH__
    return static_cast<double>(__powf(__fdividef(static_cast<float>(tol), static_cast<float>(err)), 0.2f));
#else
    return static_cast<double>(powf(static_cast<float>(tol) / static_cast<float>(err), 0.2f));
#endif
}

GRRT_HD StepDecision pi_control_f32(double err, double tol, double dl, int retry,
                                                   double r5) {
    constexpr double safety = 0.9, grow_max = 5.0, shrink_max = 0.2, dl_min = 1e-6;
    StepDecision d;
    const double ar = fabs(r5);
    const double cap = 5.0 * ((ar < 1.0) ? 1.0 : ar);
    if (retry >= 20) {
        d.accept = true;
        d.next = dl;
        return d;
    }
    if (err <= tol) {
        double f = (err > 1e-30) ? safety * step_factor_ratio(tol, err) : grow_max;
        f = (f < 1.0) ? 1.0 : (grow_max < f) ? grow_max : f;
        const double nx = dl * f;
        d.accept = true;
        d.next = (cap < nx) ? cap : nx;
        return d;
    }
    double f = safety * step_factor_ratio(tol, err);
    f = (f < shrink_max) ? shrink_max : (1.0 < f) ? 1.0 : f;
    const double ndl = dl * f;
    if (ndl < dl_min) {
        d.accept = true;
        d.next = (cap < dl_min) ? cap : dl_min;
        return d;
    }
    d.accept = false;
    d.next = ndl;
    return d;
}

}  // namespace grrt_b200
