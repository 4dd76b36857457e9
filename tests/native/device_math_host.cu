// Host build of the device math headers, so CPU tests can check the kernels'
// right-hand side and integrator step against the oracle. Test-only.
#include "../../grrt_b200/csrc/device/integrate.cuh"

using namespace grrt_b200;

extern "C" {

// y8 = (t, r, th, ph, p_t, p_r, p_th, p_ph) -> out5 = (dr, dth, dph, dp_r, dp_th)
void devmath_rhs(double M, double a, const double* y8, double* out5) {
    const Vec5<double> y{y8[1], y8[2], y8[3], y8[5], y8[6]};
    const Vec5<double> d = kerr_rhs<double>(M, a, y8[4], y8[7], y);
    out5[0] = d.r; out5[1] = d.th; out5[2] = d.ph; out5[3] = d.pr; out5[4] = d.pth;
}

void devmath_rhs_f32(double M, double a, const double* y8, double* out5) {
    const Vec5<float> y{float(y8[1]), float(y8[2]), float(y8[3]), float(y8[5]), float(y8[6])};
    const Vec5<float> d = kerr_rhs<float>(float(M), float(a), float(y8[4]), float(y8[7]), y);
    out5[0] = d.r; out5[1] = d.th; out5[2] = d.ph; out5[3] = d.pr; out5[4] = d.pth;
}

// One DP45 attempt: returns the error norm, y5 in out5.
double devmath_dp45(double M, double a, const double* y8, double h, double* out5) {
    const Vec5<double> y{y8[1], y8[2], y8[3], y8[5], y8[6]};
    Vec5<double> y5;
    const double err = dp45_attempt<double>(M, a, y8[4], y8[7], y, h, y5);
    out5[0] = y5.r; out5[1] = y5.th; out5[2] = y5.ph; out5[3] = y5.pr; out5[4] = y5.pth;
    return err;
}

}
