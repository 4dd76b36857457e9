// Host build of the device math headers, so CPU tests can check the kernels'
// right-hand side and integrator step against the oracle. Test-only.
#include "../../grrt_b200/csrc/device/integrate.cuh"
#include "../../grrt_b200/csrc/device/mixed_spec.cuh"
#include "../../grrt_b200/csrc/device/surrogate_geom.cuh"
#include "../../grrt_b200/csrc/device/vol_steps.cuh"

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


// One tracker step of the speculative pass: tr = (disk_on, r_in, r_out,
// margin, r_near, a, p_t, p_phi), y and y5 = (r, theta, phi, p_r, p_theta),
// h the step length. Returns 1 when the step sends the sample to the re-trace.
// out[0] = cos^2 of the theta turning colatitude at y5 (Carter constant).
int devmath_tracker_step(const double* tr, const double* y, const double* y5, double h, double* out) {
    mixed::Tracker t;
    t.reset(tr[0] != 0.0, tr[1], tr[2], tr[3], tr[4], tr[5], tr[6], tr[7], y[1]);
    const Vec5<double> a{y[0], y[1], y[2], y[3], y[4]}, b{y5[0], y5[1], y5[2], y5[3], y5[4]};
    float s5, c5;
    fast_sincos(static_cast<float>(b.th), s5, c5);
    out[0] = t.turning_cos2(b.pth, s5, c5);
    return t.step(a, b, h) ? 1 : 0;
}

// The mixed form's speculative pass for one sample, as mixed_speculate_kernel
// and mixed_star_kernel run it. sc = (M, a, r_stop, r_escape, dl0, tol_fp32,
// max_steps, r_in, r_out, margin, r_near, disk_on, stars_on); star arrays may
// be null when stars_on is 0. Returns 1 when the sample goes to the FP64
// re-trace, 0 when its colour is final (exactly 0); *term_out = the
// speculative termination (-1 when it stopped early for the re-trace).
int devmath_speculate(const double* sc, const double* y8, const double* st_th, const double* st_ph,
                      const int* cells, const int* items, double tol2, int* term_out) {
    const double M = sc[0], a = sc[1], r_stop = sc[2], r_esc = sc[3], dl0 = sc[4], tol32 = sc[5];
    const int max_steps = static_cast<int>(sc[6]);
    const bool disk_on = sc[11] != 0.0, stars_on = sc[12] != 0.0;
    const double pt = y8[4], pph = y8[7];
    Vec5<double> y{y8[1], y8[2], y8[3], y8[5], y8[6]};
    double dl = dl0;
    int retry = 0, step = 0;
    mixed::Tracker trk;
    trk.reset(disk_on, sc[7], sc[8], sc[9], sc[10], a, pt, pph, y.th);
    Vec5<float> k7{};
    *term_out = -1;
    // black sky: a ray whose closed-form smallest radius lies outside the disk,
    // r_near and every photon orbit is final at once (as the kernel)
    if (!stars_on) {
        const double p[4] = {y8[4], y8[5], y8[6], y8[7]};
        const double r_gate = fmax(fmax(mixed::kEscapeRMin * M, sc[10]), disk_on ? sc[8] + 2.0 * sc[9] : 0.0);
        if (surr::camera_ray_clears(M, a, r_stop - 0.01, y8[1], y8[2], p, r_gate)) {
            *term_out = kTermEscaped;
            return 0;
        }
    }
    while (true) {
        if (retry == 0) {
            if (step >= max_steps) { *term_out = kTermMaxSteps; return 1; }
            if (y.r < r_stop) { *term_out = kTermHorizon; return 0; }
            if (y.r > r_esc) break;
        }
        Vec5<double> y5;
        const double err = mixed_attempt_impl(float(M), float(a), float(pt), float(pph), y, dl, y5, k7);
        const StepDecision d = pi_control_f32(err, tol32, dl, retry, y5.r);
        if (d.accept) {
            const bool hit = trk.step(y, y5, dl);
            y = y5;
            if (hit) return 1;
            dl = d.next;
            retry = 0;
            ++step;
            // black sky: a certain escape is final (as mixed_speculate_kernel)
            if (!stars_on && !(y.r > r_esc) &&
                mixed::certain_escape(y, fmax(fmax(mixed::kEscapeRMin * M, sc[10]), disk_on ? sc[8] + 2.0 * sc[9] : 0.0),
                                      step, max_steps)) {
                *term_out = kTermEscaped;
                return 0;
            }
        } else {
            dl = d.next;
            ++retry;
        }
    }
    *term_out = kTermEscaped;
    if (!stars_on) return 0;
    DevStars st;
    st.theta = st_th;
    st.phi = st_ph;
    st.cell_start = cells;
    st.cell_items = items;
    st.tol2 = tol2;
    return mixed::star_in_reach(st, mixed::escape_arc(r_esc, y, k7)) ? 1 : 0;
}

// A full adaptive trace of one camera ray to termination with the FP64 DP45
// attempt (mode bit 1 clear) or the FP32 mixed attempt (bit 1 set), taking k1
// from the previous attempt (bit 0 set) or evaluating it afresh every attempt
// (bit 0 clear), as the kernels do. sc = (M, a, r_stop, r_escape, dl0, tol,
// max_steps). out8 = (termination, accepted steps, attempts, r, theta, phi,
// p_r, p_theta) at the end.
void devmath_trace_final(const double* sc, const double* y8, int mode, double* out8) {
    const double M = sc[0], a = sc[1], r_stop = sc[2], r_esc = sc[3], dl0 = sc[4], tol = sc[5];
    const int max_steps = static_cast<int>(sc[6]);
    const bool reuse = (mode & 1) != 0, f32 = (mode & 2) != 0;
    const double pt = y8[4], pph = y8[7];
    Vec5<double> y{y8[1], y8[2], y8[3], y8[5], y8[6]};
    Vec5<double> k1{};
    Vec5<float> k1f{};
    bool k1_ok = false;
    double dl = dl0;
    int retry = 0, step = 0, attempts = 0, term = -1;
    while (true) {
        if (retry == 0) {
            if (step >= max_steps) { term = kTermMaxSteps; break; }
            if (y.r < r_stop) { term = kTermHorizon; break; }
            if (y.r > r_esc) { term = kTermEscaped; break; }
        }
        Vec5<double> y5;
        double err;
        if (f32) {
            Vec5<float> k7;
            if (!reuse || !k1_ok) k1f = mixed_k1(float(M), float(a), float(pt), float(pph), y);
            err = mixed_attempt_k1(float(M), float(a), float(pt), float(pph), y, dl, k1f, y5, k7);
            k1_ok = reuse;
            const StepDecision d = pi_control(err, tol, dl, retry, y5.r);
            ++attempts;
            if (d.accept) {
                y = y5;
                k1f = k7;
                dl = d.next;
                retry = 0;
                ++step;
            } else {
                dl = d.next;
                ++retry;
            }
        } else {
            Vec5<double> k7;
            if (!reuse || !k1_ok) k1 = kerr_rhs<double>(M, a, pt, pph, y);
            err = dp45_attempt_k1<double>(M, a, pt, pph, y, dl, k1, y5, k7);
            k1_ok = reuse;
            const StepDecision d = pi_control(err, tol, dl, retry, y5.r);
            ++attempts;
            if (d.accept) {
                y = y5;
                k1 = k7;
                dl = d.next;
                retry = 0;
                ++step;
            } else {
                dl = d.next;
                ++retry;
            }
        }
    }
    out8[0] = term;
    out8[1] = step;
    out8[2] = attempts;
    out8[3] = y.r;
    out8[4] = y.th;
    out8[5] = y.ph;
    out8[6] = y.pr;
    out8[7] = y.pth;
}

// Closed-form margins of the surrogate for a camera ray y8 = (t, r, th, ph,
// p_t, p_r, p_th, p_ph): out2 = (capture margin, graze margin).
void devmath_ray_margins(double M, double a, double r_h, const double* y8, double* out2) {
    const double p[4] = {y8[4], y8[5], y8[6], y8[7]};
    const surr::RayConstants k = surr::constants(a, y8[2], p);
    out2[0] = (p[1] < 0.0) ? surr::capture_margin(M, a, k, r_h, y8[1]) : -1.0;
    out2[1] = surr::graze_margin(a, k);
}

// The black-sky gate both ways for a camera ray: out2 = (smallest radius by
// the full scan and bisection, whether the scan stopped at r_gate clears it).
void devmath_gate(double M, double a, double r_h, const double* y8, double r_gate, double* out2) {
    const double p[4] = {y8[4], y8[5], y8[6], y8[7]};
    out2[0] = surr::camera_ray_min_radius(M, a, r_h, y8[1], y8[2], p);
    out2[1] = surr::camera_ray_clears(M, a, r_h, y8[1], y8[2], p, r_gate) ? 1.0 : 0.0;
}

// The surrogate's training trace (the FP64 method, as the thin-disk kernel)
// of one camera ray: sc = (M, a, r_stop, r_escape, dl0, tol, max_steps, r_cut).
// out = (termination, crossings outside r_cut, first and second such radius,
// accepted steps, crossings after the second in time order outside r_cut).
void devmath_trace_crossings(const double* sc, const double* y8, double* out) {
    const double M = sc[0], a = sc[1], r_stop = sc[2], r_esc = sc[3], dl0 = sc[4], tol = sc[5], r_cut = sc[7];
    const int max_steps = static_cast<int>(sc[6]);
    const double pt = y8[4], pph = y8[7];
    Vec5<double> y{y8[1], y8[2], y8[3], y8[5], y8[6]};
    double dl = dl0, r1 = 0.0, r2 = 0.0;
    int retry = 0, step = 0, nc = 0, term = -1, n_all = 0, n_extra = 0;
    while (true) {
        if (retry == 0) {
            if (step >= max_steps) { term = kTermMaxSteps; break; }
            if (y.r < r_stop) { term = kTermHorizon; break; }
            if (y.r > r_esc) { term = kTermEscaped; break; }
        }
        Vec5<double> y5;
        const double err = dp45_attempt<double>(M, a, pt, pph, y, dl, y5);
        const StepDecision d = pi_control(err, tol, dl, retry, y5.r);
        if (d.accept) {
            const double dp = y.th - 0.5 * mixed::kPi, dn = y5.th - 0.5 * mixed::kPi;
            if (dp * dn < 0.0 && fabs(dp - dn) > 1e-12) {
                const double rc = y.r + (-dp / (dn - dp)) * (y5.r - y.r);
                if (n_all >= 2 && rc >= r_cut) ++n_extra;
                ++n_all;
                if (rc >= r_cut) {
                    if (nc == 0) r1 = rc;
                    else if (nc == 1) r2 = rc;
                    ++nc;
                }
            }
            y = y5;
            dl = d.next;
            retry = 0;
            ++step;
        } else {
            dl = d.next;
            ++retry;
        }
    }
    out[0] = term;
    out[1] = nc;
    out[2] = r1;
    out[3] = r2;
    out[4] = step;
    out[5] = n_extra;
}

// The spectral kernel's work order: out[k] = the item taken k-th, k < total.
void devmath_vol_spread_order(unsigned total, unsigned* out) {
    for (unsigned k = 0; k < total; ++k) out[k] = vol_spread_order(k, total);
}

unsigned devmath_vol_spread() { return kVolSpread; }
}
