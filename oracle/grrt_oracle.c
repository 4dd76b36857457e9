/*
 * grrt_oracle.c — CPU restatement of the reference's per-pixel path.
 *
 * TEST INFRASTRUCTURE ONLY (see grrt_oracle.h). Parity pinned: tests compare
 * this file, compiled strict, bit for bit against the reference library built
 * from its own sources (oracle/_ref/libgrrt_ref_strict.so) on every table and
 * on per-sample traces.
 *
 * Each function cites the reference code it restates. Expressions keep the
 * reference's operand order and parenthesisation, so that the same IEEE
 * operations happen in the same order. min/max/clamp are written out with the
 * comparison direction of the C++ standard library so NaN propagates the same
 * way.
 */
#include "grrt_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define HALF_PI (3.141592653589793 / 2.0)
#define PI_D 3.141592653589793

static inline double max_d(double a, double b) { return (a < b) ? b : a; }   /* std::max */
static inline double min_d(double a, double b) { return (b < a) ? b : a; }   /* std::min */
static inline double clamp_d(double v, double lo, double hi) {               /* std::clamp */
    return (v < lo) ? lo : (hi < v) ? hi : v;
}
static inline int min_i(int a, int b) { return (b < a) ? b : a; }
static inline int clamp_i(int v, int lo, int hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

/* ------------------------------------------------------------------------ */
/* src/renderer.cpp:14-20                                                    */
double oracle_pixel_hash(int i, int j, int s, int ch) {
    uint32_t h = ((uint32_t)i * 73856093u) ^ ((uint32_t)j * 19349663u) ^ ((uint32_t)s * 83492791u)
                 ^ ((uint32_t)ch * 45678917u);
    h ^= h >> 16;
    h *= 0x45d9f3bu;
    h ^= h >> 16;
    return (h & 0xFFFFu) / 65536.0;
}

/* ------------------------------------------------------------------------ */
/* include/grrt/math/fast_trig.h:21-82: Cody-Waite reduction to [-pi/4, pi/4]
 * and Cephes minimax polynomials for sin and cos.                           */
void oracle_fast_sincos(double x, double* s, double* c) {
    const double DP1 = 7.85398125648498535156e-1, DP2 = 3.77489470793079817668e-8,
                 DP3 = 2.69515142907905952645e-15, FOPI = 1.27323954473516268615;
    const double S0 = -1.66666666666666324348e-01, S1 = 8.33333333332248946124e-03,
                 S2 = -1.98412698298579493134e-04, S3 = 2.75573137070700676789e-06,
                 S4 = -2.50507602534068634195e-08, S5 = 1.58969099521155010221e-10;
    const double C0 = 4.16666666666666019037e-02, C1 = -1.38888888888741095749e-03,
                 C2 = 2.48015872894767294178e-05, C3 = -2.75573143513906633035e-07,
                 C4 = 2.08757232129817482790e-09, C5 = -1.13596475577881948265e-11;
    double ax = fabs(x);
    int sign_s = (x < 0.0) ? -1 : 1;
    int sign_c = 1;
    int j = (int)(ax * FOPI);
    j = (j + 1) & ~1;
    double y = (double)j;
    ax = ((ax - y * DP1) - y * DP2) - y * DP3;
    int oct = j & 7;
    if (oct > 3) { sign_s = -sign_s; sign_c = -sign_c; oct -= 4; }
    if (oct > 1) sign_c = -sign_c;
    double z = ax * ax;
    double ps = ((((S5 * z + S4) * z + S3) * z + S2) * z + S1) * z + S0;
    double pc = (((((C5 * z + C4) * z + C3) * z + C2) * z + C1) * z + C0);
    double sr = ax + ax * z * ps;
    double cr = 1.0 - 0.5 * z + z * z * pc;
    if (oct == 1 || oct == 2) { *s = sign_s * cr; *c = sign_c * sr; }
    else { *s = sign_s * sr; *c = sign_c * cr; }
}

/* ------------------------------------------------------------------------ */
/* include/grrt/spacetime/kerr.h:31-109. y = (t, r, th, ph, p_t, p_r, p_th, p_ph). */
static void kerr_rhs(double M, double a, const double* y, double* dy) {
    const double r = y[1], theta = y[2];
    const double* p = y + 4;
    const double r2 = r * r, a2 = a * a;
    double st, ct;
    oracle_fast_sincos(theta, &st, &ct);
    if (fabs(st) < 1e-10) st = (st >= 0.0) ? 1e-10 : -1e-10;
    const double sin2 = st * st, cos2 = ct * ct, sin4 = sin2 * sin2;
    const double sin2theta = 2.0 * st * ct;
    const double Sigma = r2 + a2 * cos2;
    const double Delta = r2 - 2.0 * M * r + a2;
    const double Sigma2 = Sigma * Sigma, Delta2 = Delta * Delta;
    const double Mr = M * r;
    const double g_tt = -(1.0 - 2.0 * Mr / Sigma);
    const double g_tphi = -2.0 * M * a * r * sin2 / Sigma;
    const double g_rr = Sigma / Delta;
    const double g_thth = Sigma;
    const double g_phph = (r2 + a2 + 2.0 * M * a2 * r * sin2 / Sigma) * sin2;
    const double det_tf = g_tt * g_phph - g_tphi * g_tphi;
    const double ginv_tt = g_phph / det_tf;
    const double ginv_tphi = -g_tphi / det_tf;
    const double ginv_rr = 1.0 / g_rr;
    const double ginv_thth = 1.0 / g_thth;
    const double ginv_phph = g_tt / det_tf;
    double dx0 = ginv_tt * p[0] + ginv_tphi * p[3];
    double dx1 = ginv_rr * p[1];
    double dx2 = ginv_thth * p[2];
    double dx3 = ginv_tphi * p[0] + ginv_phph * p[3];
    const double Sm = Sigma - 2.0 * r2;
    const double dg_tt_dr = 2.0 * M * Sm / Sigma2;
    const double dg_tphi_dr = -2.0 * M * a * sin2 * Sm / Sigma2;
    const double dg_rr_dr = (2.0 * r * Delta - 2.0 * Sigma * (r - M)) / Delta2;
    const double dg_phph_dr = 2.0 * r * sin2 + 2.0 * M * a2 * sin4 * Sm / Sigma2;
    const double dp_r = 0.5 * (dg_tt_dr * dx0 * dx0 + 2.0 * dg_tphi_dr * dx0 * dx3
                               + dg_rr_dr * dx1 * dx1 + 2.0 * r * dx2 * dx2
                               + dg_phph_dr * dx3 * dx3);
    const double dg_tt_dth = 2.0 * Mr * a2 * sin2theta / Sigma2;
    const double dg_tphi_dth = -2.0 * Mr * a * sin2theta * (Sigma + a2 * sin2) / Sigma2;
    const double dg_rr_dth = -a2 * sin2theta / Delta;
    const double dg_phph_dth = (r2 + a2) * sin2theta
                               + 2.0 * Mr * a2 * sin2theta * sin2 * (2.0 * Sigma + a2 * sin2) / Sigma2;
    const double dp_th = 0.5 * (dg_tt_dth * dx0 * dx0 + 2.0 * dg_tphi_dth * dx0 * dx3
                                + dg_rr_dth * dx1 * dx1 + (-a2 * sin2theta) * dx2 * dx2
                                + dg_phph_dth * dx3 * dx3);
    dy[0] = dx0; dy[1] = dx1; dy[2] = dx2; dy[3] = dx3;
    dy[4] = 0.0; dy[5] = dp_r; dy[6] = dp_th; dy[7] = 0.0;
}

void oracle_derivatives(const OracleScene* sc, const double* y, double* dy) { kerr_rhs(sc->M, sc->a, y, dy); }

/* include/grrt/geodesic/rk4.h:34-52 — classic RK4 (ray-march steps). */
static void rk4_step(double M, double a, const double* y, double dl, double* out) {
    double k1[8], k2[8], k3[8], k4[8], t[8];
    kerr_rhs(M, a, y, k1);
    for (int i = 0; i < 8; ++i) t[i] = y[i] + k1[i] * (dl * 0.5);
    kerr_rhs(M, a, t, k2);
    for (int i = 0; i < 8; ++i) t[i] = y[i] + k2[i] * (dl * 0.5);
    kerr_rhs(M, a, t, k3);
    for (int i = 0; i < 8; ++i) t[i] = y[i] + k3[i] * dl;
    kerr_rhs(M, a, t, k4);
    for (int i = 0; i < 8; ++i) out[i] = y[i] + (k1[i] + k2[i] * 2.0 + k3[i] * 2.0 + k4[i]) * (dl / 6.0);
}

/* include/grrt/geodesic/rk4.h:73-177 — one Dormand-Prince 5(4) attempt with the
 * embedded error estimate (k7 evaluated at y5). Returns the error norm. */
static double dp45_attempt(double M, double a, const double* y, double dl, double* y5) {
    double k1[8], k2[8], k3[8], k4[8], k5[8], k6[8], k7[8], s[8];
    kerr_rhs(M, a, y, k1);
    for (int i = 0; i < 8; ++i) s[i] = y[i] + k1[i] * (dl / 5.0);
    kerr_rhs(M, a, s, k2);
    for (int i = 0; i < 8; ++i) s[i] = y[i] + k1[i] * (dl * 3.0 / 40.0) + k2[i] * (dl * 9.0 / 40.0);
    kerr_rhs(M, a, s, k3);
    for (int i = 0; i < 8; ++i)
        s[i] = y[i] + k1[i] * (dl * 44.0 / 45.0) + k2[i] * (dl * -56.0 / 15.0) + k3[i] * (dl * 32.0 / 9.0);
    kerr_rhs(M, a, s, k4);
    for (int i = 0; i < 8; ++i)
        s[i] = y[i] + k1[i] * (dl * 19372.0 / 6561.0) + k2[i] * (dl * -25360.0 / 2187.0)
               + k3[i] * (dl * 64448.0 / 6561.0) + k4[i] * (dl * -212.0 / 729.0);
    kerr_rhs(M, a, s, k5);
    for (int i = 0; i < 8; ++i)
        s[i] = y[i] + k1[i] * (dl * 9017.0 / 3168.0) + k2[i] * (dl * -355.0 / 33.0)
               + k3[i] * (dl * 46732.0 / 5247.0) + k4[i] * (dl * 49.0 / 176.0)
               + k5[i] * (dl * -5103.0 / 18656.0);
    kerr_rhs(M, a, s, k6);
    for (int i = 0; i < 8; ++i)
        y5[i] = y[i] + k1[i] * (dl * 35.0 / 384.0) + k3[i] * (dl * 500.0 / 1113.0)
                + k4[i] * (dl * 125.0 / 192.0) + k5[i] * (dl * -2187.0 / 6784.0)
                + k6[i] * (dl * 11.0 / 84.0);
    kerr_rhs(M, a, y5, k7);
    double e[8];
    for (int i = 0; i < 8; ++i)
        e[i] = k1[i] * (dl * 71.0 / 57600.0) + k3[i] * (dl * -71.0 / 16695.0)
               + k4[i] * (dl * 71.0 / 1920.0) + k5[i] * (dl * -17253.0 / 339200.0)
               + k6[i] * (dl * 22.0 / 525.0) + k7[i] * (dl * -1.0 / 40.0);
    double err = 0.0;
    for (int i = 1; i < 4; ++i) err = max_d(err, fabs(e[i]) / (fabs(y5[i]) + 1e-10));
    for (int i = 4; i < 8; ++i) err = max_d(err, fabs(e[i]) / (fabs(y5[i]) + 1e-10));
    return err;
}

/* src/rk4.cpp:87-136 — PI-controlled adaptive DP45. */
static double dp45_adaptive(double M, double a, const double* y, double dlambda, double tol,
                            double* out, long long* attempts) {
    const double dl_min = 1e-6, safety = 0.9, p_exp = 0.2, grow_max = 5.0, shrink_max = 0.2;
    double dl = dlambda;
    for (int retry = 0; retry < 20; ++retry) {
        const double err = dp45_attempt(M, a, y, dl, out);
        ++*attempts;
        if (err <= tol) {
            double f = (err > 1e-30) ? safety * pow(tol / err, p_exp) : grow_max;
            f = clamp_d(f, 1.0, grow_max);
            double next = dl * f;
            const double r = fabs(out[1]);
            next = min_d(next, 5.0 * max_d(r, 1.0));
            return next;
        }
        double f = safety * pow(tol / err, p_exp);
        f = clamp_d(f, shrink_max, 1.0);
        dl *= f;
        if (dl < dl_min) {
            const double r = fabs(out[1]);
            return min_d(dl_min, 5.0 * max_d(r, 1.0));
        }
    }
    dp45_attempt(M, a, y, dl, out);
    ++*attempts;
    return dl;
}

/* ------------------------------------------------------------------------ */
/* src/camera.cpp:69-96 */
void oracle_camera_ray(const OracleScene* sc, double x, double y, double* out) {
    const double alpha = (x - sc->width / 2.0) * sc->fov / sc->width;
    const double beta = (y - sc->height / 2.0) * sc->fov / sc->width;
    const double ca = cos(beta) * sin(alpha);
    const double cb = sin(beta);
    const double cc = cos(beta) * cos(alpha);
    double pu[4];
    for (int m = 0; m < 4; ++m) {
        const double d = -ca * sc->e1[m] - cb * sc->e2[m] + cc * sc->e3[m];
        pu[m] = -sc->e0[m] + d;
    }
    for (int m = 0; m < 4; ++m) {
        double sum = 0.0;
        for (int n = 0; n < 4; ++n) sum += sc->g[4 * m + n] * pu[n];
        out[4 + m] = sum;
        out[m] = sc->cam_pos[m];
    }
}

/* ------------------------------------------------------------------------ */
/* Thin disk: src/accretion_disk.cpp:96-147, src/spectrum.cpp:115-131 */
static double disk_flux(const OracleScene* sc, double r) {
    if (r <= sc->disk_r_inner || r >= sc->disk_r_outer || sc->flux_max <= 0.0) return 0.0;
    const int n = sc->flux_n;
    const double frac = (r - sc->disk_r_inner) / (sc->disk_r_outer - sc->disk_r_inner) * (n - 1);
    const int idx = (int)frac;
    const double t = frac - idx;
    if (idx >= n - 1) return sc->flux[n - 1];
    return sc->flux[idx] * (1.0 - t) + sc->flux[idx + 1] * t;
}

static void disk_emission(const OracleScene* sc, double r, double p0, double p3, double* col) {
    col[0] = col[1] = col[2] = 0.0;
    const double F = disk_flux(sc, r);
    if (F <= 0.0 || sc->flux_max <= 0.0) return;
    const double T = sc->peak_temperature * pow(F / sc->flux_max, 0.25);
    if (T <= 0.0) return;
    const double M = sc->M, a = sc->a;
    /* redshift */
    double g;
    {
        const double u_t_obs = 1.0 / sqrt(1.0 - 2.0 * M / sc->observer_r);
        const double pu_obs = p0 * u_t_obs;
        const double w = sqrt(M / (r * r * r));
        const double aw = a * w;
        const double u_t_emit = 1.0 / sqrt(1.0 - 3.0 * M / r + 2.0 * aw);
        const double w2 = sqrt(M / (r * r * r));
        const double Om = w2 / (1.0 + a * w2);
        const double u_phi_emit = Om * u_t_emit;
        const double pu_emit = p0 * u_t_emit + p3 * u_phi_emit;
        g = (fabs(pu_obs) < 1e-30) ? 1.0 : pu_emit / pu_obs;
    }
    const double T_obs = g * T;
    if (T_obs < 100.0) return;
    /* chromaticity */
    const double Tc = clamp_d(T_obs, sc->t_min, sc->t_max);
    const double frac = (Tc - sc->t_min) / (sc->t_max - sc->t_min) * (sc->spec_n - 1);
    const int idx = (int)frac;
    const double t = frac - idx;
    double chroma[3];
    for (int k = 0; k < 3; ++k)
        chroma[k] = (idx >= sc->spec_n - 1) ? sc->spec_color[3 * (sc->spec_n - 1) + k]
                                            : sc->spec_color[3 * idx + k] * (1.0 - t)
                                                  + sc->spec_color[3 * (idx + 1) + k] * t;
    const double ratio = T / sc->t_max;
    const double lum = ratio * ratio * ratio * ratio;
    const double g4 = g * g * g * g;
    for (int k = 0; k < 3; ++k) col[k] = chroma[k] * (lum * g4);
}

/* src/celestial_sphere.cpp:48-90: first star (scan order) within tolerance. */
static double star_sample(const OracleScene* sc, double theta, double phi) {
    theta = fmod(theta, 2.0 * PI_D);
    if (theta < 0.0) theta += 2.0 * PI_D;
    if (theta > PI_D) { theta = 2.0 * PI_D - theta; phi += PI_D; }
    phi = fmod(phi, 2.0 * PI_D);
    if (phi > PI_D) phi -= 2.0 * PI_D;
    if (phi < -PI_D) phi += 2.0 * PI_D;
    const int nt = 180, np = 360;
    const int tb = (int)(theta * nt / PI_D);
    const int pb = (int)((phi + PI_D) * np / (2.0 * PI_D));
    const double tol2 = sc->star_tol * sc->star_tol;
    for (int dt = -1; dt <= 1; ++dt)
        for (int dp = -1; dp <= 1; ++dp) {
            const int t = clamp_i(tb + dt, 0, nt - 1);
            const int p = (((pb + dp) % np) + np) % np;
            const int cell = t * np + p;
            for (int q = sc->cell_start[cell]; q < sc->cell_start[cell + 1]; ++q) {
                const int si = sc->cell_items[q];
                const double dth = theta - sc->star_theta[si];
                double dph = phi - sc->star_phi[si];
                if (dph > PI_D) dph -= 2.0 * PI_D;
                if (dph < -PI_D) dph += 2.0 * PI_D;
                const double s = sin(theta);
                const double d2 = dth * dth + dph * dph * s * s;
                if (d2 < tol2) return sc->star_b[si];
            }
        }
    return 0.0;
}

/* ------------------------------------------------------------------------ */
/* Volumetric disk queries: src/volumetric_disk.cpp:97-273 */
static double v_interp_radial(const OracleScene* sc, const double* lut, double r) {
    if (r <= sc->v_r_min) return lut[0];
    if (r >= sc->v_r_outer) return lut[sc->v_n_r - 1];
    const double frac = (r - sc->v_r_min) / (sc->v_r_outer - sc->v_r_min) * (sc->v_n_r - 1);
    const int idx = clamp_i((int)frac, 0, sc->v_n_r - 2);
    const double t = frac - idx;
    return lut[idx] * (1.0 - t) + lut[idx + 1] * t;
}

static double v_interp_2d(const OracleScene* sc, const double* lut, double r, double z_abs) {
    const int nr = sc->v_n_r, nz = sc->v_n_z;
    const double r_frac = clamp_d((r - sc->v_r_min) / (sc->v_r_outer - sc->v_r_min) * (nr - 1), 0.0,
                                  (double)(nr - 1));
    const int ri = min_i((int)r_frac, nr - 2);
    const double tr = r_frac - ri;
    const double zm_lo = sc->v_zmax[ri];
    const double zm_hi = sc->v_zmax[min_i(ri + 1, nr - 1)];
    if ((zm_lo <= 0.0 || z_abs >= zm_lo) && (zm_hi <= 0.0 || z_abs >= zm_hi)) return 0.0;
    double lo = 0.0;
    if (zm_lo > 0.0 && z_abs < zm_lo) {
        const double zf = clamp_d(z_abs / zm_lo * (nz - 1), 0.0, (double)(nz - 1));
        const int zi = min_i((int)zf, nz - 2);
        const double tz = zf - zi;
        lo = (1.0 - tz) * lut[ri * nz + zi] + tz * lut[ri * nz + zi + 1];
    }
    double hi = 0.0;
    const int ri1 = min_i(ri + 1, nr - 1);
    if (zm_hi > 0.0 && z_abs < zm_hi) {
        const double zf = clamp_d(z_abs / zm_hi * (nz - 1), 0.0, (double)(nz - 1));
        const int zi = min_i((int)zf, nz - 2);
        const double tz = zf - zi;
        hi = (1.0 - tz) * lut[ri1 * nz + zi] + tz * lut[ri1 * nz + zi + 1];
    }
    return (1.0 - tr) * lo + tr * hi;
}

static double v_scale_height(const OracleScene* sc, double r) { return v_interp_radial(sc, sc->v_H, r); }
static double v_zmax_at(const OracleScene* sc, double r) { return v_interp_radial(sc, sc->v_zmax, r); }

static int v_inside(const OracleScene* sc, double r, double z) {
    if (r <= sc->v_r_horizon || r > sc->v_r_outer) return 0;
    const double zm = v_zmax_at(sc, r);
    const double H = v_scale_height(sc, r);
    return fabs(z) < zm + 1.5 * H;
}

static double v_taper(const OracleScene* sc, double r) {
    if (r >= sc->v_r_isco) return 1.0;
    const double dr = sc->v_r_isco - r;
    return exp(-(dr * dr) / (sc->v_taper_width * sc->v_taper_width));
}

/* src/noise.cpp:38-96, 105-115 */
static const double kGrad3[12][3] = {{1, 1, 0}, {-1, 1, 0}, {1, -1, 0}, {-1, -1, 0},
                                     {1, 0, 1}, {-1, 0, 1}, {1, 0, -1}, {-1, 0, -1},
                                     {0, 1, 1}, {0, -1, 1}, {0, 1, -1}, {0, -1, -1}};
static double simplex_corner(double cx, double cy, double cz, int gi) {
    double t0 = 0.6 - cx * cx - cy * cy - cz * cz;
    if (t0 < 0.0) return 0.0;
    t0 *= t0;
    const double* g = kGrad3[gi % 12];
    return t0 * t0 * (g[0] * cx + g[1] * cy + g[2] * cz);
}

double oracle_noise(const OracleScene* sc, double x, double y, double z) {
    const double F3 = 1.0 / 3.0, G3 = 1.0 / 6.0;
    const int* P = sc->v_perm;
    const double s = (x + y + z) * F3;
    const int i = (int)floor(x + s), j = (int)floor(y + s), k = (int)floor(z + s);
    const double t = (i + j + k) * G3;
    const double X0 = i - t, Y0 = j - t, Z0 = k - t;
    const double x0 = x - X0, y0 = y - Y0, z0 = z - Z0;
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

static double noise_fbm(const OracleScene* sc, double x, double y, double z, int octaves) {
    double result = 0.0, amp = 1.0, freq = 1.0;
    for (int o = 0; o < octaves; ++o) {
        result += amp * oracle_noise(sc, x * freq, y * freq, z * freq);
        amp *= 0.5;
        freq *= 2.0;
    }
    return result;
}

double oracle_vol_density(const OracleScene* sc, double r, double z, double phi) {
    if (r <= sc->v_r_horizon || r > sc->v_r_outer) return 0.0;
    const double z_abs = fabs(z);
    const double zm = v_zmax_at(sc, r);
    const double H = v_scale_height(sc, r);
    double edge = 1.0, z_look = z_abs;
    if (z_abs >= zm) {
        const double dz = z_abs - zm;
        if (dz >= 1.5 * H) return 0.0;
        edge = exp(-2.0 * (dz / H) * (dz / H));
        z_look = zm * 0.9999;
    }
    const double rho_mid = v_interp_radial(sc, sc->v_rho_mid, r);
    const double rho_norm = v_interp_2d(sc, sc->v_rho_prof, r, z_look);
    const double base = rho_mid * rho_norm * sc->v_rho_scale * v_taper(sc, r) * edge;
    const double nx = r * cos(phi) / sc->v_noise_scale;
    const double ny = r * sin(phi) / sc->v_noise_scale;
    const double nz = z / sc->v_noise_scale;
    const double n = noise_fbm(sc, nx, ny, nz, sc->v_octaves);
    return max_d(0.0, base * (1.0 + sc->v_turbulence * n));
}

double oracle_vol_temperature(const OracleScene* sc, double r, double z) {
    if (r <= sc->v_r_horizon || r > sc->v_r_outer) return 0.0;
    const double z_abs = fabs(z);
    const double zm = v_zmax_at(sc, r);
    const double H = v_scale_height(sc, r);
    if (z_abs >= zm + 1.5 * H) return 0.0;
    const double z_look = min_d(z_abs, zm * 0.9999);
    return v_interp_2d(sc, sc->v_T_prof, r, z_look);
}

static void v_circular(const OracleScene* sc, double r, double* ut, double* uphi) {
    const double M = sc->v_M, a = sc->v_a;
    const double Omg = sqrt(M) / (r * sqrt(r) + a * sqrt(M));
    const double g_tt = -(1.0 - 2.0 * M / r);
    const double g_tphi = -2.0 * M * a / r;
    const double g_phph = r * r + a * a + 2.0 * M * a * a / r;
    const double den = -(g_tt + 2.0 * g_tphi * Omg + g_phph * Omg * Omg);
    *ut = 1.0 / sqrt(max_d(den, 1e-30));
    *uphi = Omg * *ut;
}

static void v_plunging(const OracleScene* sc, double r, double theta, double* ut, double* ur,
                       double* uphi) {
    const double M = sc->v_M, a = sc->v_a, E = sc->v_E_isco, L = sc->v_L_isco;
    const double Delta = r * r - 2.0 * M * r + a * a;
    const double Sigma = r * r + a * a * cos(theta) * cos(theta);
    *ut = (E * (r * r + a * a + 2.0 * M * a * a / r) - 2.0 * M * a * L / r) / Delta;
    *uphi = (L * (1.0 - 2.0 * M / r) + 2.0 * M * a * E / r) / Delta;
    const double EaL = E * (r * r + a * a) - a * L;
    const double LaE = L - a * E;
    const double R = EaL * EaL - Delta * (r * r + LaE * LaE);
    *ur = -sqrt(max_d(0.0, R)) / Sigma;
}

/* src/opacity.cpp:218-224, 307-345, 209-214 */
static void log_locate(double v, double lo, double hi, int n, int* idx, double* frac) {
    double t = (v - lo) / (hi - lo) * (n - 1);
    t = clamp_d(t, 0.0, (double)(n - 2));
    *idx = (int)t;
    *frac = t - *idx;
}

static double safe_ln(double x) { return log(max_d(x, 1e-100)); }

double oracle_kappa_abs(const OracleScene* sc, double nu, double rho, double T) {
    int inu, ir, iT;
    double fnu, fr, fT;
    log_locate(log10(nu), sc->o_log_nu_min, sc->o_log_nu_max, sc->o_n_nu, &inu, &fnu);
    log_locate(log10(rho), sc->o_log_rho_min, sc->o_log_rho_max, sc->o_n_rho, &ir, &fr);
    log_locate(log10(T), sc->o_log_T_min, sc->o_log_T_max, sc->o_n_T, &iT, &fT);
    const int nr = sc->o_n_rho, nt = sc->o_n_T;
    const double* L = sc->o_kabs;
#define KIDX(i, j, k) ((size_t)(i) * nr * nt + (size_t)(j) * nt + (k))
    const double c000 = L[KIDX(inu, ir, iT)], c001 = L[KIDX(inu, ir, iT + 1)];
    const double c010 = L[KIDX(inu, ir + 1, iT)], c011 = L[KIDX(inu, ir + 1, iT + 1)];
    const double c100 = L[KIDX(inu + 1, ir, iT)], c101 = L[KIDX(inu + 1, ir, iT + 1)];
    const double c110 = L[KIDX(inu + 1, ir + 1, iT)], c111 = L[KIDX(inu + 1, ir + 1, iT + 1)];
#undef KIDX
    const double l00 = safe_ln(c000) * (1 - fT) + safe_ln(c001) * fT;
    const double l01 = safe_ln(c010) * (1 - fT) + safe_ln(c011) * fT;
    const double l10 = safe_ln(c100) * (1 - fT) + safe_ln(c101) * fT;
    const double l11 = safe_ln(c110) * (1 - fT) + safe_ln(c111) * fT;
    const double l0 = l00 * (1 - fr) + l01 * fr;
    const double l1 = l10 * (1 - fr) + l11 * fr;
    return exp(l0 * (1 - fnu) + l1 * fnu);
}

double oracle_kappa_es(const OracleScene* sc, double rho, double T) {
    int ir, iT;
    double fr, fT;
    log_locate(log10(rho), sc->o_log_rho_min, sc->o_log_rho_max, sc->o_n_rho, &ir, &fr);
    log_locate(log10(T), sc->o_log_T_min, sc->o_log_T_max, sc->o_n_T, &iT, &fT);
    const int nt = sc->o_n_T;
    const double* L = sc->o_kes;
    const double v00 = L[ir * nt + iT], v01 = L[ir * nt + iT + 1];
    const double v10 = L[(ir + 1) * nt + iT], v11 = L[(ir + 1) * nt + iT + 1];
    return v00 * (1 - fr) * (1 - fT) + v01 * (1 - fr) * fT + v10 * fr * (1 - fT) + v11 * fr * fT;
}

static double planck_nu(double nu, double T) {
    const double h = 6.626070e-27, k = 1.380649e-16, c = 2.997924e10;
    if (nu <= 0.0 || T <= 0.0) return 0.0;
    const double x = h * nu / (k * T);
    if (x > 500.0) return 0.0;
    return (2.0 * h * nu * nu * nu / (c * c)) / (exp(x) - 1.0);
}

/* Shared part of both ray-marches: emitter velocity and redshift at new state. */
static void v_emitter(const OracleScene* sc, const double* ns, double r, double theta, double ut_obs,
                      double* g_out, double* pue_out) {
    double ut = 0.0, ur = 0.0, uphi = 0.0;
    if (r >= sc->v_r_isco) v_circular(sc, r, &ut, &uphi);
    else v_plunging(sc, r, theta, &ut, &ur, &uphi);
    const double pue = ns[4] * ut + ns[5] * ur + ns[7] * uphi;
    const double puo = ns[4] * ut_obs;
    *g_out = pue / puo;
    *pue_out = pue;
}

/* src/geodesic_tracer.cpp:183-337 — RGB ray-march through the volume. */
static void march_rgb(const OracleScene* sc, double* state, double J[3], double Tt[3], OracleCounters* cnt) {
    const double c = 2.997924e10;
    const double nu_obs[3] = {c / 450e-7, c / 550e-7, c / 650e-7};
    double Jl[3] = {J[0], J[1], J[2]}, T[3] = {Tt[0], Tt[1], Tt[2]};
    const double ut_obs = 1.0 / sqrt(1.0 - 2.0 / sc->observer_r);
    double r = state[1];
    const double z0 = r * cos(state[2]);
    const double H0 = v_scale_height(sc, r);
    double ds = v_inside(sc, r, z0) ? H0 / 16.0 : min_d(fabs(z0) / 8.0, H0 * 2.0);
    int steps = 0;
    int been_inside = v_inside(sc, r, z0);
    double ns[8];
    while (steps < 4096) {
        rk4_step(sc->M, sc->a, state, ds, ns);
        ++steps;
        cnt->march_steps++;
        r = ns[1];
        const double theta = ns[2], phi = ns[3];
        const double z = r * cos(theta);
        if (r < sc->v_r_horizon) { memcpy(state, ns, sizeof ns); break; }
        if (r > sc->v_r_outer) { memcpy(state, ns, sizeof ns); break; }
        if (T[0] < 1e-6 && T[1] < 1e-6 && T[2] < 1e-6) { memcpy(state, ns, sizeof ns); break; }
        const double H = v_scale_height(sc, r);
        if (!v_inside(sc, r, z)) {
            const double zm = v_zmax_at(sc, r);
            if (been_inside && fabs(z) > zm + 3.0 * H) { memcpy(state, ns, sizeof ns); break; }
            if (!been_inside) {
                ds = min_d(fabs(z) / 8.0, H * 2.0);
                ds = max_d(ds, H / 64.0);
            } else {
                ds = clamp_d(H / 4.0, H / 64.0, H);
            }
            memcpy(state, ns, sizeof ns);
            continue;
        }
        been_inside = 1;
        const double rho = oracle_vol_density(sc, r, z, phi);
        const double Tl = oracle_vol_temperature(sc, r, fabs(z));
        if (rho <= 0.0 || Tl <= 0.0) { memcpy(state, ns, sizeof ns); continue; }
        cnt->physics_steps++;
        double g, pue;
        v_emitter(sc, ns, r, theta, ut_obs, &g, &pue);
        const double dsp = fabs(pue) * fabs(ds);
        for (int ch = 0; ch < 3; ++ch) {
            const double nu = fabs(g) * nu_obs[ch];
            const double ka = oracle_kappa_abs(sc, nu, rho, Tl);
            const double ke = oracle_kappa_es(sc, rho, Tl);
            const double kt = ka + ke;
            const double eps = (kt > 0.0) ? ka / kt : 1.0;
            const double dtau = kt * rho * dsp;
            const double B = planck_nu(nu, Tl);
            const double S = eps * B / (nu * nu * nu);
            const double e = exp(-dtau);
            Jl[ch] += T[ch] * S * (1.0 - e);
            T[ch] *= e;
        }
        const double at = (oracle_kappa_abs(sc, fabs(g) * nu_obs[1], rho, Tl) + oracle_kappa_es(sc, rho, Tl)) * rho;
        const double ds_tau = (at > 0.0) ? 0.05 / at : ds * 2.0;
        const double ds_geo = 0.1 * max_d(r - sc->v_r_horizon, 0.5);
        ds = min_d(ds_tau, ds_geo);
        ds = clamp_d(ds, H / 64.0, H);
        memcpy(state, ns, sizeof ns);
    }
    for (int k = 0; k < 3; ++k) { J[k] = Jl[k]; Tt[k] = T[k]; }
}

/* src/geodesic_tracer.cpp:605-746 — spectral ray-march (nb bins). */
static void march_spectral(const OracleScene* sc, double* state, int nb, const double* nu_obs, double* J,
                           double* Tt, double* tau, OracleCounters* cnt) {
    const double ut_obs = 1.0 / sqrt(1.0 - 2.0 / sc->observer_r);
    double r = state[1];
    const double z0 = r * cos(state[2]);
    const double H0 = v_scale_height(sc, r);
    double ds = v_inside(sc, r, z0) ? H0 / 16.0 : min_d(fabs(z0) / 8.0, H0 * 2.0);
    int steps = 0;
    int been_inside = v_inside(sc, r, z0);
    const int med = nb / 2;
    double ns[8];
    while (steps < 4096) {
        rk4_step(sc->M, sc->a, state, ds, ns);
        ++steps;
        cnt->march_steps++;
        r = ns[1];
        const double theta = ns[2], phi = ns[3];
        const double z = r * cos(theta);
        if (r < sc->v_r_horizon) { memcpy(state, ns, sizeof ns); break; }
        if (r > sc->v_r_outer) { memcpy(state, ns, sizeof ns); break; }
        int thick = 1;
        for (int b = 0; b < nb; ++b)
            if (tau[b] <= 10.0) { thick = 0; break; }
        if (thick) { memcpy(state, ns, sizeof ns); break; }
        const double H = v_scale_height(sc, r);
        if (!v_inside(sc, r, z)) {
            const double zm = v_zmax_at(sc, r);
            if (been_inside && fabs(z) > zm + 3.0 * H) { memcpy(state, ns, sizeof ns); break; }
            if (!been_inside) {
                ds = min_d(fabs(z) / 8.0, H * 2.0);
                ds = max_d(ds, H / 64.0);
            } else {
                ds = clamp_d(H / 4.0, H / 64.0, H);
            }
            memcpy(state, ns, sizeof ns);
            continue;
        }
        been_inside = 1;
        const double rho = oracle_vol_density(sc, r, z, phi);
        const double Tl = oracle_vol_temperature(sc, r, fabs(z));
        if (rho <= 0.0 || Tl <= 0.0) { memcpy(state, ns, sizeof ns); continue; }
        cnt->physics_steps++;
        double g, pue;
        v_emitter(sc, ns, r, theta, ut_obs, &g, &pue);
        const double dsp = fabs(pue) * fabs(ds);
        for (int b = 0; b < nb; ++b) {
            const double nu = fabs(g) * nu_obs[b];
            const double ka = oracle_kappa_abs(sc, nu, rho, Tl);
            const double ke = oracle_kappa_es(sc, rho, Tl);
            const double kt = ka + ke;
            const double eps = (kt > 0.0) ? ka / kt : 1.0;
            const double dtau = kt * rho * dsp;
            tau[b] += dtau;
            const double B = planck_nu(nu, Tl);
            const double S = eps * B / (nu * nu * nu);
            const double e = exp(-dtau);
            J[b] += Tt[b] * S * (1.0 - e);
            Tt[b] *= e;
        }
        const double nu_med = fabs(g) * nu_obs[med];
        const double at = (oracle_kappa_abs(sc, nu_med, rho, Tl) + oracle_kappa_es(sc, rho, Tl)) * rho;
        const double ds_tau = (at > 0.0) ? 0.05 / at : ds * 2.0;
        const double ds_geo = 0.1 * max_d(r - sc->v_r_horizon, 0.5);
        ds = min_d(ds_tau, ds_geo);
        ds = clamp_d(ds, H / 64.0, H);
        memcpy(state, ns, sizeof ns);
    }
}

/* src/geodesic_tracer.cpp:71-95 — step clamp near the volume. */
static void v_step_clamp(const OracleScene* sc, const double* state, double* dlambda, OracleCounters* cnt) {
    const double r = state[1];
    const double theta = state[2];
    const double z = r * cos(theta);
    if (r >= sc->v_r_horizon * 0.9 && r <= sc->v_r_outer * 1.5) {
        const double H = v_scale_height(sc, r);
        const double zm = v_zmax_at(sc, r);
        if (fabs(z) < zm + 6.0 * H) {
            double d[8];
            kerr_rhs(sc->M, sc->a, state, d);
            cnt->clamp_evals++;
            const double dz_dl = fabs(cos(theta) * d[1] - r * sin(theta) * d[2]);
            if (dz_dl > 1e-20) {
                const double dl_max = max_d(0.25 * H / dz_dl, H / 64.0);
                *dlambda = min_d(*dlambda, dl_max);
            }
        }
    }
}

/* src/geodesic_tracer.cpp:105-153 — does this step hand over to the ray-march? */
static int v_should_march(const OracleScene* sc, const double* prev, const double* state) {
    const double d_prev = prev[2] - HALF_PI;
    const double d_new = state[2] - HALF_PI;
    const double r_new = state[1], r_prev = prev[1];
    const double z_new = r_new * cos(state[2]);
    const double z_prev = r_prev * cos(prev[2]);
    const int crossed = (d_prev * d_new < 0.0) && fabs(d_prev - d_new) > 1e-12;
    const int inside_now = v_inside(sc, r_new, z_new);
    const double zm_new = v_zmax_at(sc, r_new);
    const double H_new = v_scale_height(sc, r_new);
    const double H_prev = v_scale_height(sc, r_prev);
    const int near = (fabs(z_new) < zm_new + 2.0 * H_new || fabs(z_prev) < v_zmax_at(sc, r_prev) + 2.0 * H_prev)
                     && r_new >= sc->v_r_horizon && r_new <= sc->v_r_outer;
    if (!(crossed || inside_now || near)) return 0;
    const double r_lo = min_d(r_prev, r_new);
    const double r_hi = max_d(r_prev, r_new);
    if (!(r_hi >= sc->v_r_horizon && r_lo <= sc->v_r_outer)) return 0;
    const double re = prev[1];
    return re >= sc->v_r_horizon * 0.9 && re <= sc->v_r_outer * 1.5;
}

/* src/geodesic_tracer.cpp:23-181 (+ star lookup of src/renderer.cpp:61-63). */
static int trace_one(const OracleScene* sc, const double* init, double* rgb, int* ncross, double* fin,
                     OracleCounters* cnt) {
    const double c = 2.997924e10;
    const double nu_rgb[3] = {c / 450e-7, c / 550e-7, c / 650e-7};
    double y[8], prev[8];
    memcpy(y, init, sizeof y);
    double col[3] = {0, 0, 0};
    double J[3] = {0, 0, 0}, T[3] = {1, 1, 1};
    double dlambda = 0.01 * sc->observer_r;
    int term = 2;
    int nc = 0;
    for (int step = 0; step < sc->max_steps; ++step) {
        const double r = y[1];
        if (r < sc->r_horizon + sc->horizon_eps) { term = 0; break; }
        if (r > sc->r_escape) { term = 1; break; }
        memcpy(prev, y, sizeof y);
        if (sc->vol_on) v_step_clamp(sc, y, &dlambda, cnt);
        double out[8];
        dlambda = dp45_adaptive(sc->M, sc->a, prev, dlambda, sc->tolerance, out, &cnt->attempts);
        memcpy(y, out, sizeof y);
        cnt->accepted++;
        if (sc->vol_on) {
            const int opaque = (T[0] < 1e-6 && T[1] < 1e-6 && T[2] < 1e-6);
            if (!opaque && v_should_march(sc, prev, y)) {
                double entry[8];
                memcpy(entry, prev, sizeof entry);
                march_rgb(sc, entry, J, T, cnt);
                memcpy(y, entry, sizeof y);
                ++nc;  /* with a volumetric disk the fate counts ray-march entries */
                continue;
            }
        }
        if (!sc->vol_on && sc->disk_on) {
            const double d_prev = prev[2] - HALF_PI;
            const double d_new = y[2] - HALF_PI;
            if (d_prev * d_new < 0.0 && fabs(d_prev - d_new) > 1e-12) {
                const double frac = -d_prev / (d_new - d_prev);
                const double r_cross = prev[1] + frac * (y[1] - prev[1]);
                double pc[4];
                for (int m = 0; m < 4; ++m) pc[m] = prev[4 + m] + frac * (y[4 + m] - prev[4 + m]);
                if (r_cross >= sc->disk_r_inner && r_cross <= sc->disk_r_outer) {
                    double e[3];
                    disk_emission(sc, r_cross, pc[0], pc[3], e);
                    for (int k = 0; k < 3; ++k) col[k] += e[k];
                    ++nc;
                    cnt->crossings++;
                }
            }
        }
    }
    for (int k = 0; k < 3; ++k) col[k] += J[k] * nu_rgb[k] * nu_rgb[k] * nu_rgb[k];
    if (term == 1 && sc->stars_on) {
        const double b = star_sample(sc, y[2], y[3]);
        for (int k = 0; k < 3; ++k) col[k] += b;
    }
    for (int k = 0; k < 3; ++k) rgb[k] = col[k];
    if (ncross) *ncross = nc;
    if (fin) memcpy(fin, y, sizeof y);
    return term;
}

static void add_counters(OracleCounters* dst, const OracleCounters* src) {
#pragma omp atomic
    dst->attempts += src->attempts;
#pragma omp atomic
    dst->accepted += src->accepted;
#pragma omp atomic
    dst->crossings += src->crossings;
#pragma omp atomic
    dst->clamp_evals += src->clamp_evals;
#pragma omp atomic
    dst->march_steps += src->march_steps;
#pragma omp atomic
    dst->physics_steps += src->physics_steps;
}

void oracle_trace_rgb(const OracleScene* sc, int n, const double* px, const double* py, double* rgb,
                      int* term, int* ncross, double* fin, OracleCounters* cnt) {
#pragma omp parallel
    {
        OracleCounters local = {0, 0, 0, 0, 0, 0};
#pragma omp for schedule(dynamic, 8)
        for (int k = 0; k < n; ++k) {
            double init[8];
            oracle_camera_ray(sc, px[k], py[k], init);
            int nc = 0;
            term[k] = trace_one(sc, init, rgb + 3 * (size_t)k, &nc, fin ? fin + 8 * (size_t)k : NULL, &local);
            if (ncross) ncross[k] = nc;
        }
        if (cnt) add_counters(cnt, &local);
    }
}

void oracle_render_pixels(const OracleScene* sc, int spp, int n, const int* pix, double* rgb,
                          OracleCounters* cnt) {
    int grid = (int)sqrt((double)spp);
    if (grid < 1) grid = 1;
    const double inv = 1.0 / (grid * grid);
    const double cell = 1.0 / grid;
#pragma omp parallel
    {
        OracleCounters local = {0, 0, 0, 0, 0, 0};
#pragma omp for schedule(dynamic, 4)
        for (int q = 0; q < n; ++q) {
            const int j = pix[q] / sc->width, i = pix[q] % sc->width;
            double acc[3] = {0, 0, 0};
            for (int sy = 0; sy < grid; ++sy)
                for (int sx = 0; sx < grid; ++sx) {
                    const int s = sy * grid + sx;
                    const double x = i + (sx + oracle_pixel_hash(i, j, s, 0)) * cell;
                    const double yy = j + (sy + oracle_pixel_hash(i, j, s, 1)) * cell;
                    double init[8], c[3];
                    oracle_camera_ray(sc, x, yy, init);
                    trace_one(sc, init, c, NULL, NULL, &local);
                    for (int k = 0; k < 3; ++k) acc[k] = acc[k] + c[k];
                }
            for (int k = 0; k < 3; ++k) rgb[3 * (size_t)q + k] = acc[k] * inv;
        }
        if (cnt) add_counters(cnt, &local);
    }
}

/* src/geodesic_tracer.cpp:495-603 */
static int trace_spectral_one(const OracleScene* sc, const double* init, int nb, const double* freqs,
                              double* out, double* J, double* Tt, double* tau, OracleCounters* cnt) {
    for (int b = 0; b < nb; ++b) out[b] = 0.0;
    if (!sc->vol_on || nb == 0) return 1;
    for (int b = 0; b < nb; ++b) { J[b] = 0.0; Tt[b] = 1.0; tau[b] = 0.0; }
    double y[8], prev[8];
    memcpy(y, init, sizeof y);
    double dlambda = 0.01 * sc->observer_r;
    int term = 2;
    for (int step = 0; step < sc->max_steps; ++step) {
        const double r = y[1];
        if (r < sc->r_horizon + sc->horizon_eps) { term = 0; break; }
        if (r > sc->r_escape) { term = 1; break; }
        memcpy(prev, y, sizeof y);
        v_step_clamp(sc, y, &dlambda, cnt);
        double o[8];
        dlambda = dp45_adaptive(sc->M, sc->a, prev, dlambda, sc->tolerance, o, &cnt->attempts);
        memcpy(y, o, sizeof y);
        cnt->accepted++;
        if (v_should_march(sc, prev, y)) {
            double entry[8];
            memcpy(entry, prev, sizeof entry);
            march_spectral(sc, entry, nb, freqs, J, Tt, tau, cnt);
            memcpy(y, entry, sizeof y);
            continue;
        }
    }
    for (int b = 0; b < nb; ++b) out[b] = J[b] * freqs[b] * freqs[b] * freqs[b];
    return term;
}

void oracle_trace_spectral(const OracleScene* sc, int nb, const double* freqs, int n, const double* px,
                           const double* py, double* spec, int* term, OracleCounters* cnt) {
#pragma omp parallel
    {
        OracleCounters local = {0, 0, 0, 0, 0, 0};
        double* work = (double*)malloc(sizeof(double) * 3 * (size_t)(nb > 0 ? nb : 1));
#pragma omp for schedule(dynamic, 4)
        for (int k = 0; k < n; ++k) {
            double init[8];
            oracle_camera_ray(sc, px[k], py[k], init);
            term[k] = trace_spectral_one(sc, init, nb, freqs, spec + (size_t)k * nb, work, work + nb,
                                         work + 2 * nb, &local);
        }
        free(work);
        if (cnt) add_counters(cnt, &local);
    }
}

void oracle_render_spectral_pixels(const OracleScene* sc, int spp, int nb, const double* freqs, int n,
                                   const int* pix, double* spec, OracleCounters* cnt) {
    int grid = (int)sqrt((double)spp);
    if (grid < 1) grid = 1;
    const double inv = 1.0 / (grid * grid);
    const double cell = 1.0 / grid;
#pragma omp parallel
    {
        OracleCounters local = {0, 0, 0, 0, 0, 0};
        double* work = (double*)malloc(sizeof(double) * 5 * (size_t)(nb > 0 ? nb : 1));
        double* acc = work + 3 * nb;
        double* one = work + 4 * nb;
#pragma omp for schedule(dynamic, 2)
        for (int q = 0; q < n; ++q) {
            const int j = pix[q] / sc->width, i = pix[q] % sc->width;
            for (int b = 0; b < nb; ++b) acc[b] = 0.0;
            for (int sy = 0; sy < grid; ++sy)
                for (int sx = 0; sx < grid; ++sx) {
                    const int s = sy * grid + sx;
                    const double x = i + (sx + oracle_pixel_hash(i, j, s, 0)) * cell;
                    const double yy = j + (sy + oracle_pixel_hash(i, j, s, 1)) * cell;
                    double init[8];
                    oracle_camera_ray(sc, x, yy, init);
                    trace_spectral_one(sc, init, nb, freqs, one, work, work + nb, work + 2 * nb, &local);
                    for (int b = 0; b < nb; ++b) acc[b] += one[b];
                }
            for (int b = 0; b < nb; ++b) spec[(size_t)q * nb + b] = acc[b] * inv;
        }
        free(work);
        if (cnt) add_counters(cnt, &local);
    }
}
