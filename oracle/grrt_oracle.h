/*
 * grrt_oracle.h — CPU restatement of the reference's per-pixel path.
 *
 * TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py load this library, as the checker. The product
 * (libgrrt.so) never links or calls it.
 *
 * The scene tables are inputs (plain arrays); the per-ray arithmetic follows
 * the reference expressions term by term, so compiled without FMA contraction
 * (liboracle.so) it reproduces the reference's strict build bit for bit. The
 * same source compiled with contraction (liboracle_fma.so) measures how
 * sensitive each pixel is to rounding.
 */
#ifndef GRRT_ORACLE_H
#define GRRT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    /* spacetime and integrator */
    double M, a, r_horizon, r_escape, horizon_eps, tolerance, observer_r;
    int max_steps;
    /* camera (include/grrt/camera/camera.h: tetrad at the observer) */
    double cam_pos[4], e0[4], e1[4], e2[4], e3[4], g[16];
    double fov;
    int width, height;
    /* thin disk (disk_on = 0: none) */
    int disk_on;
    double disk_r_inner, disk_r_outer, flux_max, peak_temperature;
    int flux_n;
    const double* flux;
    /* chromaticity table */
    double t_min, t_max;
    int spec_n;
    const double* spec_color; /* 3*spec_n */
    /* stars (stars_on = 0: black background) */
    int stars_on;
    const double *star_theta, *star_phi, *star_b;
    const int *cell_start, *cell_items;
    double star_tol;
    /* volumetric disk (vol_on = 0: none) */
    int vol_on;
    double v_M, v_a; /* the volumetric disk's own mass and spin (src/api.cpp:122-126) */
    double v_r_min, v_r_outer, v_r_isco, v_r_horizon, v_taper_width, v_E_isco, v_L_isco;
    double v_rho_scale, v_noise_scale, v_turbulence;
    int v_octaves, v_n_r, v_n_z;
    const double *v_H, *v_rho_mid, *v_rho_prof, *v_T_prof, *v_zmax;
    const int* v_perm; /* 512 */
    int o_n_nu, o_n_rho, o_n_T;
    double o_log_nu_min, o_log_nu_max, o_log_rho_min, o_log_rho_max, o_log_T_min, o_log_T_max;
    const double *o_kabs, *o_kes;
} OracleScene;

/* Per-sample counters (summed over the call). */
typedef struct {
    long long attempts;     /* DP45 attempts, accepted and rejected */
    long long accepted;     /* outer integration steps */
    long long crossings;    /* thin-disk emission events */
    long long clamp_evals;  /* volumetric pre-step derivative evaluations */
    long long march_steps;  /* volumetric classic-RK4 steps */
    long long physics_steps;/* volumetric steps with matter (per-bin work) */
} OracleCounters;

/* The reference's jitter hash (src/renderer.cpp:14-20). */
double oracle_pixel_hash(int i, int j, int s, int ch);

/* Initial covariant state of a camera sample (src/camera.cpp:69-96). out[8]. */
void oracle_camera_ray(const OracleScene* sc, double x, double y, double* out);

/* Trace n camera samples at fractional pixel coordinates (GeodesicTracer::trace
 * plus the star lookup of Renderer::render). rgb[3n], term[n] (0 horizon,
 * 1 escaped, 2 max steps), ncross[n] emitting disk crossings (with a
 * volumetric disk: ray-march entries), fin[8n] final state (may be NULL).
 * OpenMP over samples. */
void oracle_trace_rgb(const OracleScene* sc, int n, const double* px, const double* py,
                      double* rgb, int* term, int* ncross, double* fin, OracleCounters* cnt);

/* Render pixels (Renderer::render loop body in double): for each pixel index in
 * pix[0..n) with the reference's stratified jitter and spp grid, rgb[3n] is the
 * spp-averaged double colour before the float cast. */
void oracle_render_pixels(const OracleScene* sc, int spp, int n, const int* pix, double* rgb,
                          OracleCounters* cnt);

/* Spectral trace (GeodesicTracer::trace_spectral): spec[n*nb] observed
 * intensity per bin, term[n]. */
void oracle_trace_spectral(const OracleScene* sc, int nb, const double* freqs, int n,
                           const double* px, const double* py, double* spec, int* term,
                           OracleCounters* cnt);

/* Spectral pixels (Renderer::render_spectral loop body): spec[n*nb]. */
void oracle_render_spectral_pixels(const OracleScene* sc, int spp, int nb, const double* freqs,
                                   int n, const int* pix, double* spec, OracleCounters* cnt);

/* Pieces exposed for unit tests. */
void oracle_fast_sincos(double x, double* s, double* c);
void oracle_derivatives(const OracleScene* sc, const double* y, double* dy);
double oracle_vol_density(const OracleScene* sc, double r, double z, double phi);
double oracle_vol_temperature(const OracleScene* sc, double r, double z);
double oracle_kappa_abs(const OracleScene* sc, double nu, double rho, double T);
double oracle_kappa_es(const OracleScene* sc, double rho, double T);
double oracle_noise(const OracleScene* sc, double x, double y, double z);

#ifdef __cplusplus
}
#endif
#endif
