// Pieces of the volumetric trace shared by the volumetric kernels: the
// near-disk clamp at the start of an outer step, the hand-over test from the
// outer DP45 loop to the ray-march, the march's starting step, and the
// per-launch counters (src/geodesic_tracer.cpp:71-153 and 495-603).
#pragma once

#include "integrate.cuh"
#include "shading.cuh"
#include "volume.cuh"

namespace grrt_b200 {

struct VolCounters {
    unsigned long long attempts = 0, accepted = 0, rays = 0, horizon = 0, escaped = 0, maxsteps = 0;
    unsigned long long clamp = 0, march = 0, physics = 0, bins = 0, fp64 = 0;
};

// Order in which the spectral kernel takes its work items: within each full
// block of kVolSpread^2 items the order is transposed, so the 32 items a warp
// takes at once lie kVolSpread items apart in the image. Neighbouring pixels
// trace alike, and the costliest rays (near the photon orbit, grazing the
// volume for thousands of clamped steps) come in clusters; a cluster taken by
// one warp serves its lanes' physics steps one after another, while spread
// over different warps the long rays run side by side. Items past the last
// full block keep their index. A bijection on [0, total).
#ifndef GRRT_VOL_SPREAD
#define GRRT_VOL_SPREAD 64
#endif
constexpr unsigned kVolSpread = GRRT_VOL_SPREAD;
__host__ __device__ __forceinline__ unsigned vol_spread_order(unsigned k, unsigned total) {
    constexpr unsigned kBlock = kVolSpread * kVolSpread;
    if (k >= (total / kBlock) * kBlock) return k;
    const unsigned base = k - k % kBlock, j = k % kBlock;
    return base + (j % kVolSpread) * kVolSpread + j / kVolSpread;
}

// Warp sum of the counters, one atomic per counter per warp.
__device__ __forceinline__ void flush_vol(DevStats* st, const VolCounters& c, bool cancelled) {
    unsigned long long v[11] = {c.attempts, c.accepted, c.rays, c.horizon, c.escaped, c.maxsteps,
                                c.clamp, c.march, c.physics, c.bins, c.fp64};
#pragma unroll
    for (int k = 0; k < 11; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&st->attempts, v[0]);
        atomicAdd(&st->accepted, v[1]);
        atomicAdd(&st->rays, v[2]);
        atomicAdd(&st->horizon, v[3]);
        atomicAdd(&st->escaped, v[4]);
        atomicAdd(&st->max_steps, v[5]);
        atomicAdd(&st->clamp_evals, v[6]);
        atomicAdd(&st->march_steps, v[7]);
        atomicAdd(&st->physics_steps, v[8]);
        atomicAdd(&st->bin_updates, v[9]);
        atomicAdd(&st->fp64_attempts, v[10]);
        if (cancelled && threadIdx.x == 0) atomicAdd(&st->cancelled, 1ull);
    }
}

// Pixel sum += J nu^3 (I_obs = J nu^3, src/geodesic_tracer.cpp:598-600), each
// operation rounded on its own (no contraction into a fused multiply-add), so
// every spectral kernel and the mixed form's resolve produce the same bits.
__device__ __forceinline__ double add_intensity(double sum, double J, double f) {
    return __dadd_rn(sum, __dmul_rn(__dmul_rn(__dmul_rn(J, f), f), f));
}

// Near-disk clamp at the start of an outer step (src/geodesic_tracer.cpp:71-95):
// for r in [0.9 r_h, 1.5 r_outer] and |z| < z_max + 6 H, dlambda is capped at
// max(H / (4 |dz/dlambda|), H / 64). d = f(y), the right-hand side the step's
// first DP45 stage uses too (the reference evaluates it here once more).
// Returns whether the clamp applied (the clamp counter).
__device__ __forceinline__ bool vol_clamp(const DevScene& S, const Vec5<double>& d, const Vec5<double>& y,
                                          double& dlambda) {
    const DevVolume& V = S.vol;
    const double r = y.r;
    if (!(r >= V.r_horizon * 0.9 && r <= V.r_outer * 1.5)) return false;
    double st, ct;
    sincos(y.th, &st, &ct);
    const double z = r * ct;
    const double H = v_scale_height(V, r);
    const double zm = v_zmax(V, r);
    if (!(fabs(z) < zm + 6.0 * H)) return false;
    const double dz_dl = fabs(ct * d.r - r * st * d.th);
    if (dz_dl > 1e-20) {
        const double dl_max = vmax(0.25 * H / dz_dl, H / 64.0);
        dlambda = vmin(dlambda, dl_max);
    }
    return true;
}

// Hand-over after an accepted outer step prev -> y (src/geodesic_tracer.cpp:105-153):
// the step crossed the equator, ends inside the volume, or either end is
// within z_max + 2H of the plane over the disk's radii; and the step's radii
// reach [r_h, r_outer] from a start inside [0.9 r_h, 1.5 r_outer]. The march
// then starts from prev.
__device__ __forceinline__ bool vol_enters(const DevVolume& V, const Vec5<double>& prev, const Vec5<double>& y) {
    const double hp = kHalfPi;
    const double d_prev = prev.th - hp, d_new = y.th - hp;
    const double r_new = y.r, r_prev = prev.r;
    const double z_new = r_new * cos(y.th);
    const double z_prev = r_prev * cos(prev.th);
    const bool crossed = (d_prev * d_new < 0.0) && fabs(d_prev - d_new) > 1e-12;
    const bool inside_now = v_inside(V, r_new, z_new);
    const double zm_new = v_zmax(V, r_new), H_new = v_scale_height(V, r_new);
    const double H_prev = v_scale_height(V, r_prev);
    const bool near = (fabs(z_new) < zm_new + 2.0 * H_new || fabs(z_prev) < v_zmax(V, r_prev) + 2.0 * H_prev) &&
                      r_new >= V.r_horizon && r_new <= V.r_outer;
    if (!(crossed || inside_now || near)) return false;
    const double r_lo = vmin(r_prev, r_new), r_hi = vmax(r_prev, r_new);
    return r_hi >= V.r_horizon && r_lo <= V.r_outer && r_prev >= V.r_horizon * 0.9 && r_prev <= V.r_outer * 1.5;
}

// First march step length from the start state s: H/16 inside the volume,
// else min(|z|/8, 2H).
__device__ __forceinline__ double vol_march_start(const DevVolume& V, const Vec5<double>& s, bool& been_inside) {
    const double r0 = s.r;
    const double z0 = r0 * cos(s.th);
    const double H0 = v_scale_height(V, r0);
    been_inside = v_inside(V, r0, z0);
    return been_inside ? H0 / 16.0 : vmin(fabs(z0) / 8.0, H0 * 2.0);
}

// Observer-frame RGB frequencies (450, 550, 650 nm) of the RGB transfer.
__device__ __forceinline__ double rgb_nu(int ch) {
    constexpr double c = 2.997924e10;
    return ch == 0 ? c / 450e-7 : (ch == 1 ? c / 550e-7 : c / 650e-7);
}

// One RK4 step of the RGB ray-march (src/geodesic_tracer.cpp:183-337): ms
// advances by ds; inside the volume the three channels' emission and
// absorption update J and Tt and the next ds follows the optical depth and
// the radius; outside it ds approaches the volume (never inside yet) or holds
// at H/4 (after being inside). Returns whether the march ends here: outside
// [r_h, r_outer], all channels opaque, or beyond z_max + 3H after being
// inside. The 4096-step cap is the caller's.
__device__ __forceinline__ bool vol_march_rgb_step(const DevScene& S, double pt, double pph, Vec5<double>& ms,
                                                   double& ds, bool& been_inside, double* J, double* Tt,
                                                   VolCounters& cnt) {
    const DevVolume& V = S.vol;
    const Vec5<double> ns = rk4_step<double>(S.M, S.a, pt, pph, ms, ds);
    ++cnt.march;
    const double r = ns.r, theta = ns.th;
    double st, ct;
    sincos(theta, &st, &ct);
    const double z = r * ct;
    bool end = false;
    if (r < V.r_horizon || r > V.r_outer) {
        end = true;
    } else if (Tt[0] < 1e-6 && Tt[1] < 1e-6 && Tt[2] < 1e-6) {
        end = true;
    } else {
        const double H = v_scale_height(V, r);
        if (!v_inside(V, r, z)) {
            const double zm = v_zmax(V, r);
            if (been_inside && fabs(z) > zm + 3.0 * H) {
                end = true;
            } else if (!been_inside) {
                ds = vmax(vmin(fabs(z) / 8.0, H * 2.0), H / 64.0);
            } else {
                ds = vclamp(H / 4.0, H / 64.0, H);
            }
        } else {
            been_inside = true;
            const double rho = v_density(V, V.perm, r, z, ns.ph);
            const double Tl = v_temperature(V, r, fabs(z));
            if (rho > 0.0 && Tl > 0.0) {
                ++cnt.physics;
                double g, pue;
                v_redshift(V, pt, ns.pr, pph, r, theta, g, pue);
                const double dsp = fabs(pue) * fabs(ds);
                int ir, iT;
                double fr, fT;
                log_locate(log10(rho), V.log_rho_min, V.log_rho_max, V.n_rho, ir, fr);
                log_locate(log10(Tl), V.log_T_min, V.log_T_max, V.n_T, iT, fT);
                const double ke = v_kappa_es(V, ir, fr, iT, fT);
                const double ag = fabs(g);
                double ka_med = 0.0;
                for (int b = 0; b < 3; ++b) {
                    const double nu = ag * rgb_nu(b);
                    const double ka = v_kappa_abs(V, nu, ir, fr, iT, fT);
                    if (b == 1) ka_med = ka;
                    const double kt = ka + ke;
                    const double eps = (kt > 0.0) ? ka / kt : 1.0;
                    const double dtau = kt * rho * dsp;
                    const double B = planck_nu(nu, Tl);
                    const double Sv = eps * B / (nu * nu * nu);
                    const double e = exp(-dtau);
                    J[b] += Tt[b] * Sv * (1.0 - e);
                    Tt[b] *= e;
                }
                cnt.bins += 3;
                const double at = (ka_med + ke) * rho;
                const double ds_tau = (at > 0.0) ? 0.05 / at : ds * 2.0;
                const double ds_geo = 0.1 * vmax(r - V.r_horizon, 0.5);
                ds = vclamp(vmin(ds_tau, ds_geo), H / 64.0, H);
            }
        }
    }
    ms = ns;
    return end;
}

}  // namespace grrt_b200
