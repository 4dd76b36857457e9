// Spectral volumetric render with warp-cooperative radiative transfer, and
// the mixed-precision form built on it.
//
// Per ray the method is the spectral path of the reference
// (GeodesicTracer::trace_spectral and raymarch_volumetric_spectral,
// src/geodesic_tracer.cpp:495-746): the outer adaptive DP45 loop with the
// near-disk clamp and the hand-over, then the fixed-step RK4 march with a
// per-bin transfer update at every physics step. One lane owns one ray and
// computes its geometry (outer attempts, march steps, density, temperature,
// redshift and the table coordinates of rho and T). The per-bin part of a
// physics step (opacity, Planck function, the J / T / tau update: nb bins) is
// done by the whole warp, one bin per lane: each loop iteration, the lanes
// that reached a physics step are served in turn, so the cost is one pass
// over the bins instead of nb serial passes while 31 lanes wait. Ray starts
// and sample finishes (reset of the ray's row, the J nu^3 sum and the
// coalesced store of a pixel's spectrum) are served the same way.
//
// A ray's transfer state is a row of 4 x nb doubles per lane slot
// [J | T | tau | pixel sum], so the warp's accesses to one row are
// contiguous. Every bin sees the plain kernel's arithmetic in the same order,
// so the spectra are bit-identical to it.
//
// Mixed form: an FP32 speculative pass (FP32 right-hand sides, FP64 state,
// relaxed tolerance) traces every sample and keeps those whose trajectory
// stays away from the volume: no clamp, no hand-over, no near-critical orbit,
// so the FP64 form would give them zero intensity and the same termination.
// The rest are listed and re-traced from the camera by the FP64 kernel; a
// resolve pass sums each pixel's samples in order.
// The volumetric kernels end on a few long rays, one warp per SM, where
// instruction fetch stalls as much as arithmetic: one shared body of the FP64
// right-hand side instead of twelve inlined copies (Kerr a=0.9, 512x512, 32
// bins: 82 -> 74-79 ms for the FP64 form on B200).
#define GRRT_RHS_CALL_F64 1
#include <cuda_runtime.h>

#include <cstdint>

#include "launch_cache.h"
#include "integrate.cuh"
#include "mixed_spec.cuh"
#include "render_launch.h"
#include "shading.cuh"
#include "surrogate_geom.cuh"
#include "vol_steps.cuh"
#include "volume.cuh"

namespace grrt_b200 {

namespace {

constexpr int kSpecThreads = kVolSpectralThreads;
constexpr unsigned kWarp = 0xffffffffu;

}  // namespace

// kList = false: work item = pixel of the tile (list[k] when a pixel order
// is given); its spp samples are traced in order, summed in the row's
// pixel-sum part, and out_spec[pixel][nb] is written. kList = true: work item k = sample list[k] (pixel * grid^2 + s)
// of the tile; out_spec[sample][nb] receives the sample's J (its term of the
// pixel sum is J nu^3).
// kBatch = true (with kList = false): the batched form over many volumetric
// cameras. Work index -> (chunk, offset) through the batch's chunk table, as
// in the thin-disk batch; each lane reads its camera's scene, bins and output
// offset from the batch's items, and a served lane's bins are those of its
// own camera. nb is then the largest bin count of the batch (the row stride);
// tile, freqs and out_fate are unused.
template <bool kList, bool kBatch = false>
__global__ void __launch_bounds__(kSpecThreads)
vol_spectral_kernel(const __grid_constant__ DevScene S0, const DevTile tile, const double* __restrict__ freqs0,
                    int nb0, double* __restrict__ out_spec, uint32_t* __restrict__ out_fate,
                    double* __restrict__ scratch, unsigned int* __restrict__ queue, DevStats* __restrict__ stats,
                    const volatile int* __restrict__ cancel, const unsigned* __restrict__ list,
                    const unsigned* __restrict__ list_count, const __grid_constant__ DevBatch B) {
    static_assert(!(kList && kBatch), "the batched form has no list mode");
    // the scene of the lane's current pixel (batch: per lane, in global memory)
    const DevScene* sp = &S0;
#define S (kBatch ? *sp : S0)
#define V (S.vol)
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const unsigned total = kList ? *list_count
                                 : kBatch ? static_cast<unsigned>(B.n_chunks) * static_cast<unsigned>(B.chunk_size)
                                          : static_cast<unsigned>(tile.w) * static_cast<unsigned>(tile.h);
    const size_t slot = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    // a row is [J | T | tau | pixel sum], each part `seg` doubles
    const int seg = nb0;
    const size_t row_len = 4 * static_cast<size_t>(seg);
    // row of lane `src` of this warp: lane slots of a warp are consecutive
    double* const my_row = scratch + slot * row_len;
    auto row_of = [&](int src) { return my_row + (static_cast<ptrdiff_t>(src) - lane) * static_cast<ptrdiff_t>(row_len); };
    // the lane's camera (batch): its item, bins and bin count
    int item = 0;
    int nb = nb0;
    const double* freqs = freqs0;

    VolCounters cnt;
    int pix = -1, smp = 0;  // kList: pix = the listed sample
    bool live = false, need_start = false, marching = false;
    Vec5<double> y{}, prev{};
    Vec5<double> k1{};  // f(y) while k1_ok: the last accepted attempt's k7 or this step's first stage
    bool k1_ok = false;
    double pt = 0.0, pph = 0.0, dl = 0.0, dlambda = 0.0;
    int retry = 0, step = 0, entries = 0, n_thick = 0;
    Vec5<double> ms{};
    double ds = 0.0;
    int mcount = 0;
    bool been_inside = false, cancelled = false;
    unsigned iter = 0;

    while (true) {
        // ---- refill ----
        const bool want = (pix == -1);
        const unsigned want_mask = __ballot_sync(kWarp, want);
        bool fresh_pixel = false;
        if (want_mask) {
            unsigned base = 0;
            const int leader = __ffs(want_mask) - 1;
            if (lane == leader) base = atomicAdd(queue, static_cast<unsigned>(__popc(want_mask)));
            base = __shfl_sync(kWarp, base, leader);
            if (want) {
                const unsigned k = base + __popc(want_mask & lt_mask);
                if (k < total) {
                    if (kBatch) {
                        const DevBatchChunk ch = B.chunks[k / B.chunk_size];
                        const int within = static_cast<int>(k % B.chunk_size);
                        if (within < ch.count) {
                            item = ch.item;
                            const DevBatchItem& it = B.items[item];
                            sp = B.scenes + it.scene;
                            nb = it.nb;
                            freqs = it.freqs;
                            pix = ch.start + within;
                            smp = 0;
                            fresh_pixel = true;
                        }  // else: padding slot of a short chunk, fetch again
                    } else {
                        // list: the listed samples (kList), or the pixel order;
                        // taken in the spread order (vol_spread_order)
                        const unsigned ks = vol_spread_order(k, total);
                        pix = static_cast<int>(list ? list[ks] : ks);
                        smp = 0;
                        fresh_pixel = true;
                    }
                } else {
                    pix = -2;
                }
            }
        }
        bool fresh_ray = false;
        if (!live && pix >= 0) {
            const int grid2 = S.grid * S.grid;
            const int pixel = kList ? pix / grid2 : pix;
            const int s = kList ? pix % grid2 : smp;
            int i, j;
            if (kBatch) {
                const DevBatchItem& it = B.items[item];
                i = it.x0 + pixel % it.w;
                j = it.y0 + pixel / it.w;
            } else {
                const int qx = pixel % tile.w, qy = pixel / tile.w;
                i = tile.x0 + qx;
                j = tile.y0 + qy * tile.row_step;
            }
            const int sy = s / S.grid, sx = s % S.grid;
            const double x = i + (sx + pixel_hash(i, j, s, 0)) * S.cell;
            const double yy = j + (sy + pixel_hash(i, j, s, 1)) * S.cell;
            double p[4];
            camera_momentum(S, x, yy, p);
            y = Vec5<double>{S.cam_pos[1], S.cam_pos[2], S.cam_pos[3], p[1], p[2]};
            pt = p[0];
            pph = p[3];
            dlambda = S.dl0;
            step = 0;
            entries = 0;
            marching = false;
            n_thick = 0;
            k1_ok = false;
            live = true;
            need_start = true;
            fresh_ray = true;
        }
        // ---- reset the new rays' rows (J = 0, T = 1, tau = 0; a new pixel's sum = 0) ----
        {
            const unsigned rm = __ballot_sync(kWarp, fresh_ray);
            const unsigned pm = __ballot_sync(kWarp, fresh_pixel);
            for (unsigned m = rm; m; m &= m - 1) {
                const int src = __ffs(m) - 1;
                double* row = row_of(src);
                const bool new_pixel = !kList && ((pm >> src) & 1u);
                const int snb = kBatch ? __shfl_sync(kWarp, nb, src) : nb;
                for (int b = lane; b < snb; b += 32) {
                    row[b] = 0.0;
                    row[seg + b] = 1.0;
                    row[2 * seg + b] = 0.0;
                    if (new_pixel) row[3 * seg + b] = 0.0;
                }
            }
        }

        int term = -1;
        // ---- start of an outer step: termination tests, then the near-disk clamp ----
        if (live && need_start) {
            if (step >= S.max_steps) term = kTermMaxSteps;
            else if (y.r < S.r_stop) term = kTermHorizon;
            else if (y.r > S.r_escape) term = kTermEscaped;
            if (term < 0) {
                if (!k1_ok) {
                    k1 = kerr_rhs<double>(S.M, S.a, pt, pph, y);
                    k1_ok = true;
                }
                if (vol_clamp(S, k1, y, dlambda)) ++cnt.clamp;
                prev = y;
                dl = dlambda;
                retry = 0;
                need_start = false;
            }
        }

        // physics step inputs handed to the warp (bin-independent)
        bool phys = false;
        double ph_ag = 0.0, ph_rho = 0.0, ph_T = 0.0, ph_dsp = 0.0, ph_ke = 0.0, ph_fr = 0.0, ph_fT = 0.0;
        double ph_r = 0.0, ph_H = 0.0, ph_kamed = 0.0;
        int ph_ir = 0, ph_iT = 0;
        bool marched = false, mend = false;
        Vec5<double> ns{};
        if (live && term < 0 && !marching) {
            // ---- one DP45 attempt ----
            Vec5<double> y5, k7;
            const double err = dp45_attempt_k1<double>(S.M, S.a, pt, pph, y, dl, k1, y5, k7);
            ++cnt.fp64;
            ++cnt.attempts;
            const StepDecision d = pi_control(err, S.tol, dl, retry, y5.r);
            if (!d.accept) {
                dl = d.next;
                ++retry;
            } else {
                ++cnt.accepted;
                y = y5;
                k1 = k7;
                dlambda = d.next;
                ++step;  // the reference's loop counter advances on every outer iteration
                // hand-over to the ray-march (src/geodesic_tracer.cpp:105-153)
                if (vol_enters(V, prev, y)) {
                    marching = true;
                    ++entries;
                    ms = prev;  // march from the pre-step state
                    ds = vol_march_start(V, ms, been_inside);
                    mcount = 0;
                }
                if (!marching) need_start = true;
            }
        } else if (live && term < 0 && marching) {
            // ---- one RK4 march step (geometry; the bins follow below) ----
            marched = true;
            ns = rk4_step<double>(S.M, S.a, pt, pph, ms, ds);
            ++mcount;
            ++cnt.march;
            const double r = ns.r, theta = ns.th;
            double st, ct;
            sincos(theta, &st, &ct);
            const double z = r * ct;
            if (r < V.r_horizon || r > V.r_outer) {
                mend = true;
            } else if (n_thick == nb) {
                mend = true;
            } else {
                const double H = v_scale_height(V, r);
                if (!v_inside(V, r, z)) {
                    const double zm = v_zmax(V, r);
                    if (been_inside && fabs(z) > zm + 3.0 * H) {
                        mend = true;
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
                        ph_dsp = fabs(pue) * fabs(ds);
                        log_locate(log10(rho), V.log_rho_min, V.log_rho_max, V.n_rho, ph_ir, ph_fr);
                        log_locate(log10(Tl), V.log_T_min, V.log_T_max, V.n_T, ph_iT, ph_fT);
                        ph_ke = v_kappa_es(V, ph_ir, ph_fr, ph_iT, ph_fT);
                        ph_ag = fabs(g);
                        ph_rho = rho;
                        ph_T = Tl;
                        ph_r = r;
                        ph_H = H;
                        phys = true;
                    }
                }
            }
        }

        // ---- per-bin transfer of this iteration's physics steps, one bin per lane ----
        {
            const unsigned pm = __ballot_sync(kWarp, phys);
            for (unsigned m = pm; m; m &= m - 1) {
                const int src = __ffs(m) - 1;
                const double ag = __shfl_sync(kWarp, ph_ag, src);
                const double rho = __shfl_sync(kWarp, ph_rho, src);
                const double Tl = __shfl_sync(kWarp, ph_T, src);
                const double dsp = __shfl_sync(kWarp, ph_dsp, src);
                const double ke = __shfl_sync(kWarp, ph_ke, src);
                const double fr = __shfl_sync(kWarp, ph_fr, src);
                const double fT = __shfl_sync(kWarp, ph_fT, src);
                const int ir = __shfl_sync(kWarp, ph_ir, src);
                const int iT = __shfl_sync(kWarp, ph_iT, src);
                // the served lane's camera: its opacity tables and bins
                const int sitem = kBatch ? __shfl_sync(kWarp, item, src) : 0;
                const DevVolume& Vs = kBatch ? B.scenes[B.items[sitem].scene].vol : S0.vol;
                const double* sfreqs = kBatch ? B.items[sitem].freqs : freqs0;
                const int snb = kBatch ? B.items[sitem].nb : nb0;
                const int smed = snb / 2;
                double* row = row_of(src);
                double kam = 0.0;
                int thick = 0;
                for (int b0 = 0; b0 < snb; b0 += 32) {
                    const int b = b0 + lane;
                    double ka = 0.0;
                    bool thk = false;
                    if (b < snb) {
                        const double nu = ag * __ldg(sfreqs + b);
                        ka = v_kappa_abs(Vs, nu, ir, fr, iT, fT);
                        const double kt = ka + ke;
                        const double eps = (kt > 0.0) ? ka / kt : 1.0;
                        const double dtau = kt * rho * dsp;
                        const double B_nu = planck_nu(nu, Tl);
                        const double Sv = eps * B_nu / (nu * nu * nu);
                        const double e = exp(-dtau);
                        double tau = row[2 * seg + b];
                        tau += dtau;
                        row[2 * seg + b] = tau;
                        thk = !(tau <= 10.0);
                        const double Tb = row[seg + b];
                        row[b] += Tb * Sv * (1.0 - e);
                        row[seg + b] = Tb * e;
                    }
                    thick += __popc(__ballot_sync(kWarp, thk));
                    if (smed >= b0 && smed < b0 + 32) kam = __shfl_sync(kWarp, ka, smed - b0);
                }
                if (lane == src) {
                    ph_kamed = kam;
                    n_thick = thick;  // bins with tau > 10 (tau only grows)
                }
            }
        }
        if (phys) {
            cnt.bins += static_cast<unsigned long long>(nb);
            const double at = (ph_kamed + ph_ke) * ph_rho;
            const double ds_tau = (at > 0.0) ? 0.05 / at : ds * 2.0;
            const double ds_geo = 0.1 * vmax(ph_r - V.r_horizon, 0.5);
            ds = vclamp(vmin(ds_tau, ds_geo), ph_H / 64.0, ph_H);
        }
        if (marched) {
            ms = ns;
            if (!mend && mcount >= 4096) mend = true;
            if (mend) {
                marching = false;
                y = ms;  // the outer loop continues from the march's end state
                k1_ok = false;
                need_start = true;
            }
        }

        // ---- finish a terminated sample ----
        bool finish = false, pixel_done = false;
        size_t out_elem = 0;  // first output element of the finished pixel (list: sample)
        if (live && term >= 0) {
            live = false;
            finish = true;
            ++cnt.rays;
            if (term == kTermEscaped) ++cnt.escaped;
            else if (term == kTermHorizon) ++cnt.horizon;
            else ++cnt.maxsteps;
            const int grid2 = S.grid * S.grid;
            if (!kBatch && out_fate) {
                const unsigned ne = (entries > 0x3fffffff) ? 0x3fffffffu : static_cast<unsigned>(entries);
                const size_t q = kList ? static_cast<size_t>(pix) : static_cast<size_t>(pix) * grid2 + smp;
                out_fate[q] = static_cast<unsigned>(term) | (ne << 2);
            }
            if (kList) {
                out_elem = static_cast<size_t>(pix) * nb;
                pixel_done = true;
                pix = -1;
            } else if (++smp == grid2) {
                if (kBatch) {
                    out_elem = B.items[item].spec_offset + static_cast<size_t>(pix) * nb;
                } else {
                    const int qx = pix % tile.w, qy = pix / tile.w;
                    out_elem = (static_cast<size_t>(qy) * tile.out_pitch + qx) * nb;
                }
                pixel_done = true;
                pix = -1;
            }
        }
        {
            // I nu^3 of the finished samples into the pixel sums; finished pixels stored
            const unsigned fm = __ballot_sync(kWarp, finish);
            const unsigned dm = __ballot_sync(kWarp, pixel_done);
            // finished work items, for progress reports (the work counter
            // counts items taken; the long rays finish long after)
            if (dm && lane == 0) atomicAdd(queue + 1, static_cast<unsigned>(__popc(dm)));
            for (unsigned m = fm; m; m &= m - 1) {
                const int src = __ffs(m) - 1;
                const size_t o = __shfl_sync(kWarp, static_cast<unsigned long long>(out_elem), src);
                double* row = row_of(src);
                const bool done = (dm >> src) & 1u;
                const int sitem = kBatch ? __shfl_sync(kWarp, item, src) : 0;
                const double* sfreqs = kBatch ? B.items[sitem].freqs : freqs0;
                const int snb = kBatch ? B.items[sitem].nb : nb0;
                const double inv_spp = kBatch ? B.scenes[B.items[sitem].scene].inv_spp : S0.inv_spp;
                double* dst = out_spec + o;
                for (int b = lane; b < snb; b += 32) {
                    if (kList) {
                        dst[b] = row[b];  // the sample's J; the resolve forms the sum
                    } else {
                        const double sum = add_intensity(row[3 * seg + b], row[b], __ldg(sfreqs + b));
                        if (done)
                            dst[b] = __dmul_rn(sum, inv_spp);
                        else
                            row[3 * seg + b] = sum;
                    }
                }
            }
        }

        if (cancel && ((++iter & 1023u) == 0)) {
            int c = 0;
            if (lane == 0) c = *cancel;
            c = __shfl_sync(kWarp, c, 0);
            if (c) {
                cancelled = true;
                break;
            }
        }
        if (!__any_sync(kWarp, live || pix >= -1)) break;
    }
#undef S
#undef V
    flush_vol(stats, cnt, cancelled);
}

// ---------------------------------------------------------------------------
// Mixed form
// ---------------------------------------------------------------------------

// Speculative pass: every sample of the tile with FP32 right-hand sides
// against tol_fp32. A sample whose trajectory may come into the volume's
// region of influence (VolReach), sweeps more than mixed::kSweptMax radians
// inside r_near, or exhausts the step budget is listed for the FP64 re-trace;
// the others end with zero intensity and their termination.
//
// The FP64 form departs from plain DP45 stepping only at the near-disk clamp
// (a step starting at r <= 1.5 r_outer with |z| < z_max + 6H) and at the
// hand-over (a step starting at r <= 1.5 r_outer that crosses the equator or
// ends within z_max + 2H of it). So a trajectory that never enters
// {r <= R, |z| <= Z} (R = 1.5 r_outer, Z = max_r z_max + 6H) and never
// crosses the equator inside r <= R is traced identically by plain stepping
// and gets zero intensity. Each accepted speculative step a -> b is tested
// with bounds that hold along the whole step, not only at its ends:
//   - r: monotonic between the ends when p_r keeps its sign (no radial
//     turning point inside a step outside the photon region); otherwise the
//     ray's turning radius, from the constants of motion;
//   - |cos theta|: the smaller end value when theta does not cross pi/2;
//     for Q < 0 orbits (one hemisphere) never below mu_-.
// Padded by a margin for the FP64 trajectory's distance from the FP32 one.
struct VolReach {
    double R = 0.0;  // 1.5 r_outer
    double Z = 0.0;  // max over r of z_max(r) + 6 H(r)
    double margin = 0.05;
};

struct ReachRay {
    double r_turn = 0.0;  // smallest radius on the ray (r_h when it falls in)
    double mu_lo = 0.0;   // |cos theta| floor of a Q < 0 orbit, else 0
    bool far = false;     // never inside r <= R: no step test needed
};

__device__ ReachRay reach_ray(const DevScene& S, const VolReach& v, const double p[4]) {
    ReachRay rr;
    const double r_cam = S.cam_pos[1];
    const surr::RayConstants kc = surr::constants(S.a, S.cam_pos[2], p);
    rr.r_turn = (p[1] >= 0.0) ? r_cam : surr::turning_radius(S.M, S.a, kc, S.r_stop - 0.01, r_cam);
    rr.mu_lo = (kc.Q < 0.0) ? surr::graze_margin(S.a, kc) : 0.0;
    rr.far = rr.r_turn - (v.margin + 1e-3 * v.R) > v.R;
    return rr;
}

// True when the accepted step a -> b may touch the region.
__device__ __forceinline__ bool vol_reach(const VolReach& v, const ReachRay& rr, const Vec5<double>& a,
                                          const Vec5<double>& b) {
    if (rr.far) return false;
    const double pad = v.margin + 1e-3 * fmax(a.r, b.r);
    const double r_lo = (a.pr * b.pr > 0.0) ? fmin(a.r, b.r) : rr.r_turn;
    if (r_lo - pad > v.R) return false;
    const double ca = cos(a.th), cb = cos(b.th);
    if ((ca > 0.0) != (cb > 0.0)) return true;  // crosses the equator inside r <= R
    double c_lo = fmin(fabs(ca), fabs(cb));
    if (a.pth * b.pth <= 0.0 && rr.mu_lo > 0.0) c_lo = fmin(c_lo, rr.mu_lo);
    return fmax(r_lo - pad, 0.0) * c_lo - pad <= v.Z;
}

// kRGB = false (spectral): a settled sample gets its fate in out_fate (the
// spectra, zeroed, carry no sky). kRGB = true: the mixed form's sample
// buffers of the RGB render: a settled sample gets colour 0 and its fate, or,
// escaping under a star sky, its sky arc for the star pass (mixed_star_kernel)
// in sample_rgb and kFateStarPending; rays are counted here and terminations
// by the resolve, as in the thin-disk mixed form.
template <bool kRGB>
__global__ void __launch_bounds__(kSpecThreads, 4)
vol_speculate_kernel(const __grid_constant__ DevScene S, const DevTile tile, const VolReach reach,
                     uint32_t* __restrict__ out_fate, unsigned* __restrict__ queue,
                     unsigned* __restrict__ list, unsigned* __restrict__ list_count, double* __restrict__ sample_rgb,
                     DevStats* __restrict__ stats) {
    const int lane = threadIdx.x & 31;
    const bool sky = kRGB && S.stars_on;  // escapes look a star up: no early ends
    const int g2 = S.grid * S.grid;
    const unsigned total = static_cast<unsigned>(tile.w) * tile.h * g2;
    const float Mf = static_cast<float>(S.M), af = static_cast<float>(S.a);
    VolCounters cnt;
    unsigned q = ~0u;
    bool live = false, exhausted = false;
    Vec5<double> y{};
    double pt = 0.0, pph = 0.0, dl = 0.0;
    int retry = 0, step = 0;
    mixed::Tracker trk;
    ReachRay rr;
    Vec5<float> k1;  // FP32 f(y), kept from the previous attempt when k1_ok
    bool k1_ok = false;
    while (true) {
        const bool want = !live && !exhausted;
        const unsigned m = __ballot_sync(kWarp, want);
        unsigned base = 0;
        if (m) {
            const int leader = __ffs(m) - 1;
            if (lane == leader) base = atomicAdd(queue, static_cast<unsigned>(__popc(m)));
            base = __shfl_sync(kWarp, base, leader);
        }
        if (want) {
            const unsigned k = base + __popc(m & ((1u << lane) - 1u));
            if (k >= total) {
                exhausted = true;
            } else {
                q = k;
                const int pixel = static_cast<int>(q / g2), s = static_cast<int>(q % g2);
                const int i = tile.x0 + pixel % tile.w, j = tile.y0 + (pixel / tile.w) * tile.row_step;
                const int sy = s / S.grid, sx = s % S.grid;
                const double x = i + (sx + pixel_hash(i, j, s, 0)) * S.cell;
                const double yy = j + (sy + pixel_hash(i, j, s, 1)) * S.cell;
                double p[4];
                camera_momentum(S, x, yy, p);
                y = Vec5<double>{S.cam_pos[1], S.cam_pos[2], S.cam_pos[3], p[1], p[2]};
                pt = p[0];
                pph = p[3];
                rr = reach_ray(S, reach, p);
                dl = S.dl0;
                retry = 0;
                step = 0;
                trk.reset(false, 0.0, 0.0, 0.0, S.r_near_mixed, S.a, pt, pph, y.th);
                k1_ok = false;
                live = true;
            }
        }
        if (!__any_sync(kWarp, live)) break;
        int term = -1;
        bool retrace = false;
        if (live && retry == 0) {
            if (step >= S.max_steps) term = kTermMaxSteps;
            else if (y.r < S.r_stop) term = kTermHorizon;
            else if (y.r > S.r_escape) term = kTermEscaped;
            // never inside R: a turning point there, so it escapes, and the
            // plain stepping it gets has zero intensity; nothing to trace
            else if (!sky && step == 0 && rr.far) term = kTermEscaped;
        }
        if (live && term < 0) {
            if (!k1_ok) {
                k1 = mixed_k1(Mf, af, static_cast<float>(pt), static_cast<float>(pph), y);
                k1_ok = true;
            }
            Vec5<double> y5;
            Vec5<float> k7;
            const double err =
                mixed_attempt_k1(Mf, af, static_cast<float>(pt), static_cast<float>(pph), y, dl, k1, y5, k7);
            ++cnt.attempts;
            const StepDecision d = pi_control(err, S.tol_fp32, dl, retry, y5.r);
            if (d.accept) {
                ++cnt.accepted;
                retrace = vol_reach(reach, rr, y, y5) || trk.step(y, y5, dl);
                y = y5;
                k1 = k7;
                dl = d.next;
                retry = 0;
                ++step;
                if (retrace)
                    term = kTermMaxSteps;
                else if (!sky && mixed::certain_escape(y,
                                               fmax(fmax(mixed::kEscapeRMin * S.M, S.r_near_mixed),
                                                    reach.R + 2.0 * reach.margin + 2e-3 * y.r),
                                               step, S.max_steps))
                    term = kTermEscaped;  // no sky lookup: the escape is final once certain
            } else {
                dl = d.next;
                ++retry;
            }
        }
        bool queue_it = false;
        if (live && term >= 0) {
            live = false;
            if (kRGB) ++cnt.rays;
            if (retrace || term == kTermMaxSteps) {
                queue_it = true;
            } else if (kRGB) {
                const size_t o = 3 * static_cast<size_t>(q);
                if (term == kTermEscaped && S.stars_on) {
                    // k1 is the FP32 right-hand side at the escape state
                    const mixed::EscapeArc e = mixed::escape_arc(S.r_escape, y, k1);
                    sample_rgb[o + 0] = e.th0;
                    sample_rgb[o + 1] = e.ph0;
                    sample_rgb[o + 2] = __hiloint2double(__float_as_int(e.dth), __float_as_int(e.dph));
                    out_fate[q] = mixed::kFateStarPending;
                } else {
                    sample_rgb[o + 0] = 0.0;
                    sample_rgb[o + 1] = 0.0;
                    sample_rgb[o + 2] = 0.0;
                    out_fate[q] = static_cast<unsigned>(term);
                }
            } else {
                ++cnt.rays;
                if (term == kTermEscaped) ++cnt.escaped;
                else ++cnt.horizon;
                if (out_fate) out_fate[q] = static_cast<unsigned>(term);
            }
        }
        const unsigned qm = __ballot_sync(kWarp, queue_it);
        if (qm) {
            const int leader = __ffs(qm) - 1;
            unsigned b = 0;
            if (lane == leader) b = atomicAdd(list_count, static_cast<unsigned>(__popc(qm)));
            b = __shfl_sync(kWarp, b, leader);
            if (queue_it) list[b + __popc(qm & ((1u << lane) - 1u))] = q;
        }
    }
    flush_vol(stats, cnt, false);
}

// Per pixel and bin: the samples' J nu^3 summed in sample order from 0, then
// scaled by 1/spp, as the plain kernel's pixel sum. Grid-stride over pixel x bin.
__global__ void vol_resolve_kernel(const __grid_constant__ DevScene S, const DevTile tile, const double* freqs,
                                   int nb, const double* __restrict__ sample_J, double* __restrict__ out_spec) {
    const int g2 = S.grid * S.grid;
    const size_t n = static_cast<size_t>(tile.w) * tile.h * nb;
    for (size_t k = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t p = k / nb;
        const int b = static_cast<int>(k % nb);
        const double f = __ldg(freqs + b);
        double acc = 0.0;
        for (int s = 0; s < g2; ++s) acc = add_intensity(acc, sample_J[(p * g2 + s) * nb + b], f);
        const int qx = static_cast<int>(p % tile.w), qy = static_cast<int>(p / tile.w);
        out_spec[(static_cast<size_t>(qy) * tile.out_pitch + qx) * nb + b] = __dmul_rn(acc, S.inv_spp);
    }
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
namespace {
struct SpecShape {
    int sms = 0, per_fp64 = 1, per_list = 1, per_spec = 1, per_spec_rgb = 1;
};
const SpecShape& spec_shape() {
    return per_device_shape<SpecShape>([](int dev) {
        SpecShape sh;
        cudaDeviceGetAttribute(&sh.sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sh.per_fp64, vol_spectral_kernel<false>, kSpecThreads, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sh.per_list, vol_spectral_kernel<true>, kSpecThreads, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sh.per_spec, vol_speculate_kernel<false>, kSpecThreads, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sh.per_spec_rgb, vol_speculate_kernel<true>, kSpecThreads, 0);
        if (sh.per_spec_rgb < 1) sh.per_spec_rgb = 1;
        if (sh.per_fp64 < 1) sh.per_fp64 = 1;
        if (sh.per_list < 1) sh.per_list = 1;
        if (sh.per_spec < 1) sh.per_spec = 1;
        return sh;
    });
}
}  // namespace

size_t volume_spectral_scratch_elems(int nb) {
    const SpecShape& sh = spec_shape();
    const int per = sh.per_fp64 > sh.per_list ? sh.per_fp64 : sh.per_list;
    return static_cast<size_t>(4) * nb * sh.sms * per * kSpecThreads;
}

cudaError_t launch_vol_spectral_on(const DevScene& S, const DevTile& tile, const double* freqs, int nb,
                                   double* out_spec, uint32_t* out_fate, double* scratch, unsigned* queue,
                                   DevStats* stats, const volatile int* cancel, int blocks, cudaStream_t stream) {
    vol_spectral_kernel<false><<<blocks, kSpecThreads, 0, stream>>>(S, tile, freqs, nb, out_spec, out_fate, scratch,
                                                                     queue, stats, cancel, nullptr, nullptr,
                                                                     DevBatch{});
    return cudaGetLastError();
}

cudaError_t launch_volume_spectral(const DevScene& S, const DevTile& tile, const double* freqs, int nb,
                                   const SpectralOutputs& out, const LaunchResources& res, cudaStream_t stream) {
    const SpecShape& sh = spec_shape();
    const unsigned total = static_cast<unsigned>(tile.w) * static_cast<unsigned>(tile.h);
    if (total == 0) return cudaSuccess;
    int blocks = sh.sms * sh.per_fp64;
    const int needed = static_cast<int>((total + kSpecThreads - 1) / kSpecThreads);
    if (needed < blocks) blocks = needed;
    if (!res.spectral_scratch || res.spectral_scratch_elems < static_cast<size_t>(4) * nb * blocks * kSpecThreads)
        return cudaErrorInvalidValue;
    // work counter and finished-items counter
    cudaError_t e = cudaMemsetAsync(res.queue, 0, 2 * sizeof(unsigned int), stream);
    if (e != cudaSuccess) return e;
    return launch_vol_spectral_on(S, tile, freqs, nb, out.spec, out.fate, res.spectral_scratch, res.queue, res.stats,
                                  res.cancel, blocks, stream);
}

int vol_spectral_batch_max_blocks_per_sm() {
    return per_device_shape<int>([](int) {
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, vol_spectral_kernel<false, true>, kSpecThreads, 0);
        return n < 1 ? 1 : n;
    });
}

int vol_spectral_batch_threads() { return kSpecThreads; }

cudaError_t launch_vol_spectral_batch(const DevBatch& B, int nb_max, double* out_spec, double* scratch,
                                      size_t scratch_elems, unsigned* queue, DevStats* stats, int blocks,
                                      cudaStream_t stream) {
    if (B.n_chunks <= 0) return cudaSuccess;
    if (nb_max < 1 || !scratch || scratch_elems < static_cast<size_t>(4) * nb_max * blocks * kSpecThreads)
        return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(queue, 0, 2 * sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    vol_spectral_kernel<false, true><<<blocks, kSpecThreads, 0, stream>>>(
        DevScene{}, DevTile{}, nullptr, nb_max, out_spec, nullptr, scratch, queue, stats, nullptr, nullptr, nullptr, B);
    return cudaGetLastError();
}

size_t volume_mixed_scratch_bytes(const DevTile& tile, int g2, int nb) {
    const size_t n = static_cast<size_t>(tile.w) * tile.h * g2;
    // header (counters), the re-trace list (rounded up to 256 B), per-sample J
    // (rounded up to 256 B), the list ordering's bitmap and block sums
    return 1024 + ((n * sizeof(unsigned) + 255) / 256) * 256 + ((n * nb * sizeof(double) + 255) / 256) * 256 +
           order_list_scratch_bytes(n);
}

cudaError_t launch_volume_spectral_mixed(const DevScene& S, const DevTile& tile, const double* freqs, int nb,
                                         const SpectralOutputs& out, const LaunchResources& res, void* scratch,
                                         size_t scratch_bytes, double reach_z, cudaEvent_t* phase_events,
                                         cudaStream_t stream) {
    auto mark = [&](int k) {
        if (phase_events) cudaEventRecord(phase_events[k], stream);
    };
    const SpecShape& sh = spec_shape();
    const int g2 = S.grid * S.grid;
    const size_t n = static_cast<size_t>(tile.w) * tile.h * g2;
    if (n == 0) return cudaSuccess;
    if (scratch_bytes < volume_mixed_scratch_bytes(tile, g2, nb)) return cudaErrorInvalidValue;
    auto* base = static_cast<unsigned char*>(scratch);
    unsigned* queue2 = reinterpret_cast<unsigned*>(base + 256);
    unsigned* list_count = reinterpret_cast<unsigned*>(base + 512);
    unsigned* list = reinterpret_cast<unsigned*>(base + 1024);
    auto* sample_spec = reinterpret_cast<double*>(base + 1024 + ((n * sizeof(unsigned) + 255) / 256) * 256);
    unsigned char* order_scratch =
        reinterpret_cast<unsigned char*>(sample_spec) + ((n * nb * sizeof(double) + 255) / 256) * 256;
    if (static_cast<size_t>(order_scratch - base) + order_list_scratch_bytes(n) > scratch_bytes)
        return cudaErrorInvalidValue;
    int lb = sh.sms * sh.per_list;
    if (!res.spectral_scratch || res.spectral_scratch_elems < static_cast<size_t>(4) * nb * lb * kSpecThreads)
        return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(scratch, 0, 1024, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(res.queue, 0, sizeof(unsigned), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(sample_spec, 0, n * nb * sizeof(double), stream);
    if (e != cudaSuccess) return e;
    VolReach reach;
    reach.R = 1.5 * S.vol.r_outer;
    reach.Z = reach_z;
    reach.margin = S.mixed_margin;
    mark(0);
    const int need = static_cast<int>((n + kSpecThreads - 1) / kSpecThreads);
    int sb = sh.sms * sh.per_spec;
    if (need < sb) sb = need;
    vol_speculate_kernel<false><<<sb, kSpecThreads, 0, stream>>>(S, tile, reach, out.fate, res.queue, list,
                                                                list_count, nullptr, res.stats);
    e = cudaGetLastError();
    // the re-trace takes its samples in the FP64 form's order (the speculation
    // lists them in the order it finds them, the longest last)
    if (e == cudaSuccess) e = order_sample_list(list, list_count, n, order_scratch, stream);
    if (e != cudaSuccess) return e;
    mark(1);
    vol_spectral_kernel<true><<<lb, kSpecThreads, 0, stream>>>(S, tile, freqs, nb, sample_spec, out.fate,
                                                                res.spectral_scratch, queue2, res.stats, res.cancel,
                                                                list, list_count, DevBatch{});
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    mark(2);
    const size_t work = static_cast<size_t>(tile.w) * tile.h * nb;
    int rb = static_cast<int>((work + 255) / 256);
    if (rb > sh.sms * 8) rb = sh.sms * 8;
    if (rb < 1) rb = 1;
    vol_resolve_kernel<<<rb, 256, 0, stream>>>(S, tile, freqs, nb, sample_spec, out.spec);
    e = cudaGetLastError();
    mark(3);
    return e;
}

cudaError_t launch_volume_rgb_mixed(const DevScene& S, const DevTile& tile, const ThinOutputs& out,
                                    const LaunchResources& res, void* scratch, size_t scratch_bytes, double reach_z,
                                    cudaEvent_t* phase_events, cudaStream_t stream) {
    auto mark = [&](int k) {
        if (phase_events) cudaEventRecord(phase_events[k], stream);
    };
    const SpecShape& sh = spec_shape();
    const int g2 = S.grid * S.grid;
    const size_t n = static_cast<size_t>(tile.w) * tile.h * g2;
    if (n == 0) return cudaSuccess;
    if (scratch_bytes < mixed_scratch_bytes(tile, g2)) return cudaErrorInvalidValue;
    const DevMixedBuffers mb = mixed_buffers(scratch, n, res.queue);
    cudaError_t e = cudaMemsetAsync(scratch, 0, 1024, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(res.queue, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    VolReach reach;
    reach.R = 1.5 * S.vol.r_outer;
    reach.Z = reach_z;
    reach.margin = S.mixed_margin;
    mark(0);
    const int need = static_cast<int>((n + kSpecThreads - 1) / kSpecThreads);
    int sb = sh.sms * sh.per_spec_rgb;
    if (need < sb) sb = need;
    vol_speculate_kernel<true><<<sb, kSpecThreads, 0, stream>>>(S, tile, reach, mb.sample_fate, res.queue,
                                                               mb.retrace_list, mb.retrace_count, mb.sample_rgb,
                                                               res.stats);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    mark(1);
    e = launch_mixed_stars(S, tile, mb, stream);
    if (e != cudaSuccess) return e;
    mark(2);
    // the re-trace takes its samples in the FP64 form's order (the longest rays
    // would otherwise start last)
    e = order_sample_list(mb.retrace_list, mb.retrace_count, n, mixed_order_scratch(scratch, n), stream);
    if (e != cudaSuccess) return e;
    e = launch_volume_rgb_retrace(S, tile, mb, res.stats, res.cancel, stream);
    if (e != cudaSuccess) return e;
    mark(3);
    e = launch_mixed_resolve(S, tile, mb, out, res.stats, stream);
    mark(4);
    return e;
}

}  // namespace grrt_b200
