// Volumetric disk renders, RGB and spectral: the outer adaptive DP45 loop with
// the near-disk step clamp and the ray-march hand-over
// (src/geodesic_tracer.cpp:23-181 and 495-603), and the fixed-step RK4 march
// with per-channel or per-bin radiative transfer
// (src/geodesic_tracer.cpp:183-337 and 605-746).
//
// Same persistent execution model as the thin-disk kernel: a lane owns one
// pixel, one loop iteration advances each live ray by one DP45 attempt (outer
// phase) or one RK4 march step (march phase). Spectral transfer state
// (J, T, tau and the pixel sum, per bin) sits in a global scratch laid out
// [array][bin][lane slot], so the 32 lanes of a warp touch consecutive words.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "integrate.cuh"
#include "render_launch.h"
#include "shading.cuh"
#include "volume.cuh"

namespace grrt_b200 {

namespace {

constexpr int kVolThreads = 128;
constexpr unsigned kFullMask = 0xffffffffu;

struct VolCounters {
    unsigned long long attempts = 0, accepted = 0, rays = 0, horizon = 0, escaped = 0, maxsteps = 0;
    unsigned long long clamp = 0, march = 0, physics = 0, bins = 0, fp64 = 0;
};

__device__ __forceinline__ void flush_vol(DevStats* st, const VolCounters& c, bool cancelled) {
    unsigned long long v[11] = {c.attempts, c.accepted, c.rays, c.horizon, c.escaped, c.maxsteps,
                                c.clamp, c.march, c.physics, c.bins, c.fp64};
#pragma unroll
    for (int k = 0; k < 11; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(kFullMask, v[k], o);
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

// Observer-frame RGB frequencies (450, 550, 650 nm) of the RGB transfer.
__device__ __forceinline__ double rgb_nu(int ch) {
    constexpr double c = 2.997924e10;
    return ch == 0 ? c / 450e-7 : (ch == 1 ? c / 550e-7 : c / 650e-7);
}

}  // namespace

// kSpectral = false: three channels in registers, opaque when all T < 1e-6.
// kSpectral = true: nb bins in scratch, optically thick when all tau > 10.
template <bool kSpectral, int kForm>
__global__ void __launch_bounds__(kVolThreads)
vol_render_kernel(const __grid_constant__ DevScene S, const DevTile tile, const double* __restrict__ freqs,
                  int nb, float4* __restrict__ out_rgba, double* __restrict__ out_d, uint32_t* __restrict__ out_fate,
                  double* __restrict__ scratch, unsigned int* __restrict__ queue, DevStats* __restrict__ stats,
                  const volatile int* __restrict__ cancel) {
    const DevVolume& V = S.vol;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const unsigned total = static_cast<unsigned>(tile.w) * static_cast<unsigned>(tile.h);
    const int grid2 = S.grid * S.grid;
    const size_t slot = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    const size_t nslot = static_cast<size_t>(gridDim.x) * blockDim.x;
    // spectral scratch: J, T, tau, pixel sum; element (array, bin) at [(array*nb + bin)*nslot + slot]
    auto sc = [&](int arr, int b) -> double& { return scratch[(static_cast<size_t>(arr) * nb + b) * nslot + slot]; };
    const int med = nb / 2;

    VolCounters cnt;
    int pix = -1, smp = 0;
    double acc[3] = {0.0, 0.0, 0.0};
    bool live = false, need_start = false, marching = false;
    Vec5<double> y{}, prev{};
    double pt = 0.0, pph = 0.0, dl = 0.0, dlambda = 0.0;
    int retry = 0, step = 0, entries = 0;
    // transfer state (RGB in registers)
    double J[3] = {0.0, 0.0, 0.0}, Tt[3] = {1.0, 1.0, 1.0};
    int n_thick = 0;
    // march state
    Vec5<double> ms{};
    double ds = 0.0;
    int mcount = 0;
    bool been_inside = false;
    bool cancelled = false;
    unsigned iter = 0;

    while (true) {
        // ---- refill ----
        const bool want = (pix == -1);
        const unsigned want_mask = __ballot_sync(kFullMask, want);
        if (want_mask) {
            unsigned base = 0;
            const int leader = __ffs(want_mask) - 1;
            if (lane == leader) base = atomicAdd(queue, static_cast<unsigned>(__popc(want_mask)));
            base = __shfl_sync(kFullMask, base, leader);
            if (want) {
                const unsigned q = base + __popc(want_mask & lt_mask);
                if (q < total) {
                    pix = static_cast<int>(q);
                    smp = 0;
                    acc[0] = acc[1] = acc[2] = 0.0;
                    if (kSpectral)
                        for (int b = 0; b < nb; ++b) sc(3, b) = 0.0;
                } else {
                    pix = -2;
                }
            }
        }
        if (!live && pix >= 0) {
            const int qx = pix % tile.w, qy = pix / tile.w;
            const int i = tile.x0 + qx, j = tile.y0 + qy;
            const int sy = smp / S.grid, sx = smp % S.grid;
            const double x = i + (sx + pixel_hash(i, j, smp, 0)) * S.cell;
            const double yy = j + (sy + pixel_hash(i, j, smp, 1)) * S.cell;
            double p[4];
            camera_momentum(S, x, yy, p);
            y = Vec5<double>{S.cam_pos[1], S.cam_pos[2], S.cam_pos[3], p[1], p[2]};
            pt = p[0];
            pph = p[3];
            dlambda = S.dl0;
            step = 0;
            entries = 0;
            marching = false;
            J[0] = J[1] = J[2] = 0.0;
            Tt[0] = Tt[1] = Tt[2] = 1.0;
            n_thick = 0;
            if (kSpectral)
                for (int b = 0; b < nb; ++b) {
                    sc(0, b) = 0.0;
                    sc(1, b) = 1.0;
                    sc(2, b) = 0.0;
                }
            live = true;
            need_start = true;
        }

        int term = -1;
        // ---- start of an outer step: termination tests, then the near-disk clamp ----
        if (live && need_start) {
            if (step >= S.max_steps) term = kTermMaxSteps;
            else if (y.r < S.r_stop) term = kTermHorizon;
            else if (y.r > S.r_escape) term = kTermEscaped;
            if (term < 0) {
                const double r = y.r;
                if (r >= V.r_horizon * 0.9 && r <= V.r_outer * 1.5) {
                    double st, ct;
                    sincos(y.th, &st, &ct);
                    const double z = r * ct;
                    const double H = v_scale_height(V, r);
                    const double zm = v_zmax(V, r);
                    if (fabs(z) < zm + 6.0 * H) {
                        const Vec5<double> d = kerr_rhs<double>(S.M, S.a, pt, pph, y);
                        ++cnt.clamp;
                        const double dz_dl = fabs(ct * d.r - r * st * d.th);
                        if (dz_dl > 1e-20) {
                            const double dl_max = vmax(0.25 * H / dz_dl, H / 64.0);
                            dlambda = vmin(dlambda, dl_max);
                        }
                    }
                }
                prev = y;
                dl = dlambda;
                retry = 0;
                need_start = false;
            }
        }

        if (live && term < 0 && !marching) {
            // ---- one DP45 attempt ----
            Vec5<double> y5;
            double err, tol = S.tol;
            if (kForm == kFormMixed && y.r > S.fp32_r_min) {
                Vec5<float> k7;
                err = mixed_attempt_impl(static_cast<float>(S.M), static_cast<float>(S.a), static_cast<float>(pt),
                                         static_cast<float>(pph), y, dl, y5, k7);
                tol = S.tol_fp32;
            } else {
                err = dp45_attempt<double>(S.M, S.a, pt, pph, y, dl, y5);
                ++cnt.fp64;
            }
            ++cnt.attempts;
            const StepDecision d = pi_control(err, tol, dl, retry, y5.r);
            if (!d.accept) {
                dl = d.next;
                ++retry;
            } else {
                ++cnt.accepted;
                y = y5;
                dlambda = d.next;
                ++step;  // the reference's loop counter advances on every outer iteration
                // hand-over to the ray-march (src/geodesic_tracer.cpp:105-153)
                bool opaque = false;
                if (!kSpectral) opaque = (Tt[0] < 1e-6 && Tt[1] < 1e-6 && Tt[2] < 1e-6);
                if (!opaque) {
                    const double hp = kHalfPi;
                    const double d_prev = prev.th - hp, d_new = y.th - hp;
                    const double r_new = y.r, r_prev = prev.r;
                    const double z_new = r_new * cos(y.th);
                    const double z_prev = r_prev * cos(prev.th);
                    const bool crossed = (d_prev * d_new < 0.0) && fabs(d_prev - d_new) > 1e-12;
                    const bool inside_now = v_inside(V, r_new, z_new);
                    const double zm_new = v_zmax(V, r_new), H_new = v_scale_height(V, r_new);
                    const double H_prev = v_scale_height(V, r_prev);
                    const bool near = (fabs(z_new) < zm_new + 2.0 * H_new ||
                                       fabs(z_prev) < v_zmax(V, r_prev) + 2.0 * H_prev) &&
                                      r_new >= V.r_horizon && r_new <= V.r_outer;
                    if (crossed || inside_now || near) {
                        const double r_lo = vmin(r_prev, r_new), r_hi = vmax(r_prev, r_new);
                        if (r_hi >= V.r_horizon && r_lo <= V.r_outer && r_prev >= V.r_horizon * 0.9 &&
                            r_prev <= V.r_outer * 1.5) {
                            // march from the pre-step state
                            marching = true;
                            ++entries;
                            ms = prev;
                            const double r0 = ms.r;
                            const double z0 = r0 * cos(ms.th);
                            const double H0 = v_scale_height(V, r0);
                            been_inside = v_inside(V, r0, z0);
                            ds = been_inside ? H0 / 16.0 : vmin(fabs(z0) / 8.0, H0 * 2.0);
                            mcount = 0;
                        }
                    }
                }
                // the next outer step starts now, or when the march ends
                if (!marching) need_start = true;
            }
        } else if (live && term < 0 && marching) {
            // ---- one RK4 march step ----
            const Vec5<double> ns = rk4_step<double>(S.M, S.a, pt, pph, ms, ds);
            ++mcount;
            ++cnt.march;
            const double r = ns.r, theta = ns.th;
            double st, ct;
            sincos(theta, &st, &ct);
            const double z = r * ct;
            bool end = false;
            if (r < V.r_horizon || r > V.r_outer) {
                end = true;
            } else if (kSpectral ? (n_thick == nb) : (Tt[0] < 1e-6 && Tt[1] < 1e-6 && Tt[2] < 1e-6)) {
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
                        const int nbins = kSpectral ? nb : 3;
                        for (int b = 0; b < nbins; ++b) {
                            const double nu = ag * (kSpectral ? __ldg(freqs + b) : rgb_nu(b));
                            const double ka = v_kappa_abs(V, nu, ir, fr, iT, fT);
                            if (b == (kSpectral ? med : 1)) ka_med = ka;
                            const double kt = ka + ke;
                            const double eps = (kt > 0.0) ? ka / kt : 1.0;
                            const double dtau = kt * rho * dsp;
                            const double B = planck_nu(nu, Tl);
                            const double Sv = eps * B / (nu * nu * nu);
                            const double e = exp(-dtau);
                            if (kSpectral) {
                                double& tau = sc(2, b);
                                const bool was = !(tau <= 10.0);
                                tau += dtau;
                                n_thick += (!(tau <= 10.0)) - was;
                                double& Tb = sc(1, b);
                                sc(0, b) += Tb * Sv * (1.0 - e);
                                Tb *= e;
                            } else {
                                J[b] += Tt[b] * Sv * (1.0 - e);
                                Tt[b] *= e;
                            }
                        }
                        cnt.bins += static_cast<unsigned long long>(nbins);
                        const double at = (ka_med + ke) * rho;
                        const double ds_tau = (at > 0.0) ? 0.05 / at : ds * 2.0;
                        const double ds_geo = 0.1 * vmax(r - V.r_horizon, 0.5);
                        ds = vclamp(vmin(ds_tau, ds_geo), H / 64.0, H);
                    }
                }
            }
            ms = ns;
            if (!end && mcount >= 4096) end = true;
            if (end) {
                marching = false;
                y = ms;  // the outer loop continues from the march's end state
                need_start = true;
            }
        }

        // ---- finish a terminated sample ----
        if (live && term >= 0) {
            live = false;
            ++cnt.rays;
            if (term == kTermEscaped) ++cnt.escaped;
            else if (term == kTermHorizon) ++cnt.horizon;
            else ++cnt.maxsteps;
            if (kSpectral) {
                for (int b = 0; b < nb; ++b) {
                    const double f = __ldg(freqs + b);
                    sc(3, b) += sc(0, b) * f * f * f;
                }
            } else {
                double col[3];
                for (int ch = 0; ch < 3; ++ch) {
                    const double nu = rgb_nu(ch);
                    col[ch] = 0.0 + J[ch] * nu * nu * nu;
                }
                if (term == kTermEscaped && S.stars_on) {
                    const double bright = star_brightness(S.stars, y.th, y.ph);
                    for (int ch = 0; ch < 3; ++ch) col[ch] += bright;
                }
                for (int ch = 0; ch < 3; ++ch) acc[ch] = acc[ch] + col[ch];
            }
            if (out_fate) {
                const unsigned ne = (entries > 0x3fffffff) ? 0x3fffffffu : static_cast<unsigned>(entries);
                out_fate[static_cast<size_t>(pix) * grid2 + smp] = static_cast<unsigned>(term) | (ne << 2);
            }
            if (++smp == grid2) {
                const int qx = pix % tile.w, qy = pix / tile.w;
                const size_t o = static_cast<size_t>(qy) * tile.out_pitch + qx;
                if (kSpectral) {
                    double* dst = out_d + o * nb;
                    for (int b = 0; b < nb; ++b) dst[b] = sc(3, b) * S.inv_spp;
                } else {
                    const double r0 = acc[0] * S.inv_spp, r1 = acc[1] * S.inv_spp, r2 = acc[2] * S.inv_spp;
                    if (out_rgba)
                        out_rgba[o] = make_float4(static_cast<float>(r0), static_cast<float>(r1),
                                                  static_cast<float>(r2), 1.0f);
                    if (out_d) {
                        out_d[3 * o + 0] = r0;
                        out_d[3 * o + 1] = r1;
                        out_d[3 * o + 2] = r2;
                    }
                }
                pix = -1;
            }
        }

        if (cancel && ((++iter & 1023u) == 0)) {
            int c = 0;
            if (lane == 0) c = *cancel;
            c = __shfl_sync(kFullMask, c, 0);
            if (c) {
                cancelled = true;
                break;
            }
        }
        if (!__any_sync(kFullMask, live || pix >= -1)) break;
    }
    flush_vol(stats, cnt, cancelled);
}

namespace {

template <bool kSpectral, int kForm>
cudaError_t launch_vol(const DevScene& S, const DevTile& tile, const double* freqs, int nb, float4* rgba,
                       double* out_d, uint32_t* fate, const LaunchResources& res, cudaStream_t stream) {
    static int blocks_per_sm = 0, num_sms = 0;
    if (blocks_per_sm == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, vol_render_kernel<kSpectral, kForm>,
                                                      kVolThreads, 0);
        if (blocks_per_sm < 1) blocks_per_sm = 1;
    }
    const unsigned total = static_cast<unsigned>(tile.w) * static_cast<unsigned>(tile.h);
    if (total == 0) return cudaSuccess;
    int blocks = num_sms * blocks_per_sm;
    const int needed = static_cast<int>((total + kVolThreads - 1) / kVolThreads);
    if (needed < blocks) blocks = needed;
    double* scratch = nullptr;
    if (kSpectral) {
        // J, T, tau and the pixel sum per bin and lane slot.
        const size_t need = static_cast<size_t>(4) * nb * blocks * kVolThreads;
        scratch = res.spectral_scratch;
        if (!scratch || res.spectral_scratch_elems < need) return cudaErrorInvalidValue;
    }
    cudaError_t e = cudaMemsetAsync(res.queue, 0, sizeof(unsigned int), stream);
    if (e != cudaSuccess) return e;
    vol_render_kernel<kSpectral, kForm><<<blocks, kVolThreads, 0, stream>>>(
        S, tile, freqs, nb, rgba, out_d, fate, scratch, res.queue, res.stats, res.cancel);
    return cudaGetLastError();
}

}  // namespace

size_t volume_spectral_scratch_elems(int nb) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vol_render_kernel<true, kFormFP64>, kVolThreads, 0);
    int per_sm_m = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_m, vol_render_kernel<true, kFormMixed>, kVolThreads, 0);
    if (per_sm_m > per_sm) per_sm = per_sm_m;
    if (per_sm < 1) per_sm = 1;
    return static_cast<size_t>(4) * nb * sms * per_sm * kVolThreads;
}

cudaError_t launch_volume_rgb(const DevScene& S, const DevTile& tile, const ThinOutputs& out,
                              const LaunchResources& res, int form, cudaStream_t stream) {
    if (form == kFormMixed)
        return launch_vol<false, kFormMixed>(S, tile, nullptr, 0, out.rgba, out.rgb64, out.fate, res, stream);
    return launch_vol<false, kFormFP64>(S, tile, nullptr, 0, out.rgba, out.rgb64, out.fate, res, stream);
}

cudaError_t launch_volume_spectral(const DevScene& S, const DevTile& tile, const double* freqs, int nb,
                                   const SpectralOutputs& out, const LaunchResources& res, int form,
                                   cudaStream_t stream) {
    if (form == kFormMixed)
        return launch_vol<true, kFormMixed>(S, tile, freqs, nb, nullptr, out.spec, out.fate, res, stream);
    return launch_vol<true, kFormFP64>(S, tile, freqs, nb, nullptr, out.spec, out.fate, res, stream);
}

// ---------------------------------------------------------------------------
// Spectral render without any device allocation.
//
// For callers that must not allocate device memory while they render: a host
// application that hands the renderer a fixed memory budget and forbids
// driver allocations during a frame, a pipeline recorded into a CUDA graph
// (cudaMalloc cannot be captured), or a process running near the device
// memory limit where an allocation could fail mid-frame. The per-launch
// scratch (work counter, counters, and the per-lane J, T, tau and pixel-sum
// transfer state) lives in the file-scope array below instead of cudaMalloc'd
// memory. Every GPU that loads the library holds this array until the process
// exits.
//
// Limits: at most kNoAllocMaxBins frequency bins, one fixed grid of
// kNoAllocBlocks x kVolThreads lanes. All calls share the one array, which
// keeps the last call's contents; launches of this entry point that overlap on
// the GPU (two streams, or two threads) race on it and must be serialised by
// the caller.
// ---------------------------------------------------------------------------
namespace {
constexpr int kNoAllocMaxBins = 32;
constexpr int kNoAllocBlocks = 148;  // one block per B200 SM
constexpr size_t kNoAllocSlots = static_cast<size_t>(kNoAllocBlocks) * kVolThreads;
constexpr size_t kNoAllocHeader = 512;  // [0,256): work counter, [256,512): DevStats
constexpr size_t kNoAllocBytes = kNoAllocHeader + sizeof(double) * 4 * kNoAllocMaxBins * kNoAllocSlots;
static_assert(sizeof(DevStats) <= 256, "stats must fit the header");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
unsigned char* g_noalloc_ptr[kMaxDevices] = {};
std::mutex g_noalloc_mutex;
}  // namespace

int volume_spectral_noalloc_max_bins() { return kNoAllocMaxBins; }
size_t volume_spectral_noalloc_bytes() { return kNoAllocBytes; }

cudaError_t launch_volume_spectral_noalloc(const DevScene& S, const DevTile& tile, const double* freqs, int nb,
                                           double* out_spec, int form, cudaStream_t stream) {
    if (nb < 1 || nb > kNoAllocMaxBins) return cudaErrorInvalidValue;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    unsigned char* base = nullptr;
    {
        // Set-up, once per device with that device current: the host-side name
        // of the array is not a device address, so ask the runtime for it.
        std::lock_guard<std::mutex> lk(g_noalloc_mutex);
        if (!g_noalloc_ptr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) return e;
            g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
        }
        base = g_noalloc_ptr[dev];
    }
    const unsigned total = static_cast<unsigned>(tile.w) * static_cast<unsigned>(tile.h);
    if (total == 0) return cudaSuccess;
    // The work counter must start at zero; the counters are cleared with it.
    e = cudaMemsetAsync(base, 0, kNoAllocHeader, stream);
    if (e != cudaSuccess) return e;
    auto* queue = reinterpret_cast<unsigned int*>(base);
    auto* stats = reinterpret_cast<DevStats*>(base + 256);
    auto* transfer = reinterpret_cast<double*>(base + kNoAllocHeader);
    if (form == kFormMixed)
        vol_render_kernel<true, kFormMixed><<<kNoAllocBlocks, kVolThreads, 0, stream>>>(
            S, tile, freqs, nb, nullptr, out_spec, nullptr, transfer, queue, stats, nullptr);
    else
        vol_render_kernel<true, kFormFP64><<<kNoAllocBlocks, kVolThreads, 0, stream>>>(
            S, tile, freqs, nb, nullptr, out_spec, nullptr, transfer, queue, stats, nullptr);
    return cudaGetLastError();
}

}  // namespace grrt_b200
