// Volumetric disk, RGB render: the outer adaptive DP45 loop with the
// near-disk step clamp and the ray-march hand-over
// (src/geodesic_tracer.cpp:23-181), and the fixed-step RK4 march with
// three-channel radiative transfer (src/geodesic_tracer.cpp:183-337). The
// spectral render is vol_spectral.cu; the spectral entry point without device
// allocation (below) launches that kernel on a fixed scratch.
//
// Same persistent execution model as the thin-disk kernel: a lane owns one
// pixel, one loop iteration advances each live ray by one DP45 attempt (outer
// phase) or one RK4 march step (march phase); the three channels' transfer
// state sits in registers. The list instantiation is the FP64 re-trace of the
// mixed form (its speculation is in vol_spectral.cu).
// One shared body of the FP64 right-hand side instead of inlined copies: the
// launches end on a few long rays, where instruction fetch stalls (Kerr
// a=0.9, 512x512 RGB: 49 -> 41 ms for the FP64 form on B200). The FP64 form
// and the mixed form's re-trace are both in this file, so their arithmetic is
// identical.
#define GRRT_RHS_CALL_F64 1
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "launch_cache.h"
#include "integrate.cuh"
#include "render_launch.h"
#include "shading.cuh"
#include "vol_steps.cuh"
#include "volume.cuh"

namespace grrt_b200 {

namespace {

constexpr int kVolThreads = 128;
constexpr unsigned kFullMask = 0xffffffffu;

}  // namespace

// Three channels in registers; the march ends when all T < 1e-6.
// kList = false: work item = pixel of the tile, spp samples summed into the
// outputs. kList = true (the mixed form's re-trace): work item k = sample
// list[k] (pixel * grid^2 + s); out_d[3 q ..] receives the sample's colour and
// out_fate[q] its fate; rays and terminations are counted by the mixed form's
// other passes.
template <bool kList>
__global__ void __launch_bounds__(kVolThreads)
vol_render_kernel(const __grid_constant__ DevScene S, const DevTile tile, float4* __restrict__ out_rgba,
                  double* __restrict__ out_d, uint32_t* __restrict__ out_fate, unsigned int* __restrict__ queue,
                  DevStats* __restrict__ stats, const volatile int* __restrict__ cancel,
                  const unsigned* __restrict__ list, const unsigned* __restrict__ list_count) {
    const DevVolume& V = S.vol;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const unsigned total = kList ? *list_count : static_cast<unsigned>(tile.w) * static_cast<unsigned>(tile.h);
    const int grid2 = S.grid * S.grid;

    VolCounters cnt;
    int pix = -1, smp = 0;
    double acc[3] = {0.0, 0.0, 0.0};
    bool live = false, need_start = false, marching = false;
    Vec5<double> y{}, prev{};
    Vec5<double> k1{};  // f(y) while k1_ok: the last accepted attempt's k7 or this step's first stage
    bool k1_ok = false;
    double pt = 0.0, pph = 0.0, dl = 0.0, dlambda = 0.0;
    int retry = 0, step = 0, entries = 0;
    // transfer state (RGB in registers)
    double J[3] = {0.0, 0.0, 0.0}, Tt[3] = {1.0, 1.0, 1.0};
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
                    pix = static_cast<int>(kList ? list[q] : q);  // kList: the listed sample
                    smp = 0;
                    acc[0] = acc[1] = acc[2] = 0.0;
                } else {
                    pix = -2;
                }
            }
        }
        if (!live && pix >= 0) {
            const int pixel = kList ? pix / grid2 : pix;
            const int s = kList ? pix % grid2 : smp;
            const int qx = pixel % tile.w, qy = pixel / tile.w;
            const int i = tile.x0 + qx, j = tile.y0 + qy * tile.row_step;
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
            J[0] = J[1] = J[2] = 0.0;
            Tt[0] = Tt[1] = Tt[2] = 1.0;
            k1_ok = false;
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
                const bool opaque = (Tt[0] < 1e-6 && Tt[1] < 1e-6 && Tt[2] < 1e-6);
                if (!opaque && vol_enters(V, prev, y)) {
                    // march from the pre-step state
                    marching = true;
                    ++entries;
                    ms = prev;
                    ds = vol_march_start(V, ms, been_inside);
                    mcount = 0;
                }
                // the next outer step starts now, or when the march ends
                if (!marching) need_start = true;
            }
        } else if (live && term < 0 && marching) {
            // ---- one RK4 march step ----
            bool end = vol_march_rgb_step(S, pt, pph, ms, ds, been_inside, J, Tt, cnt);
            ++mcount;
            if (!end && mcount >= 4096) end = true;
            if (end) {
                marching = false;
                y = ms;  // the outer loop continues from the march's end state
                k1_ok = false;
                need_start = true;
            }
        }

        // ---- finish a terminated sample ----
        if (live && term >= 0) {
            live = false;
            if (!kList) {
                ++cnt.rays;
                if (term == kTermEscaped) ++cnt.escaped;
                else if (term == kTermHorizon) ++cnt.horizon;
                else ++cnt.maxsteps;
            }
            double col[3];
            for (int ch = 0; ch < 3; ++ch) {
                const double nu = rgb_nu(ch);
                col[ch] = 0.0 + J[ch] * nu * nu * nu;
            }
            if (term == kTermEscaped && S.stars_on) {
                const double bright = star_brightness(S.stars, y.th, y.ph);
                for (int ch = 0; ch < 3; ++ch) col[ch] += bright;
            }
            if (kList) {
                const size_t q = static_cast<size_t>(pix);
                for (int ch = 0; ch < 3; ++ch) out_d[3 * q + ch] = col[ch];
                const unsigned ne = (entries > 0x3fffffff) ? 0x3fffffffu : static_cast<unsigned>(entries);
                out_fate[q] = static_cast<unsigned>(term) | (ne << 2);
                pix = -1;
                atomicAdd(queue + 1, 1u);  // finished items, for progress reports
            } else {
                for (int ch = 0; ch < 3; ++ch) acc[ch] = acc[ch] + col[ch];
                if (out_fate) {
                    const unsigned ne = (entries > 0x3fffffff) ? 0x3fffffffu : static_cast<unsigned>(entries);
                    out_fate[static_cast<size_t>(pix) * grid2 + smp] = static_cast<unsigned>(term) | (ne << 2);
                }
                if (++smp == grid2) {
                    const int qx = pix % tile.w, qy = pix / tile.w;
                    const size_t o = static_cast<size_t>(qy) * tile.out_pitch + qx;
                    const double r0 = acc[0] * S.inv_spp, r1 = acc[1] * S.inv_spp, r2 = acc[2] * S.inv_spp;
                    if (out_rgba)
                        out_rgba[o] = make_float4(static_cast<float>(r0), static_cast<float>(r1),
                                                  static_cast<float>(r2), 1.0f);
                    if (out_d) {
                        out_d[3 * o + 0] = r0;
                        out_d[3 * o + 1] = r1;
                        out_d[3 * o + 2] = r2;
                    }
                    pix = -1;
                    atomicAdd(queue + 1, 1u);  // finished items, for progress reports
                }
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
struct VolRgbShape {
    int sms = 0, per[2] = {1, 1};
};
int vol_rgb_blocks_per_sm(bool list, int& sms) {
    const VolRgbShape& sh = per_device_shape<VolRgbShape>([](int dev) {
        VolRgbShape v;
        cudaDeviceGetAttribute(&v.sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v.per[0], vol_render_kernel<false>, kVolThreads, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v.per[1], vol_render_kernel<true>, kVolThreads, 0);
        for (int& p : v.per)
            if (p < 1) p = 1;
        return v;
    });
    sms = sh.sms;
    return sh.per[list ? 1 : 0];
}
}  // namespace

cudaError_t launch_volume_rgb(const DevScene& S, const DevTile& tile, const ThinOutputs& out,
                              const LaunchResources& res, cudaStream_t stream) {
    int sms = 0;
    const int per = vol_rgb_blocks_per_sm(false, sms);
    const unsigned total = static_cast<unsigned>(tile.w) * static_cast<unsigned>(tile.h);
    if (total == 0) return cudaSuccess;
    int blocks = sms * per;
    const int needed = static_cast<int>((total + kVolThreads - 1) / kVolThreads);
    if (needed < blocks) blocks = needed;
    cudaError_t e = cudaMemsetAsync(res.queue, 0, 2 * sizeof(unsigned int), stream);
    if (e != cudaSuccess) return e;
    vol_render_kernel<false><<<blocks, kVolThreads, 0, stream>>>(S, tile, out.rgba, out.rgb64, out.fate, res.queue,
                                                                 res.stats, res.cancel, nullptr, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_volume_rgb_retrace(const DevScene& S, const DevTile& tile, const DevMixedBuffers& mb,
                                      DevStats* stats, const volatile int* cancel, cudaStream_t stream) {
    int sms = 0;
    const int per = vol_rgb_blocks_per_sm(true, sms);
    vol_render_kernel<true><<<sms * per, kVolThreads, 0, stream>>>(S, tile, nullptr, mb.sample_rgb, mb.sample_fate,
                                                                   mb.queue2, stats, cancel, mb.retrace_list,
                                                                   mb.retrace_count);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Spectral render without any device allocation.
//
// For callers that must not allocate device memory while they render: a host
// application that hands the renderer a fixed memory budget and forbids
// driver allocations during a frame, or a process running near the device
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
constexpr size_t kNoAllocSlots = static_cast<size_t>(kNoAllocBlocks) * kVolSpectralThreads;
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
    // Both forms: the FP64 kernel. The mixed form's output is bit-identical to
    // it, and its per-sample buffers would need an allocation.
    (void)form;
    return launch_vol_spectral_on(S, tile, freqs, nb, out_spec, nullptr, transfer, queue, stats, nullptr,
                                  kNoAllocBlocks, stream);
}

}  // namespace grrt_b200
