// Mixed-precision form of the thin-disk render: speculate in FP32, re-trace in
// FP64 the samples whose colour depends on the FP64 step sequence (the tests
// are in mixed_spec.cuh).
//
//   speculate: every sample is integrated with FP32 right-hand sides and FP64
//     state (mixed_attempt_k1) against a relaxed tolerance. A sample that
//     needs the FP64 step sequence is queued for the re-trace and dropped; a
//     horizon sample is final (colour 0); an escape stores its sky arc for the
//     star pass.
//   stars: each pending escape checks the star catalogue along its arc; a
//     star in reach queues it for the re-trace, otherwise its colour is 0.
//     (Its own pass, so the speculative warps never diverge into the star scan.)
//   re-trace: the queued samples are traced from the camera with the plain
//     form's arithmetic, lanes pulling from the queue (converged FP64 warps).
//   resolve: per pixel, the spp samples are summed in order and scaled, as
//     Renderer::render does (src/renderer.cpp:47-72).
//
// The batched form runs the same four phases over the samples of many
// cameras at once (one sample space, items in order), so each phase is one
// launch for the whole batch and every sample gets the arithmetic of its own
// camera's single render.
// One shared body of the FP64 right-hand side instead of seven inlined copies
// per attempt: less code to fetch (Kerr a=0.998, 1024x1024, 4 spp: 46.4 ->
// 43.4 ms for the FP64 form on B200). The FP64 form and the mixed form's
// re-trace must use the same setting, so that their arithmetic is identical.
#define GRRT_RHS_CALL_F64 1
#include <cuda_runtime.h>

#include <cstdint>

#include "launch_cache.h"
#include "integrate.cuh"
#include "mixed_spec.cuh"
#include "render_launch.h"
#include "shading.cuh"
#include "surrogate_geom.cuh"

namespace grrt_b200 {

namespace {

constexpr int kMixThreads = 128;
constexpr unsigned kMask = 0xffffffffu;
// Most samples one launch takes: the work counters run up to 32 items per
// warp past the end, and a cancel pushes them to 0x7f7f7f7f.
constexpr size_t kMaxSamples = 0x7f000000u;

__device__ __forceinline__ void sample_start(const DevScene& S, const DevTile& tile, unsigned q, int g2,
                                             Vec5<double>& y, double& pt, double& pph) {
    const int pix = static_cast<int>(q / g2), s = static_cast<int>(q % g2);
    const int i = tile.x0 + pix % tile.w, j = tile.y0 + (pix / tile.w) * tile.row_step;
    const int sy = s / S.grid, sx = s % S.grid;
    const double x = i + (sx + pixel_hash(i, j, s, 0)) * S.cell;
    const double yy = j + (sy + pixel_hash(i, j, s, 1)) * S.cell;
    double p[4];
    camera_momentum(S, x, yy, p);
    y = Vec5<double>{S.cam_pos[1], S.cam_pos[2], S.cam_pos[3], p[1], p[2]};
    pt = p[0];
    pph = p[3];
}

// Batch item holding sample q (kBySample) or output pixel q: the last item
// whose first sample (first pixel) is <= q; items are stored in that order.
template <bool kBySample>
__device__ __forceinline__ const DevBatchItem& batch_item(const DevBatch& B, size_t q) {
    int lo = 0, hi = B.n_items - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const size_t first = kBySample ? B.items[mid].sample0 : B.items[mid].out_offset;
        if (first <= q)
            lo = mid;
        else
            hi = mid - 1;
    }
    return B.items[lo];
}

// Camera ray of sample q. One camera: q indexes the tile's samples (pixel-major,
// spp samples per pixel). Batch: q indexes the samples of all items in item
// order, and the lane's scene becomes the item's.
template <bool kBatch>
__device__ __forceinline__ void start_ray(const DevScene& S0, const DevTile& tile, const DevBatch& B, unsigned q,
                                          const DevScene*& sp, Vec5<double>& y, double& pt, double& pph) {
    if (kBatch) {
        const DevBatchItem& it = batch_item<true>(B, q);
        const DevTile t{it.x0, it.y0, it.w, it.h, it.out_pitch};
        const unsigned local = static_cast<unsigned>(q - it.sample0);
        sp = B.scenes + it.scene;
        sample_start(*sp, t, local, sp->grid * sp->grid, y, pt, pph);
    } else {
        sample_start(S0, tile, q, S0.grid * S0.grid, y, pt, pph);
    }
}

// Queues sample q for the FP64 re-trace (warp-aggregated over the lanes that ask).
__device__ __forceinline__ void queue_retrace(bool want, unsigned q, const DevMixedBuffers& mb) {
    const int lane = threadIdx.x & 31;
    const unsigned m = __ballot_sync(kMask, want);
    if (!m) return;
    const int leader = __ffs(m) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(mb.retrace_count, static_cast<unsigned>(__popc(m)));
    base = __shfl_sync(kMask, base, leader);
    if (want) mb.retrace_list[base + __popc(m & ((1u << lane) - 1u))] = q;
}

__device__ __forceinline__ int start_test(const DevScene& S, int step, double r) {
    if (step >= S.max_steps) return kTermMaxSteps;
    if (r < S.r_stop) return kTermHorizon;
    if (r > S.r_escape) return kTermEscaped;
    return -1;
}

__device__ __forceinline__ void warp_add(DevStats* st, unsigned long long a, unsigned long long acc,
                                         unsigned long long rays, unsigned long long f64) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(kMask, a, o);
        acc += __shfl_xor_sync(kMask, acc, o);
        rays += __shfl_xor_sync(kMask, rays, o);
        f64 += __shfl_xor_sync(kMask, f64, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&st->attempts, a);
        atomicAdd(&st->accepted, acc);
        atomicAdd(&st->rays, rays);
        atomicAdd(&st->fp64_attempts, f64);
    }
}

}  // namespace

// Every kernel below comes in two instantiations: kBatch = false renders the
// tile of one camera (scene S0, a kernel parameter); kBatch = true renders
// every item of the batch B (scenes in global memory, one per lane's sample),
// over one sample space, so one launch per phase covers all cameras.
// Inside, S names the scene of the lane's current sample.

namespace {
// Per-warp staging of the FP32 speculation's starts in shared memory (one
// slot per lane, fields as arrays): the warp takes 32 samples at once, and
// every lane forms one sample's camera ray, its black-sky closed-form test and
// the FP32 first stage f(y), so that work runs with the whole warp instead of
// one lane at a time as rays end. Samples the closed-form test settles are
// written there and then; the rest are compacted into the slots, which lanes
// whose ray ended take in order.
struct SpecStage {
    double pr[32], pth[32], pt[32], pph[32];  // start momentum (r, theta, phi are the camera's)
    float k[5][32];                           // FP32 f(y) at the start
    unsigned q[32];                           // sample index
    const DevScene* sp[32];                   // batch: the sample's scene
};
}  // namespace

// Five resident blocks per SM (at most 96 registers): the issue-bound FP32
// pass gains more from the fifth block's warps than it loses to the few
// spilled registers (four blocks: 8.8 ms, five: 8.2 ms on the 1024x1024 4-spp
// frame on B200; six, with more spills, no better).
template <bool kBatch>
__global__ void __launch_bounds__(kMixThreads, 5)
mixed_speculate_kernel(const __grid_constant__ DevScene S0, const DevTile tile, const __grid_constant__ DevBatch B,
                       DevMixedBuffers mb, DevStats* stats) {
    __shared__ SpecStage stage_all[kMixThreads / 32];
    SpecStage& W = stage_all[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const DevScene* sp = nullptr;
#define S (kBatch ? *sp : S0)
    const unsigned total = kBatch ? B.n_samples
                                  : (mb.spec_list ? *mb.spec_count
                                                  : static_cast<unsigned>(tile.w) * tile.h * (S0.grid * S0.grid));
    float Mf = static_cast<float>(S0.M), af = static_cast<float>(S0.a);
    unsigned long long n_att = 0, n_acc = 0, n_rays = 0;
    // warp-uniform: prepared slots [ring_head, ring_n) and the queue state
    int ring_head = 0, ring_n = 0;
    bool drained = false;
    unsigned q = ~0u;
    bool live = false;
    Vec5<double> y;
    Vec5<float> k1;  // FP32 f(y), kept from the previous attempt
    double pt = 0, pph = 0, dl = 0;
    int retry = 0, step = 0;
    mixed::Tracker trk;
    while (true) {
        const unsigned need = __ballot_sync(kMask, !live);
        // ---- the warp prepares its next starts (every lane one sample) ----
        while (need && ring_head == ring_n && !drained) {
            unsigned base = 0;
            if (lane == 0) base = atomicAdd(mb.queue, 32u);
            base = __shfl_sync(kMask, base, 0);
            const int n_take = base < total ? static_cast<int>(min(32u, total - base)) : 0;
            if (n_take < 32) drained = true;
            bool keep = false;
            unsigned qq = 0;
            const DevScene* ssp = nullptr;
            Vec5<double> ys;
            double pts = 0.0, pphs = 0.0;
            if (lane < n_take) {
                qq = (!kBatch && mb.spec_list) ? mb.spec_list[base + lane] : base + lane;
                start_ray<kBatch>(S0, tile, B, qq, ssp, ys, pts, pphs);
                const DevScene& Ss = kBatch ? *ssp : S0;
                // Black sky: a ray whose smallest radius (closed form, from its
                // constants of motion) lies outside the disk, r_near and every
                // photon orbit escapes with colour 0 and no crossing.
                bool settled = false;
                if (!Ss.stars_on && (kBatch || !mb.spec_list)) {
                    const double p[4] = {pts, ys.pr, ys.pth, pphs};
                    const double m = kBatch ? Ss.mixed_margin : mb.margin;
                    const double r_near = kBatch ? Ss.r_near_mixed : mb.r_near;
                    const double r_gate =
                        fmax(fmax(mixed::kEscapeRMin * Ss.M, r_near), Ss.disk_on ? Ss.r_out + 2.0 * m : 0.0);
                    settled = surr::camera_ray_clears(Ss.M, Ss.a, Ss.r_stop - 0.01, Ss.cam_pos[1], Ss.cam_pos[2],
                                                      p, r_gate);
                }
                if (settled) {
                    const size_t o = 3 * static_cast<size_t>(qq);
                    mb.sample_rgb[o + 0] = 0.0;
                    mb.sample_rgb[o + 1] = 0.0;
                    mb.sample_rgb[o + 2] = 0.0;
                    mb.sample_fate[qq] = static_cast<unsigned>(kTermEscaped);
                    ++n_rays;
                } else {
                    keep = true;
                }
            }
            const unsigned km = __ballot_sync(kMask, keep);
            if (keep) {
                const int slot = __popc(km & lt_mask);
                const DevScene& Ss = kBatch ? *ssp : S0;
                const float Ms = kBatch ? static_cast<float>(Ss.M) : Mf;
                const float as = kBatch ? static_cast<float>(Ss.a) : af;
                const Vec5<float> f = mixed_k1(Ms, as, static_cast<float>(pts), static_cast<float>(pphs), ys);
                W.q[slot] = qq;
                if (kBatch) W.sp[slot] = ssp;
                W.pr[slot] = ys.pr;
                W.pth[slot] = ys.pth;
                W.pt[slot] = pts;
                W.pph[slot] = pphs;
                W.k[0][slot] = f.r;
                W.k[1][slot] = f.th;
                W.k[2][slot] = f.ph;
                W.k[3][slot] = f.pr;
                W.k[4][slot] = f.pth;
            }
            ring_head = 0;
            ring_n = __popc(km);
            __syncwarp();
        }
        // ---- lanes without a ray take the prepared starts in order ----
        if (need && ring_head < ring_n) {
            const int avail = ring_n - ring_head;
            const int rank = __popc(need & lt_mask);
            if (!live && rank < avail) {
                const int slot = ring_head + rank;
                q = W.q[slot];
                if (kBatch) {
                    sp = W.sp[slot];
                    Mf = static_cast<float>(S.M);
                    af = static_cast<float>(S.a);
                }
                y = Vec5<double>{S.cam_pos[1], S.cam_pos[2], S.cam_pos[3], W.pr[slot], W.pth[slot]};
                pt = W.pt[slot];
                pph = W.pph[slot];
                k1 = Vec5<float>{W.k[0][slot], W.k[1][slot], W.k[2][slot], W.k[3][slot], W.k[4][slot]};
                dl = S.dl0;
                retry = 0;
                step = 0;
                if (kBatch)
                    trk.reset(S.disk_on, S.r_in, S.r_out, S.mixed_margin, S.r_near_mixed, S.a, pt, pph, y.th);
                else
                    trk.reset(S.disk_on, S.r_in, S.r_out, mb.margin, mb.r_near, S.a, pt, pph, y.th);
                live = true;
            }
            ring_head += min(__popc(need), avail);
            __syncwarp();
        }
        if (!__any_sync(kMask, live)) break;
        int term = -1;
        bool retrace = false;
        Vec5<float> k7;
        if (live && retry == 0) term = start_test(S, step, y.r);
        if (live && term < 0) {
            Vec5<double> y5;
            const double err =
                mixed_attempt_k1(Mf, af, static_cast<float>(pt), static_cast<float>(pph), y, dl, k1, y5, k7);
            ++n_att;
            const StepDecision d = pi_control_f32(err, S.tol_fp32, dl, retry, y5.r);
            if (d.accept) {
                ++n_acc;
                retrace = trk.step(y, y5, dl);
                y = y5;
                k1 = k7;
                dl = d.next;
                retry = 0;
                ++step;
                term = retrace ? kTermMaxSteps : start_test(S, step, y.r);
                // black sky: an escape is final as soon as it is certain
                if (term < 0 && !S.stars_on) {
                    const double m = kBatch ? S.mixed_margin : mb.margin;
                    const double r_near = kBatch ? S.r_near_mixed : mb.r_near;
                    const double r_min = fmax(fmax(mixed::kEscapeRMin * S.M, r_near),
                                              S.disk_on ? S.r_out + 2.0 * m : 0.0);
                    if (mixed::certain_escape(y, r_min, step, S.max_steps)) term = kTermEscaped;
                }
            } else {
                dl = d.next;
                ++retry;
            }
        }
        bool queue = false;
        if (live && term >= 0) {
            live = false;
            if (kBatch || !mb.spec_list) ++n_rays;  // a list's samples are counted by its producer
            const size_t o = 3 * static_cast<size_t>(q);
            if (retrace || term == kTermMaxSteps) {
                queue = true;
            } else if (term == kTermEscaped && S.stars_on) {
                // an escape always ends an accepted step, so k7 is the
                // right-hand side at y
                const mixed::EscapeArc e = mixed::escape_arc(S.r_escape, y, k7);
                mb.sample_rgb[o + 0] = e.th0;
                mb.sample_rgb[o + 1] = e.ph0;
                mb.sample_rgb[o + 2] = __hiloint2double(__float_as_int(e.dth), __float_as_int(e.dph));
                mb.sample_fate[q] = mixed::kFateStarPending;
            } else {
                // horizon, or an escape with stars off: colour 0
                mb.sample_rgb[o + 0] = 0.0;
                mb.sample_rgb[o + 1] = 0.0;
                mb.sample_rgb[o + 2] = 0.0;
                mb.sample_fate[q] = static_cast<unsigned>(term);
            }
        }
        queue_retrace(queue, q, mb);
    }
#undef S
    warp_add(stats, n_att, n_acc, n_rays, 0ull);
}

// Star pass over the pending escapes: colour 0, or queued for the re-trace.
template <bool kBatch>
__global__ void __launch_bounds__(256)
mixed_star_kernel(const __grid_constant__ DevScene S0, const DevTile tile, const __grid_constant__ DevBatch B,
                  DevMixedBuffers mb) {
    const unsigned n = kBatch ? B.n_samples : static_cast<unsigned>(tile.w) * tile.h * (S0.grid * S0.grid);
    const unsigned stride = gridDim.x * blockDim.x;
    // whole warps iterate together so queue_retrace can ballot
    for (unsigned base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const unsigned q = base + threadIdx.x;
        bool queue = false;
        if (q < n && mb.sample_fate[q] == mixed::kFateStarPending) {
            const DevScene& S = kBatch ? B.scenes[batch_item<true>(B, q).scene] : S0;
            const size_t o = 3 * static_cast<size_t>(q);
            mixed::EscapeArc e;
            e.th0 = mb.sample_rgb[o + 0];
            e.ph0 = mb.sample_rgb[o + 1];
            const double packed = mb.sample_rgb[o + 2];
            e.dth = __int_as_float(__double2hiint(packed));
            e.dph = __int_as_float(__double2loint(packed));
            if (mixed::star_in_reach(S.stars, e)) {
                queue = true;
            } else {
                mb.sample_rgb[o + 0] = 0.0;
                mb.sample_rgb[o + 1] = 0.0;
                mb.sample_rgb[o + 2] = 0.0;
                mb.sample_fate[q] = static_cast<unsigned>(kTermEscaped);
            }
        }
        queue_retrace(queue, q, mb);
    }
}

// FP64 re-trace of the queued samples with the plain form's arithmetic.
namespace {

// Per-warp staging of the FP64 trace in shared memory, one slot per lane,
// fields stored as arrays so that lane k touches element k (no bank
// conflicts beyond the two wavefronts of an 8-byte access).
//   Prepared starts: the warp takes 32 work items at once and every lane
//   forms one item's camera ray and the first stage f(y) of its first
//   attempt, so this work runs with the whole warp instead of one lane at a
//   time as rays end; lanes whose ray ended take the slots in order.
//   Deferred star lookups: an escape under a star sky parks its direction and
//   colour here, and the warp looks up up to 32 of them at once.
struct WarpStage {
    double pr[32], pth[32], pt[32], pph[32];  // start momentum (r, theta, phi are the camera's)
    double k[5][32];                          // f(y) at the start
    unsigned q[32];                           // sample index
    const DevScene* sp[32];                   // batch: the sample's scene
    double th[32], ph[32], c[3][32];          // escape direction and colour so far
    unsigned pq[32], pfate[32];
    const DevScene* psp[32];
};

// Writes the parked escapes' colours (colour + star brightness, the order of
// the single-lane form) and fate words; lanes below n each take one.
template <bool kBatch>
__device__ __forceinline__ void flush_star_lookups(WarpStage& W, int n, const DevScene& S0,
                                                   const DevMixedBuffers& mb) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
    if (lane < n) {
        const DevScene& Sl = kBatch ? *W.psp[lane] : S0;
        const double b = star_brightness(Sl.stars, W.th[lane], W.ph[lane]);
        const size_t q = W.pq[lane];
        mb.sample_rgb[3 * q + 0] = W.c[0][lane] + b;
        mb.sample_rgb[3 * q + 1] = W.c[1][lane] + b;
        mb.sample_rgb[3 * q + 2] = W.c[2][lane] + b;
        mb.sample_fate[q] = W.pfate[lane];
    }
    __syncwarp();
}

}  // namespace

// FP64 trace of samples into per-sample colours and fate words, the plain
// method of GeodesicTracer::trace (src/geodesic_tracer.cpp:23-181): the FP64
// form traces every sample of the tile (kList = false, work item = sample),
// the mixed form's re-trace the listed ones (kList = true, work item = entry
// of mb.retrace_list). Each loop iteration is one DP45 attempt for every lane
// with a live ray. The per-sample work around it (camera ray, first
// right-hand side, star lookup) runs for 32 samples at a time with the whole
// warp (WarpStage), not lane by lane as rays end. counter: the work counter
// (zeroed by the launcher), total: the item count for kList = false.
template <bool kList, bool kBatch>
__global__ void __launch_bounds__(kMixThreads, 4)
fp64_trace_kernel(const __grid_constant__ DevScene S0, const DevTile tile, const __grid_constant__ DevBatch B,
                  DevMixedBuffers mb, unsigned* __restrict__ counter, unsigned total_items, DevStats* stats) {
    __shared__ WarpStage stage_all[kMixThreads / 32];
    WarpStage& W = stage_all[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const DevScene* sp = nullptr;
#define S (kBatch ? *sp : S0)
    const unsigned total = kList ? *mb.retrace_count : total_items;
    unsigned long long n_att = 0, n_acc = 0, n_rays = 0;
    // warp-uniform: prepared slots [ring_head, ring_n), parked lookups, queue state
    int ring_head = 0, ring_n = 0, pend_n = 0;
    bool drained = false;
    unsigned q = 0;
    bool live = false;
    Vec5<double> y, k1;  // k1 = f(y)
    double pt = 0, pph = 0, dl = 0;
    int retry = 0, step = 0, ncross = 0;
    double c0 = 0, c1 = 0, c2 = 0;
    while (true) {
        const unsigned need = __ballot_sync(kMask, !live);
        // ---- the warp prepares its next 32 starts (every lane one) ----
        if (need && ring_head == ring_n && !drained) {
            unsigned base = 0;
            if (lane == 0) base = atomicAdd(counter, 32u);
            base = __shfl_sync(kMask, base, 0);
            ring_head = 0;
            ring_n = base < total ? static_cast<int>(min(32u, total - base)) : 0;
            if (ring_n < 32) drained = true;
            if (lane < ring_n) {
                const unsigned w = base + lane;
                const unsigned qq = kList ? mb.retrace_list[w] : w;
                const DevScene* ssp = nullptr;
                Vec5<double> ys;
                double pts, pphs;
                start_ray<kBatch>(S0, tile, B, qq, ssp, ys, pts, pphs);
                const DevScene& Ss = kBatch ? *ssp : S0;
                const Vec5<double> f = kerr_rhs<double>(Ss.M, Ss.a, pts, pphs, ys);
                W.q[lane] = qq;
                if (kBatch) W.sp[lane] = ssp;
                W.pr[lane] = ys.pr;
                W.pth[lane] = ys.pth;
                W.pt[lane] = pts;
                W.pph[lane] = pphs;
                W.k[0][lane] = f.r;
                W.k[1][lane] = f.th;
                W.k[2][lane] = f.ph;
                W.k[3][lane] = f.pr;
                W.k[4][lane] = f.pth;
            }
            __syncwarp();
        }
        // ---- lanes without a ray take the prepared starts in order ----
        if (need && ring_head < ring_n) {
            const int avail = ring_n - ring_head;
            const int rank = __popc(need & lt_mask);
            if (!live && rank < avail) {
                const int slot = ring_head + rank;
                q = W.q[slot];
                if (kBatch) sp = W.sp[slot];
                y = Vec5<double>{S.cam_pos[1], S.cam_pos[2], S.cam_pos[3], W.pr[slot], W.pth[slot]};
                pt = W.pt[slot];
                pph = W.pph[slot];
                k1 = Vec5<double>{W.k[0][slot], W.k[1][slot], W.k[2][slot], W.k[3][slot], W.k[4][slot]};
                dl = S.dl0;
                retry = 0;
                step = 0;
                ncross = 0;
                c0 = c1 = c2 = 0.0;
                live = true;
                ++n_rays;
            }
            ring_head += min(__popc(need), avail);
            __syncwarp();
        }
        // No lane holds a ray: the queue is drained (a lane without a ray
        // would have taken a prepared start, and a refill found none).
        if (!__any_sync(kMask, live)) break;
        int term = -1;
        if (live && retry == 0) term = start_test(S, step, y.r);
        if (live && term < 0) {
            Vec5<double> y5, k7;
            const double err = dp45_attempt_k1<double>(S.M, S.a, pt, pph, y, dl, k1, y5, k7);
            ++n_att;
            const StepDecision d = pi_control(err, S.tol, dl, retry, y5.r);
            if (d.accept) {
                ++n_acc;
                if (S.disk_on) {
                    const double d_prev = y.th - kHalfPi;
                    const double d_new = y5.th - kHalfPi;
                    if (d_prev * d_new < 0.0 && fabs(d_prev - d_new) > 1e-12) {
                        const double frac = -d_prev / (d_new - d_prev);
                        const double rc = y.r + frac * (y5.r - y.r);
                        if (rc >= S.r_in && rc <= S.r_out) {
                            double e0, e1, e2;
                            disk_emission(S, rc, pt, pph, e0, e1, e2);
                            c0 += e0;
                            c1 += e1;
                            c2 += e2;
                            ++ncross;
                        }
                    }
                }
                y = y5;
                k1 = k7;
                dl = d.next;
                retry = 0;
                ++step;
                term = start_test(S, step, y.r);
                // Re-trace on a black sky: once the escape is certain
                // (outgoing beyond the disk, r_near and every photon orbit,
                // far from the step budget) no crossing can follow and no star
                // is looked up, so the colour, the crossings and the fate are
                // those the FP64 trace to r_escape would give. (The FP64 form
                // traces to r_escape, as the reference does.)
                if (kList && term < 0 && !S.stars_on) {
                    const double m = kBatch ? S.mixed_margin : mb.margin;
                    const double r_near = kBatch ? S.r_near_mixed : mb.r_near;
                    const double r_min = fmax(fmax(mixed::kEscapeRMin * S.M, r_near),
                                              S.disk_on ? S.r_out + 2.0 * m : 0.0);
                    if (mixed::certain_escape(y, r_min, step, S.max_steps)) term = kTermEscaped;
                }
            } else {
                dl = d.next;
                ++retry;
            }
        }
        // ---- finished samples: park escapes under a star sky, write the rest ----
        const bool fin = live && term >= 0;
        const bool star = fin && term == kTermEscaped && S.stars_on;
        const unsigned nc = (ncross > 0x3fffffff) ? 0x3fffffffu : static_cast<unsigned>(ncross);
        const unsigned fate = static_cast<unsigned>(term) | (nc << 2);
        const unsigned smask = __ballot_sync(kMask, star);
        if (smask) {
            const int ns = __popc(smask);
            if (pend_n + ns > 32) {
                flush_star_lookups<kBatch>(W, pend_n, S0, mb);
                pend_n = 0;
            }
            if (star) {
                const int slot = pend_n + __popc(smask & lt_mask);
                W.th[slot] = y.th;
                W.ph[slot] = y.ph;
                W.c[0][slot] = c0;
                W.c[1][slot] = c1;
                W.c[2][slot] = c2;
                W.pq[slot] = q;
                W.pfate[slot] = fate;
                if (kBatch) W.psp[slot] = sp;
            }
            pend_n += ns;
            __syncwarp();
        }
        if (fin) {
            live = false;
            if (!star) {
                mb.sample_rgb[3 * static_cast<size_t>(q) + 0] = c0;
                mb.sample_rgb[3 * static_cast<size_t>(q) + 1] = c1;
                mb.sample_rgb[3 * static_cast<size_t>(q) + 2] = c2;
                mb.sample_fate[q] = fate;
            }
        }
    }
#undef S
    if (pend_n) flush_star_lookups<kBatch>(W, pend_n, S0, mb);
    warp_add(stats, n_att, n_acc, kList ? 0ull : n_rays, n_att);
}

// Per pixel: sum the spp sample colours in order, scale, write the outputs.
template <bool kBatch>
__global__ void mixed_resolve_kernel(const __grid_constant__ DevScene S0, const DevTile tile,
                                     const __grid_constant__ DevBatch B, DevMixedBuffers mb,
                                     float4* __restrict__ out_rgba, double* __restrict__ out_rgb64,
                                     uint32_t* __restrict__ out_fate, DevStats* stats) {
    const size_t npix = kBatch ? B.n_pixels : static_cast<size_t>(tile.w) * tile.h;
    unsigned long long hz = 0, es = 0, mx = 0, cr = 0;
    for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < npix;
         p += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const DevScene* sp = &S0;
        size_t q0, o;
        if (kBatch) {
            const DevBatchItem& it = batch_item<false>(B, p);
            sp = B.scenes + it.scene;
            const size_t local = p - it.out_offset;
            q0 = it.sample0 + local * static_cast<size_t>(sp->grid * sp->grid);
            const int qx = static_cast<int>(local % it.w), qy = static_cast<int>(local / it.w);
            o = it.out_offset + static_cast<size_t>(qy) * it.out_pitch + qx;
        } else {
            q0 = p * static_cast<size_t>(S0.grid * S0.grid);
            const int qx = static_cast<int>(p % tile.w), qy = static_cast<int>(p / tile.w);
            o = static_cast<size_t>(qy) * tile.out_pitch + qx;
        }
        const DevScene& S = kBatch ? *sp : S0;
        const int g2 = S.grid * S.grid;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (int s = 0; s < g2; ++s) {
            const size_t q = q0 + s;
            a0 = a0 + mb.sample_rgb[3 * q + 0];
            a1 = a1 + mb.sample_rgb[3 * q + 1];
            a2 = a2 + mb.sample_rgb[3 * q + 2];
            const unsigned f = mb.sample_fate[q];
            const unsigned t = f & 3u;
            hz += (t == kTermHorizon);
            es += (t == kTermEscaped);
            mx += (t == kTermMaxSteps);
            cr += f >> 2;
            if (out_fate) out_fate[q] = f;
        }
        const double r0 = a0 * S.inv_spp, r1 = a1 * S.inv_spp, r2 = a2 * S.inv_spp;
        if (out_rgba)
            out_rgba[o] = make_float4(static_cast<float>(r0), static_cast<float>(r1), static_cast<float>(r2), 1.0f);
        if (out_rgb64) {
            out_rgb64[3 * o + 0] = r0;
            out_rgb64[3 * o + 1] = r1;
            out_rgb64[3 * o + 2] = r2;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        hz += __shfl_xor_sync(kMask, hz, o);
        es += __shfl_xor_sync(kMask, es, o);
        mx += __shfl_xor_sync(kMask, mx, o);
        cr += __shfl_xor_sync(kMask, cr, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&stats->horizon, hz);
        atomicAdd(&stats->escaped, es);
        atomicAdd(&stats->max_steps, mx);
        atomicAdd(&stats->crossings, cr);
    }
}

// Header, per-sample colour and fate, the re-trace and speculation lists, then
// (256-byte aligned) room for ordering the re-trace list.
static size_t mixed_order_offset(size_t n_samples) {
    return ((n_samples * (3 * sizeof(double) + 3 * sizeof(unsigned)) + 1024 + 255) / 256) * 256;
}

// the longest-first re-trace list (black sky) and its ordering scratch
static size_t mixed_cost_offset(size_t n_samples) {
    return mixed_order_offset(n_samples) + ((order_list_scratch_bytes(n_samples) + 255) / 256) * 256;
}

size_t mixed_scratch_bytes_for(size_t n_samples) {
    return mixed_cost_offset(n_samples) + ((n_samples * sizeof(unsigned) + 255) / 256) * 256 +
           cost_order_scratch_bytes(n_samples);
}

void* mixed_order_scratch(void* scratch, size_t n_samples) {
    return static_cast<unsigned char*>(scratch) + mixed_order_offset(n_samples);
}

size_t mixed_scratch_bytes(const DevTile& tile, int g2) {
    return mixed_scratch_bytes_for(static_cast<size_t>(tile.w) * tile.h * g2);
}

namespace {
struct MixLaunchShape {
    int sms = 0;
    int per_spec = 1, per_retrace = 1;      // resident blocks per SM, one camera
    int per_spec_b = 1, per_retrace_b = 1;  // the batch instantiations
    int per_fp64 = 1, per_fp64_b = 1;       // the FP64 form's trace of every sample (one camera, batch)
};
const MixLaunchShape& mix_shape() {
    return per_device_shape<MixLaunchShape>([](int dev) {
        MixLaunchShape sh;
        cudaDeviceGetAttribute(&sh.sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sh.per_spec, mixed_speculate_kernel<false>, kMixThreads, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sh.per_retrace, fp64_trace_kernel<true, false>, kMixThreads,
                                                      0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sh.per_fp64, fp64_trace_kernel<false, false>, kMixThreads, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sh.per_fp64_b, fp64_trace_kernel<false, true>, kMixThreads,
                                                      0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sh.per_spec_b, mixed_speculate_kernel<true>, kMixThreads, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sh.per_retrace_b, fp64_trace_kernel<true, true>, kMixThreads,
                                                      0);
        if (sh.per_spec < 1) sh.per_spec = 1;
        if (sh.per_retrace < 1) sh.per_retrace = 1;
        if (sh.per_spec_b < 1) sh.per_spec_b = 1;
        if (sh.per_retrace_b < 1) sh.per_retrace_b = 1;
        if (sh.per_fp64 < 1) sh.per_fp64 = 1;
        if (sh.per_fp64_b < 1) sh.per_fp64_b = 1;
        return sh;
    });
}
}  // namespace

DevMixedBuffers mixed_buffers(void* scratch, size_t n, unsigned* queue) {
    auto* base = static_cast<unsigned char*>(scratch);
    DevMixedBuffers mb;
    mb.queue = queue;
    mb.queue2 = reinterpret_cast<unsigned*>(base + 256);
    mb.retrace_count = reinterpret_cast<unsigned*>(base + 512);
    mb.sample_rgb = reinterpret_cast<double*>(base + 1024);
    mb.sample_fate = reinterpret_cast<uint32_t*>(base + 1024 + n * 3 * sizeof(double));
    mb.retrace_list = mb.sample_fate + n;
    return mb;
}

DevMixedBuffers mixed_buffers_with_list(void* scratch, size_t n, unsigned* queue) {
    DevMixedBuffers mb = mixed_buffers(scratch, n, queue);
    mb.spec_count = reinterpret_cast<unsigned*>(static_cast<unsigned char*>(scratch) + 768);
    mb.spec_list = mb.retrace_list + n;
    return mb;
}

cudaError_t launch_mixed_speculate(const DevScene& S, const DevTile& tile, const DevMixedBuffers& mb,
                                   DevStats* stats, cudaStream_t stream) {
    const MixLaunchShape& sh = mix_shape();
    const size_t n = static_cast<size_t>(tile.w) * tile.h * S.grid * S.grid;
    // the work counters run up to 32 items per warp past the end, and a cancel
    // pushes them to 0x7f7f7f7f
    if (n > kMaxSamples) return cudaErrorInvalidValue;
    const int need = static_cast<int>((n + kMixThreads - 1) / kMixThreads);
    mixed_speculate_kernel<false>
        <<<need < sh.sms * sh.per_spec ? need : sh.sms * sh.per_spec, kMixThreads, 0, stream>>>(S, tile, DevBatch{},
                                                                                                  mb, stats);
    return cudaGetLastError();
}

cudaError_t launch_mixed_stars(const DevScene& S, const DevTile& tile, const DevMixedBuffers& mb,
                               cudaStream_t stream) {
    if (!S.stars_on) return cudaSuccess;
    const MixLaunchShape& sh = mix_shape();
    const size_t n = static_cast<size_t>(tile.w) * tile.h * S.grid * S.grid;
    int sb = static_cast<int>((n + 255) / 256);
    if (sb > sh.sms * 8) sb = sh.sms * 8;
    mixed_star_kernel<false><<<sb, 256, 0, stream>>>(S, tile, DevBatch{}, mb);
    return cudaGetLastError();
}

cudaError_t launch_mixed_retrace(const DevScene& S, const DevTile& tile, const DevMixedBuffers& mb, DevStats* stats,
                                 void* scratch, cudaStream_t stream) {
    const MixLaunchShape& sh = mix_shape();
    if (static_cast<size_t>(tile.w) * tile.h * S.grid * S.grid > kMaxSamples) return cudaErrorInvalidValue;
    DevMixedBuffers m = mb;
    if (!S.stars_on) {
        // Black sky: the list holds lit samples near the hole, whose lengths
        // follow their closed-form distance to the critical curve; taken
        // nearest first, the long ones start first (the C5 frame, 2048^2 at
        // a = 0.998: re-trace 5.47 -> 5.02 ms on B200). Under a star sky the
        // list is mostly escapes with a star in reach, and the finding order,
        // which groups rays of similar length into warps, is faster (1024^2
        // 4-spp frame: 7.58 against 8.43 ms ordered).
        const size_t n = static_cast<size_t>(tile.w) * tile.h * S.grid * S.grid;
        auto* base = static_cast<unsigned char*>(scratch) + mixed_cost_offset(n);
        auto* ordered = reinterpret_cast<unsigned*>(base);
        void* cs = base + ((n * sizeof(unsigned) + 255) / 256) * 256;
        const cudaError_t e =
            order_by_cost(S, tile, mb.retrace_list, static_cast<unsigned>(n), mb.retrace_count, true, ordered, cs, stream);
        if (e != cudaSuccess) return e;
        m.retrace_list = ordered;
    }
    fp64_trace_kernel<true, false>
        <<<sh.sms * sh.per_retrace, kMixThreads, 0, stream>>>(S, tile, DevBatch{}, m, m.queue2, 0u, stats);
    return cudaGetLastError();
}

cudaError_t launch_mixed_resolve(const DevScene& S, const DevTile& tile, const DevMixedBuffers& mb,
                                 const ThinOutputs& out, DevStats* stats, cudaStream_t stream) {
    const MixLaunchShape& sh = mix_shape();
    const size_t npix = static_cast<size_t>(tile.w) * tile.h;
    int rb = static_cast<int>((npix + 255) / 256);
    if (rb > sh.sms * 8) rb = sh.sms * 8;
    if (rb < 1) rb = 1;
    mixed_resolve_kernel<false>
        <<<rb, 256, 0, stream>>>(S, tile, DevBatch{}, mb, out.rgba, out.rgb64, out.fate, stats);
    return cudaGetLastError();
}

cudaError_t launch_thin_mixed(const DevScene& S, const DevTile& tile, const ThinOutputs& out,
                              const LaunchResources& res, void* scratch, size_t scratch_bytes, double margin,
                              double r_near, cudaEvent_t* phase_events, cudaStream_t stream) {
    auto mark = [&](int k) {
        if (phase_events) cudaEventRecord(phase_events[k], stream);
    };
    DevStats* stats = res.stats;
    const int g2 = S.grid * S.grid;
    const size_t n = static_cast<size_t>(tile.w) * tile.h * g2;
    if (n == 0) return cudaSuccess;
    if (scratch_bytes < mixed_scratch_bytes(tile, g2)) return cudaErrorInvalidValue;
    // the phase-1 counter doubles as the progress counter
    DevMixedBuffers mb = mixed_buffers(scratch, n, res.queue);
    mb.margin = margin;
    mb.r_near = r_near;
    cudaError_t e = cudaMemsetAsync(scratch, 0, 1024, stream);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(res.queue, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    mark(0);
    e = launch_mixed_speculate(S, tile, mb, stats, stream);
    if (e != cudaSuccess) return e;
    mark(1);
    e = launch_mixed_stars(S, tile, mb, stream);
    if (e != cudaSuccess) return e;
    mark(2);
    e = launch_mixed_retrace(S, tile, mb, stats, scratch, stream);
    if (e != cudaSuccess) return e;
    mark(3);
    e = launch_mixed_resolve(S, tile, mb, out, stats, stream);
    mark(4);
    return e;
}

cudaError_t launch_thin_fp64(const DevScene& S, const DevTile& tile, const ThinOutputs& out,
                             const LaunchResources& res, void* scratch, size_t scratch_bytes,
                             cudaEvent_t* phase_events, cudaStream_t stream) {
    auto mark = [&](int k) {
        if (phase_events) cudaEventRecord(phase_events[k], stream);
    };
    const int g2 = S.grid * S.grid;
    const size_t n = static_cast<size_t>(tile.w) * tile.h * g2;
    if (n == 0) return cudaSuccess;
    if (scratch_bytes < mixed_scratch_bytes(tile, g2) || n > kMaxSamples) return cudaErrorInvalidValue;
    // the work counter doubles as the progress counter (samples taken)
    const DevMixedBuffers mb = mixed_buffers(scratch, n, res.queue);
    cudaError_t e = cudaMemsetAsync(res.queue, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    const MixLaunchShape& sh = mix_shape();
    const int need = static_cast<int>((n + kMixThreads - 1) / kMixThreads);
    int blocks = sh.sms * sh.per_fp64;
    if (need < blocks) blocks = need;
    mark(0);
    fp64_trace_kernel<false, false><<<blocks, kMixThreads, 0, stream>>>(S, tile, DevBatch{}, mb, res.queue,
                                                                         static_cast<unsigned>(n), res.stats);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    mark(1);
    e = launch_mixed_resolve(S, tile, mb, out, res.stats, stream);
    mark(2);
    return e;
}

int mixed_batch_max_blocks_per_sm() { return mix_shape().per_spec_b; }

int fp64_batch_max_blocks_per_sm() { return mix_shape().per_fp64_b; }

cudaError_t launch_thin_fp64_batch(const DevBatch& B, float4* out_rgba, unsigned* queue, DevStats* stats,
                                   void* scratch, size_t scratch_bytes, int blocks_per_sm, cudaStream_t stream) {
    const size_t n = B.n_samples;
    if (n == 0) return cudaSuccess;
    if (B.n_items < 1 || scratch_bytes < mixed_scratch_bytes_for(n) || n > kMaxSamples) return cudaErrorInvalidValue;
    const DevMixedBuffers mb = mixed_buffers(scratch, n, queue);
    cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    const MixLaunchShape& sh = mix_shape();
    const int per = (blocks_per_sm > 0 && blocks_per_sm < sh.per_fp64_b) ? blocks_per_sm : sh.per_fp64_b;
    const int need = static_cast<int>((n + kMixThreads - 1) / kMixThreads);
    int blocks = sh.sms * per;
    if (need < blocks) blocks = need;
    const DevScene none{};
    const DevTile no_tile{};
    fp64_trace_kernel<false, true>
        <<<blocks, kMixThreads, 0, stream>>>(none, no_tile, B, mb, queue, static_cast<unsigned>(n), stats);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    int rb = static_cast<int>((B.n_pixels + 255) / 256);
    if (rb > sh.sms * 8) rb = sh.sms * 8;
    if (rb < 1) rb = 1;
    mixed_resolve_kernel<true><<<rb, 256, 0, stream>>>(none, no_tile, B, mb, out_rgba, nullptr, nullptr, stats);
    return cudaGetLastError();
}

cudaError_t launch_thin_mixed_batch(const DevBatch& B, bool any_stars, float4* out_rgba, unsigned* queue,
                                    DevStats* stats, void* scratch, size_t scratch_bytes, int blocks_per_sm,
                                    cudaStream_t stream) {
    const size_t n = B.n_samples;
    if (n == 0) return cudaSuccess;
    if (B.n_items < 1 || scratch_bytes < mixed_scratch_bytes_for(n)) return cudaErrorInvalidValue;
    const DevMixedBuffers mb = mixed_buffers(scratch, n, queue);
    cudaError_t e = cudaMemsetAsync(scratch, 0, 1024, stream);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(queue, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    const MixLaunchShape& sh = mix_shape();
    auto per = [&](int maxb) { return (blocks_per_sm > 0 && blocks_per_sm < maxb) ? blocks_per_sm : maxb; };
    const DevScene none{};
    const DevTile no_tile{};
    const int need = static_cast<int>((n + kMixThreads - 1) / kMixThreads);
    int sb = sh.sms * per(sh.per_spec_b);
    if (need < sb) sb = need;
    mixed_speculate_kernel<true><<<sb, kMixThreads, 0, stream>>>(none, no_tile, B, mb, stats);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (any_stars) {
        int b = static_cast<int>((n + 255) / 256);
        if (b > sh.sms * 8) b = sh.sms * 8;
        mixed_star_kernel<true><<<b, 256, 0, stream>>>(none, no_tile, B, mb);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    fp64_trace_kernel<true, true><<<sh.sms * per(sh.per_retrace_b), kMixThreads, 0, stream>>>(none, no_tile, B, mb,
                                                                                               mb.queue2, 0u, stats);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    int rb = static_cast<int>((B.n_pixels + 255) / 256);
    if (rb > sh.sms * 8) rb = sh.sms * 8;
    if (rb < 1) rb = 1;
    mixed_resolve_kernel<true><<<rb, 256, 0, stream>>>(none, no_tile, B, mb, out_rgba, nullptr, nullptr, stats);
    return cudaGetLastError();
}

}  // namespace grrt_b200
