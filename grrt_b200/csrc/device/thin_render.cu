// Thin-disk RGB render: camera -> Kerr null geodesic (adaptive DP45) ->
// emission summed over every equatorial crossing inside [r_in, r_out] ->
// first-match star lookup on escape. The per-pixel path of
// GeodesicTracer::trace (src/geodesic_tracer.cpp:23-181) inside the loop of
// Renderer::render (src/renderer.cpp:30-82), in the FP64 form, one lane per
// pixel. This kernel serves the Hamiltonian diagnostic (GRRT_DIAG_HAMILTONIAN)
// and the batched form's pixel schedules; the FP64 form's renders otherwise
// trace by samples with the per-sample work staged per warp
// (fp64_trace_kernel in mixed_render.cu, the same arithmetic).
//
// Execution model: a persistent grid (resident blocks only). Each lane owns one
// pixel at a time and walks its spp samples; each loop iteration performs
// exactly one DP45 attempt for every lane with a live ray, so the warp stays
// converged in the expensive part. A lane whose pixel is done takes the next
// pixel from a global counter with one warp-aggregated atomic, which keeps
// warps full while ray lengths range from tens to thousands of steps.
// One shared body of the FP64 right-hand side instead of seven inlined copies
// per attempt: less code to fetch (Kerr a=0.998, 1024x1024, 4 spp: 46.4 ->
// 43.4 ms for the FP64 form on B200). The FP64 form and the mixed form's
// re-trace must use the same setting, so that their arithmetic is identical.
#define GRRT_RHS_CALL_F64 1
#include <cuda_runtime.h>

#include <cstdint>

#include "launch_cache.h"
#include "integrate.cuh"
#include "render_launch.h"
#include "shading.cuh"

namespace grrt_b200 {

namespace {

constexpr int kThreads = 128;
constexpr unsigned kFull = 0xffffffffu;

// Minimum resident blocks per SM the compiler must allow (register budget
// 65536 / (128 * n)). 4 (16 warps per SM, 128 registers, ~120 B of
// spills) measured faster than 3 (12 warps, 168 registers, no spills) and 2.
#ifndef GRRT_THIN_MIN_BLOCKS
#define GRRT_THIN_MIN_BLOCKS 4
#endif

// Per-lane state that is touched only when a sample starts, crosses the disk
// or ends. It lives in shared memory, so the registers hold the ray itself
// (state, kept first stage, step size) through the DP45 attempt.
struct LaneCold {
    double acc[3];        // the pixel's sum over its finished samples
    double col[3];        // the current sample's colour (disk crossings, then the star)
    size_t out;           // output index of the pixel
    int i, j;             // image coordinates of the pixel
    int smp;              // sample index within the pixel
    int ncross;           // the current sample's emitting disk crossings
    unsigned crossings, horizon, escaped, maxsteps;  // counters of the lane's samples
    double h_max;         // max |H| / p_t^2 at the final state of the lane's samples
};

// Sums the lanes' counters per warp and adds them to the launch's totals
// (every DP45 attempt of this kernel is an FP64 attempt).
__device__ __forceinline__ void flush_counters(DevStats* st, unsigned attempts, unsigned accepted,
                                               const LaneCold& c, bool cancelled) {
    unsigned long long v[6] = {attempts, accepted, c.crossings, c.horizon, c.escaped, c.maxsteps};
#pragma unroll
    for (int k = 0; k < 6; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(kFull, v[k], o);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&st->attempts, v[0]);
        atomicAdd(&st->accepted, v[1]);
        atomicAdd(&st->crossings, v[2]);
        atomicAdd(&st->rays, v[3] + v[4] + v[5]);
        atomicAdd(&st->horizon, v[3]);
        atomicAdd(&st->escaped, v[4]);
        atomicAdd(&st->max_steps, v[5]);
        atomicAdd(&st->fp64_attempts, v[0]);
        if (cancelled && threadIdx.x == 0) atomicAdd(&st->cancelled, 1ull);
    }
    double h = c.h_max;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) h = fmax(h, __shfl_xor_sync(kFull, h, o));
    if ((threadIdx.x & 31) == 0 && h > 0.0)
        atomicMax(&st->h_max_bits, static_cast<unsigned long long>(__double_as_longlong(h)));
}

// Start-of-step termination test in the reference order: step budget first
// (the loop condition), then horizon, then escape.
__device__ __forceinline__ int start_check(const DevScene& S, int step, double r) {
    if (step >= S.max_steps) return kTermMaxSteps;
    if (r < S.r_stop) return kTermHorizon;
    if (r > S.r_escape) return kTermEscaped;
    return -1;
}

}  // namespace

// The per-lane pixel loop shared by the single-camera and the batched kernels.
// kBatch = false: every lane renders pixels of one camera (scene S0, the
// kernel's parameter) in the rectangle `tile`, work index = pixel index.
// kBatch = true: work index -> (chunk, offset) through the batch's chunk table,
// so one launch covers many cameras (scenes[item.scene]) in the order the
// schedule lists the chunks.
// kDiag: also measure the Hamiltonian constraint at each sample's final state
// (the diagnostic instantiation; the render instantiation carries no cost).
template <bool kBatch, int kBlock = kThreads, bool kDiag = false>
__device__ __forceinline__ void thin_loop(const DevScene& S0, const DevBatch& B, const DevTile& tile,
                                          float4* __restrict__ out_rgba, double* __restrict__ out_rgb64,
                                          uint32_t* __restrict__ out_fate, unsigned total,
                                          unsigned int* __restrict__ queue, DevStats* __restrict__ stats,
                                          const volatile int* __restrict__ cancel) {
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    // the scene of the lane's current pixel (batch: per lane, in global memory)
    int scene = 0;
#define S (kBatch ? B.scenes[scene] : S0)
    __shared__ LaneCold cold_all[kBlock];
    LaneCold& cold = cold_all[threadIdx.x];
    cold.crossings = cold.horizon = cold.escaped = cold.maxsteps = 0;
    cold.h_max = 0.0;

    unsigned n_attempts = 0, n_accepted = 0;
    // pixel slot
    int pix = -1;        // work index of the lane's pixel; -1 = needs a pixel; -2 = queue exhausted
    // ray slot
    bool live = false;
    Vec5<double> y;      // state at the start of the current outer step
    Vec5<double> k1;     // f(y), kept from the previous attempt when k1_ok
    bool k1_ok = false;
    double pt = 0.0, pph = 0.0;
    double dl = 0.0;
    int retry = 0, step = 0;

    while (true) {
        // ---- refill: lanes without a pixel take one (warp-aggregated atomic) ----
        const bool want = (pix == -1);
        const unsigned want_mask = __ballot_sync(kFull, want);
        if (want_mask) {
            unsigned base = 0;
            const int leader = __ffs(want_mask) - 1;
            if (lane == leader) base = atomicAdd(queue, static_cast<unsigned>(__popc(want_mask)));
            base = __shfl_sync(kFull, base, leader);
            if (want) {
                const unsigned q = base + __popc(want_mask & lt_mask);
                if (q < total) {
                    if (kBatch) {
                        const DevBatchChunk ch = B.chunks[q / B.chunk_size];
                        const int within = static_cast<int>(q % B.chunk_size);
                        if (within < ch.count) {
                            const DevBatchItem it = B.items[ch.item];
                            const int local = ch.start + within;
                            const int qx = local % it.w, qy = local / it.w;
                            scene = it.scene;
                            cold.i = it.x0 + qx;
                            cold.j = it.y0 + qy;
                            cold.out = it.out_offset + static_cast<size_t>(qy) * it.out_pitch + qx;
                            pix = static_cast<int>(q);
                            cold.smp = 0;
                            cold.acc[0] = cold.acc[1] = cold.acc[2] = 0.0;
                        }  // else: padding slot of a short chunk, fetch again
                    } else {
                        const int qx = static_cast<int>(q) % tile.w, qy = static_cast<int>(q) / tile.w;
                        cold.i = tile.x0 + qx;
                        cold.j = tile.y0 + qy * tile.row_step;
                        cold.out = static_cast<size_t>(qy) * tile.out_pitch + qx;
                        pix = static_cast<int>(q);
                        cold.smp = 0;
                        cold.acc[0] = cold.acc[1] = cold.acc[2] = 0.0;
                    }
                } else {
                    pix = -2;
                }
            }
        }
        // ---- start a ray for lanes that have a pixel but no live ray ----
        if (!live && pix >= 0) {
            const int i = cold.i, j = cold.j, smp = cold.smp;
            const int sy = smp / S.grid, sx = smp % S.grid;
            const double x = i + (sx + pixel_hash(i, j, smp, 0)) * S.cell;
            const double yy = j + (sy + pixel_hash(i, j, smp, 1)) * S.cell;
            double p[4];
            camera_momentum(S, x, yy, p);
            y = Vec5<double>{S.cam_pos[1], S.cam_pos[2], S.cam_pos[3], p[1], p[2]};
            pt = p[0];
            pph = p[3];
            dl = S.dl0;
            retry = 0;
            step = 0;
            cold.ncross = 0;
            cold.col[0] = cold.col[1] = cold.col[2] = 0.0;
            k1_ok = false;
            live = true;
        }
        int term = -1;
        if (live && retry == 0) term = start_check(S, step, y.r);

        // ---- one DP45 attempt for every lane with a live, unterminated ray ----
        if (live && term < 0) {
            if (!k1_ok) {
                k1 = kerr_rhs<double>(S.M, S.a, pt, pph, y);
                k1_ok = true;
            }
            Vec5<double> y5, k7;
            const double err = dp45_attempt_k1<double>(S.M, S.a, pt, pph, y, dl, k1, y5, k7);
            ++n_attempts;
            const StepDecision d = pi_control(err, S.tol, dl, retry, y5.r);
            if (d.accept) {
                ++n_accepted;
                // equatorial crossing (src/geodesic_tracer.cpp:156-176): every
                // crossing inside the disk adds emission; r is interpolated
                // linearly in theta; p_t and p_phi are constants of motion.
                if (S.disk_on) {
                    const double d_prev = y.th - kHalfPi;
                    const double d_new = y5.th - kHalfPi;
                    if (d_prev * d_new < 0.0 && fabs(d_prev - d_new) > 1e-12) {
                        const double frac = -d_prev / (d_new - d_prev);
                        const double rc = y.r + frac * (y5.r - y.r);
                        if (rc >= S.r_in && rc <= S.r_out) {
                            double e0, e1, e2;
                            disk_emission(S, rc, pt, pph, e0, e1, e2);
                            cold.col[0] += e0;
                            cold.col[1] += e1;
                            cold.col[2] += e2;
                            ++cold.ncross;
                            ++cold.crossings;
                        }
                    }
                }
                y = y5;
                k1 = k7;
                dl = d.next;
                retry = 0;
                ++step;
                term = start_check(S, step, y.r);
            } else {
                dl = d.next;
                ++retry;
            }
        }

        // ---- finish a terminated sample ----
        if (live && term >= 0) {
            live = false;
            // the constraint at the final state of rays that do not end at the
            // horizon (there Delta -> 0 and P^2 / Delta cancels catastrophically)
            if (kDiag && term != kTermHorizon)
                cold.h_max = fmax(cold.h_max, fabs(kerr_hamiltonian<double>(S.M, S.a, pt, pph, y)) / (pt * pt));
            double c0 = cold.col[0], c1 = cold.col[1], c2 = cold.col[2];
            if (term == kTermEscaped) {
                ++cold.escaped;
                if (S.stars_on) {
                    const double b = star_brightness(S.stars, y.th, y.ph);
                    c0 += b;
                    c1 += b;
                    c2 += b;
                }
            } else if (term == kTermHorizon) {
                ++cold.horizon;
            } else {
                ++cold.maxsteps;
            }
            const double acc0 = cold.acc[0] + c0, acc1 = cold.acc[1] + c1, acc2 = cold.acc[2] + c2;
            const int grid2 = S.grid * S.grid;
            const int smp = cold.smp;
            if (out_fate) {
                const int ncross = cold.ncross;
                const unsigned nc = (ncross > 0x3fffffff) ? 0x3fffffffu : static_cast<unsigned>(ncross);
                out_fate[static_cast<size_t>(pix) * grid2 + smp] = static_cast<unsigned>(term) | (nc << 2);
            }
            if (smp + 1 == grid2) {
                const size_t o = cold.out;
                const double r0 = acc0 * S.inv_spp, r1 = acc1 * S.inv_spp, r2 = acc2 * S.inv_spp;
                if (out_rgba) out_rgba[o] = make_float4(static_cast<float>(r0), static_cast<float>(r1),
                                                         static_cast<float>(r2), 1.0f);
                if (out_rgb64) {
                    out_rgb64[3 * o + 0] = r0;
                    out_rgb64[3 * o + 1] = r1;
                    out_rgb64[3 * o + 2] = r2;
                }
                pix = -1;
            } else {
                cold.smp = smp + 1;
                cold.acc[0] = acc0;
                cold.acc[1] = acc1;
                cold.acc[2] = acc2;
            }
        }

        // (no polling for a cancel: grrt_cancel pushes the work counter past
        // every pixel, and the lanes end with their current samples)
        // ---- exit when the queue is drained and no lane holds a ray ----
        if (!__any_sync(kFull, live || pix >= -1)) break;
    }
#undef S
    flush_counters(stats, n_attempts, n_accepted, cold, false);
}

template <bool kDiag>
__global__ void __launch_bounds__(kThreads, GRRT_THIN_MIN_BLOCKS)
thin_render_kernel(const __grid_constant__ DevScene S, const DevTile tile, float4* __restrict__ out_rgba,
                   double* __restrict__ out_rgb64, uint32_t* __restrict__ out_fate,
                   unsigned int* __restrict__ queue, DevStats* __restrict__ stats,
                   const volatile int* __restrict__ cancel) {
    const unsigned total = static_cast<unsigned>(tile.w) * static_cast<unsigned>(tile.h);
    thin_loop<false, kThreads, kDiag>(S, DevBatch{}, tile, out_rgba, out_rgb64, out_fate, total, queue, stats,
                                      cancel);
}

// One launch over many cameras: the batched form. Work index space =
// n_chunks * chunk_size (short chunks padded). Instantiated for 64-, 128- and
// 256-thread blocks at the same register budget (128 per thread); the
// batch's autotuner picks one.
template <int kBlock>
__global__ void __launch_bounds__(kBlock, GRRT_THIN_MIN_BLOCKS * kThreads / kBlock)
thin_batch_kernel(const __grid_constant__ DevBatch B, float4* __restrict__ out_rgba, unsigned int* __restrict__ queue,
                  DevStats* __restrict__ stats) {
    const unsigned total = static_cast<unsigned>(B.n_chunks) * static_cast<unsigned>(B.chunk_size);
    thin_loop<true, kBlock>(B.scenes[0], B, DevTile{}, out_rgba, nullptr, nullptr, total, queue, stats, nullptr);
}

cudaError_t launch_thin(const DevScene& S, const DevTile& tile, const ThinOutputs& out,
                        const LaunchResources& res, cudaStream_t stream) {
    struct Shape {
        int sms = 0, per = 1;
    };
    const Shape& sh = per_device_shape<Shape>([](int dev) {
        Shape v;
        cudaDeviceGetAttribute(&v.sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v.per, thin_render_kernel<false>, kThreads, 0);
        if (v.per < 1) v.per = 1;
        return v;
    });
    const int num_sms = sh.sms, blocks_per_sm = sh.per;
    const unsigned total = static_cast<unsigned>(tile.w) * static_cast<unsigned>(tile.h);
    if (total == 0) return cudaSuccess;
    int blocks = num_sms * blocks_per_sm;
    const int needed = static_cast<int>((total + kThreads - 1) / kThreads);
    if (needed < blocks) blocks = needed;
    cudaError_t e = cudaMemsetAsync(res.queue, 0, sizeof(unsigned int), stream);
    if (e != cudaSuccess) return e;
    if (res.diag_hamiltonian)
        thin_render_kernel<true><<<blocks, kThreads, 0, stream>>>(S, tile, out.rgba, out.rgb64, out.fate, res.queue,
                                                                  res.stats, res.cancel);
    else
        thin_render_kernel<false><<<blocks, kThreads, 0, stream>>>(S, tile, out.rgba, out.rgb64, out.fate, res.queue,
                                                                   res.stats, res.cancel);
    return cudaGetLastError();
}

namespace {
template <int kBlock>
int thin_batch_blocks_per_sm_for() {
    return per_device_shape<int>([](int) {
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, thin_batch_kernel<kBlock>, kBlock, 0);
        return n < 1 ? 1 : n;
    });
}
}  // namespace

int thin_batch_max_blocks_per_sm(int block) {
    return block == 64 ? thin_batch_blocks_per_sm_for<64>()
           : block == 256 ? thin_batch_blocks_per_sm_for<256>()
                          : thin_batch_blocks_per_sm_for<128>();
}

cudaError_t launch_thin_batch(const DevBatch& B, float4* out_rgba, unsigned int* queue, DevStats* stats, int blocks,
                              int block, cudaStream_t stream) {
    if (B.n_chunks <= 0) return cudaSuccess;
    if (block != 64 && block != 128 && block != 256) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned int), stream);
    if (e != cudaSuccess) return e;
    if (block == 64)
        thin_batch_kernel<64><<<blocks, 64, 0, stream>>>(B, out_rgba, queue, stats);
    else if (block == 256)
        thin_batch_kernel<256><<<blocks, 256, 0, stream>>>(B, out_rgba, queue, stats);
    else
        thin_batch_kernel<128><<<blocks, 128, 0, stream>>>(B, out_rgba, queue, stats);
    return cudaGetLastError();
}

}  // namespace grrt_b200
