// Single-ray debug trace on the device: the FP64 trace of one camera sample,
// written out as a list of records in the order GeodesicTracer::trace_debug
// prints its lines (src/geodesic_tracer.cpp:339-493): one STEP record per
// accepted outer step (position, next step, and with a volumetric disk the
// scale height, z_max and the hand-over event), a THIN_HIT record per
// emitting thin-disk crossing, a MARCH_ENTRY / MARCH_EXIT pair per ray-march,
// and an END record (termination, colour, attempts).
//
// The steps are the render kernels' own: dp45_attempt_k1 with the kept k1,
// pi_control, vol_clamp, vol_enters and vol_march_rgb_step, so the record
// list describes the ray those kernels trace for the same sample. Like the
// reference's debug trace, the END colour is the disk's (and the volume's)
// emission only; the sky is not added. One thread does the work: the trace is
// bounded by max_steps outer steps of at most 21 attempts each and 4096 march
// steps per ray-march.
#include <cuda_runtime.h>

#include <cmath>

#include "integrate.cuh"
#include "render_launch.h"
#include "shading.cuh"
#include "vol_steps.cuh"
#include "volume.cuh"

namespace grrt_b200 {

namespace {

struct RecordSink {
    DevDebugRecord* rec;
    int cap;  // slots; the last one is kept for the END record
    int n;    // records produced so far (may exceed cap)

    __device__ void put(int kind, int step, int event, int aux, double v0 = 0.0, double v1 = 0.0,
                        double v2 = 0.0, double v3 = 0.0, double v4 = 0.0, double v5 = 0.0, double v6 = 0.0) {
        const bool end = (kind == kDebugEnd);
        const int slot = end ? (n < cap ? n : cap - 1) : n;
        if (slot < (end ? cap : cap - 1)) {
            DevDebugRecord& r = rec[slot];
            r.kind = kind;
            r.step = step;
            r.event = event;
            r.aux = aux;
            r.v[0] = v0;
            r.v[1] = v1;
            r.v[2] = v2;
            r.v[3] = v3;
            r.v[4] = v4;
            r.v[5] = v5;
            r.v[6] = v6;
        }
        ++n;
    }
};

// The hand-over event trace_debug labels a step with
// (src/geodesic_tracer.cpp:435-451): CROSS, else INSIDE, else NEAR.
__device__ int vol_event(const DevVolume& V, const Vec5<double>& prev, const Vec5<double>& y) {
    const double d_prev = prev.th - kHalfPi, d_new = y.th - kHalfPi;
    const double z_new = y.r * cos(y.th), z_prev = prev.r * cos(prev.th);
    if ((d_prev * d_new < 0.0) && fabs(d_prev - d_new) > 1e-12) return kDebugCross;
    if (v_inside(V, y.r, z_new)) return kDebugInside;
    const bool near = (fabs(z_new) < v_zmax(V, y.r) + 2.0 * v_scale_height(V, y.r) ||
                       fabs(z_prev) < v_zmax(V, prev.r) + 2.0 * v_scale_height(V, prev.r)) &&
                      y.r >= V.r_horizon && y.r <= V.r_outer;
    return near ? kDebugNear : kDebugNone;
}

__global__ void __launch_bounds__(32) debug_trace_kernel(const __grid_constant__ DevScene S, double x, double yy,
                                                         DevDebugRecord* __restrict__ rec, int cap,
                                                         int* __restrict__ count) {
    if (threadIdx.x != 0) return;
    RecordSink out{rec, cap, 0};
    const DevVolume& V = S.vol;
    const bool vol = S.vol_on != 0;
    double p[4];
    camera_momentum(S, x, yy, p);
    Vec5<double> y{S.cam_pos[1], S.cam_pos[2], S.cam_pos[3], p[1], p[2]};
    const double pt = p[0], pph = p[3];
    out.put(kDebugStart, 0, 0, 0, y.r, y.th, y.ph, p[0], p[1], p[2], p[3]);

    double col[3] = {0.0, 0.0, 0.0};
    double J[3] = {0.0, 0.0, 0.0}, Tt[3] = {1.0, 1.0, 1.0};
    VolCounters cnt;
    Vec5<double> k1{};
    bool k1_ok = false;
    double dlambda = S.dl0;
    int nc = 0, step = 0, term = kTermMaxSteps;
    for (;;) {
        if (step >= S.max_steps) { term = kTermMaxSteps; break; }
        if (y.r < S.r_stop) { term = kTermHorizon; break; }
        if (y.r > S.r_escape) { term = kTermEscaped; break; }
        if (!k1_ok) {
            k1 = kerr_rhs<double>(S.M, S.a, pt, pph, y);
            k1_ok = true;
        }
        if (vol && vol_clamp(S, k1, y, dlambda)) ++cnt.clamp;
        const Vec5<double> prev = y;
        double dl = dlambda;
        Vec5<double> y5, k7;
        for (int retry = 0;; ++retry) {
            const double err = dp45_attempt_k1<double>(S.M, S.a, pt, pph, y, dl, k1, y5, k7);
            ++cnt.attempts;
            const StepDecision d = pi_control(err, S.tol, dl, retry, y5.r);
            if (d.accept) {
                dlambda = d.next;
                break;
            }
            dl = d.next;
        }
        ++cnt.accepted;
        y = y5;
        k1 = k7;
        const double z = y.r * cos(y.th);
        if (vol) {
            const bool opaque = (Tt[0] < 1e-6 && Tt[1] < 1e-6 && Tt[2] < 1e-6);
            const int event = opaque ? kDebugNone : vol_event(V, prev, y);
            out.put(kDebugStep, step, event, 0, y.r, y.th, z, dlambda, v_scale_height(V, y.r), v_zmax(V, y.r), y.ph);
            if (!opaque && vol_enters(V, prev, y)) {
                out.put(kDebugMarchEntry, step, 0, 0, prev.r, prev.r * cos(prev.th));
                Vec5<double> ms = prev;
                bool been_inside = false;
                double ds = vol_march_start(V, ms, been_inside);
                int mcount = 0;
                bool end = false;
                while (!end) {
                    end = vol_march_rgb_step(S, pt, pph, ms, ds, been_inside, J, Tt, cnt);
                    ++mcount;
                    if (!end && mcount >= 4096) end = true;
                }
                double c[3];
                for (int ch = 0; ch < 3; ++ch) {
                    const double nu = rgb_nu(ch);
                    c[ch] = J[ch] * nu * nu * nu;
                }
                out.put(kDebugMarchExit, step, 0, mcount, c[0], c[1], c[2], ms.r, ms.r * cos(ms.th));
                ++nc;
                y = ms;  // the outer loop continues from the march's end state
                k1_ok = false;
            }
        } else {
            const double nan = __longlong_as_double(0x7ff8000000000000ll);
            out.put(kDebugStep, step, kDebugNone, 0, y.r, y.th, z, dlambda, nan, nan, y.ph);
            if (S.disk_on) {
                const double d_prev = prev.th - kHalfPi;
                const double d_new = y.th - kHalfPi;
                if (d_prev * d_new < 0.0 && fabs(d_prev - d_new) > 1e-12) {
                    const double frac = -d_prev / (d_new - d_prev);
                    const double rc = prev.r + frac * (y.r - prev.r);
                    if (rc >= S.r_in && rc <= S.r_out) {
                        double e0, e1, e2;
                        disk_emission(S, rc, pt, pph, e0, e1, e2);
                        col[0] += e0;
                        col[1] += e1;
                        col[2] += e2;
                        ++nc;
                        out.put(kDebugThinHit, step, 0, 0, rc, e0, e1, e2);
                    }
                }
            }
        }
        ++step;
    }
    double c[3];
    for (int ch = 0; ch < 3; ++ch) {
        const double nu = rgb_nu(ch);
        c[ch] = vol ? 0.0 + J[ch] * nu * nu * nu : col[ch];
    }
    out.put(kDebugEnd, step, term, nc, y.r, y.th, y.ph, c[0], c[1], c[2], static_cast<double>(cnt.attempts));
    *count = out.n;
}

}  // namespace

int debug_trace_capacity(int max_steps) {
    // per outer step at most a STEP record and a THIN_HIT or a MARCH pair
    const long long n = 3LL * (max_steps > 0 ? max_steps : 0) + 2;
    return static_cast<int>(n < kDebugMaxRecords ? n : kDebugMaxRecords);
}

cudaError_t launch_debug_trace(const DevScene& S, double x, double y, DevDebugRecord* rec, int cap, int* count,
                               cudaStream_t stream) {
    if (!rec || !count || cap < 1) return cudaErrorInvalidValue;
    debug_trace_kernel<<<1, 32, 0, stream>>>(S, x, y, rec, cap, count);
    return cudaGetLastError();
}

}  // namespace grrt_b200
