"""The surrogate's closed-form ray classification
(grrt_b200/csrc/device/surrogate_geom.cuh), compiled as host code, against
the FP64 method's traces of the same camera rays. CPU only.

A camera ray falls in iff the radial potential R(r) stays positive between the
horizon and the camera; the minimum of R / (E^2 r^4) is the distance to the
critical curve. Bars: the closed-form fate equals the integrated one (any
disagreement lies within 0.01 of the curve and is rare), and every ray with an
equatorial crossing outside 0.9 r_in after its second crossing that does not
graze the plane lies inside the default critical band (|margin| < 0.15), so
the network, which models two crossings, never has to model one.
"""
import ctypes as C
import math
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from oracle_bind import Oracle, jittered_samples
from test_device_math import devmath  # noqa: F401  (fixture)

CASES = [
    ("kerr 0.998 80deg", dict(spin=0.998)),
    ("schwarzschild 80deg", dict(metric_type=0, spin=0.0)),
    ("kerr 0.9 67deg", dict(spin=0.9, observer_theta=math.radians(67.3))),
    ("kerr 0.998 33deg", dict(spin=0.998, observer_theta=math.radians(33.3))),
    ("kerr 0.5 edge-on", dict(spin=0.5, observer_theta=math.pi / 2)),
]
CRITICAL_BAND = 0.15  # surr::RenderBands::capture
GRAZE_BAND = 0.02


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_closed_form_margins(grrt, devmath, name, kw):  # noqa: F811
    n = 64
    R = grrt.Renderer(grrt.config_params(2, width=n, height=n, spp=1, background_type=0, **kw))
    M, a, rh, _isco, robs, tol, max_steps = R.table("scalars")[:7]
    r_in = R.table("flux_meta")[1]
    sc = np.array([M, a, rh + 0.01, 1000.0, 0.01 * robs, tol, max_steps, 0.9 * r_in])
    PD = C.POINTER(C.c_double)
    devmath.devmath_ray_margins.argtypes = [C.c_double, C.c_double, C.c_double, PD, PD]
    devmath.devmath_trace_crossings.argtypes = [PD, PD, PD]
    px, py = jittered_samples(n, n, 1, np.arange(n * n))
    O = Oracle(R)

    def one(k):
        y8 = O.camera_ray(px[k], py[k])
        m, o = np.zeros(2), np.zeros(6)
        devmath.devmath_ray_margins(M, a, rh, y8.ctypes.data_as(PD), m.ctypes.data_as(PD))
        devmath.devmath_trace_crossings(sc.ctypes.data_as(PD), y8.ctypes.data_as(PD), o.ctypes.data_as(PD))
        return np.concatenate([m, o])

    with ThreadPoolExecutor(8) as ex:
        res = np.array(list(ex.map(one, range(n * n), chunksize=64)))
    cap, graze, term, extra = res[:, 0], res[:, 1], res[:, 2].astype(int), res[:, 7]
    # the host trace is the oracle's method: its fates are the oracle's
    _, oterm, _, _, _ = O.trace_rgb(px, py)
    assert np.mean(oterm == term) > 0.998
    ok = term != 2
    bad = ok & ((cap > 0) != (term == 0))
    multi = (extra >= 1) & (graze >= GRAZE_BAND)
    worst_bad = float(np.max(np.abs(cap[bad]))) if bad.any() else 0.0
    worst_multi = float(np.max(np.abs(cap[multi]))) if multi.any() else 0.0
    print(f"\n  [{name}] captured {np.mean(term == 0):.3f}; fate disagreements {int(bad.sum())} (|m| <= {worst_bad:.2e}); "
          f"relevant crossings after the second {int(multi.sum())} (|m| <= {worst_multi:.3f}); in critical band {np.mean(np.abs(cap) < CRITICAL_BAND):.4f}")
    assert worst_bad < 0.01 and bad.mean() < 0.005
    assert worst_multi < CRITICAL_BAND


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_gate_scan_stops_at_gate_radius(grrt, devmath, name, kw):  # noqa: F811
    """The black-sky gate (camera_ray_clears: scan stopped at r_gate, bracket
    settled by the sign of R there) gives the same answer as comparing the
    full scan-and-bisection smallest radius with r_gate, on every camera ray of
    a frame and several gate radii."""
    n = 96
    R = grrt.Renderer(grrt.config_params(2, width=n, height=n, spp=1, background_type=0, **kw))
    M, a, rh = R.table("scalars")[:3]
    PD = C.POINTER(C.c_double)
    devmath.devmath_gate.argtypes = [C.c_double, C.c_double, C.c_double, PD, C.c_double, PD]
    px, py = jittered_samples(n, n, 1, np.arange(n * n))
    O = Oracle(R)
    rays = [O.camera_ray(x, y) for x, y in zip(px, py)]
    cleared = 0
    for r_gate in (5.0, 10.0, 20.1, 30.0):
        for y8 in rays:
            out = np.zeros(2)
            devmath.devmath_gate(M, a, rh, y8.ctypes.data_as(PD), r_gate, out.ctypes.data_as(PD))
            r_min = out[0]
            if abs(r_min - r_gate) < 1e-9 * r_gate:
                continue  # the root at the gate radius itself (bisection precision)
            assert (out[1] == 1.0) == (r_min > r_gate), (name, r_gate, r_min)
            cleared += int(out[1])
    assert cleared > 0
