"""The mixed form's speculative pass (grrt_b200/csrc/device/mixed_spec.cuh),
compiled as host code, against the oracle. CPU only.

The mixed form keeps a speculative FP32 result only when it is exactly 0
(horizon, or escape with no star within reach of the lookup); everything else
is re-traced with the FP64 method. So the bar is one-sided and exact: every
sample whose oracle colour is non-zero, or that crosses the disk inside
[r_in, r_out], must be sent to the re-trace. The flagged fraction is bounded
too, so a pass that re-traces everything cannot meet the bar.
"""
import ctypes as C
import math

import numpy as np
import pytest

from oracle_bind import Oracle, jittered_samples
from test_device_math import devmath  # noqa: F401  (fixture)

STAR_TOL = 0.003  # the star catalogue's angular tolerance (rad)


def speculate_all(L, R, px, py, margin=0.05, r_factor=3.0, tol32=3e-6):
    sc = R.table("scalars")
    M, a, rh, isco, robs, _tol, max_steps = sc[:7]
    disk = R.values["disk_enabled"] != 0
    r_in, r_out = (R.table("flux_meta")[1], R.table("flux_meta")[2]) if disk else (0.0, 0.0)
    stars = R.values["background_type"] == 1
    # near-critical radius: r_factor r_h, at least 1.25 x the outermost photon orbit (as the library)
    r_ph = 2.0 * M * (1.0 + math.cos(2.0 / 3.0 * math.acos(min(abs(a) / M, 1.0))))
    r_near = max(r_factor * rh, 1.25 * r_ph)
    v = np.array([M, a, rh + 0.01, 1000.0, 0.01 * robs, tol32, max_steps, r_in, r_out, margin, r_near,
                  1.0 if disk else 0.0, 1.0 if stars else 0.0])
    PD, PI = C.POINTER(C.c_double), C.POINTER(C.c_int)
    hold = []
    if stars:
        st = R.table("stars").reshape(-1, 3)
        th, ph = np.ascontiguousarray(st[:, 0]), np.ascontiguousarray(st[:, 1])
        cells = R.table("star_cells").astype(np.int32)
        items = R.table("star_items").astype(np.int32)
        hold = [th, ph, cells, items]
        args = (th.ctypes.data_as(PD), ph.ctypes.data_as(PD), cells.ctypes.data_as(PI), items.ctypes.data_as(PI))
    else:
        args = (None, None, None, None)
    O = Oracle(R)
    flags = np.zeros(len(px), dtype=np.int32)
    terms = np.zeros(len(px), dtype=np.int32)
    t = C.c_int()
    for k, (x, y) in enumerate(zip(px, py)):
        y8 = O.camera_ray(x, y)
        flags[k] = L.devmath_speculate(v.ctypes.data_as(PD), y8.ctypes.data_as(PD), *args, STAR_TOL ** 2,
                                       C.byref(t))
        terms[k] = t.value
    del hold
    return flags, terms


CASES = [
    ("schwarzschild 80deg", 1, 72, {}),
    ("kerr 0.998 80deg stars", 2, 56, {}),
    ("kerr 0.998 edge-on stars", 2, 56, {"observer_theta": math.pi / 2}),
    ("kerr 0.5 30deg stars", 2, 48, {"spin": 0.5, "observer_theta": math.radians(30.0)}),
    # black sky: certain escapes end the speculative trace early
    ("kerr 0.998 80deg black sky", 2, 56, {"background_type": 0}),
    ("kerr 0.9 edge-on black sky", 2, 48, {"spin": 0.9, "observer_theta": math.pi / 2, "background_type": 0}),
]


@pytest.mark.parametrize("name,cfg,n,kw", CASES, ids=[c[0] for c in CASES])
def test_speculation_flags_every_sample_with_colour(grrt, devmath, name, cfg, n, kw):  # noqa: F811
    L = devmath
    L.devmath_speculate.restype = C.c_int
    L.devmath_speculate.argtypes = [C.POINTER(C.c_double)] * 4 + [C.POINTER(C.c_int)] * 2 + [C.c_double,
                                                                                            C.POINTER(C.c_int)]
    R = grrt.Renderer(grrt.config_params(cfg, width=n, height=n, spp=1, **kw))
    px, py = jittered_samples(n, n, 1, np.arange(n * n))
    flags, terms = speculate_all(L, R, px, py)
    O = Oracle(R)
    rgb, term, ncross, _fin, _cnt = O.trace_rgb(px, py)
    coloured = np.any(rgb != 0.0, axis=1) | (ncross > 0) | (term == 2)
    missed = np.nonzero(coloured & (flags == 0))[0]
    assert len(missed) == 0, f"{name}: {len(missed)} samples with colour kept as 0, e.g. {missed[:5]}"
    # a final speculative zero keeps the oracle's termination
    keep = flags == 0
    assert np.all(terms[keep] == term[keep]), f"{name}: termination differs on kept samples"
    frac = flags.mean()
    print(f"\n  [{name}] flagged {frac:.3f} of samples; coloured {coloured.mean():.3f}")
    assert frac <= max(0.5, 1.6 * coloured.mean())


def tracker_step(L, tr, y, y5, h):
    PD = C.POINTER(C.c_double)
    L.devmath_tracker_step.restype = C.c_int
    L.devmath_tracker_step.argtypes = [PD, PD, PD, C.c_double, PD]
    tr, y, y5, out = (np.ascontiguousarray(v, dtype=np.float64) for v in (tr, y, y5, [0.0]))
    hit = L.devmath_tracker_step(tr.ctypes.data_as(PD), y.ctypes.data_as(PD), y5.ctypes.data_as(PD), h,
                                 out.ctypes.data_as(PD))
    return hit, out[0]


def test_tracker_polar_and_turning_rules(devmath):  # noqa: F811
    """The speculation's polar and turning-point rules on hand-made steps
    (mixed_spec.cuh): a step ending near a pole, a step across the axis, a
    theta turning point closer to the axis than the threshold inside a long
    step, and an equatorial crossing whose chord misses the disk band while
    the step holds a radial turning point inside it. Plain steps away from
    all of these are not flagged."""
    L = devmath
    half = math.pi / 2
    # disk [2, 20], margin 0.05, r_near 5; a = 0.9, p_t = -1, p_phi = 0.1
    tr = [1.0, 2.0, 20.0, 0.05, 5.0, 0.9, -1.0, 0.1]
    # an ordinary step high above the plane: not flagged
    hit, _ = tracker_step(L, tr, [40, 0.8, 0, 0.5, 0.3], [41, 0.81, 0.1, 0.5, 0.3], 1.0)
    assert hit == 0
    # ends within |sin theta| < 0.02 of the pole
    hit, _ = tracker_step(L, tr, [40, 0.05, 0, 0.5, -0.3], [41, 0.01, 0.1, 0.5, -0.3], 1.0)
    assert hit == 1
    # steps across the axis (theta changes sign)
    hit, _ = tracker_step(L, tr, [40, 0.05, 0, 0.5, -0.3], [41, -0.04, 0.1, 0.5, -0.3], 1.0)
    assert hit == 1
    # theta turns inside the step, both ends 0.1 from the axis: flagged when
    # the Carter-constant turning point lies within 0.02 of the axis
    hit, u = tracker_step(L, tr, [40, 0.1, 0, 0.5, -0.05], [41, 0.1, 0.1, 0.5, 0.05], 1.0)
    assert (1.0 - u < 0.02 ** 2) == (hit == 1)
    tr_lz = list(tr)
    tr_lz[7] = 0.0  # zero angular momentum: the ray passes over the pole itself
    hit, u = tracker_step(L, tr_lz, [40, 0.1, 0, 0.5, -0.05], [41, 0.1, 0.1, 0.5, 0.05], 1.0)
    assert hit == 1 and u == pytest.approx(1.0)
    tr_big = list(tr)
    tr_big[7] = 40.0  # large p_phi: turns far from the axis
    hit, u = tracker_step(L, tr_big, [40, 0.6, 0, 0.5, -0.05], [41, 0.6, 0.1, 0.5, 0.05], 1.0)
    assert hit == 0 and 1.0 - u > 0.02 ** 2
    # an equatorial crossing whose chord lands at 20.40, outside [1.95, 20.05]
    # widened by 0.2 |dr| = 0.02 ...
    y = [20.30, half - 0.01, 0, -0.02, 0.0]
    y5 = [20.40, half + 0.01, 0.1, -0.01, 0.0]
    hit, _ = tracker_step(L, tr, y, y5, 3.0)
    assert hit == 0
    # ... is flagged when p_r changes sign in the step (radial turning point:
    # the radii dip by up to h min|p_r| below the smaller end)
    y5_turn = [20.40, half + 0.01, 0.1, 0.2, 0.0]
    hit, _ = tracker_step(L, tr, [20.30, half - 0.01, 0, -0.2, 0.0], y5_turn, 3.0)
    assert hit == 1
