"""The mixed-precision thin-disk form (FP32 speculation + FP64 re-trace)
through the C ABI.

Bar of the mixed form (relative linear intensity <= 1e-4 against the FP64
form, identical fates outside the caustic band): here every pixel must be
within MIX_TOL of the FP64 form's device render, every sample's fate must
equal it, and the mixed render must pass the FP64 form's own parity check
against the oracle. The re-trace's FP64 attempts are bounded by half of the
FP64 form's, so that a form that re-traces everything fails.
"""
import math

import numpy as np
import pytest

from parity_util import device_render_rgb
from test_gpu_parity import check_rgb

pytestmark = pytest.mark.gpu

MIX_TOL = 1e-4


def both_forms(grrt, params):
    R = grrt.Renderer(params)
    spp = params.get("samples_per_pixel", 1)
    R.set_precision(grrt.FORM_FP64)
    f = device_render_rgb(R, spp)
    R.set_precision(grrt.FORM_MIXED)
    m = device_render_rgb(R, spp)
    return R, f, m


def compare(f, m, name):
    _, f64, ffate, fst = f
    _, m64, mfate, mst = m
    scale = float(np.max(f64))
    rel = np.abs(m64 - f64) / np.maximum(np.abs(f64), 1e-6 * scale)
    worst = float(rel.max())
    nfate = int(np.sum(ffate != mfate))
    share = mst["fp64_attempts"] / mst["attempts"]
    fp64_work = mst["fp64_attempts"] / fst["attempts"]
    print(f"\n  [{name}] max rel {worst:.2e}; fate differences {nfate}; pixels differing "
          f"{int(np.sum(np.any(m64 != f64, axis=2)))}; re-trace share of attempts {share:.3f}; "
          f"attempts mixed/fp64 {mst['attempts'] / fst['attempts']:.3f}; FP64 attempts mixed/fp64 {fp64_work:.3f}")
    assert worst <= MIX_TOL, f"{name}: max relative error {worst:.3e} against the FP64 form"
    assert nfate == 0, f"{name}: {nfate} sample fates differ from the FP64 form"
    assert mst["rays"] == fst["rays"]
    assert mst["crossings"] == fst["crossings"]
    # the re-trace does less than half of the FP64 form's FP64 work
    assert fp64_work < 0.5


CASES = [
    ("schwarzschild 256 1spp", 1, dict(width=256, height=256)),
    ("kerr 0.998 256 4spp stars", 2, dict(width=256, height=256)),
    ("kerr 0.998 edge-on 192", 2, dict(width=192, height=192, observer_theta=math.pi / 2)),
    ("kerr 0.9 20deg 160", 2, dict(width=160, height=160, spin=0.9, observer_theta=math.radians(20.0))),
    ("schwarzschild 9spp 96", 1, dict(width=96, height=96, spp=9)),
]


@pytest.mark.parametrize("name,cfg,kw", CASES, ids=[c[0] for c in CASES])
def test_mixed_matches_fp64_form(grrt, need_gpu, name, cfg, kw):
    p = grrt.config_params(cfg, **kw)
    _, f, m = both_forms(grrt, p)
    compare(f, m, name)


def test_mixed_parity_against_oracle(grrt, need_gpu):
    R = grrt.Renderer(grrt.config_params(1))
    R.set_precision(grrt.FORM_MIXED)
    # the speculative pass does other work than the method (fewer, FP32 attempts)
    check_rgb(grrt, R, same_work=False)


def test_mixed_tile_equals_crop(grrt, need_gpu):
    p = grrt.config_params(2, width=160, height=120)
    R = grrt.Renderer(p)
    R.set_precision(grrt.FORM_MIXED)
    full = R.render()
    tile = R.render_tile(37, 21, 64, 50)
    np.testing.assert_array_equal(tile, full[21:71, 37:101])


def test_mixed_knobs(grrt, need_gpu):
    """A wider disk margin and a tighter FP32 tolerance re-trace more and give
    the same image; the knobs are rejected when out of range."""
    p = grrt.config_params(2, width=128, height=128)
    R = grrt.Renderer(p)
    R.set_precision(grrt.FORM_FP64)
    want = R.render()
    R.set_precision(grrt.FORM_MIXED)
    R.set_mixed_params(3.0, 1e-6)
    a = R.render()
    s1 = R.stats()
    R.set_mixed_params(6.0, 1e-7)
    b = R.render()
    s2 = R.stats()
    np.testing.assert_allclose(a, want, rtol=MIX_TOL, atol=0)
    np.testing.assert_allclose(b, want, rtol=MIX_TOL, atol=0)
    assert s2["attempts"] != s1["attempts"]
    with pytest.raises(RuntimeError):
        R.set_mixed_params(0.5, 1e-6)
    with pytest.raises(RuntimeError):
        R.set_mixed_params(3.0, 0.0)
