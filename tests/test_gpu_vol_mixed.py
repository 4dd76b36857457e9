"""Mixed form of the volumetric spectral render through the C ABI.

The speculative FP32 pass keeps only samples whose trajectory stays away from
the volume (no near-disk clamp, no hand-over, no near-critical orbit); every
other sample is re-traced from the camera by the FP64 kernel, and a resolve
pass sums each pixel's samples in order. So the spectra and every sample's
fate (termination | march entries << 2) must equal the FP64 form's bit for
bit, for one and several samples per pixel. The speculation must also keep a
real share of the samples, or the form would only add work.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def render(grrt, R, W, H, nb, g2):
    import torch
    spec = torch.full((H, W, nb), float("nan"), dtype=torch.float64, device="cuda")
    fate = torch.full((H * W * g2,), -1, dtype=torch.int32, device="cuda")
    R.render_spectral_device(spec, W, H, fate)
    torch.cuda.synchronize()
    return spec.cpu().numpy(), fate.cpu().numpy(), R.stats()


CASES = [
    ("a=0.9 80deg 96x96", dict(width=96, height=96)),
    ("a=0.9 edge-on 4spp 48x40", dict(width=48, height=40, samples_per_pixel=4, observer_theta=math.pi / 2)),
    ("a=0.5 30deg 64x64", dict(width=64, height=64, spin=0.5, observer_theta=math.radians(30.0))),
]


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_volumetric_mixed_equals_fp64(grrt, need_gpu, name, kw):
    freqs = grrt.log_bins(1e14, 1e18, 32)
    R = grrt.Renderer(grrt.config_params(3, **kw), freqs=freqs)
    W, H, nb = kw["width"], kw["height"], len(freqs)
    g2 = int(math.isqrt(kw.get("samples_per_pixel", 1))) ** 2
    R.set_precision(grrt.FORM_FP64)
    f, ff, fs = render(grrt, R, W, H, nb, g2)
    R.set_precision(grrt.FORM_MIXED)
    m, mf, ms = render(grrt, R, W, H, nb, g2)
    assert np.isfinite(f).all() and (f > 0).any()
    np.testing.assert_array_equal(m, f, err_msg=name)
    np.testing.assert_array_equal(mf, ff, err_msg=name)
    assert ms["rays"] == fs["rays"] == W * H * g2
    assert ms["horizon"] == fs["horizon"] and ms["escaped"] == fs["escaped"]
    # FP64 attempts of the re-trace against the FP64 form's
    share = ms["fp64_attempts"] / fs["fp64_attempts"]
    print(f"\n  [{name}] re-traced FP64 attempts / FP64 form's {share:.3f}; "
          f"speculative attempts {ms['attempts'] - ms['fp64_attempts']}")
    assert share < 0.95


@pytest.mark.parametrize("bg", [0, 1], ids=["black sky", "stars"])
def test_volumetric_rgb_mixed_equals_fp64(grrt, need_gpu, bg):
    """The volumetric RGB render's mixed form (the same speculation, plus the
    thin-disk form's star pass for escapes under a star sky, then the FP64
    re-trace and the ordered resolve) gives the FP64 form's image and fates
    bit for bit."""
    from parity_util import device_render_rgb
    R = grrt.Renderer(grrt.config_params(3, width=64, height=48, background_type=bg, samples_per_pixel=4))
    R.set_precision(grrt.FORM_FP64)
    f_rgba, f64, ffate, fst = device_render_rgb(R, 4)
    R.set_precision(grrt.FORM_MIXED)
    m_rgba, m64, mfate, mst = device_render_rgb(R, 4)
    assert (f64 > 0).any()
    np.testing.assert_array_equal(m64, f64)
    np.testing.assert_array_equal(m_rgba, f_rgba)
    np.testing.assert_array_equal(mfate, ffate)
    assert mst["rays"] == fst["rays"] == 64 * 48 * 4
    assert mst["horizon"] == fst["horizon"] and mst["escaped"] == fst["escaped"]
    share = mst["fp64_attempts"] / fst["fp64_attempts"]
    print(f"\n  [{'stars' if bg else 'black'}] re-traced FP64 attempts / FP64 form's {share:.3f}")
    assert share < 0.95
