"""The oracle and the host-built tables against the reference's own outputs.

tests/golden/reference_vectors.json was produced by tests/golden/make_golden.py
from the reference library compiled from its own sources (strict IEEE build);
every double is stored as float.hex(), so these comparisons are bit-exact.
CPU only.
"""
import hashlib
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def unhex(lst):
    return np.array([float.fromhex(x) for x in lst])


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


SCENES = ["schwarzschild_thin", "kerr0998_thin_stars", "kerr09_volumetric"]


def make_renderer(grrt, rec):
    vals = dict(rec["params"])
    freqs = unhex(rec["freqs"]) if "freqs" in rec else None
    return grrt.Renderer(vals, freqs=freqs), freqs


@pytest.mark.parametrize("scene", SCENES)
def test_host_tables_match_reference(grrt, golden, scene):
    rec = golden["scenes"][scene]
    R, _ = make_renderer(grrt, rec)
    for name, want in rec["tables"].items():
        assert digest(R.table(name)) == want, f"{scene}: table {name} differs from the reference"
    meta = R.table("flux_meta")
    np.testing.assert_array_equal(meta[:3], unhex(rec["flux_meta"]))
    if "vol_scalars" in rec:
        np.testing.assert_array_equal(R.table("vol_scalars")[:11], unhex(rec["vol_scalars"]))


@pytest.mark.parametrize("scene", SCENES)
def test_camera_rays_match_reference(grrt, oracle_lib, golden, scene):
    rec = golden["scenes"][scene]
    R, _ = make_renderer(grrt, rec)
    px, py = unhex(rec["px"]), unhex(rec["py"])
    want = unhex(rec["camera"]).reshape(-1, 8)
    got = np.array([R.camera_ray(x, y) for x, y in zip(px, py)])
    np.testing.assert_array_equal(got, want)
    O = oracle_lib.Oracle(R)
    got_o = np.array([O.camera_ray(x, y) for x, y in zip(px, py)])
    np.testing.assert_array_equal(got_o, want)


@pytest.mark.parametrize("scene", ["schwarzschild_thin", "kerr0998_thin_stars"])
def test_oracle_thin_traces_bit_exact(grrt, oracle_lib, golden, scene):
    rec = golden["scenes"][scene]
    R, _ = make_renderer(grrt, rec)
    O = oracle_lib.Oracle(R)
    rgb, term, nc, fin, _ = O.trace_rgb(unhex(rec["px"]), unhex(rec["py"]))
    np.testing.assert_array_equal(rgb.ravel(), unhex(rec["rgb"]))
    np.testing.assert_array_equal(term, np.array(rec["term"]))
    np.testing.assert_array_equal(fin.ravel(), unhex(rec["final"]))
    assert (term == 1).any() and (term == 0).any(), "fixture should cover escape and horizon"
    assert (nc > 0).any(), "fixture should include disk crossings"


def test_oracle_volumetric_traces_bit_exact(grrt, oracle_lib, golden):
    rec = golden["scenes"]["kerr09_volumetric"]
    R, freqs = make_renderer(grrt, rec)
    O = oracle_lib.Oracle(R)
    px, py = unhex(rec["px"]), unhex(rec["py"])
    spec, term, cnt = O.trace_spectral(freqs, px, py)
    np.testing.assert_array_equal(spec.ravel(), unhex(rec["spectra"]))
    np.testing.assert_array_equal(term, np.array(rec["term"]))
    rgb, term_rgb, _, _, _ = O.trace_rgb(px, py)
    np.testing.assert_array_equal(rgb.ravel(), unhex(rec["rgb"]))
    np.testing.assert_array_equal(term_rgb, np.array(rec["term_rgb"]))
    assert cnt["physics_steps"] > 0, "fixture should march through matter"


def test_oracle_matches_reference_c_api_render(grrt, oracle_lib, golden):
    """Renderer::render end to end (jitter hash, 2x2 grid, spp mean, float cast)."""
    rec = golden["api_render"]
    vals = dict(rec["params"])
    R = grrt.Renderer(vals)
    O = oracle_lib.Oracle(R)
    W, H = vals["width"], vals["height"]
    rgb, _ = O.render_pixels(np.arange(W * H), spp=vals["samples_per_pixel"])
    want = unhex(rec["rgba_f32"]).astype(np.float32).reshape(H, W, 4)
    np.testing.assert_array_equal(rgb.reshape(H, W, 3).astype(np.float32), want[..., :3])
    assert np.all(want[..., 3] == 1.0)


def test_pixel_hash(oracle_lib, golden):
    L = oracle_lib.load_oracle()
    for i, j, s, ch, want in golden["pixel_hash"]:
        assert float(L.oracle_pixel_hash(i, j, s, ch)) == float.fromhex(want)


def test_fast_sincos_accuracy(oracle_lib):
    """The Cephes sin/cos of the integrator: error ~1e-16 over the range rays visit."""
    import ctypes as C
    L = oracle_lib.load_oracle()
    xs = np.linspace(-8.0, 8.0, 20001)
    s, c = C.c_double(), C.c_double()
    err = 0.0
    for x in xs:
        L.oracle_fast_sincos(x, C.byref(s), C.byref(c))
        err = max(err, abs(s.value - np.sin(x)), abs(c.value - np.cos(x)))
    assert err < 1e-15


GOLDEN_FITS = os.path.join(os.path.dirname(__file__), "golden", "reference_fits.json")


@pytest.mark.parametrize("case", ["log32_16x12", "linear5_13x7_spp4", "table3_9x5"])
def test_oracle_matches_reference_fits_data(grrt, oracle_lib, case):
    """The reference's grrt_render_spectral_to_fits_cb (src/api.cpp:283-332):
    its cube, decoded (big-endian, FITS row = height-1-j, plane-major), equals
    the oracle's spp-mean spectra bit for bit."""
    with open(GOLDEN_FITS) as f:
        rec = json.load(f)["cases"][case]
    vals = dict(rec["params"])
    freqs = unhex(rec["freqs"])
    W, H, nb = vals["width"], vals["height"], len(freqs)
    R = grrt.Renderer(vals, freqs=freqs)
    O = oracle_lib.Oracle(R)
    spec, _ = O.render_spectral_pixels(freqs, np.arange(W * H), spp=vals["samples_per_pixel"])
    planes = unhex(rec["data"]).reshape(nb, H, W)
    want = planes[:, ::-1, :].transpose(1, 2, 0).reshape(W * H, nb)
    np.testing.assert_array_equal(spec, want)
    assert (want > 0).any(), "fixture should hold emission"
    hdr = rec["header"]
    assert len(hdr) % 2880 == 0 and hdr.startswith("SIMPLE  =")
    data = 8 * W * H * nb
    assert rec["size"] == len(hdr) + (data + 2879) // 2880 * 2880
