"""Generate tests/golden/reference_vectors.json from the reference itself.

The reference library is compiled from its own sources by oracle/Makefile
(`make -C oracle ref`, needs the reference tree) into oracle/_ref/. This script
drives it through oracle/_ref/libref_harness_strict.so and records, with
every double written as float.hex() so the comparison is bit-exact:

  * SHA-256 digests of every host-built table for the benchmark scenes
    (small image sizes; tables do not depend on the image size except the
    camera),
  * per-sample traces (colour, termination, final state) of a fixed set of
    camera samples for the thin-disk scenes, and spectra for the volumetric
    scene,
  * the stratified-jitter hash on a few arguments.

It also writes tests/golden/reference_fits.json: FITS cubes written by the
reference's own grrt_render_spectral_to_fits_cb (src/api.cpp:283-332, the
streaming writer of src/fits_writer.cpp:315-395) for three frequency-axis
kinds (log-uniform, linear-uniform, tabulated), each with its header bytes
(latin-1 text), file size and data section (big-endian doubles as hex).

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import grrt_b200 as G  # noqa: E402
from oracle_bind import RefScene, jittered_samples  # noqa: E402

OUT = os.path.join(HERE, "reference_vectors.json")
OUT_FITS = os.path.join(HERE, "reference_fits.json")

# (name, scene overrides of the volumetric scene (config 3), frequencies)
FITS_CASES = [
    ("log32_16x12", dict(width=16, height=12), ("log", 1e14, 1e18, 32)),
    ("linear5_13x7_spp4", dict(width=13, height=7, samples_per_pixel=4), ("list", 1e14, 2e14, 3e14, 4e14, 5e14)),
    ("table3_9x5", dict(width=9, height=5, spin=0.5), ("list", 1e14, 3e15, 2e17)),
]


def fits_case_freqs(spec) -> np.ndarray:
    if spec[0] == "log":
        return G.log_bins(spec[1], spec[2], spec[3])
    return np.array(spec[1:], dtype=np.float64)


def fits_vectors() -> None:
    """FITS files written by the reference's C API (strict build)."""
    import ctypes as C
    import tempfile
    ref_api = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libgrrt_ref_strict.so"))
    ref_api.grrt_create.restype = C.c_void_p
    ref_api.grrt_create.argtypes = [C.POINTER(G.GRRTParams)]
    ref_api.grrt_set_frequency_bins.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int]
    ref_api.grrt_render_spectral_to_fits_cb.restype = C.c_int
    ref_api.grrt_render_spectral_to_fits_cb.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int, C.c_void_p,
                                                        C.c_void_p]
    ref_api.grrt_destroy.argtypes = [C.c_void_p]
    out = {"generator": "tests/golden/make_golden.py", "build": "oracle/_ref/libgrrt_ref_strict.so", "cases": {}}
    for name, over, fspec in FITS_CASES:
        vals = G.config_params(3, **over)
        freqs = fits_case_freqs(fspec)
        prm = G.make_params(vals, freqs)
        ctx = ref_api.grrt_create(C.byref(prm))
        assert ctx, name
        ref_api.grrt_set_frequency_bins(ctx, freqs.ctypes.data_as(C.POINTER(C.c_double)), len(freqs))
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "ref.fits")
            rc = ref_api.grrt_render_spectral_to_fits_cb(ctx, path.encode(), vals["width"], vals["height"], None,
                                                         None)
            assert rc == 0, name
            raw = open(path, "rb").read()
        ref_api.grrt_destroy(ctx)
        # header: 80-character cards up to END, padded to 2880-byte blocks
        end = 0
        while raw[end:end + 3] != b"END":
            end += 80
        hdr_len = (end // 2880 + 1) * 2880
        n = vals["width"] * vals["height"] * len(freqs)
        data = np.frombuffer(raw[hdr_len:hdr_len + 8 * n], dtype=">f8")
        out["cases"][name] = {"params": vals, "freqs": hexlist(freqs), "size": len(raw),
                              "header": raw[:hdr_len].decode("latin-1"), "data": hexlist(data)}
    with open(OUT_FITS, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT_FITS, os.path.getsize(OUT_FITS), "bytes")


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def hexlist(a) -> list:
    return [float(x).hex() for x in np.ravel(a)]


def sample_coords(W: int, H: int, n: int, seed: int):
    # jittered samples of a fixed pixel set: a third anywhere (mostly sky), a
    # third around the shadow, a third in the band where the disk projects
    rng = np.random.default_rng(seed)
    k = n // 3
    anywhere = rng.choice(W * H, size=n - 2 * k, replace=False)
    r = max(2, W // 10)
    cx, cy = W // 2, H // 2
    shadow = [(cy + rng.integers(-r, r)) * W + cx + rng.integers(-r, r) for _ in range(k)]
    band = [(cy + rng.integers(-max(1, H // 12), max(1, H // 12))) * W + rng.integers(0, W) for _ in range(k)]
    pix = np.concatenate([anywhere, np.array(shadow), np.array(band)]).astype(np.int64)
    return jittered_samples(W, H, 1, pix)


def main() -> None:
    out = {"generator": "tests/golden/make_golden.py", "build": "oracle/_ref/libgrrt_ref_strict.so",
           "scenes": {}}
    scenes = {
        "schwarzschild_thin": dict(cfg=1, W=64, H=64, n=48),
        "kerr0998_thin_stars": dict(cfg=2, W=64, H=64, n=48),
        "kerr09_volumetric": dict(cfg=3, W=48, H=48, n=24),
    }
    for name, s in scenes.items():
        vals = G.config_params(s["cfg"], width=s["W"], height=s["H"], spp=1)
        freqs = G.log_bins(1e14, 1e18, 32) if s["cfg"] == 3 else None
        ref = RefScene(vals, freqs=freqs)
        rec = {"params": {k: v for k, v in vals.items()}, "tables": {}}
        flux, meta = ref.flux()
        rec["tables"]["flux"] = digest(flux)
        rec["flux_meta"] = hexlist(meta[:3])
        color, lum = ref.spectrum()
        rec["tables"]["spectrum_color"] = digest(color)
        rec["tables"]["spectrum_lum"] = digest(lum)
        if vals["background_type"] == G.BG_STARS:
            rec["tables"]["stars"] = digest(ref.stars())
        vt = ref.vol_tables()
        if vt is not None:
            for k in ("vol_H", "vol_rho_mid", "vol_rho_prof", "vol_T_prof", "vol_zmax", "op_kabs", "op_kes",
                      "op_kross", "op_mu"):
                rec["tables"][k] = digest(vt[k])
            rec["tables"]["vol_perm"] = digest(vt["vol_perm"].astype(np.float64))
            rec["vol_scalars"] = hexlist(vt["scal"][:11])
        px, py = sample_coords(s["W"], s["H"], s["n"], seed=11 + s["cfg"])
        rec["px"] = hexlist(px)
        rec["py"] = hexlist(py)
        rec["camera"] = hexlist(ref.camera_rays(px, py))
        if freqs is None:
            rgb, term, fin = ref.trace_rgb(px, py)
            rec["rgb"] = hexlist(rgb)
            rec["term"] = [int(t) for t in term]
            rec["final"] = hexlist(fin)
        else:
            rec["freqs"] = hexlist(freqs)
            spec, term = ref.trace_spectral(px, py)
            rec["spectra"] = hexlist(spec)
            rec["term"] = [int(t) for t in term]
            rgb, term_rgb, fin = ref.trace_rgb(px, py)
            rec["rgb"] = hexlist(rgb)
            rec["term_rgb"] = [int(t) for t in term_rgb]
        out["scenes"][name] = rec
    # The reference's own C API end to end (Renderer::render with its file-static
    # jitter hash and spp averaging, float framebuffer) on a 4-spp scene.
    import ctypes as C
    import oracle_bind
    ref_api = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libgrrt_ref_strict.so"))
    ref_api.grrt_create.restype = C.c_void_p
    ref_api.grrt_create.argtypes = [C.POINTER(G.GRRTParams)]
    ref_api.grrt_render.restype = C.c_int
    ref_api.grrt_render.argtypes = [C.c_void_p, C.POINTER(C.c_float)]
    ref_api.grrt_destroy.argtypes = [C.c_void_p]
    vals = G.config_params(2, width=16, height=16, spp=4)
    prm = G.make_params(vals)
    ctx = ref_api.grrt_create(C.byref(prm))
    fb = np.zeros((16, 16, 4), dtype=np.float32)
    ref_api.grrt_render(ctx, fb.ctypes.data_as(C.POINTER(C.c_float)))
    ref_api.grrt_destroy(ctx)
    out["api_render"] = {"params": vals, "rgba_f32": [float(x).hex() for x in fb.ravel()]}
    L = oracle_bind.load_oracle()
    hashes = []
    for (i, j, s_, ch) in [(0, 0, 0, 0), (1, 0, 0, 1), (17, 33, 2, 0), (1023, 1023, 3, 1), (511, 7, 1, 0)]:
        hashes.append([i, j, s_, ch, float(L.oracle_pixel_hash(i, j, s_, ch)).hex()])
    out["pixel_hash"] = hashes
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")
    fits_vectors()


if __name__ == "__main__":
    main()
