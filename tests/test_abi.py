"""The C-ABI boundary: libgrrt.so loads, exports every symbol include/*.h
declares, keeps GRRTParams byte-identical to the reference's, and follows the
reference's error conventions. No compute calls (CPU only)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for dirpath, _, files in os.walk(INCLUDE):
        for fn in files:
            if fn.endswith(".h"):
                text = open(os.path.join(dirpath, fn)).read()
                names.update(re.findall(r"GRRT_EXPORT\s+[^;(]*?\b(grrt_\w+)\s*\(", text, flags=re.S))
    return sorted(names)


def test_every_declared_symbol_is_exported(grrt):
    names = declared_functions()
    assert len(names) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", grrt.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [n for n in names if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    L = grrt.lib()
    for n in names:
        assert hasattr(L, n)


def test_reference_api_surface_complete(grrt):
    """Every entry point of the reference's include/grrt/api.h:11-51."""
    ref_api = ["grrt_create", "grrt_destroy", "grrt_update_params", "grrt_render", "grrt_render_cb",
               "grrt_render_tile", "grrt_cancel", "grrt_progress", "grrt_error", "grrt_cuda_available",
               "grrt_last_error", "grrt_tonemap", "grrt_debug_pixel", "grrt_set_frequency_bins",
               "grrt_render_spectral", "grrt_render_spectral_cb", "grrt_render_spectral_to_fits_cb"]
    names = set(declared_functions())
    assert set(ref_api) <= names


def header_layout():
    """offsetof each GRRTParams member as compiled from include/grrt_api.h."""
    fields = [f for f, _ in __import__("grrt_b200").GRRTParams._fields_]
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "grrt_api.h"', "int main(void){",
           'printf("%zu\\n", sizeof(GRRTParams));']
    src += [f'printf("%zu\\n", offsetof(GRRTParams, {f}));' for f in fields]
    src += ["return 0;}"]
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "l.c")
        exe = os.path.join(d, "l")
        open(c, "w").write("\n".join(src))
        subprocess.run(["/usr/bin/gcc", "-I", INCLUDE, c, "-o", exe], check=True)
        vals = [int(x) for x in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    return vals


def test_params_layout_matches_ctypes(grrt):
    vals = header_layout()
    P = grrt.GRRTParams
    assert vals[0] == C.sizeof(P)
    for (name, _), off in zip(P._fields_, vals[1:]):
        assert getattr(P, name).offset == off, name


def test_params_layout_matches_reference(grrt):
    import oracle_bind
    if not oracle_bind.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    L = oracle_bind.load_ref()
    L.rh_params_layout.restype = C.c_int
    L.rh_params_layout.argtypes = [C.POINTER(C.c_long)]
    buf = (C.c_long * 64)()
    n = L.rh_params_layout(buf)
    ref = list(buf[: n + 1])
    assert ref == header_layout()


def test_create_errors(grrt):
    L = grrt.lib()
    assert not L.grrt_create(None)
    assert b"NULL" in L.grrt_last_error()
    p = grrt.make_params(grrt.config_params(1, width=0))
    assert not L.grrt_create(C.byref(p))
    assert b"width" in L.grrt_last_error()


def test_create_resolves_reference_defaults(grrt):
    """Zero fields take src/api.cpp:47-57 defaults; spin <= 0 with KERR -> 0.998."""
    vals = dict(width=8, height=8, metric_type=1, mass=0.0, spin=0.0, observer_r=0.0, observer_theta=0.0,
                fov=0.0, disk_enabled=1, integrator_tolerance=0.0, integrator_max_steps=0, samples_per_pixel=0)
    R = grrt.Renderer(vals)
    M, a, r_h, isco, r_obs, tol, max_steps, spp = R.table("scalars")
    assert (M, a, r_obs, tol, max_steps, spp) == (1.0, 0.998, 50.0, 1e-8, 10000, 1)
    cam = R.table("camera")
    assert cam[2] == 1.396 and cam[36] == 1.047
    meta = R.table("flux_meta")
    assert meta[1] == isco and meta[2] == 20.0 and meta[3] == 1e7
    # Schwarzschild metric ignores the spin parameter
    R2 = grrt.Renderer(dict(vals, metric_type=0, spin=0.5))
    assert R2.table("scalars")[1] == 0.0
    assert R2.table("scalars")[2] == 2.0 and R2.table("scalars")[3] == 6.0


def test_error_conventions_without_render(grrt):
    R = grrt.Renderer(grrt.config_params(1, width=16, height=16))
    L = grrt.lib()
    assert L.grrt_set_precision(R.ctx, 7) == -1
    assert b"unknown form" in L.grrt_error(R.ctx)
    assert L.grrt_scene_table(R.ctx, b"no_such_table", None, 0) == -1
    assert L.grrt_scene_table(R.ctx, b"vol_H", None, 0) == -1  # thin disk: no volumetric tables
    buf = np.zeros(16 * 16 * 4)
    # spectral render without bins: -1 and the reference's message, before any device work
    rc = L.grrt_render_spectral(R.ctx, buf.ctypes.data_as(C.POINTER(C.c_double)), 16, 16)
    assert rc == -1
    assert L.grrt_error(R.ctx).decode() == "No frequency bins set -- call grrt_set_frequency_bins first"
    # FITS path checks
    L.grrt_set_frequency_bins(R.ctx, np.array([1e14, 1e15]).ctypes.data_as(C.POINTER(C.c_double)), 2)
    rc = L.grrt_render_spectral_to_fits_cb(R.ctx, b"", 16, 16, grrt.PROGRESS_FN(0), None)
    assert rc == -1 and b"output_path" in L.grrt_error(R.ctx)
    assert L.grrt_progress(R.ctx) == 0.0


def test_render_without_gpu_fails_loudly(grrt):
    if grrt.cuda_available():
        pytest.skip("a GPU is present")
    R = grrt.Renderer(grrt.config_params(1, width=8, height=8))
    with pytest.raises(RuntimeError, match="no CUDA device"):
        R.render()


def test_tonemap_matches_reference_algorithm(grrt):
    """grrt_tonemap (host post-process) against a restatement of src/tonemapper.cpp:7-71."""
    rng = np.random.default_rng(3)
    fb = rng.lognormal(0.0, 2.0, size=(12, 9, 4)).astype(np.float32)
    fb[0, 0, :3] = 0.0
    want = fb.astype(np.float64).copy()
    rgb = np.maximum(want[..., :3], 0.0)
    L = 0.2126 * rgb[..., 0] + 0.7152 * rgb[..., 1] + 0.0722 * rgb[..., 2]
    lit = L > 1e-10
    L_avg = np.exp(np.sum(np.log(1e-6 + L[lit])) / lit.sum())
    exposure = 0.18 / L_avg
    Lw2 = (L.max() * exposure) ** 2
    Ls = L * exposure
    Lm = np.clip(Ls * (1 + Ls / Lw2) / (1 + Ls), 0, 1)
    scale = np.where(L > 0, Lm / np.where(L > 0, L, 1), 0)
    out = np.clip(rgb * scale[..., None], 0, 1) ** (1 / 2.2)
    got = fb.copy()
    grrt.lib().grrt_tonemap(got.ctypes.data_as(C.POINTER(C.c_float)), 9, 12)
    np.testing.assert_allclose(got[..., :3], out.astype(np.float32), rtol=1e-6, atol=1e-7)
