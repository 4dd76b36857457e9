"""grrt_b200 — Python binding of libgrrt.so, the B200-native GRRT renderer.

The library exports the reference's pure C API unchanged (include/grrt_api.h:
grrt_create / grrt_render* / grrt_destroy, GRRTParams) plus additive entry
points (include/grrt_b200.h). This module binds both with ctypes so Python
callers (tests, bench.py) use exactly the C ABI a C/C++ host would.

Every render runs on the GPU through the sm_100a kernels in
grrt_b200/csrc/device; there is no CPU fallback. Importing this module fails
loudly if the shared library has not been built.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

__all__ = [
    "GRRTParams", "GRRTStats", "Renderer", "lib", "load_library", "build",
    "FORM_FP64", "FORM_MIXED", "config_params", "LIB_PATH", "Surrogate", "multi",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libgrrt.so")

FORM_FP64 = 0
FORM_MIXED = 1
DIAG_HAMILTONIAN = 1

METRIC_SCHWARZSCHILD = 0
METRIC_KERR = 1
BG_BLACK = 0
BG_STARS = 1
BG_TEXTURE = 2


DEBUG_START, DEBUG_STEP, DEBUG_THIN_HIT, DEBUG_MARCH_ENTRY, DEBUG_MARCH_EXIT, DEBUG_END = range(6)
DEBUG_EVENT_NONE, DEBUG_EVENT_CROSS, DEBUG_EVENT_INSIDE, DEBUG_EVENT_NEAR = range(4)


class GRRTDebugRecord(C.Structure):
    """Mirror of GRRTDebugRecord (include/grrt_b200.h)."""

    _fields_ = [("kind", C.c_int), ("step", C.c_int), ("event", C.c_int), ("aux", C.c_int),
                ("v", C.c_double * 7)]


class GRRTParams(C.Structure):
    """Mirror of GRRTParams (include/grrt/types.h:20-64, include/grrt_api.h)."""

    _fields_ = [
        ("width", C.c_int), ("height", C.c_int),
        ("metric_type", C.c_int), ("mass", C.c_double), ("spin", C.c_double),
        ("observer_r", C.c_double), ("observer_theta", C.c_double), ("observer_phi", C.c_double),
        ("fov", C.c_double),
        ("cam_yaw", C.c_double), ("cam_pitch", C.c_double), ("cam_roll", C.c_double),
        ("disk_enabled", C.c_int), ("disk_inner", C.c_double), ("disk_outer", C.c_double),
        ("disk_temperature", C.c_double),
        ("disk_volumetric", C.c_int), ("disk_alpha", C.c_double), ("disk_turbulence", C.c_double),
        ("disk_seed", C.c_int), ("disk_noise_scale", C.c_double), ("disk_noise_octaves", C.c_int),
        ("mass_solar", C.c_double), ("eddington_fraction", C.c_double),
        ("background_type", C.c_int), ("background_texture_path", C.c_char_p),
        ("integrator_tolerance", C.c_double), ("integrator_max_steps", C.c_int),
        ("samples_per_pixel", C.c_int), ("thread_count", C.c_int), ("backend", C.c_int),
        ("num_frequency_bins", C.c_int), ("frequency_bins_hz", C.POINTER(C.c_double)),
    ]


class GRRTStats(C.Structure):
    """Mirror of GRRTStats (include/grrt_b200.h)."""

    _fields_ = [
        ("attempts", C.c_ulonglong), ("accepted", C.c_ulonglong), ("crossings", C.c_ulonglong),
        ("rays", C.c_ulonglong), ("horizon", C.c_ulonglong), ("escaped", C.c_ulonglong),
        ("max_steps", C.c_ulonglong), ("clamp_evals", C.c_ulonglong), ("march_steps", C.c_ulonglong),
        ("physics_steps", C.c_ulonglong), ("bin_updates", C.c_ulonglong),
        ("fp64_attempts", C.c_ulonglong), ("kernel_ms", C.c_double), ("hamiltonian_max", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


PROGRESS_FN = C.CFUNCTYPE(None, C.c_float, C.c_void_p)

_lib: Optional[C.CDLL] = None


def build(jobs: int = 8) -> None:
    """Compile libgrrt.so in-tree (host C++ and sm_100a CUDA)."""
    import subprocess
    subprocess.run(["make", "-j", str(jobs)], cwd=os.path.join(_HERE, "csrc"), check=True,
                   stdout=subprocess.DEVNULL)


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load libgrrt.so and declare every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libgrrt.so not built ({path}); run grrt_b200.build() or make -C grrt_b200/csrc")
    L = C.CDLL(path)
    P = C.POINTER
    vp = C.c_void_p
    sig = {
        "grrt_create": (vp, [P(GRRTParams)]),
        "grrt_destroy": (None, [vp]),
        "grrt_update_params": (None, [vp, P(GRRTParams)]),
        "grrt_render": (C.c_int, [vp, P(C.c_float)]),
        "grrt_render_cb": (C.c_int, [vp, P(C.c_float), PROGRESS_FN, vp]),
        "grrt_render_tile": (C.c_int, [vp, P(C.c_float), C.c_int, C.c_int, C.c_int, C.c_int]),
        "grrt_cancel": (None, [vp]),
        "grrt_progress": (C.c_float, [vp]),
        "grrt_error": (C.c_char_p, [vp]),
        "grrt_cuda_available": (C.c_int, []),
        "grrt_last_error": (C.c_char_p, []),
        "grrt_tonemap": (None, [P(C.c_float), C.c_int, C.c_int]),
        "grrt_debug_pixel": (None, [vp, C.c_int, C.c_int]),
        "grrt_set_frequency_bins": (None, [vp, P(C.c_double), C.c_int]),
        "grrt_render_spectral": (C.c_int, [vp, P(C.c_double), C.c_int, C.c_int]),
        "grrt_render_spectral_cb": (C.c_int, [vp, P(C.c_double), C.c_int, C.c_int, PROGRESS_FN, vp]),
        "grrt_render_spectral_to_fits_cb": (C.c_int, [vp, C.c_char_p, C.c_int, C.c_int, PROGRESS_FN, vp]),
        "grrt_set_precision": (C.c_int, [vp, C.c_int]),
        "grrt_set_diagnostics": (C.c_int, [vp, C.c_int]),
        "grrt_get_precision": (C.c_int, [vp]),
        "grrt_set_mixed_params": (C.c_int, [vp, C.c_double, C.c_double]),
        "grrt_render_device": (C.c_int, [vp, vp, vp, vp, vp]),
        "grrt_render_rows_device": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp]),
        "grrt_tonemap_device": (C.c_int, [vp, C.c_int, C.c_int, vp]),
        "grrt_render_spectral_device": (C.c_int, [vp, vp, C.c_int, C.c_int, vp, vp]),
        "grrt_render_spectral_rows_device": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, vp, vp, vp]),
        "grrt_render_spectral_tile_device": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp]),
        "grrt_render_spectral_device_noalloc": (C.c_int, [vp, vp, C.c_int, vp, C.c_int, C.c_int, vp]),
        "grrt_get_stats": (C.c_int, [vp, P(GRRTStats)]),
        "grrt_get_phase_ms": (C.c_int, [vp, P(C.c_double), C.c_int]),
        "grrt_surrogate_create": (vp, [C.c_uint]),
        "grrt_surrogate_destroy": (None, [vp]),
        "grrt_surrogate_error": (C.c_char_p, [vp]),
        "grrt_surrogate_generate": (C.c_int, [vp, vp, C.c_int, C.c_int]),
        "grrt_surrogate_dataset": (C.c_longlong, [vp, P(C.c_float), P(C.c_float), C.c_longlong]),
        "grrt_surrogate_train": (C.c_int, [vp, C.c_int, C.c_int, C.c_double, P(C.c_float)]),
        "grrt_surrogate_calibrate": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_double, C.c_double, P(C.c_double)]),
        "grrt_surrogate_set_bands": (C.c_int, [vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]),
        "grrt_surrogate_get_bands": (C.c_int, [vp, P(C.c_double)]),
        "grrt_surrogate_params": (C.c_longlong, [vp, P(C.c_float), C.c_longlong]),
        "grrt_surrogate_set_params": (C.c_int, [vp, P(C.c_float), C.c_longlong]),
        "grrt_surrogate_forward": (C.c_int, [vp, vp, C.c_longlong, vp]),
        "grrt_surrogate_gradients": (C.c_int, [vp, P(C.c_float), P(C.c_float), C.c_int, P(C.c_float),
                                               P(C.c_double)]),
        "grrt_surrogate_render_device": (C.c_int, [vp, vp, vp, vp, vp, vp]),
        "grrt_surrogate_render": (C.c_int, [vp, vp, P(C.c_float)]),
        "grrt_surrogate_last_exact": (C.c_int, [vp, P(C.c_longlong), P(C.c_longlong)]),
        "grrt_surrogate_last_counts": (C.c_int, [vp, P(C.c_longlong), P(C.c_longlong), P(C.c_longlong),
                                                 P(C.c_longlong)]),
        "grrt_surrogate_save": (C.c_int, [vp, C.c_char_p]),
        "grrt_surrogate_load": (C.c_int, [vp, C.c_char_p]),
        "grrt_surrogate_gemm_bf16": (C.c_int, [vp, C.c_int, vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp,
                                               C.c_int, C.c_int, vp, C.c_int, vp, C.c_int, vp]),
        "grrt_batch_create": (vp, [P(GRRTParams), C.c_int]),
        "grrt_batch_destroy": (None, [vp]),
        "grrt_batch_error": (C.c_char_p, [vp]),
        "grrt_batch_set_precision": (C.c_int, [vp, C.c_int]),
        "grrt_batch_set_schedule": (C.c_int, [vp, C.c_int, C.c_int, C.c_int]),
        "grrt_batch_get_schedule": (C.c_int, [vp, P(C.c_int), P(C.c_int), P(C.c_int)]),
        "grrt_batch_autotune": (C.c_int, [vp, C.c_char_p, P(C.c_double)]),
        "grrt_batch_render": (C.c_int, [vp, P(P(C.c_float))]),
        "grrt_batch_render_device": (C.c_int, [vp, vp, vp]),
        "grrt_batch_get_stats": (C.c_int, [vp, P(GRRTStats)]),
        "grrt_batch_set_frequency_bins": (C.c_int, [vp, C.c_int, P(C.c_double), C.c_int]),
        "grrt_batch_set_tuning": (C.c_int, [vp, C.c_int, C.c_double, C.c_double]),
        "grrt_batch_get_tuning": (C.c_int, [vp, P(C.c_int), P(C.c_double), P(C.c_double)]),
        "grrt_batch_spectral_offset": (C.c_longlong, [vp, C.c_int]),
        "grrt_batch_render_spectral_device": (C.c_int, [vp, vp, vp]),
        "grrt_batch_render_spectral": (C.c_int, [vp, P(P(C.c_double))]),
        "grrt_scene_table": (C.c_longlong, [vp, C.c_char_p, P(C.c_double), C.c_longlong]),
        "grrt_camera_ray": (C.c_int, [vp, C.c_double, C.c_double, P(C.c_double)]),
        "grrt_debug_trace": (C.c_int, [vp, C.c_double, C.c_double, P(GRRTDebugRecord), C.c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def lib() -> C.CDLL:
    return load_library()


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def config_params(config: int = 1, *, width: Optional[int] = None, height: Optional[int] = None,
                  spp: Optional[int] = None, **overrides) -> dict:
    """GRRTParams field values of the benchmark scenes.

    1: Schwarzschild (M=1) 256x256, 1 spp, thin disk ISCO..20, black background.
    2: Kerr a=0.998 1024x1024, 4 spp, thin disk ISCO..20, stars (seed 42).
    3: volumetric Kerr a=0.9 512x512, 1 spp, alpha 0.1, turbulence 0.4, 2 octaves,
       seed 42, outer 20, M=10 M_sun at 0.1 Eddington; 32 log-spaced bins 1e14..1e18 Hz.
    Observer r=50, theta=80 deg, phi=0, FOV 90 deg, tolerance 1e-8, 10000 steps.
    """
    p = dict(width=256, height=256, metric_type=METRIC_KERR, mass=1.0, spin=0.998, observer_r=50.0,
             observer_theta=math.radians(80.0), observer_phi=0.0, fov=math.radians(90.0),
             disk_enabled=1, disk_inner=0.0, disk_outer=20.0, disk_temperature=0.0, disk_volumetric=0,
             disk_alpha=0.1, disk_turbulence=0.4, disk_seed=42, disk_noise_scale=0.0,
             disk_noise_octaves=2, mass_solar=0.0, eddington_fraction=0.0, background_type=BG_STARS,
             integrator_tolerance=1e-8, integrator_max_steps=10000, samples_per_pixel=1)
    if config == 1:
        p.update(metric_type=METRIC_SCHWARZSCHILD, spin=0.0, background_type=BG_BLACK)
    elif config == 2:
        p.update(width=1024, height=1024, samples_per_pixel=4)
    elif config == 3:
        p.update(width=512, height=512, spin=0.9, disk_volumetric=1, mass_solar=10.0,
                 eddington_fraction=0.1, background_type=BG_BLACK)
    else:
        raise ValueError(f"unknown config {config}")
    if width is not None:
        p["width"] = width
    if height is not None:
        p["height"] = height
    if spp is not None:
        p["samples_per_pixel"] = spp
    p.update(overrides)
    return p


def log_bins(lo: float = 1e14, hi: float = 1e18, n: int = 32) -> np.ndarray:
    """n log-spaced frequencies in [lo, hi] (the CLI's --freq-range)."""
    if n == 1:
        return np.array([lo], dtype=np.float64)
    llo, lhi = math.log10(lo), math.log10(hi)
    return np.array([10.0 ** (llo + (lhi - llo) * i / (n - 1)) for i in range(n)], dtype=np.float64)


def make_params(values: dict, freqs: Optional[np.ndarray] = None) -> GRRTParams:
    p = GRRTParams()
    for k, v in values.items():
        if k in ("frequency_bins_hz", "num_frequency_bins"):
            continue
        setattr(p, k, v)
    if freqs is not None:
        p.num_frequency_bins = len(freqs)
        p.frequency_bins_hz = _dptr(freqs)
    return p


class Renderer:
    """One GRRT context (grrt_create ... grrt_destroy)."""

    def __init__(self, values: Optional[dict] = None, freqs: Optional[Sequence[float]] = None, **kw):
        self._L = lib()
        vals = dict(values or {})
        vals.update(kw)
        self.values = vals
        self.freqs = None if freqs is None else np.ascontiguousarray(freqs, dtype=np.float64)
        params = make_params(vals, self.freqs)
        self.ctx = self._L.grrt_create(C.byref(params))
        if not self.ctx:
            err = self._L.grrt_last_error()
            raise RuntimeError("grrt_create failed: " + (err.decode() if err else "unknown"))
        if self.freqs is not None:
            self._L.grrt_set_frequency_bins(self.ctx, _dptr(self.freqs), len(self.freqs))
        self.width = vals.get("width", 0)
        self.height = vals.get("height", 0)

    def close(self) -> None:
        if getattr(self, "ctx", None):
            self._L.grrt_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            err = self._L.grrt_error(self.ctx)
            raise RuntimeError(f"{what} failed: " + (err.decode() if err else f"rc={rc}"))

    # --- reference API ---------------------------------------------------
    def render(self) -> np.ndarray:
        fb = np.empty((self.height, self.width, 4), dtype=np.float32)
        self._check(self._L.grrt_render(self.ctx, fb.ctypes.data_as(C.POINTER(C.c_float))), "grrt_render")
        return fb

    def render_tile(self, x: int, y: int, w: int, h: int) -> np.ndarray:
        fb = np.empty((h, w, 4), dtype=np.float32)
        self._check(self._L.grrt_render_tile(self.ctx, fb.ctypes.data_as(C.POINTER(C.c_float)), x, y, w, h),
                    "grrt_render_tile")
        return fb

    def render_spectral(self, width: Optional[int] = None, height: Optional[int] = None) -> np.ndarray:
        w = width or self.width
        h = height or self.height
        nb = 0 if self.freqs is None else len(self.freqs)
        out = np.empty((h, w, max(nb, 1)), dtype=np.float64)
        self._check(self._L.grrt_render_spectral(self.ctx, _dptr(out), w, h), "grrt_render_spectral")
        return out

    def render_fits(self, path: str, width: Optional[int] = None, height: Optional[int] = None) -> None:
        w = width or self.width
        h = height or self.height
        self._check(self._L.grrt_render_spectral_to_fits_cb(self.ctx, path.encode(), w, h, PROGRESS_FN(0), None),
                    "grrt_render_spectral_to_fits_cb")

    # --- additive API ----------------------------------------------------
    def set_precision(self, form: int) -> None:
        self._check(self._L.grrt_set_precision(self.ctx, form), "grrt_set_precision")

    def set_diagnostics(self, flags: int) -> None:
        self._check(self._L.grrt_set_diagnostics(self.ctx, flags), "grrt_set_diagnostics")

    def set_mixed_params(self, r_factor: float, tol_fp32: float) -> None:
        self._check(self._L.grrt_set_mixed_params(self.ctx, r_factor, tol_fp32), "grrt_set_mixed_params")

    def render_device(self, d_rgba=None, d_rgb64=None, d_fate=None, stream=None) -> None:
        """Render into device buffers given as raw pointers (int) or torch tensors."""
        def ptr(x):
            if x is None:
                return None
            return x if isinstance(x, int) else x.data_ptr()
        s = stream if (stream is None or isinstance(stream, int)) else stream.cuda_stream
        self._check(self._L.grrt_render_device(self.ctx, ptr(d_rgba), ptr(d_rgb64), ptr(d_fate), s),
                    "grrt_render_device")

    def render_rows_device(self, row0: int, row_step: int, n_rows: int, d_rgba=None, d_rgb64=None, d_fate=None,
                           stream=None) -> None:
        """Render image rows row0, row0 + row_step, ... (n_rows, full width) densely into device buffers."""
        def ptr(x):
            if x is None:
                return None
            return x if isinstance(x, int) else x.data_ptr()
        s = stream if (stream is None or isinstance(stream, int)) else stream.cuda_stream
        self._check(self._L.grrt_render_rows_device(self.ctx, row0, row_step, n_rows, ptr(d_rgba), ptr(d_rgb64),
                                                    ptr(d_fate), s), "grrt_render_rows_device")

    def render_spectral_device(self, d_spec, width: int, height: int, d_fate=None, stream=None) -> None:
        def ptr(x):
            if x is None:
                return None
            return x if isinstance(x, int) else x.data_ptr()
        s = stream if (stream is None or isinstance(stream, int)) else stream.cuda_stream
        self._check(self._L.grrt_render_spectral_device(self.ctx, ptr(d_spec), width, height, ptr(d_fate), s),
                    "grrt_render_spectral_device")

    def render_spectral_rows_device(self, row0: int, row_step: int, n_rows: int, d_spec, d_fate=None,
                                    stream=None) -> None:
        """Spectral render of image rows row0, row0 + row_step, ... (n_rows, full width) into device buffers."""
        def ptr(x):
            if x is None:
                return None
            return x if isinstance(x, int) else x.data_ptr()
        s = stream if (stream is None or isinstance(stream, int)) else stream.cuda_stream
        self._check(self._L.grrt_render_spectral_rows_device(self.ctx, row0, row_step, n_rows, ptr(d_spec),
                                                             ptr(d_fate), s), "grrt_render_spectral_rows_device")

    def render_spectral_tile_device(self, x: int, y: int, w: int, h: int, d_spec, d_fate=None, stream=None) -> None:
        """Spectral render of the w x h tile at image pixel (x, y) into device buffers."""
        def ptr(v):
            if v is None:
                return None
            return v if isinstance(v, int) else v.data_ptr()
        s = stream if (stream is None or isinstance(stream, int)) else stream.cuda_stream
        self._check(self._L.grrt_render_spectral_tile_device(self.ctx, x, y, w, h, ptr(d_spec), ptr(d_fate), s),
                    "grrt_render_spectral_tile_device")

    def render_spectral_device_noalloc(self, d_freqs, nb: int, d_spec, width: int, height: int,
                                       stream=None) -> None:
        """The spectral render that allocates no device memory (fixed in-library scratch)."""
        fp = d_freqs if isinstance(d_freqs, int) else d_freqs.data_ptr()
        sp = d_spec if isinstance(d_spec, int) else d_spec.data_ptr()
        s = stream if (stream is None or isinstance(stream, int)) else stream.cuda_stream
        self._check(self._L.grrt_render_spectral_device_noalloc(self.ctx, fp, nb, sp, width, height, s),
                    "grrt_render_spectral_device_noalloc")

    def stats(self) -> dict:
        st = GRRTStats()
        self._check(self._L.grrt_get_stats(self.ctx, C.byref(st)), "grrt_get_stats")
        return st.as_dict()

    def phase_ms(self) -> list:
        """Device time of each kernel phase of the last render (ms)."""
        out = np.zeros(8, dtype=np.float64)
        n = self._L.grrt_get_phase_ms(self.ctx, _dptr(out), 8)
        if n < 0:
            err = self._L.grrt_error(self.ctx)
            raise RuntimeError("grrt_get_phase_ms failed: " + (err.decode() if err else f"rc={n}"))
        return [float(x) for x in out[:n]]

    def table(self, name: str) -> np.ndarray:
        n = self._L.grrt_scene_table(self.ctx, name.encode(), None, 0)
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, dtype=np.float64)
        self._L.grrt_scene_table(self.ctx, name.encode(), _dptr(out), n)
        return out

    def camera_ray(self, x: float, y: float) -> np.ndarray:
        out = np.empty(8, dtype=np.float64)
        self._L.grrt_camera_ray(self.ctx, x, y, _dptr(out))
        return out

    def debug_trace(self, x: float, y: float, capacity: Optional[int] = None) -> list:
        """The FP64 device trace of the sample at fractional pixel (x, y) as
        records (grrt_debug_trace): dicts with kind, step, event, aux and v."""
        if capacity is None:
            n = self._L.grrt_debug_trace(self.ctx, x, y, None, 0)
            if n < 0:
                err = self._L.grrt_error(self.ctx)
                raise RuntimeError("grrt_debug_trace failed: " + (err.decode() if err else f"rc={n}"))
            capacity = n
        buf = (GRRTDebugRecord * max(1, capacity))()
        n = self._L.grrt_debug_trace(self.ctx, x, y, buf, capacity)
        if n < 0:
            err = self._L.grrt_error(self.ctx)
            raise RuntimeError("grrt_debug_trace failed: " + (err.decode() if err else f"rc={n}"))
        return [{"kind": r.kind, "step": r.step, "event": r.event, "aux": r.aux, "v": list(r.v)}
                for r in buf[:min(n, capacity)]]

    def debug_pixel(self, px: int, py: int) -> None:
        """Print the pixel centre's trace (grrt_debug_pixel) to the process's stdout."""
        self._L.grrt_debug_pixel(self.ctx, px, py)


class Batch:
    """Many cameras rendered by one persistent launch (grrt_batch_*): thin-disk
    cameras (RGB) or volumetric cameras (spectra, each with its own bins)."""

    ORDER_CAMERA_MAJOR = 0
    ORDER_ROUND_ROBIN = 1
    ORDER_SAMPLES = 2  # FP64 thin-disk batches: traced by samples (chunk size and block size do not apply)

    def __init__(self, cameras: Sequence[dict], freqs: Optional[Sequence] = None):
        """freqs: per camera, the bins (Hz) of a volumetric camera or None. As
        for a Renderer, they widen the camera's opacity tables at creation and
        become its render bins."""
        self._L = lib()
        self.cameras = [dict(c) for c in cameras]
        fl = [None if (freqs is None or f is None) else np.ascontiguousarray(f, dtype=np.float64)
              for f in (freqs if freqs is not None else [None] * len(cameras))]
        arr = (GRRTParams * len(cameras))()
        for i, c in enumerate(cameras):
            arr[i] = make_params(c, fl[i])
        self.b = self._L.grrt_batch_create(arr, len(cameras))
        if not self.b:
            err = self._L.grrt_batch_error(None)
            raise RuntimeError("grrt_batch_create failed: " + (err.decode() if err else "unknown"))
        self.sizes = [(c["width"], c["height"]) for c in cameras]
        self.offsets = np.cumsum([0] + [w * h for w, h in self.sizes])
        for i, f in enumerate(fl):
            if f is not None:
                self.set_frequency_bins(f, i)

    def close(self) -> None:
        if getattr(self, "b", None):
            self._L.grrt_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            err = self._L.grrt_batch_error(self.b)
            raise RuntimeError(f"{what} failed: " + (err.decode() if err else f"rc={rc}"))

    def set_precision(self, form: int) -> None:
        self._check(self._L.grrt_batch_set_precision(self.b, form), "grrt_batch_set_precision")

    def set_frequency_bins(self, freqs, camera: int = -1) -> None:
        """Bins (Hz) of one camera, or of every camera (camera = -1)."""
        f = np.ascontiguousarray(freqs, dtype=np.float64)
        self._check(self._L.grrt_batch_set_frequency_bins(self.b, camera, _dptr(f), len(f)),
                    "grrt_batch_set_frequency_bins")

    def set_tuning(self, block: int = 128, tol_fp32: float = 3e-6, r_factor: float = 3.0) -> None:
        self._check(self._L.grrt_batch_set_tuning(self.b, block, tol_fp32, r_factor), "grrt_batch_set_tuning")

    def tuning(self) -> dict:
        a, t, r = C.c_int(), C.c_double(), C.c_double()
        self._L.grrt_batch_get_tuning(self.b, C.byref(a), C.byref(t), C.byref(r))
        return {"block": a.value, "tol_fp32": t.value, "r_factor": r.value}

    def spectral_offset(self, camera: int) -> int:
        """Element offset of camera's cube in the batch's spectral output (camera = count: total size)."""
        return int(self._L.grrt_batch_spectral_offset(self.b, camera))

    def render_spectral_device(self, d_spec, stream=None) -> None:
        p = d_spec if isinstance(d_spec, int) else d_spec.data_ptr()
        s = stream if (stream is None or isinstance(stream, int)) else stream.cuda_stream
        self._check(self._L.grrt_batch_render_spectral_device(self.b, p, s), "grrt_batch_render_spectral_device")

    def render_spectral(self) -> list:
        n = len(self.cameras)
        sizes = [self.spectral_offset(i + 1) - self.spectral_offset(i) for i in range(n)]
        cubes = [np.empty(k, dtype=np.float64) for k in sizes]
        ptrs = (C.POINTER(C.c_double) * n)(*[_dptr(c) for c in cubes])
        self._check(self._L.grrt_batch_render_spectral(self.b, ptrs), "grrt_batch_render_spectral")
        return [c.reshape(h, w, -1) for c, (w, h) in zip(cubes, self.sizes)]

    def set_schedule(self, chunk: int, order: int, blocks_per_sm: int = 0) -> None:
        self._check(self._L.grrt_batch_set_schedule(self.b, chunk, order, blocks_per_sm), "grrt_batch_set_schedule")

    def schedule(self) -> tuple:
        a, b_, c = C.c_int(), C.c_int(), C.c_int()
        self._L.grrt_batch_get_schedule(self.b, C.byref(a), C.byref(b_), C.byref(c))
        return a.value, b_.value, c.value

    def autotune(self, cache_path: Optional[str] = None) -> float:
        ms = C.c_double()
        self._check(self._L.grrt_batch_autotune(self.b, cache_path.encode() if cache_path else None, C.byref(ms)),
                    "grrt_batch_autotune")
        return ms.value

    def render(self) -> list:
        fbs = [np.empty((h, w, 4), dtype=np.float32) for w, h in self.sizes]
        ptrs = (C.POINTER(C.c_float) * len(fbs))(*[f.ctypes.data_as(C.POINTER(C.c_float)) for f in fbs])
        self._check(self._L.grrt_batch_render(self.b, ptrs), "grrt_batch_render")
        return fbs

    def render_device(self, d_rgba, stream=None) -> None:
        p = d_rgba if isinstance(d_rgba, int) else d_rgba.data_ptr()
        s = stream if (stream is None or isinstance(stream, int)) else stream.cuda_stream
        self._check(self._L.grrt_batch_render_device(self.b, p, s), "grrt_batch_render_device")

    def stats(self) -> dict:
        st = GRRTStats()
        self._check(self._L.grrt_batch_get_stats(self.b, C.byref(st)), "grrt_batch_get_stats")
        return st.as_dict()


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Surrogate:
    """The learned surrogate (include/grrt_surrogate.h): MLP 4 -> 256 x 4 -> 6,
    trained on the GPU by the library's tensor-core kernels."""

    N_PARAMS = 256 * 4 + 256 + 3 * (256 * 256 + 256) + 16 * 256 + 16
    Y_COLS = 10

    def __init__(self, seed: int = 0):
        self._L = lib()
        self.s = self._L.grrt_surrogate_create(seed)
        if not self.s:
            err = self._L.grrt_surrogate_error(None)
            raise RuntimeError("grrt_surrogate_create failed: " + (err.decode() if err else "unknown"))

    def close(self) -> None:
        if getattr(self, "s", None):
            self._L.grrt_surrogate_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            err = self._L.grrt_surrogate_error(self.s)
            raise RuntimeError(f"{what} failed: " + (err.decode() if err else f"rc={rc}"))

    @staticmethod
    def _cams(cameras: Sequence[dict]):
        arr = (GRRTParams * len(cameras))()
        for i, c in enumerate(cameras):
            arr[i] = make_params(c)
        return arr

    def generate(self, cameras: Sequence[dict], n_side: int) -> None:
        arr = self._cams(cameras)
        self._check(self._L.grrt_surrogate_generate(self.s, arr, len(cameras), n_side), "grrt_surrogate_generate")

    def dataset(self):
        n = self._L.grrt_surrogate_dataset(self.s, None, None, 0)
        X = np.empty((n, 4), dtype=np.float32)
        Y = np.empty((n, self.Y_COLS), dtype=np.float32)
        if n:
            self._L.grrt_surrogate_dataset(self.s, _fptr(X), _fptr(Y), n)
        return X, Y

    def train(self, steps: int, batch: int = 16384, lr: float = 1e-3) -> np.ndarray:
        hist = np.empty(steps, dtype=np.float32)
        self._check(self._L.grrt_surrogate_train(self.s, steps, batch, lr, _fptr(hist)), "grrt_surrogate_train")
        return hist

    def calibrate(self, cameras: Sequence[dict], n_side: int, quantile: float = 0.999, safety: float = 1.5) -> dict:
        arr = self._cams(cameras)
        rep = np.zeros(8)
        self._check(self._L.grrt_surrogate_calibrate(self.s, arr, len(cameras), n_side, quantile, safety, _dptr(rep)),
                    "grrt_surrogate_calibrate")
        keys = ["du", "dir", "capture", "graze", "samples", "fate_disagreements", "band_fraction", "median_du"]
        return dict(zip(keys, rep.tolist()))

    def set_bands(self, du: float, dir: float, capture: float, graze: float, tol_rel: float = 1e-3) -> None:
        self._check(self._L.grrt_surrogate_set_bands(self.s, du, dir, capture, graze, tol_rel),
                    "grrt_surrogate_set_bands")

    def bands(self) -> dict:
        out = np.zeros(5)
        self._L.grrt_surrogate_get_bands(self.s, _dptr(out))
        return dict(zip(["du", "dir", "capture", "graze", "tol_rel"], out.tolist()))

    def params(self) -> np.ndarray:
        p = np.empty(self.N_PARAMS, dtype=np.float32)
        n = self._L.grrt_surrogate_params(self.s, _fptr(p), self.N_PARAMS)
        assert n == self.N_PARAMS
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._check(self._L.grrt_surrogate_set_params(self.s, _fptr(p), len(p)), "grrt_surrogate_set_params")

    def forward(self, d_in, d_out, n: int) -> None:
        """Device pointers (int) or torch tensors: inputs float[n][4] -> outputs float[n][16]."""
        pi = d_in if isinstance(d_in, int) else d_in.data_ptr()
        po = d_out if isinstance(d_out, int) else d_out.data_ptr()
        self._check(self._L.grrt_surrogate_forward(self.s, pi, n, po), "grrt_surrogate_forward")

    def gradients(self, X: np.ndarray, Y: np.ndarray):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        g = np.empty(self.N_PARAMS, dtype=np.float32)
        loss = C.c_double()
        self._check(self._L.grrt_surrogate_gradients(self.s, _fptr(X), _fptr(Y), len(X), _fptr(g), C.byref(loss)),
                    "grrt_surrogate_gradients")
        return loss.value, g

    def render_device(self, R: "Renderer", d_rgba=None, d_rgb64=None, d_fate=None, stream=None) -> None:
        def ptr(x):
            if x is None:
                return None
            return x if isinstance(x, int) else x.data_ptr()
        s = stream if (stream is None or isinstance(stream, int)) else stream.cuda_stream
        rc = self._L.grrt_surrogate_render_device(self.s, R.ctx, ptr(d_rgba), ptr(d_rgb64), ptr(d_fate), s)
        self._check(rc, "grrt_surrogate_render_device")

    def render(self, R: "Renderer") -> np.ndarray:
        fb = np.empty((R.height, R.width, 4), dtype=np.float32)
        self._check(self._L.grrt_surrogate_render(self.s, R.ctx, _fptr(fb)), "grrt_surrogate_render")
        return fb

    def last_exact(self):
        e, n = C.c_longlong(), C.c_longlong()
        self._L.grrt_surrogate_last_exact(self.s, C.byref(e), C.byref(n))
        return e.value, n.value

    def last_counts(self) -> dict:
        """Samples of the last render: re-traced exactly, sent to the FP32 speculation,
        evaluated by the network (the rest settled in closed form), total."""
        e, sp, nw, n = C.c_longlong(), C.c_longlong(), C.c_longlong(), C.c_longlong()
        self._check(self._L.grrt_surrogate_last_counts(self.s, C.byref(e), C.byref(sp), C.byref(nw), C.byref(n)),
                    "grrt_surrogate_last_counts")
        return {"exact": e.value, "speculated": sp.value, "network": nw.value, "samples": n.value}

    def save(self, path: str) -> None:
        self._check(self._L.grrt_surrogate_save(self.s, path.encode()), "grrt_surrogate_save")

    def load(self, path: str) -> None:
        self._check(self._L.grrt_surrogate_load(self.s, path.encode()), "grrt_surrogate_load")


def sweep_cameras(width: int = 256, height: int = 256, spins=(0.0, 0.5, 0.9, 0.998), n_incl: int = 16,
                  incl_lo_deg: float = 5.0, incl_hi_deg: float = 90.0) -> list:
    """The batched benchmark sweep: spins x evenly spaced inclinations, thin disk
    ISCO..20 M, stars seed 42, tolerance 1e-8. Spin 0 uses the Schwarzschild
    metric (with GRRT_METRIC_KERR a spin of 0 selects 0.998)."""
    cams = []
    for spin in spins:
        for k in range(n_incl):
            th = incl_lo_deg + k * (incl_hi_deg - incl_lo_deg) / (n_incl - 1)
            p = config_params(2, width=width, height=height, spp=1, observer_theta=math.radians(th))
            if spin == 0.0:
                p.update(metric_type=METRIC_SCHWARZSCHILD, spin=0.0)
            else:
                p.update(spin=spin)
            cams.append(p)
    return cams


def tonemap_device(d_rgba, width: int, height: int, stream=None) -> None:
    """In-place tone mapping of a device RGBA float frame (raw pointer or torch tensor)."""
    p = d_rgba if isinstance(d_rgba, int) else d_rgba.data_ptr()
    s = stream if (stream is None or isinstance(stream, int)) else stream.cuda_stream
    if lib().grrt_tonemap_device(p, width, height, s) != 0:
        raise RuntimeError("grrt_tonemap_device failed")


def cuda_available() -> bool:
    return bool(lib().grrt_cuda_available())


from . import multi  # noqa: E402  (frame sharding across ranks)
