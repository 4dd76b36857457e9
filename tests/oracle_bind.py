"""ctypes bindings of the test oracle (oracle/_build/liboracle*.so) and of the
harness over the reference library compiled from its own sources
(oracle/_ref/libref_harness_*.so).

Test infrastructure: the product (grrt_b200) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "_build", "liboracle.so")
ORACLE_FMA_SO = os.path.join(ORACLE_DIR, "_build", "liboracle_fma.so")
REF_HARNESS = {
    "strict": os.path.join(ORACLE_DIR, "_ref", "libref_harness_strict.so"),
    "fast": os.path.join(ORACLE_DIR, "_ref", "libref_harness_fast.so"),
}

D = C.c_double
I = C.c_int
PD = C.POINTER(C.c_double)
PI = C.POINTER(C.c_int)


class OracleScene(C.Structure):
    _fields_ = [
        ("M", D), ("a", D), ("r_horizon", D), ("r_escape", D), ("horizon_eps", D), ("tolerance", D),
        ("observer_r", D), ("max_steps", I),
        ("cam_pos", D * 4), ("e0", D * 4), ("e1", D * 4), ("e2", D * 4), ("e3", D * 4), ("g", D * 16),
        ("fov", D), ("width", I), ("height", I),
        ("disk_on", I), ("disk_r_inner", D), ("disk_r_outer", D), ("flux_max", D), ("peak_temperature", D),
        ("flux_n", I), ("flux", PD),
        ("t_min", D), ("t_max", D), ("spec_n", I), ("spec_color", PD),
        ("stars_on", I), ("star_theta", PD), ("star_phi", PD), ("star_b", PD),
        ("cell_start", PI), ("cell_items", PI), ("star_tol", D),
        ("vol_on", I), ("v_M", D), ("v_a", D),
        ("v_r_min", D), ("v_r_outer", D), ("v_r_isco", D), ("v_r_horizon", D), ("v_taper_width", D),
        ("v_E_isco", D), ("v_L_isco", D),
        ("v_rho_scale", D), ("v_noise_scale", D), ("v_turbulence", D),
        ("v_octaves", I), ("v_n_r", I), ("v_n_z", I),
        ("v_H", PD), ("v_rho_mid", PD), ("v_rho_prof", PD), ("v_T_prof", PD), ("v_zmax", PD),
        ("v_perm", PI),
        ("o_n_nu", I), ("o_n_rho", I), ("o_n_T", I),
        ("o_log_nu_min", D), ("o_log_nu_max", D), ("o_log_rho_min", D), ("o_log_rho_max", D),
        ("o_log_T_min", D), ("o_log_T_max", D),
        ("o_kabs", PD), ("o_kes", PD),
    ]


class OracleCounters(C.Structure):
    _fields_ = [("attempts", C.c_longlong), ("accepted", C.c_longlong), ("crossings", C.c_longlong),
                ("clamp_evals", C.c_longlong), ("march_steps", C.c_longlong),
                ("physics_steps", C.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _dp(a):
    return a.ctypes.data_as(PD)


def _ip(a):
    return a.ctypes.data_as(PI)


def build_oracle() -> None:
    subprocess.run(["make", "oracle"], cwd=ORACLE_DIR, check=True, stdout=subprocess.DEVNULL)


_oracles = {}


def load_oracle(fma: bool = False) -> C.CDLL:
    key = "fma" if fma else "strict"
    if key in _oracles:
        return _oracles[key]
    path = ORACLE_FMA_SO if fma else ORACLE_SO
    if not os.path.exists(path):
        build_oracle()
    L = C.CDLL(path)
    P = C.POINTER
    L.oracle_pixel_hash.restype = D
    L.oracle_pixel_hash.argtypes = [I, I, I, I]
    L.oracle_camera_ray.argtypes = [P(OracleScene), D, D, PD]
    L.oracle_trace_rgb.argtypes = [P(OracleScene), I, PD, PD, PD, PI, PI, PD, P(OracleCounters)]
    L.oracle_render_pixels.argtypes = [P(OracleScene), I, I, PI, PD, P(OracleCounters)]
    L.oracle_trace_spectral.argtypes = [P(OracleScene), I, PD, I, PD, PD, PD, PI, P(OracleCounters)]
    L.oracle_render_spectral_pixels.argtypes = [P(OracleScene), I, I, PD, I, PI, PD, P(OracleCounters)]
    L.oracle_fast_sincos.argtypes = [D, PD, PD]
    L.oracle_derivatives.argtypes = [P(OracleScene), PD, PD]
    for fn in ("oracle_vol_density",):
        getattr(L, fn).restype = D
        getattr(L, fn).argtypes = [P(OracleScene), D, D, D]
    L.oracle_vol_temperature.restype = D
    L.oracle_vol_temperature.argtypes = [P(OracleScene), D, D]
    L.oracle_kappa_abs.restype = D
    L.oracle_kappa_abs.argtypes = [P(OracleScene), D, D, D]
    L.oracle_kappa_es.restype = D
    L.oracle_kappa_es.argtypes = [P(OracleScene), D, D]
    L.oracle_noise.restype = D
    L.oracle_noise.argtypes = [P(OracleScene), D, D, D]
    _oracles[key] = L
    return L


class Oracle:
    """An OracleScene filled from a product context's exported tables."""

    def __init__(self, renderer, fma: bool = False):
        self.L = load_oracle(fma)
        self.keep = []
        sc = OracleScene()
        s = renderer.table("scalars")
        M, a, r_h, isco, r_obs, tol, max_steps, spp = s
        sc.M, sc.a, sc.r_horizon, sc.r_escape, sc.horizon_eps = M, a, r_h, 1000.0, 0.01
        sc.tolerance, sc.observer_r, sc.max_steps = tol, r_obs, int(max_steps)
        self.spp = int(spp)
        cam = renderer.table("camera")
        for i in range(4):
            sc.cam_pos[i] = cam[i]
            sc.e0[i] = cam[4 + i]
            sc.e1[i] = cam[8 + i]
            sc.e2[i] = cam[12 + i]
            sc.e3[i] = cam[16 + i]
        for i in range(16):
            sc.g[i] = cam[20 + i]
        sc.fov, sc.width, sc.height = cam[36], int(cam[37]), int(cam[38])
        spec = self._hold(renderer.table("spectrum_color"))
        sc.t_min, sc.t_max, sc.spec_n, sc.spec_color = 1000.0, 100000.0, len(spec) // 3, _dp(spec)
        try:
            flux = self._hold(renderer.table("flux"))
            meta = renderer.table("flux_meta")
            sc.disk_on, sc.flux_n, sc.flux = 1, len(flux), _dp(flux)
            sc.flux_max, sc.disk_r_inner, sc.disk_r_outer, sc.peak_temperature = meta
        except KeyError:
            sc.disk_on = 0
        try:
            st = renderer.table("stars").reshape(-1, 3)
            th = self._hold(np.ascontiguousarray(st[:, 0]))
            ph = self._hold(np.ascontiguousarray(st[:, 1]))
            b = self._hold(np.ascontiguousarray(st[:, 2]))
            cs = self._hold(renderer.table("star_cells").astype(np.int32))
            ci = self._hold(renderer.table("star_items").astype(np.int32))
            sc.stars_on, sc.star_theta, sc.star_phi, sc.star_b = 1, _dp(th), _dp(ph), _dp(b)
            sc.cell_start, sc.cell_items, sc.star_tol = _ip(cs), _ip(ci), 0.003
        except KeyError:
            sc.stars_on = 0
        try:
            vs = renderer.table("vol_scalars")
        except KeyError:
            vs = None
        if vs is not None:
            (sc.v_r_min, sc.v_r_outer, sc.v_r_isco, sc.v_r_horizon, sc.v_rho_scale, sc.v_E_isco, sc.v_L_isco,
             sc.v_taper_width, sc.v_noise_scale, _peak, sc.v_turbulence, sc.v_M, sc.v_a, octv, nr, nz) = vs
            sc.vol_on, sc.v_octaves, sc.v_n_r, sc.v_n_z = 1, int(octv), int(nr), int(nz)
            for name, attr in (("vol_H", "v_H"), ("vol_rho_mid", "v_rho_mid"), ("vol_rho_prof", "v_rho_prof"),
                               ("vol_T_prof", "v_T_prof"), ("vol_zmax", "v_zmax"), ("op_kabs", "o_kabs"),
                               ("op_kes", "o_kes")):
                setattr(sc, attr, _dp(self._hold(renderer.table(name))))
            sc.v_perm = _ip(self._hold(renderer.table("vol_perm").astype(np.int32)))
            os_ = renderer.table("op_scalars")
            sc.o_n_nu, sc.o_n_rho, sc.o_n_T = int(os_[0]), int(os_[1]), int(os_[2])
            (sc.o_log_nu_min, sc.o_log_nu_max, sc.o_log_rho_min, sc.o_log_rho_max, sc.o_log_T_min,
             sc.o_log_T_max) = os_[3:9]
        self.sc = sc

    def _hold(self, a):
        a = np.ascontiguousarray(a)
        self.keep.append(a)
        return a

    def camera_ray(self, x: float, y: float) -> np.ndarray:
        out = np.empty(8)
        self.L.oracle_camera_ray(C.byref(self.sc), x, y, _dp(out))
        return out

    def trace_rgb(self, px, py):
        px = np.ascontiguousarray(px, dtype=np.float64)
        py = np.ascontiguousarray(py, dtype=np.float64)
        n = len(px)
        rgb = np.zeros((n, 3))
        term = np.zeros(n, dtype=np.int32)
        nc = np.zeros(n, dtype=np.int32)
        fin = np.zeros((n, 8))
        cnt = OracleCounters()
        self.L.oracle_trace_rgb(C.byref(self.sc), n, _dp(px), _dp(py), _dp(rgb), _ip(term), _ip(nc), _dp(fin),
                                C.byref(cnt))
        return rgb, term, nc, fin, cnt.as_dict()

    def render_pixels(self, pix, spp: Optional[int] = None):
        pix = np.ascontiguousarray(pix, dtype=np.int32)
        rgb = np.zeros((len(pix), 3))
        cnt = OracleCounters()
        self.L.oracle_render_pixels(C.byref(self.sc), spp or self.spp, len(pix), _ip(pix), _dp(rgb), C.byref(cnt))
        return rgb, cnt.as_dict()

    def trace_spectral(self, freqs, px, py):
        freqs = np.ascontiguousarray(freqs, dtype=np.float64)
        px = np.ascontiguousarray(px, dtype=np.float64)
        py = np.ascontiguousarray(py, dtype=np.float64)
        n, nb = len(px), len(freqs)
        spec = np.zeros((n, nb))
        term = np.zeros(n, dtype=np.int32)
        cnt = OracleCounters()
        self.L.oracle_trace_spectral(C.byref(self.sc), nb, _dp(freqs), n, _dp(px), _dp(py), _dp(spec), _ip(term),
                                     C.byref(cnt))
        return spec, term, cnt.as_dict()

    def render_spectral_pixels(self, freqs, pix, spp: Optional[int] = None):
        freqs = np.ascontiguousarray(freqs, dtype=np.float64)
        pix = np.ascontiguousarray(pix, dtype=np.int32)
        spec = np.zeros((len(pix), len(freqs)))
        cnt = OracleCounters()
        self.L.oracle_render_spectral_pixels(C.byref(self.sc), spp or self.spp, len(freqs), _dp(freqs), len(pix),
                                             _ip(pix), _dp(spec), C.byref(cnt))
        return spec, cnt.as_dict()


# ---------------------------------------------------------------------------
# Reference harness
# ---------------------------------------------------------------------------
_harness = {}


def ref_available(kind: str = "strict") -> bool:
    return os.path.exists(REF_HARNESS[kind])


def load_ref(kind: str = "strict") -> C.CDLL:
    if kind in _harness:
        return _harness[kind]
    from grrt_b200 import GRRTParams
    L = C.CDLL(REF_HARNESS[kind])
    vp = C.c_void_p
    L.rh_create.restype = vp
    L.rh_create.argtypes = [C.POINTER(GRRTParams)]
    L.rh_destroy.argtypes = [vp]
    L.rh_set_frequency_bins.argtypes = [vp, PD, I]
    L.rh_horizon.restype = D
    L.rh_horizon.argtypes = [vp]
    L.rh_isco.restype = D
    L.rh_isco.argtypes = [vp]
    L.rh_flux_lut.restype = I
    L.rh_flux_lut.argtypes = [vp, PD, PD]
    L.rh_spectrum_lut.restype = I
    L.rh_spectrum_lut.argtypes = [vp, PD, PD]
    L.rh_stars.restype = I
    L.rh_stars.argtypes = [vp, PD]
    L.rh_vol_sizes.restype = I
    L.rh_vol_sizes.argtypes = [vp, PI]
    L.rh_vol_tables.restype = I
    L.rh_vol_tables.argtypes = [vp, PD, PD, PD, PD, PD, PD, PD, PD, PD, PI, PD]
    L.rh_camera_rays.argtypes = [vp, I, PD, PD, PD]
    L.rh_trace_rgb.argtypes = [vp, I, PD, PD, PD, PI, PD]
    L.rh_trace_spectral.argtypes = [vp, I, PD, PD, PD, PI]
    L.rh_render_rows.restype = D
    L.rh_render_rows.argtypes = [vp, I, I, C.POINTER(C.c_float), PI]
    L.rh_render_spectral_rows.restype = D
    L.rh_render_spectral_rows.argtypes = [vp, I, I, PD, PI]
    _harness[kind] = L
    return L


class RefScene:
    """The reference's own scene objects, built as grrt_create builds them."""

    def __init__(self, values: dict, freqs=None, kind: str = "strict"):
        from grrt_b200 import make_params
        self.L = load_ref(kind)
        self.freqs = None if freqs is None else np.ascontiguousarray(freqs, dtype=np.float64)
        self.params = make_params(values, self.freqs)
        self.values = values
        self.h = self.L.rh_create(C.byref(self.params))
        if self.freqs is not None:
            self.L.rh_set_frequency_bins(self.h, _dp(self.freqs), len(self.freqs))

    def __del__(self):
        try:
            self.L.rh_destroy(self.h)
        except Exception:
            pass

    def flux(self):
        meta = np.zeros(4)
        n = self.L.rh_flux_lut(self.h, None, _dp(meta))
        out = np.zeros(n)
        self.L.rh_flux_lut(self.h, _dp(out), _dp(meta))
        return out, meta

    def spectrum(self):
        color = np.zeros(3000)
        lum = np.zeros(1000)
        self.L.rh_spectrum_lut(self.h, _dp(color), _dp(lum))
        return color, lum

    def stars(self):
        out = np.zeros(3 * 5000)
        n = self.L.rh_stars(self.h, _dp(out))
        return out[: 3 * n]

    def vol_tables(self):
        sz = np.zeros(5, dtype=np.int32)
        if not self.L.rh_vol_sizes(self.h, _ip(sz)):
            return None
        nr, nz, nnu, nrho, nT = (int(x) for x in sz)
        t = {"vol_H": np.zeros(nr), "vol_rho_mid": np.zeros(nr), "vol_rho_prof": np.zeros(nr * nz),
             "vol_T_prof": np.zeros(nr * nz), "vol_zmax": np.zeros(nr), "op_kabs": np.zeros(nnu * nrho * nT),
             "op_kes": np.zeros(nrho * nT), "op_kross": np.zeros(nrho * nT), "op_mu": np.zeros(nrho * nT)}
        perm = np.zeros(512, dtype=np.int32)
        scal = np.zeros(17)
        self.L.rh_vol_tables(self.h, _dp(t["vol_H"]), _dp(t["vol_rho_mid"]), _dp(t["vol_rho_prof"]),
                             _dp(t["vol_T_prof"]), _dp(t["vol_zmax"]), _dp(t["op_kabs"]), _dp(t["op_kes"]),
                             _dp(t["op_kross"]), _dp(t["op_mu"]), _ip(perm), _dp(scal))
        t["vol_perm"] = perm
        t["scal"] = scal
        return t

    def camera_rays(self, px, py):
        px = np.ascontiguousarray(px, dtype=np.float64)
        py = np.ascontiguousarray(py, dtype=np.float64)
        out = np.zeros((len(px), 8))
        self.L.rh_camera_rays(self.h, len(px), _dp(px), _dp(py), _dp(out))
        return out

    def trace_rgb(self, px, py):
        px = np.ascontiguousarray(px, dtype=np.float64)
        py = np.ascontiguousarray(py, dtype=np.float64)
        n = len(px)
        rgb = np.zeros((n, 3))
        term = np.zeros(n, dtype=np.int32)
        fin = np.zeros((n, 8))
        self.L.rh_trace_rgb(self.h, n, _dp(px), _dp(py), _dp(rgb), _ip(term), _dp(fin))
        return rgb, term, fin

    def trace_spectral(self, px, py):
        px = np.ascontiguousarray(px, dtype=np.float64)
        py = np.ascontiguousarray(py, dtype=np.float64)
        n, nb = len(px), len(self.freqs)
        spec = np.zeros((n, nb))
        term = np.zeros(n, dtype=np.int32)
        self.L.rh_trace_spectral(self.h, n, _dp(px), _dp(py), _dp(spec), _ip(term))
        return spec, term

    def render_rows(self, row0: int, stride: int):
        W, H = self.values["width"], self.values["height"]
        fb = np.zeros((H, W, 4), dtype=np.float32)
        th = np.zeros(1, dtype=np.int32)
        secs = self.L.rh_render_rows(self.h, row0, stride, fb.ctypes.data_as(C.POINTER(C.c_float)), _ip(th))
        return fb, secs, int(th[0])

    def render_spectral_rows(self, row0: int, stride: int):
        W, H = self.values["width"], self.values["height"]
        out = np.zeros((H, W, len(self.freqs)))
        th = np.zeros(1, dtype=np.int32)
        secs = self.L.rh_render_spectral_rows(self.h, row0, stride, _dp(out), _ip(th))
        return out, secs, int(th[0])


def jittered_samples(W: int, H: int, spp: int, pix):
    """Fractional coordinates of every sample of the given pixels, in the
    reference's order (src/renderer.cpp:48-56)."""
    import math
    L = load_oracle()
    grid = max(1, int(math.sqrt(spp)))
    cell = 1.0 / grid
    xs, ys = [], []
    for p in pix:
        j, i = divmod(int(p), W)
        for sy in range(grid):
            for sx in range(grid):
                s = sy * grid + sx
                xs.append(i + (sx + L.oracle_pixel_hash(i, j, s, 0)) * cell)
                ys.append(j + (sy + L.oracle_pixel_hash(i, j, s, 1)) * cell)
    return np.array(xs), np.array(ys)
