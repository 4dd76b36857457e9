"""Parity helpers shared by the GPU tests: run a render on the device through
the C ABI, run the same samples through the oracle, and derive the
rounding-sensitive ("caustic") band from the oracle itself.

Image-integrated flux. The volumetric march amplifies rounding: the probes
move a volumetric frame's flux per bin by ~1e-3 relative (the reference's own
strict and as-shipped builds differ per pixel by a median of ~5%), so the
flux bar of a device render is data-driven: within a few times the largest
move of any probe (OracleRGB / OracleSpectral.probe_flux_spread).

Band definition. A sample is rounding-sensitive when the strict oracle and a
rounding-level probe disagree on the fate or differ by more than the test
tolerance. The probes are the same oracle compiled with FMA contraction and
the strict oracle with the sample position moved by +-1e-12 pixel in x and in
y. The reference's own answer is only determined to this level: its PI step
controller forms the error estimate near the rounding floor, so the next step
size carries ~1e-8 relative noise, which moves the step endpoints along the
ray and, through the linear crossing interpolation, a lit pixel's colour by
~1e-10 (median) to ~1e-7. A pixel is in the band when any of its samples is.
"""
from __future__ import annotations

import math

import numpy as np

import oracle_bind

# rounding-level shifts of the sample position (pixels)
PROBE_SHIFTS = [(1e-12, 0.0), (-1e-12, 0.0), (0.0, 1e-12), (0.0, -1e-12)]


def device_render_rgb(R, spp: int):
    import torch
    W, H = R.width, R.height
    grid = max(1, int(math.sqrt(spp)))
    rgba = torch.full((H, W, 4), float("nan"), dtype=torch.float32, device="cuda")
    rgb64 = torch.full((H, W, 3), float("nan"), dtype=torch.float64, device="cuda")
    fate = torch.full((H * W * grid * grid,), -1, dtype=torch.int32, device="cuda")
    R.render_device(rgba, rgb64, fate)
    torch.cuda.synchronize()
    return rgba.cpu().numpy(), rgb64.cpu().numpy(), fate.cpu().numpy().view(np.uint32), R.stats()


def device_render_spectral(R, nb: int):
    import torch
    W, H = R.width, R.height
    spp = R.values.get("samples_per_pixel", 1) or 1
    grid = max(1, int(math.sqrt(spp)))
    spec = torch.full((H, W, nb), float("nan"), dtype=torch.float64, device="cuda")
    fate = torch.full((H * W * grid * grid,), -1, dtype=torch.int32, device="cuda")
    R.render_spectral_device(spec, W, H, fate)
    torch.cuda.synchronize()
    return spec.cpu().numpy(), fate.cpu().numpy().view(np.uint32), R.stats()


def rel_err(a, b, floor=1e-300):
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


def hull_error(got: np.ndarray, lo: np.ndarray, hi: np.ndarray, floor: float = 1e-300) -> np.ndarray:
    """Per pixel, the largest relative distance (over channels or bins) of
    `got` outside [lo, hi]: the range spanned by the oracle and its rounding
    probes. 0 when every channel lies inside it."""
    scale = np.maximum(np.maximum(np.abs(lo), np.abs(hi)), floor)
    out = np.maximum(lo - got, got - hi)
    return np.max(np.maximum(out, 0.0) / scale, axis=1)


def flux_spread(a: np.ndarray, b: np.ndarray) -> float:
    """Largest relative difference over channels (or bins) of the image-
    integrated flux of two sets of pixels."""
    fa, fb = a.sum(axis=0), b.sum(axis=0)
    floor = 1e-300 + 1e-12 * float(np.max(np.abs(fb))) if fb.size else 1e-300
    return float(np.max(np.abs(fa - fb) / np.maximum(np.abs(fb), floor))) if fb.size else 0.0


def pixel_mean(per_sample: np.ndarray, spp: int) -> np.ndarray:
    """The reference's spp mean: accumulate samples in order from 0, then scale."""
    grid = max(1, int(math.sqrt(spp)))
    g2 = grid * grid
    s = per_sample.reshape(-1, g2, *per_sample.shape[1:])
    acc = np.zeros_like(s[:, 0])
    for k in range(g2):
        acc = acc + s[:, k]
    return acc * (1.0 / g2)


class OracleRGB:
    """Oracle traces of every sample of the given pixels, strict and sensitivity runs."""

    def __init__(self, R, pix, tol: float, band: bool = True):
        self.R = R
        W, H = R.width, R.height
        spp = R.values.get("samples_per_pixel", 1) or 1
        self.spp = spp
        self.g2 = max(1, int(math.sqrt(spp))) ** 2
        px, py = oracle_bind.jittered_samples(W, H, spp, pix)
        O = oracle_bind.Oracle(R)
        self.rgb, self.term, self.ncross, self.fin, self.counters = O.trace_rgb(px, py)
        spreads = []
        self.sensitive = np.zeros(len(px), dtype=bool)
        self.fate_sensitive = np.zeros(len(px), dtype=bool)
        lo, hi = self.rgb.copy(), self.rgb.copy()
        if band:
            F = oracle_bind.Oracle(R, fma=True)
            probes = [F.trace_rgb(px, py)]
            for dx, dy in PROBE_SHIFTS:
                probes.append(O.trace_rgb(px + dx, py + dy))
            for r2, t2, n2, _, _ in probes:
                fs = (t2 != self.term) | (n2 != self.ncross)
                self.fate_sensitive |= fs
                self.sensitive |= fs
                self.sensitive |= np.any(np.abs(r2 - self.rgb) > tol * np.abs(self.rgb), axis=1)
                lo, hi = np.minimum(lo, r2), np.maximum(hi, r2)
                spreads.append(flux_spread(pixel_mean(r2, spp), pixel_mean(self.rgb, spp)))
        self.pixel_rgb = pixel_mean(self.rgb, spp)
        # how far rounding-level probes move the image-integrated flux (per channel, relative)
        self.probe_flux_spread = max(spreads) if spreads else 0.0
        # per pixel, the range the oracle and its rounding probes span
        self.pixel_lo, self.pixel_hi = pixel_mean(lo, spp), pixel_mean(hi, spp)
        self.pixel_band = self.sensitive.reshape(-1, self.g2).any(axis=1)
        self.pixel_fate_band = self.fate_sensitive.reshape(-1, self.g2).any(axis=1)
        self.fate = (self.term.astype(np.uint32) | (self.ncross.astype(np.uint32) << 2))


class OracleSpectral:
    def __init__(self, R, freqs, pix, tol: float, band: bool = True):
        W, H = R.width, R.height
        spp = R.values.get("samples_per_pixel", 1) or 1
        self.g2 = max(1, int(math.sqrt(spp))) ** 2
        px, py = oracle_bind.jittered_samples(W, H, spp, pix)
        O = oracle_bind.Oracle(R)
        self.spec, self.term, self.counters = O.trace_spectral(freqs, px, py)
        spreads = []
        self.sensitive = np.zeros(len(px), dtype=bool)
        self.fate_sensitive = np.zeros(len(px), dtype=bool)
        lo, hi = self.spec.copy(), self.spec.copy()
        if band:
            F = oracle_bind.Oracle(R, fma=True)
            probes = [F.trace_spectral(freqs, px, py)]
            for dx, dy in PROBE_SHIFTS:
                probes.append(O.trace_spectral(freqs, px + dx, py + dy))
            for s2, t2, _ in probes:
                self.fate_sensitive |= t2 != self.term
                self.sensitive |= t2 != self.term
                self.sensitive |= np.any(np.abs(s2 - self.spec) > tol * np.abs(self.spec), axis=1)
                lo, hi = np.minimum(lo, s2), np.maximum(hi, s2)
                spreads.append(flux_spread(pixel_mean(s2, spp), pixel_mean(self.spec, spp)))
        self.pixel_spec = pixel_mean(self.spec, spp)
        # how far rounding-level probes move the image-integrated flux (per bin, relative)
        self.probe_flux_spread = max(spreads) if spreads else 0.0
        self.pixel_lo, self.pixel_hi = pixel_mean(lo, spp), pixel_mean(hi, spp)
        self.pixel_band = self.sensitive.reshape(-1, self.g2).any(axis=1)
        self.pixel_fate_band = self.fate_sensitive.reshape(-1, self.g2).any(axis=1)
