#!/usr/bin/env python3
"""Benchmark: Kerr rays/s of the 1024x1024, 4-spp thin-disk render.

Workload (one step = one full frame): Kerr a=0.998, M=1, observer r=50,
theta=80 deg, phi=0, horizontal FOV 90 deg; thin disk ISCO..20 M,
T_peak 1e7 K, blackbody chromaticity with redshift and g^4 beaming; star
background (5000 stars, seed 42); adaptive Dormand-Prince 5(4) at tolerance
1e-8, at most 10000 steps; 2x2 stratified jitter from the reference's hash.
1024*1024*4 = 4,194,304 rays per step. Inputs are synthetic (the scene is
generated from its parameters; no dataset).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--form mixed|fp64]
  python bench.py --impl reference   # the reference's own CPU code, same workload

The line also carries "surrogate": the learned form, trained in the same run
on the 64-camera sweep and timed on its evaluation frame (Kerr a=0.998, 80
deg, 2048^2, 1 spp, thin disk, black background) beside the FP64 and mixed
forms of that frame, with its colour-tolerance Pareto (--surrogate-steps 0
skips it); "volumetric": the spectral render (Kerr a=0.9, 512^2, 32 bins) in
both forms, its FITS output time and the context creation time
(--no-volumetric skips it); and "batch": the 64-camera sweep in one
persistent launch, mixed and FP64 forms, against 64 separate launches
(--no-batch-section skips it).

`value` is rays/s of the headline form (default: mixed, whose output is held
to <=1e-4 relative of the FP64 form and reported against it) with the scene
and the output resident on the device (CUDA events around each render launch
on its stream; a 256 MiB buffer is written between steps to flush the 126 MB
L2). Both forms are timed; "forms" reports each, with per-kernel phase times
from the library's own CUDA events. `e2e` is the same metric through the
reference C entry point grrt_render with a host framebuffer (launch
parameters in, the float RGBA frame out, every step): a page-locked buffer,
which the library copies into directly, and, under e2e.pageable, a pageable
one, which it fills through its pinned staging buffer.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Kerr rays/s at 1024^2: plain FP64 vs mixed vs surrogate at <=1e-4 rel intensity"
WORKLOAD = "kerr_a0.998_1024x1024_4spp_thin_disk_isco_20M_stars_seed42_tol1e-8"
W = H = 1024
SPP = 4
RAYS = W * H * SPP

# Algorithmic FLOPs of the reference method (binary + - * / and sqrt, counted
# in the reference source; transcendental calls counted apart):
#   one Kerr right-hand side (include/grrt/spacetime/kerr.h:31-109): 133
#   fast_sincos (include/grrt/math/fast_trig.h:21-82): 37
#   one DP45 attempt (include/grrt/geodesic/rk4.h:73-177): 7 right-hand sides
#   + 480 for the stage sums, the 5th-order solution and the error norm over
#   the reference's 8-component state
# The kernels take an attempt's first right-hand side from the previous
# attempt (the same value), so they execute 6 per attempt plus one per ray
# start; the rooflines count what is executed (F_ATTEMPT_EXEC per attempt +
# F_EVAL per ray).
F_EVAL = 133 + 37
F_ATTEMPT_EXEC = 6 * F_EVAL + 480
# Operations the kernels execute per attempt (all of a kernel's floating-point
# operations divided by its attempts; a fused multiply-add counts 2), from the
# ncu instruction counters of a 512x512 4-spp frame
# (profiles/executed_flops_thin_mixed_kernels_kerr_512x512_4spp.md): the FP64
# kernels (fp64_trace_kernel in both forms) and the FP32 speculation
# (packed two-wide instructions count once there: a lower bound).
F_EXEC_FP64_ATTEMPT = 1022.8
F_EXEC_FP32_ATTEMPT = 479.4
# DRAM bytes (read + write) of one mixed_speculate_kernel launch on the
# 1024x1024 4-spp frame, from ncu (single-pass dram__bytes_read.sum +
# dram__bytes_write.sum, the warp-staged kernel): 0.52 MB read + 55.17 MB
# written. The launch writes 28 B per sample (colour, 3 doubles, and fate
# word: 117 MB); the rest of it is still in the 126 MB L2 when the launch ends.
TRAFFIC_SPECULATE_C2 = 55_685_580


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    # headline form; the other form is timed too and reported under "forms"
    ap.add_argument("--form", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # smaller frames of the same scene, for profiler captures (default: the benchmark frame)
    ap.add_argument("--width", type=int, default=1024)
    ap.add_argument("--height", type=int, default=1024)
    # the batched sweep (64 cameras, one persistent launch) instead of the headline frame
    ap.add_argument("--batch", action="store_true")
    # the default line also carries the batched sweep (mixed and FP64 forms); this skips it
    ap.add_argument("--no-batch-section", action="store_true")
    # the learned surrogate (trained in this run) on its evaluation frame; 0 skips it
    ap.add_argument("--surrogate-steps", type=int, default=20000)
    ap.add_argument("--surrogate-size", type=int, default=2048)
    # the volumetric spectral render (both forms) reported beside the headline
    ap.add_argument("--no-volumetric", action="store_true")
    ap.add_argument("--volumetric", action="store_true", help="run only the volumetric spectral section")
    ap.add_argument("--vol-size", type=int, default=512, help="volumetric frame side (profiler captures)")
    # N > 1: "frames" renders one whole frame per GPU per step (weak scaling);
    # "rows" splits one frame by interleaved rows and all-gathers it (strong scaling)
    ap.add_argument("--shard", default="frames", choices=["frames", "rows"])
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# peaks
# ---------------------------------------------------------------------------
def measured_peaks(torch) -> dict:
    peaks = {}
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        peaks.update(json.load(open(path)))
        peaks["source"] = "MEASURED_PEAKS.json"
    else:
        # an earlier measurement on this pool's B200s (copy bandwidth, cuBLAS
        # bf16 burst), used when the measured file is absent
        peaks.update({"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"})
    # FP64 roofline denominator: cuBLAS DGEMM measured here (the same method
    # the driver uses for its bf16 figure), best of 5.
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    peaks["fp64_tflops_dgemm"] = best
    return peaks


# ---------------------------------------------------------------------------
# the reference's CPU implementation (oracle/_ref, built from its own sources)
# ---------------------------------------------------------------------------
def cpu_reference_sample(row_offset: int = 0, stride: int = 16):
    """Render rows row_offset, row_offset+stride, ... of the benchmark frame with
    the reference's own code (as-shipped optimisation flags) on all host cores."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import grrt_b200 as G
    import oracle_bind
    kind = "fast" if oracle_bind.ref_available("fast") else "strict"
    ref = oracle_bind.RefScene(G.config_params(2), kind=kind)  # the 1024x1024 benchmark frame
    _, secs, threads = ref.render_rows(row_offset, stride)
    rows = len(range(row_offset, 1024, stride))
    rays = rows * 1024 * SPP
    return rays, secs, threads, kind, rows


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    stride = 16
    for w in range(args.warmup):
        cpu_reference_sample(w % stride, stride * 4)
    total_rays, total_secs, threads, kind, rows = 0, 0.0, 1, "fast", 0
    for k in range(args.steps):
        rays, secs, threads, kind, rows = cpu_reference_sample(k % stride, stride)
        total_rays += rays
        total_secs += secs
    value = total_rays / total_secs
    sample = (f"every {stride}th row of the 1024x1024 4-spp frame ({rows} rows, {rows * 1024 * SPP} rays) per step, "
              f"row offset = step mod {stride}; reference src/*.cpp built with its shipped flags "
              f"(minus -march=native and LTO), OpenMP over all host threads")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            # the GPU arm's workload keys; the rays of each step are a sample of the frame
            "config": {"workload": WORKLOAD, "width": W, "height": H, "spp": SPP, "rays_per_step": RAYS,
                       "form": "reference FP64 (src/*.cpp)", "l2": "not applicable (host CPU)",
                       "parallelism": "OpenMP over all host threads (rank 0 only)",
                       "row_sampling": f"every {stride}th row per step, offset rotating with the step "
                                       f"({rows} rows = {rows * 1024 * SPP} rays per step)"},
            "cpu_baseline": {"value": value, "unit": "rays/s", "cores": threads,
                             "kind": "reference" if kind else "port", "sample": sample},
            "e2e": {"value": value, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def batch_section(args, torch, G, stream, flush, form_name="mixed"):
    """Batched sweep: spins {0 (Schwarzschild), 0.5, 0.9, 0.998} x 16 inclinations
    5..90 deg, 256x256 each, thin disk ISCO..20 M, stars seed 42, tolerance 1e-8:
    one persistent launch (CUDA graph, autotuned schedule and thresholds)
    against 64 separate single-camera launches of the same cameras; in the
    mixed form also the FP64 batch and the mixed images' error against it."""
    form = G.FORM_MIXED if form_name == "mixed" else G.FORM_FP64
    cams = G.sweep_cameras()
    rays = sum(c["width"] * c["height"] for c in cams)
    cache = os.path.join(ROOT, "_build", "batch_schedule_cache.jsonl")
    os.makedirs(os.path.dirname(cache), exist_ok=True)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.mean(ts))

    B = G.Batch(cams)
    B.set_precision(form)
    tuned_ms = B.autotune(cache)
    out = torch.empty((rays, 4), dtype=torch.float32, device="cuda")
    ms = timed(lambda: B.render_device(out, stream))
    st = B.stats()
    got = out.cpu().numpy()
    # the same 64 cameras as 64 separate launches (one context each)
    ctxs = [G.Renderer(c) for c in cams]
    for R in ctxs:
        R.set_precision(form)
    bufs = [torch.empty((c["height"], c["width"], 4), dtype=torch.float32, device="cuda") for c in cams]

    def separate():
        for R, bb in zip(ctxs, bufs):
            R.render_device(bb, None, None, stream)
    sep_ms = timed(separate)
    for R in ctxs:
        R.close()
    res = {"metric": "batched sweep rays/s (64 Kerr cameras x 256^2, one persistent launch)",
           "value": rays / (ms * 1e-3), "unit": "rays/s", "ms_per_step": ms, "form": form_name,
           "dtype": "f64" if form == G.FORM_FP64 else "f32+f64",
           "config": {"workload": "sweep_64cams_spins0_0.5_0.9_0.998_x16incl_5to90deg_256x256_thin_disk_stars",
                      "rays_per_step": rays, "l2": "flushed between steps (256 MiB write)"},
           "schedule": dict(zip(("chunk", "order", "blocks_per_sm"), B.schedule()), autotune_ms=tuned_ms,
                            **B.tuning()),
           "separate_launches_ms_per_step": sep_ms, "batched_speedup": sep_ms / ms,
           "work": {"attempts_per_ray": st["attempts"] / max(1, st["rays"]),
                    "fp64_attempt_share": st["fp64_attempts"] / max(1, st["attempts"])},
           # FP64: one persistent launch; mixed: speculate, stars, re-trace, resolve
           "gpu_launches_per_step": 4 if form == G.FORM_MIXED else 1}
    if form == G.FORM_MIXED:
        B64 = G.Batch(cams)
        t64 = B64.autotune(cache)
        out64 = torch.empty_like(out)
        ms64 = timed(lambda: B64.render_device(out64, stream))
        ref = out64.cpu().numpy()
        worst, over = 0.0, 0
        for k in range(len(cams)):
            a, b = int(B.offsets[k]), int(B.offsets[k + 1])
            r, g = ref[a:b, :3], got[a:b, :3]
            scale = float(r.max())
            rel = np.abs(g - r) / np.maximum(np.abs(r), 1e-6 * scale)
            worst = max(worst, float(rel.max()))
            over += int(np.sum(rel.max(axis=1) > 1e-4))
        res["fp64_batch"] = {"ms_per_step": ms64, "value": rays / (ms64 * 1e-3), "autotune_ms": t64,
                             "schedule": dict(zip(("chunk", "order", "blocks_per_sm"), B64.schedule()),
                                              **B64.tuning())}
        res["speedup_mixed_vs_fp64_batch"] = ms64 / ms
        res["mixed_error_vs_fp64"] = {"max_rel": worst, "pixels_above_1e-4": over,
                                      "rel_floor": "max(|fp64|, 1e-6 x camera max)"}
        B64.close()
    B.close()
    return res


def run_batch(args):
    import torch
    import grrt_b200 as G
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    stream = torch.cuda.Stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    res = batch_section(args, torch, G, stream, flush, args.form)
    res.update(n_gpus=1, steps=args.steps, warmup=args.warmup, higher_is_better=True, data="synthetic",
               gpu_launches=args.steps * res["gpu_launches_per_step"])
    print(json.dumps(res), flush=True)


def time_form(torch, R, form, stream, flush, render, steps, warmup, dist):
    """W warm-up frames, then K timed frames of one precision form: CUDA events
    around each frame's work (render(), enqueued on `stream`: the render
    launches, and with rows sharded the all-gather), plus the library's
    per-phase events."""
    R.set_precision(form)

    def step(ev=None):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)  # evict L2 between frames
            if ev is not None:
                ev[0].record(stream)
            render()
            if ev is not None:
                ev[1].record(stream)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    phases = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(steps):
        step(evs[k])
        phases.append(R.phase_ms())  # waits for this frame; the next frame is enqueued after
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    st = R.stats()  # the last timed frame's work counters (every frame does the same work)
    if dist:
        dist.barrier()
    kernel_ms = [a.elapsed_time(b) for a, b in evs]
    ms = float(np.mean(kernel_ms))
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    phase_mean = [float(np.mean([p[k] for p in phases])) for k in range(len(phases[0]))]
    return {"ms": ms, "kernel_ms": kernel_ms, "stats": st, "phase_ms": phase_mean, "wall": wall}


def form_error(torch, grrt, params):
    """Mixed against FP64 on the benchmark frame: per-pixel relative error of the
    double colour and the number of samples whose fate differs."""
    R = grrt.Renderer(params)
    g2 = SPP
    out = {}
    for name, form in (("fp64", grrt.FORM_FP64), ("mixed", grrt.FORM_MIXED)):
        R.set_precision(form)
        rgb = torch.empty((H, W, 3), dtype=torch.float64, device="cuda")
        fate = torch.empty((H * W * g2,), dtype=torch.int32, device="cuda")
        R.render_device(None, rgb, fate)
        torch.cuda.synchronize()
        out[name] = (rgb, fate)
    f, m = out["fp64"][0], out["mixed"][0]
    scale = float(f.max())
    rel = (m - f).abs() / torch.clamp(f.abs(), min=1e-6 * scale)
    R.close()
    return {"max_rel": float(rel.max()), "pixels_over_1e-4": int((rel.amax(dim=2) > 1e-4).sum()),
            "pixels_differing": int(((m != f).any(dim=2)).sum()),
            "sample_fates_differing": int((out["fp64"][1] != out["mixed"][1]).sum()),
            "rel_floor": "max(|fp64|, 1e-6 x frame max)"}


# counted FP64 operations of the volumetric spectral path (transcendental
# calls not counted): an RK4 march step (4 right-hand sides + stage sums), a
# clamp evaluation (one right-hand side), one bin of a physics step (opacity
# trilinear in ln kappa, Planck function, transfer update: 56 plus log10 and 3 exp)
F_RK4 = 4 * F_EVAL + 70
F_BIN = 56


def run_volumetric(args, torch, G, stream, flush, p64):
    """Volumetric spectral render: Kerr a=0.9, 512x512, 1 spp, Shakura-Sunyaev
    alpha 0.1, fBm turbulence 0.4, 2 octaves, seed 42, outer radius 20 M,
    M = 10 M_sun at 0.1 Eddington, 32 log-spaced bins 1e14..1e18 Hz. Both
    precision forms, through grrt_render_spectral_device on device buffers,
    CUDA events on the launching stream, L2 flushed between frames."""
    freqs = G.log_bins(1e14, 1e18, 32)
    vw = vh = args.vol_size
    nb = len(freqs)
    # context creation (host tables: Saha/opacity grid, disk structure, noise),
    # timed on the host; the reference's constructor is timed beside it below
    t_create = time.perf_counter()
    R = G.Renderer(G.config_params(3, width=vw, height=vh), freqs=freqs)
    create_ms = 1e3 * (time.perf_counter() - t_create)
    spec = torch.empty((vh, vw, nb), dtype=torch.float64, device="cuda")
    fate = torch.empty((vh * vw,), dtype=torch.int32, device="cuda")
    out = {}
    for name, form in (("fp64", G.FORM_FP64), ("mixed", G.FORM_MIXED)):
        R.set_precision(form)
        for _ in range(args.warmup):
            R.render_spectral_device(spec, vw, vh, fate, stream)
        torch.cuda.synchronize()
        ts, phases = [], []
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                R.render_spectral_device(spec, vw, vh, fate, stream)
                e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
            phases.append(R.phase_ms())
        ms = float(np.mean(ts))
        st = R.stats()
        out[name] = {"ms_per_step": ms, "pixel_freq_per_s": vw * vh * nb / (ms * 1e-3),
                     "rays_per_s": vw * vh / (ms * 1e-3), "phase_ms": [float(x) for x in np.mean(phases, axis=0)],
                     "stats": {k: st[k] for k in ("attempts", "fp64_attempts", "march_steps", "clamp_evals",
                                                  "physics_steps", "bin_updates", "rays", "horizon", "escaped")},
                     "spec": spec.cpu().numpy(), "fate": fate.cpu().numpy()}
    # the same frame to a FITS cube (grrt_render_spectral_to_fits_cb, mixed
    # form): host wall clock per call, written to tmpfs so the disk is not timed
    fits_dir = "/dev/shm" if os.path.isdir("/dev/shm") else tempfile.gettempdir()
    fits_path = os.path.join(fits_dir, f"grrt_bench_{os.getpid()}.fits")
    R.set_precision(G.FORM_MIXED)
    R.render_fits(fits_path, vw, vh)  # warm-up: pinned staging and device buffers
    tf = []
    for _ in range(max(3, args.steps // 2)):
        t0 = time.perf_counter()
        R.render_fits(fits_path, vw, vh)
        tf.append(1e3 * (time.perf_counter() - t0))
    fits_bytes = os.path.getsize(fits_path)
    os.unlink(fits_path)
    f, m = out["fp64"], out["mixed"]
    scale = float(f["spec"].max())
    rel = np.abs(m["spec"] - f["spec"]) / np.maximum(np.abs(f["spec"]), 1e-6 * scale)
    flux_f = f["spec"].sum(axis=(0, 1))
    flux_m = m["spec"].sum(axis=(0, 1))
    err = {"bit_identical": bool(np.array_equal(m["spec"], f["spec"])), "max_rel": float(rel.max()),
           "pixels_above_1e-4": int(np.sum(rel.max(axis=2) > 1e-4)),
           "flux_max_rel_per_bin": float(np.max(np.abs(flux_m - flux_f) / np.maximum(np.abs(flux_f), 1e-300))),
           "fate_differences": int(np.sum(m["fate"] != f["fate"]))}
    st = f["stats"]
    # the clamp reuses the step's first right-hand side: no FLOPs of its own
    flops = st["attempts"] * F_ATTEMPT_EXEC + st["rays"] * F_EVAL + st["march_steps"] * F_RK4 + \
        st["bin_updates"] * F_BIN
    kms = f["phase_ms"][0]
    ach = flops / (kms * 1e-3) / 1e12
    cube = vw * vh * nb * 8
    res = {"config": {"workload": f"volumetric_kerr_a0.9_{vw}x{vh}_1spp_32bins_1e14-1e18Hz_alpha0.1_turb0.4_oct2",
                      "bins": nb, "width": vw, "height": vh, "l2": "flushed between steps (256 MiB write)"},
           "metric": "pixel*frequency/s", "value": m["pixel_freq_per_s"], "headline_form": "mixed",
           "forms": {k: {kk: vv for kk, vv in v.items() if kk not in ("spec", "fate")} for k, v in out.items()},
           "speedup_mixed_vs_fp64": f["ms_per_step"] / m["ms_per_step"], "mixed_error_vs_fp64": err,
           "roofline_fp64": {"kernel": "vol_spectral_kernel<false>", "bound": "fp64", "achieved": ach, "peak": p64,
                             "unit": "TFLOP/s", "frac": ach / p64,
                             "flop_count": f"{F_ATTEMPT_EXEC}/attempt + {F_EVAL}/ray (first right-hand side), "
                                           f"{F_RK4}/march step, {F_BIN}/bin update (transcendentals and the "
                                           f"right-hand sides after march ends not counted), device counters"},
           "cube_store": {"bytes": cube, "GB_per_s": cube / (kms * 1e-3) / 1e9},
           "create_ms": {"ours": create_ms, "host_threads": os.cpu_count()},
           "to_fits": {"ms_per_frame": float(np.median(tf)), "device_ms_per_frame": m["ms_per_step"],
                       "file_bytes": fits_bytes, "target": fits_dir,
                       "api": "grrt_render_spectral_to_fits_cb (mixed form), host wall clock"}}
    if not args.no_cpu_baseline:
        try:
            sys.path.insert(0, os.path.join(ROOT, "tests"))
            import oracle_bind
            kind = "fast" if oracle_bind.ref_available("fast") else "strict"
            t_ref = time.perf_counter()
            ref = oracle_bind.RefScene(G.config_params(3, width=vw, height=vh), freqs=freqs, kind=kind)
            res["create_ms"]["reference"] = 1e3 * (time.perf_counter() - t_ref)
            res["create_ms"]["reference_build"] = kind
            stride = 8
            _, secs, threads = ref.render_spectral_rows(0, stride)
            npf = len(range(0, vh, stride)) * vw * nb
            res["cpu_baseline"] = {"value": npf / secs, "unit": "pixel*frequency/s", "cores": threads,
                                   "kind": "reference",
                                   "sample": f"rows 0,{stride},...,{vh - stride} of the frame, reference src/*.cpp "
                                             f"({kind} build) via oracle/_ref, OpenMP, {secs:.2f} s"}
        except Exception as ex:
            res["cpu_baseline"] = {"value": None, "sample": f"unavailable: {ex}"}
    R.close()
    try:
        res["batch"] = volumetric_batch(args, torch, G, stream, flush)
    except Exception as ex:  # reported, the section stands on its own
        res["batch"] = {"error": str(ex)}
    return res


def volumetric_batch(args, torch, G, stream, flush):
    """The batched form over volumetric cameras: 8 cameras (spins 0.5, 0.9 x
    inclinations 60, 70, 80, 85 deg), 256x256 each, each with its own bins
    (32 or 16 log-spaced, 1e14..1e18 Hz), in one persistent launch of the
    spectral kernel (autotuned chunk schedule) against the same cameras as 8
    separate spectral launches. Both are the FP64 form."""
    cams, bins = [], []
    for spin in (0.5, 0.9):
        for k, inc in enumerate((60.0, 70.0, 80.0, 85.0)):
            cams.append(G.config_params(3, width=256, height=256, spin=spin, observer_theta=math.radians(inc)))
            bins.append(G.log_bins(1e14, 1e18, 32 if k % 2 == 0 else 16))
    B = G.Batch(cams, freqs=bins)
    cache = os.path.join(ROOT, "_build", "batch_schedule_cache.jsonl")
    os.makedirs(os.path.dirname(cache), exist_ok=True)
    tuned = B.autotune(cache)
    total = B.spectral_offset(len(cams))
    out = torch.empty((total,), dtype=torch.float64, device="cuda")
    Rs = [G.Renderer(c, freqs=f) for c, f in zip(cams, bins)]
    bufs = [torch.empty((256, 256, len(f)), dtype=torch.float64, device="cuda") for f in bins]

    def timed(fn):
        for _ in range(max(1, args.warmup)):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    ms = timed(lambda: B.render_spectral_device(out, stream))

    def separate():
        for R, b in zip(Rs, bufs):
            R.render_spectral_device(b, 256, 256, None, stream)
    sep = timed(separate)
    st = B.stats()
    sched = dict(zip(("chunk", "order", "blocks_per_sm"), B.schedule()))
    for R in Rs:
        R.close()
    B.close()
    pf = sum(256 * 256 * len(f) for f in bins)
    return {"workload": "8 volumetric cameras (spins 0.5, 0.9 x 60/70/80/85 deg), 256x256, 32 or 16 bins",
            "ms_per_step": ms, "pixel_freq_per_s": pf / (ms * 1e-3), "separate_launches_ms_per_step": sep,
            "batched_speedup": sep / ms, "autotune_ms": tuned,
            "schedule": sched, "rays": st["rays"], "statistic": "median of the timed steps"}


def sgemm_peak(torch) -> float:
    """FP32 (non-tensor) roofline denominator: cuBLAS SGEMM 8192^3 with TF32 off, best of 5."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, dtype=torch.float32, device="cuda")
    b = torch.randn(n, n, dtype=torch.float32, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    torch.cuda.empty_cache()
    return best


# One forward pass of the surrogate MLP per sample, algorithmic FLOPs:
# 2 x (4 x 256 + 3 x 256 x 256 + 256 x 9) multiply-adds (9 outputs used).
F_MLP = 2 * (4 * 256 + 3 * 256 * 256 + 256 * 9)


def run_surrogate(args, torch, G, stream, flush, peaks):
    """Learned surrogate: trained here on the 64-camera sweep (4 spins x 16
    inclinations, 512^2 samples each, black background) by the library's own
    kernels, calibrated on the same cameras at 256^2 (other jitter), then
    timed on its evaluation frame (Kerr a=0.998, 80 deg, thin disk, 1 spp,
    black background) against the FP64 and mixed forms of the same frame."""
    n = args.surrogate_size
    cams = [dict(c, background_type=0) for c in G.sweep_cameras(width=512, height=512)]
    S = G.Surrogate(11)
    t = time.perf_counter()
    S.generate(cams, 512)
    t_gen = time.perf_counter() - t
    t = time.perf_counter()
    hist = S.train(args.surrogate_steps, batch=16384, lr=1e-3)
    t_train = time.perf_counter() - t
    cal = S.calibrate(cams, 256)
    frame = G.config_params(2, width=n, height=n, spp=1, background_type=0)
    R = G.Renderer(frame)
    ref = torch.empty((n, n, 3), dtype=torch.float64, device="cuda")
    rfate = torch.empty((n * n,), dtype=torch.int32, device="cuda")
    out = torch.empty_like(ref)
    ofate = torch.empty_like(rfate)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.mean(ts))

    R.set_precision(G.FORM_FP64)
    ms_fp64 = timed(lambda: R.render_device(None, ref, rfate, stream))
    st64 = R.stats()
    R.set_precision(G.FORM_MIXED)
    mix = torch.empty_like(ref)
    ms_mixed = timed(lambda: R.render_device(None, mix, None, stream))
    ms_surr = timed(lambda: S.render_device(R, None, out, ofate, stream))
    phases = R.phase_ms()
    st = R.stats()
    exact, samples = S.last_exact()
    # network alone on the frame's sample count (CUDA events around the fused kernel)
    xin = torch.rand((n * n, 4), device="cuda") * 2 - 1
    xo = torch.empty((n * n, 16), device="cuda")
    S.forward(xin, xo, n * n)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    S.forward(xin, xo, n * n)
    e1.record()
    torch.cuda.synchronize()
    ms_mlp = e0.elapsed_time(e1)
    a, b = out.cpu().numpy(), ref.cpu().numpy()
    scale = float(b.max())
    rel = (np.abs(a - b) / np.maximum(np.abs(b), 1e-6 * scale)).max(axis=2)
    lit = b.max(axis=2) > 1e-6 * scale
    fates_fp64 = rfate.cpu().numpy()
    # the default operating point's fates and routing, read before the sweep
    # below reuses the output buffers
    fates_diff = int(np.sum(ofate.cpu().numpy() != fates_fp64))
    speculated = S.last_counts()["speculated"]
    # Speed against colour error. Which samples the network decides is set by
    # the calibrated bands (the u error band in multiples of each sample's
    # predicted sigma, the critical-curve and graze bands around the
    # closed-form classification) and the colour tolerance tol_rel (a lit
    # sample is shaded by the network when its crossing band moves the colour
    # by at most tol_rel); the rest are re-traced in FP64. The sweep narrows
    # the bands by a factor and widens tol_rel. Errors are against the FP64
    # form, on lit pixels (colour above 1e-6 x the frame maximum), so they are
    # the network's own errors on the samples it decides.
    bands0 = S.bands()
    pareto = []
    for shrink, tol in ((1.0, 1e-3), (1.0, 1e-2), (0.5, 1e-3), (0.5, 1e-2), (0.25, 1e-2), (0.1, 1e-2),
                        (0.1, 1e-1)):
        S.set_bands(bands0["du"] * shrink, bands0["dir"] * shrink, bands0["capture"] * shrink,
                    bands0["graze"] * shrink, tol)
        ms_t = timed(lambda: S.render_device(R, None, out, ofate, stream))
        c_t = S.last_counts()
        o_t = out.cpu().numpy()
        rel_t = (np.abs(o_t - b) / np.maximum(np.abs(b), 1e-6 * scale)).max(axis=2)
        pareto.append({"band_scale": shrink, "tol_rel": tol, "ms_per_step": ms_t, "speedup_vs_fp64": ms_fp64 / ms_t,
                       "exact_fraction": c_t["exact"] / max(1, c_t["samples"]),
                       "lit_rel_quantiles_50_90_99_100": [float(x) for x in
                                                          np.quantile(rel_t[lit], [0.5, 0.9, 0.99, 1.0])],
                       "pixels_over_1e-3": int((rel_t > 1e-3).sum()),
                       "pixels_over_1e-2": int((rel_t > 1e-2).sum()),
                       "sample_fates_differing": int(np.sum(ofate.cpu().numpy() != fates_fp64))})
    S.set_bands(bands0["du"], bands0["dir"], bands0["capture"], bands0["graze"], bands0["tol_rel"])
    mlp_tflops = F_MLP * n * n / (ms_mlp * 1e-3) / 1e12
    peak = peaks.get("bf16_tflops")
    rays = n * n
    return {
        "config": {"workload": f"kerr_a0.998_80deg_{n}x{n}_1spp_thin_disk_isco_20M_black_background",
                   "rays_per_step": rays, "training": "64 cameras (spins 0, 0.5, 0.9, 0.998 x 16 inclinations "
                   "5..90 deg) x 512^2 samples traced by the FP64 form", "train_steps": args.surrogate_steps,
                   "batch": 16384, "l2": "flushed between steps (256 MiB write)"},
        "value": rays / (ms_surr * 1e-3), "unit": "rays/s", "ms_per_step": ms_surr,
        "fp64": {"value": rays / (ms_fp64 * 1e-3), "ms_per_step": ms_fp64},
        "mixed": {"value": rays / (ms_mixed * 1e-3), "ms_per_step": ms_mixed},
        "speedup_vs_fp64": ms_fp64 / ms_surr, "speedup_vs_mixed": ms_mixed / ms_surr,
        "phase_ms": {"network_and_shading": phases[0], "fp32_speculation": phases[1], "exact_retrace": phases[2],
                     "resolve": phases[3]},
        "exact_fraction": exact / max(1, samples),
        "speculated_fraction": speculated / max(1, samples),
        "attempts": {"surrogate": st["attempts"], "fp64": st64["attempts"]},
        "error_vs_fp64": {"max_rel": float(rel.max()), "pixels_over_1e-3": int((rel > 1e-3).sum()),
                          "lit_pixels": int(lit.sum()),
                          "lit_rel_quantiles_50_99_100": [float(x) for x in np.quantile(rel[lit], [0.5, 0.99, 1.0])],
                          "sample_fates_differing": fates_diff,
                          "rel_floor": "max(|fp64|, 1e-6 x frame max)"},
        "calibration": cal,
        "colour_tolerance_pareto": pareto,
        "train": {"seconds": t_train, "generate_seconds": t_gen, "loss_first": float(np.mean(hist[:20])),
                  "loss_last": float(np.mean(hist[-20:])),
                  "samples_per_s": args.surrogate_steps * 16384 / t_train,
                  "tflops": 3 * F_MLP * 16384 * args.surrogate_steps / t_train / 1e12},
        "mlp_roofline": {"kernel": "mlp_fused_kernel", "bound": "tensor", "achieved": mlp_tflops,
                         "peak": peak, "unit": "TFLOP/s", "frac": (mlp_tflops / peak) if peak else None,
                         "launch_ms": ms_mlp, "flops_per_launch": F_MLP * rays,
                         "flop_count": f"{F_MLP} per sample (4x256 + 3x256x256 + 256x9 multiply-adds, x2) x {rays}",
                         "peak_source": (f"{peaks.get('source')} bf16_tflops (cuBLAS bf16 burst)"
                                         + ("" if peaks.get("source") == "MEASURED_PEAKS.json" else
                                            ", of fallback: MEASURED_PEAKS.json absent"))},
        "gpu_launches_per_step": 6,
    }


def main():
    global W, H, RAYS, WORKLOAD
    args = parse()
    if args.batch:
        run_batch(args)
        return
    if args.volumetric:
        # the volumetric spectral render alone (one GPU), as its own JSON line
        import torch
        import grrt_b200 as G
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        stream = torch.cuda.Stream()
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        p64 = measured_peaks(torch)["fp64_tflops_dgemm"]
        clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
        clocks.start()
        res = run_volumetric(args, torch, G, stream, flush, p64)
        res["clocks"] = clocks.stop()
        res.update(n_gpus=1, steps=args.steps, warmup=args.warmup, unit="pixel*frequency/s",
                   higher_is_better=True, data="synthetic", dtype="f32+f64",
                   # mixed form per frame: speculation, the longest-first ordering's three kernels,
                   # re-trace, resolve
                   gpu_launches=args.steps * 6)
        print(json.dumps(res), flush=True)
        return
    if (args.width, args.height) != (W, H):
        W, H = args.width, args.height
        RAYS = W * H * SPP
        WORKLOAD = WORKLOAD.replace("1024x1024", f"{W}x{H}")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args)
        return
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    import grrt_b200 as G

    params = G.config_params(2, width=W, height=H)
    R = G.Renderer(params)
    stream = torch.cuda.Stream()
    rgba = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    rows = args.shard == "rows"
    if rows:
        # this rank's interleaved rows of the one frame, then the all-gather
        row0, row_step, n_rows = G.multi.shard_rows(H, world, rank)
        part = torch.empty((n_rows, W, 4), dtype=torch.float32, device="cuda")

        def render():
            R.render_rows_device(row0, row_step, n_rows, part, None, None, stream)
            return G.multi.gather_frame(part, H, dist, world) if world > 1 else part
        my_rays = n_rows * W * SPP
        frames_per_step = 1
    else:
        def render():
            R.render_device(rgba, None, None, stream)
            return rgba
        my_rays = RAYS
        frames_per_step = world

    head_form = G.FORM_MIXED if args.form == "mixed" else G.FORM_FP64
    other_form = G.FORM_FP64 if head_form == G.FORM_MIXED else G.FORM_MIXED
    clocks = ClockSampler(local)
    clocks.start()
    res = {other_form: time_form(torch, R, other_form, stream, flush, render, args.steps, args.warmup, dist),
           head_form: time_form(torch, R, head_form, stream, flush, render, args.steps, args.warmup, dist)}
    clk = clocks.stop()
    head = res[head_form]
    ms = head["ms"]
    value = frames_per_step * RAYS / (ms * 1e-3)

    # end to end, headline form: whole frames through the reference C entry
    # point (host framebuffer); with rows sharded, each rank's rows, the
    # all-gather and rank 0's copy of the frame to the host
    # The framebuffer is page-locked host memory (the library copies into it
    # directly); the same call into pageable memory (numpy) is timed beside it.
    import ctypes as C
    L = G.lib()
    host_pinned = torch.empty((H, W, 4), dtype=torch.float32).pin_memory()
    host_pageable = np.empty((H, W, 4), dtype=np.float32)

    def e2e_frame(fb_t, fbp):
        if rows:
            with torch.cuda.stream(stream):
                frame = render()
            stream.synchronize()
            if rank == 0:
                fb_t.copy_(frame.reshape(fb_t.shape))
        else:
            rc = L.grrt_render(R.ctx, fbp)
            assert rc == 0, L.grrt_error(R.ctx)

    def e2e_time(fb_t, fbp):
        for _ in range(2):
            e2e_frame(fb_t, fbp)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = time.perf_counter()
        n_e2e = max(3, args.steps // 2)
        for _ in range(n_e2e):
            e2e_frame(fb_t, fbp)
        t = (time.perf_counter() - e0) / n_e2e
        if dist:
            t = G.multi.max_over_ranks(t, dist, "cuda")
        return t

    e2e_s = e2e_time(host_pinned, C.cast(host_pinned.data_ptr(), C.POINTER(C.c_float)))
    e2e_pageable_s = e2e_time(torch.from_numpy(host_pageable),
                              host_pageable.ctypes.data_as(C.POINTER(C.c_float)))
    e2e = {"value": frames_per_step * RAYS / e2e_s, "unit": "rays/s",
           "h2d_bytes_per_step": 1536,  # launch parameters (scene description) per frame
           "d2h_bytes_per_step": W * H * 16,  # float RGBA frame
           "api": ("grrt_render_rows_device + all-gather + copy to host" if rows
                   else "grrt_render(ctx, float* host_framebuffer)"),
           "host_buffer": "page-locked (pinned)",
           "form": args.form, "ms_per_step": 1e3 * e2e_s,
           "pageable": {"value": frames_per_step * RAYS / e2e_pageable_s, "ms_per_step": 1e3 * e2e_pageable_s}}

    if rank == 0:
        peaks = measured_peaks(torch)
        p64 = peaks["fp64_tflops_dgemm"]
        p32 = sgemm_peak(torch)
        forms = {}
        for name, form in (("fp64", G.FORM_FP64), ("mixed", G.FORM_MIXED)):
            r = res[form]
            st = r["stats"]
            forms[name] = {"value": frames_per_step * RAYS / (r["ms"] * 1e-3), "unit": "rays/s",
                           "ms_per_step": r["ms"],
                           "phase_ms": r["phase_ms"], "attempts_per_ray": st["attempts"] / my_rays,
                           "fp64_attempt_share": st["fp64_attempts"] / max(1, st["attempts"])}
        # FP64 form: fp64_trace_kernel (phase 0; phase 1 is the resolve), FP64
        # FLOPs against the DGEMM peak
        st64 = res[G.FORM_FP64]["stats"]
        fl64 = st64["attempts"] * F_ATTEMPT_EXEC + my_rays * F_EVAL
        a64 = fl64 / (res[G.FORM_FP64]["phase_ms"][0] * 1e-3) / 1e12
        forms["fp64"]["roofline"] = {"kernel": "fp64_trace_kernel<false, false>", "bound": "fp64", "achieved": a64,
                                     "peak": p64, "unit": "TFLOP/s", "frac": a64 / p64}
        e64 = st64["attempts"] * F_EXEC_FP64_ATTEMPT / (res[G.FORM_FP64]["phase_ms"][0] * 1e-3) / 1e12
        forms["fp64"]["roofline_executed"] = {
            "kernel": "fp64_trace_kernel<false, false>", "bound": "fp64", "achieved": e64, "peak": p64, "unit": "TFLOP/s",
            "frac": e64 / p64, "flop_count": f"{F_EXEC_FP64_ATTEMPT} executed FP64 flop per attempt (ncu counters)"}
        # mixed form: the speculation kernel (FP32 FLOPs vs the SGEMM peak) and
        # the re-trace kernel (FP64 FLOPs vs the DGEMM peak)
        stm = res[G.FORM_MIXED]["stats"]
        ph = res[G.FORM_MIXED]["phase_ms"]
        spec_att = stm["attempts"] - stm["fp64_attempts"]
        a_spec = (spec_att * F_ATTEMPT_EXEC + my_rays * F_EVAL) / (ph[0] * 1e-3) / 1e12
        a_re = stm["fp64_attempts"] * F_ATTEMPT_EXEC / (ph[2] * 1e-3) / 1e12
        forms["mixed"]["phases"] = ["mixed_speculate_kernel", "mixed_star_kernel", "fp64_trace_kernel<true, false>",
                                    "mixed_resolve_kernel"]
        forms["mixed"]["roofline"] = {
            "speculate": {"bound": "fp32", "achieved": a_spec, "peak": p32, "unit": "TFLOP/s", "frac": a_spec / p32},
            "retrace": {"bound": "fp64", "achieved": a_re, "peak": p64, "unit": "TFLOP/s", "frac": a_re / p64}}
        x_spec = spec_att * F_EXEC_FP32_ATTEMPT / (ph[0] * 1e-3) / 1e12
        x_re = stm["fp64_attempts"] * F_EXEC_FP64_ATTEMPT / (ph[2] * 1e-3) / 1e12
        forms["mixed"]["roofline_executed"] = {
            "speculate": {"bound": "fp32", "achieved": x_spec, "peak": p32, "unit": "TFLOP/s", "frac": x_spec / p32,
                          "flop_count": f"{F_EXEC_FP32_ATTEMPT} executed FP32 flop per attempt (ncu; lower bound)"},
            "retrace": {"bound": "fp64", "achieved": x_re, "peak": p64, "unit": "TFLOP/s", "frac": x_re / p64,
                        "flop_count": f"{F_EXEC_FP64_ATTEMPT} executed FP64 flop per attempt (ncu counters)"}}
        if head_form == G.FORM_MIXED:
            roof = dict(forms["mixed"]["roofline"]["speculate"])
            roof.update(kernel="mixed_speculate_kernel", flops_per_launch=spec_att * F_ATTEMPT_EXEC + my_rays * F_EVAL,
                        flop_count=f"{F_ATTEMPT_EXEC} per DP45 attempt (FP32 stages, first right-hand side kept "
                                   f"from the previous attempt) x {spec_att} speculative attempts (device counter) "
                                   f"+ {F_EVAL} per ray",
                        peak_source="cuBLAS SGEMM 8192^3, TF32 off, measured in this run (best of 5); "
                                    "MEASURED_PEAKS.json has no FP32 figure",
                        launch_ms=ph[0], executed=forms["mixed"]["roofline_executed"]["speculate"],
                        # DRAM bytes of one full-size launch: profiles/ (ncu, a single-pass metric pair)
                        traffic=TRAFFIC_SPECULATE_C2)
            launches = args.steps * (4 if params["background_type"] == G.BG_STARS else 3)
        else:
            roof = dict(forms["fp64"]["roofline"])
            roof.update(flops_per_launch=fl64, flop_count=f"{F_ATTEMPT_EXEC} per DP45 attempt (first right-hand "
                                                          f"side kept from the previous attempt) x {st64['attempts']} "
                                                          f"attempts (device counter) + {F_EVAL} per ray",
                        peak_source="cuBLAS FP64 GEMM 8192^3 measured in this run (best of 5); MEASURED_PEAKS.json "
                                    "has no FP64 figure", traffic=None)
            launches = args.steps
        err = form_error(torch, G, params)
        cpu = None
        if not args.no_cpu_baseline and world == 1:  # the CPU baseline is taken at N = 1 only
            try:
                rays, secs, threads, kind, _n_rows = cpu_reference_sample(0, 16)
                cpu = {"value": rays / secs, "unit": "rays/s", "cores": threads, "kind": "reference",
                       "sample": f"rows 0,16,...,1008 of the 1024x1024 4-spp frame ({rays} rays), reference "
                                 f"src/*.cpp ({kind} build) via oracle/_ref, OpenMP, {secs:.2f} s"}
            except Exception as ex:  # the baseline is reported, not required
                cpu = {"value": None, "unit": "rays/s", "cores": os.cpu_count(), "kind": "reference",
                       "sample": f"unavailable: {ex}"}
        line = {"metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "strong" if rows else "weak",
                "vs_baseline": None, "dtype": "f64" if head_form == G.FORM_FP64 else "f32+f64",
                "data": "synthetic",
                "config": {"workload": WORKLOAD, "width": W, "height": H, "spp": SPP, "rays_per_step": RAYS,
                           "form": args.form, "l2": "flushed between steps (256 MiB write)",
                           "parallelism": (f"one frame split by interleaved rows over {world} GPU, one "
                                           f"all-gather per frame" if rows
                                           else f"one frame per GPU per step ({world} GPU)")},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
                "gpu_launches": launches, "forms": forms,
                "speedup_mixed_vs_fp64": forms["mixed"]["value"] / forms["fp64"]["value"],
                "mixed_error_vs_fp64": err,
                "work": {"attempts_per_ray": head["stats"]["attempts"] / my_rays,
                         "accepted_per_ray": head["stats"]["accepted"] / my_rays,
                         "crossings": head["stats"]["crossings"],
                         "fp64_attempt_share": head["stats"]["fp64_attempts"] / max(1, head["stats"]["attempts"])},
                "kernel_ms_per_step": head["kernel_ms"], "wall_s_timed_region": head["wall"]}
        # the single-GPU sections run at N = 1 only (the other ranks would wait
        # for them at the closing barrier)
        if not args.no_volumetric and world == 1:
            try:
                line["volumetric"] = run_volumetric(args, torch, G, stream, flush, p64)
            except Exception as ex:  # reported, the headline stands on its own
                line["volumetric"] = {"error": str(ex)}
        if args.surrogate_steps > 0 and world == 1:
            try:
                line["surrogate"] = run_surrogate(args, torch, G, stream, flush, peaks)
            except Exception as ex:  # reported, the headline stands on its own
                line["surrogate"] = {"error": str(ex)}
        if not args.no_batch_section and world == 1:
            try:
                line["batch"] = batch_section(args, torch, G, stream, flush, "mixed")
            except Exception as ex:  # reported, the headline stands on its own
                line["batch"] = {"error": str(ex)}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
