"""The batched form (grrt_batch_*): one persistent launch over many cameras
must reproduce every camera's own render exactly (same kernel arithmetic per
pixel; only the order lanes take pixels in differs), for every schedule, and
through the CUDA-graph replay: thin-disk cameras (RGB, both precision forms)
and volumetric cameras (spectra, each camera with its own bins)."""
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def small_sweep(grrt, n_spin=2, n_incl=4, w=48, h=40):
    spins = (0.0, 0.9, 0.5, 0.998)[:n_spin]
    return grrt.sweep_cameras(width=w, height=h, spins=spins, n_incl=n_incl)


def single_renders(grrt, cams):
    out = []
    for c in cams:
        R = grrt.Renderer(c)
        out.append(R.render())
        R.close()
    return out


def test_batch_equals_single_camera_renders(grrt, need_gpu):
    cams = small_sweep(grrt)
    cams[3] = dict(cams[3], samples_per_pixel=4, width=40, height=32)  # uneven sizes and spp
    want = single_renders(grrt, cams)
    B = grrt.Batch(cams)
    schedules = [(chunk, order) for order in (B.ORDER_ROUND_ROBIN, B.ORDER_CAMERA_MAJOR)
                 for chunk in (1, 37, 256, 100000)]
    schedules.append((256, B.ORDER_SAMPLES))  # traced by samples: the chunk size does not apply
    for chunk, order in schedules:
        B.set_schedule(chunk, order, 0)
        got = B.render()
        for k, (g, w) in enumerate(zip(got, want)):
            np.testing.assert_array_equal(g, w, err_msg=f"camera {k}, chunk {chunk}, order {order}")
    st = B.stats()
    assert st["rays"] == sum(c["width"] * c["height"] * (4 if c["samples_per_pixel"] == 4 else 1) for c in cams)


def test_batch_device_graph_replay_and_autotune(grrt, need_gpu):
    import torch
    cams = small_sweep(grrt, 2, 3)
    want = single_renders(grrt, cams)
    B = grrt.Batch(cams)
    with tempfile.TemporaryDirectory() as d:
        cache = os.path.join(d, "tune.jsonl")
        ms = B.autotune(cache)
        assert ms > 0
        sched = B.schedule()
        # a second batch with the same cameras reuses the cached schedule
        B2 = grrt.Batch(cams)
        assert B2.autotune(cache) == pytest.approx(ms)
        assert B2.schedule() == sched
    total = int(B.offsets[-1])
    buf = torch.full((total, 4), float("nan"), dtype=torch.float32, device="cuda")
    for _ in range(2):  # the second call replays the captured graph
        B.render_device(buf)
        torch.cuda.synchronize()
        got = buf.cpu().numpy()
        for k, w in enumerate(want):
            a, b = int(B.offsets[k]), int(B.offsets[k + 1])
            np.testing.assert_array_equal(got[a:b].reshape(w.shape), w)


def single_renders_form(grrt, cams, form):
    out = []
    for c in cams:
        R = grrt.Renderer(c)
        R.set_precision(form)
        out.append(R.render())
        R.close()
    return out


def test_batch_mixed_equals_single_mixed_renders(grrt, need_gpu):
    """Mixed form: the batch runs the mixed pipeline over one sample space of
    all cameras, so each camera's image equals its own mixed render bit for
    bit, for any schedule and through the graph replay; and it meets the mixed
    form's bar against the FP64 render (relative 1e-4)."""
    import torch
    cams = small_sweep(grrt)
    cams[3] = dict(cams[3], samples_per_pixel=4, width=40, height=32)  # uneven sizes and spp
    cams.append(grrt.config_params(1, width=36, height=44))           # a scene without stars
    want = single_renders_form(grrt, cams, grrt.FORM_MIXED)
    f64 = single_renders_form(grrt, cams, grrt.FORM_FP64)
    B = grrt.Batch(cams)
    B.set_precision(grrt.FORM_MIXED)
    for bp in (0, 1):
        B.set_schedule(256, B.ORDER_ROUND_ROBIN, bp)
        got = B.render()
        for k, (g, w) in enumerate(zip(got, want)):
            np.testing.assert_array_equal(g, w, err_msg=f"camera {k}, blocks/SM {bp}")
    st = B.stats()
    n_samples = sum(c["width"] * c["height"] * c.get("samples_per_pixel", 1) for c in cams)
    assert st["rays"] == n_samples
    assert st["horizon"] + st["escaped"] + st["max_steps"] == n_samples
    assert 0 < st["fp64_attempts"] < 0.5 * st["attempts"]
    for k, (g, f) in enumerate(zip(got, f64)):
        scale = float(np.max(f[..., :3]))
        rel = np.abs(g[..., :3] - f[..., :3]) / np.maximum(np.abs(f[..., :3]), 1e-6 * scale)
        assert float(rel.max()) <= 1e-4, f"camera {k}: {float(rel.max()):.2e} against the FP64 form"
    total = int(B.offsets[-1])
    buf = torch.full((total, 4), float("nan"), dtype=torch.float32, device="cuda")
    for _ in range(2):  # the second call replays the captured graph
        B.render_device(buf)
        torch.cuda.synchronize()
        g = buf.cpu().numpy()
        for k, w in enumerate(want):
            a, b = int(B.offsets[k]), int(B.offsets[k + 1])
            np.testing.assert_array_equal(g[a:b].reshape(w.shape), w)
    # switching back gives the FP64 images
    B.set_precision(grrt.FORM_FP64)
    for g, f in zip(B.render(), f64):
        np.testing.assert_array_equal(g, f)


def test_batch_tuning_knobs_and_autotune(grrt, need_gpu):
    """Threads per block leave the FP64 images unchanged; the mixed-form
    autotuner picks FP32 thresholds whose images still meet the bar against
    the FP64 render, and the cache restores every knob."""
    cams = small_sweep(grrt, 2, 3)
    f64 = single_renders_form(grrt, cams, grrt.FORM_FP64)
    B = grrt.Batch(cams)
    for block in (64, 256, 128):
        B.set_tuning(block=block)
        for g, f in zip(B.render(), f64):
            np.testing.assert_array_equal(g, f)
    with pytest.raises(RuntimeError, match="block must be"):
        B.set_tuning(block=96)
    with tempfile.TemporaryDirectory() as d:
        cache = os.path.join(d, "tune.jsonl")
        assert B.autotune(cache) > 0
        assert B.tuning()["block"] in (64, 128, 256)
        M = grrt.Batch(cams)
        M.set_precision(grrt.FORM_MIXED)
        ms = M.autotune(cache)
        tun = M.tuning()
        assert tun["tol_fp32"] in (1e-6, 3e-6, 1e-5) and tun["r_factor"] in (3.0, 4.0)
        for k, (g, f) in enumerate(zip(M.render(), f64)):
            scale = float(np.max(f[..., :3]))
            rel = np.abs(g[..., :3] - f[..., :3]) / np.maximum(np.abs(f[..., :3]), 1e-6 * scale)
            assert float(rel.max()) <= 1e-4, f"camera {k}"
        M2 = grrt.Batch(cams)
        M2.set_precision(grrt.FORM_MIXED)
        assert M2.autotune(cache) == pytest.approx(ms)
        assert M2.tuning() == tun and M2.schedule() == M.schedule()


def test_batch_rejects_mixed_disk_kinds(grrt):
    cams = [grrt.config_params(1, width=16, height=16), grrt.config_params(3, width=16, height=16)]
    with pytest.raises(RuntimeError, match="either volumetric cameras"):
        grrt.Batch(cams)


def volumetric_cameras(grrt):
    """Volumetric cameras of uneven sizes, spins, inclinations, spp and
    frequency sets."""
    import math
    cams = [grrt.config_params(3, width=40, height=32, spin=0.9),
            grrt.config_params(3, width=48, height=48, spin=0.5, observer_theta=math.radians(60.0)),
            grrt.config_params(3, width=24, height=20, spin=0.9, samples_per_pixel=4),
            grrt.config_params(3, width=36, height=28, spin=0.9, observer_theta=math.radians(85.0))]
    bins = [grrt.log_bins(1e14, 1e18, 32), grrt.log_bins(1e15, 1e17, 8), np.array([1e14, 3e15, 2e17]),
            grrt.log_bins(1e14, 1e18, 45)]
    return cams, bins


def test_spectral_batch_equals_single_renders(grrt, need_gpu):
    """A batch of volumetric cameras (each with its own bins) in one persistent
    launch: every camera's cube equals its own spectral render within 1e-9
    relative (the same arithmetic per ray; the batched kernel is compiled
    separately, so FMA contraction may differ in the last bits), for any
    schedule, through the host and device entry points and the graph replay;
    the autotuner picks a schedule."""
    import torch
    cams, bins = volumetric_cameras(grrt)
    want = []
    for c, f in zip(cams, bins):
        R = grrt.Renderer(c, freqs=f)
        want.append(R.render_spectral())
        R.close()
    # bins at creation widen each camera's opacity tables, as for a single context
    B0 = grrt.Batch([dict(c) for c in cams])
    with pytest.raises(RuntimeError, match="no frequency bins"):
        B0.render_spectral()
    B0.close()
    B = grrt.Batch([dict(c) for c in cams], freqs=bins)
    B.set_frequency_bins(grrt.log_bins(1e14, 1e18, 4))  # every camera, then per camera again
    for k, f in enumerate(bins):
        B.set_frequency_bins(f, k)
    for order in (B.ORDER_ROUND_ROBIN, B.ORDER_CAMERA_MAJOR):
        for chunk in (1, 64, 100000):
            B.set_schedule(chunk, order, 0)
            got = B.render_spectral()
            for k, (g, w) in enumerate(zip(got, want)):
                assert g.shape == w.shape
                # the batched kernel is its own instantiation: FMA contraction
                # may differ in the last bits (measured ~1e-13); the FP64 form's bar
                np.testing.assert_allclose(g, w, rtol=1e-9, atol=0.0,
                                           err_msg=f"camera {k}, chunk {chunk}, order {order}")
    st = B.stats()
    assert st["rays"] == sum(c["width"] * c["height"] * c["samples_per_pixel"] for c in cams)
    assert st["physics_steps"] > 0 and st["bin_updates"] > 0
    with tempfile.TemporaryDirectory() as d:
        assert B.autotune(os.path.join(d, "tune.jsonl")) > 0
    total = B.spectral_offset(len(cams))
    assert total == sum(w.size for w in want)
    buf = torch.full((total,), float("nan"), dtype=torch.float64, device="cuda")
    for _ in range(2):  # the second call replays the captured graph
        B.render_spectral_device(buf)
        torch.cuda.synchronize()
        g = buf.cpu().numpy()
        for k, w in enumerate(want):
            a, b = B.spectral_offset(k), B.spectral_offset(k + 1)
            np.testing.assert_allclose(g[a:b].reshape(w.shape), w, rtol=1e-9, atol=0.0)
    with pytest.raises(RuntimeError, match="volumetric cameras"):
        B.render()
