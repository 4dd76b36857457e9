"""The batched form (grrt_batch_*): one persistent launch over many cameras
must reproduce every camera's own render exactly (same kernel arithmetic per
pixel; only the order lanes take pixels in differs), for every schedule, and
through the CUDA-graph replay."""
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
    for order in (B.ORDER_ROUND_ROBIN, B.ORDER_CAMERA_MAJOR):
        for chunk in (1, 37, 256, 100000):
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


def test_batch_rejects_volumetric(grrt):
    cams = [grrt.config_params(3, width=16, height=16)]
    with pytest.raises(RuntimeError, match="thin-disk"):
        grrt.Batch(cams)
