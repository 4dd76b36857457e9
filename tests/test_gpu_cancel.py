"""grrt_cancel and grrt_progress, driven from the host.

The reference's CPU versions are stubs (src/api.cpp:220-231: cancel does
nothing, progress returns 1.0); its CUDA backend cancels through a host-mapped
flag (cuda/cuda_backend.cu:31-34). Here a cancel raises a host-mapped flag,
which the volumetric kernels poll every 1024 loop iterations per warp, and
pushes the running launch's work counters past every work index with a
copy-engine write, so the thin-disk and mixed kernels take no new work. The
progress callback fires on the calling thread while the render runs.

No device fault is involved: the cancel is a plain host write that the
kernels read and then return early.
"""
import threading
import time

import ctypes as C
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fb(R):
    return np.zeros((R.height, R.width, 4), dtype=np.float32)


def _ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _render_cancelled_from_thread(grrt, R):
    """Start a render with a progress callback on this thread; another thread
    calls grrt_cancel once the first progress report has arrived."""
    L = grrt.lib()
    started = threading.Event()
    seen = []

    def on_progress(f, user):
        seen.append(float(f))
        started.set()

    cb = grrt.PROGRESS_FN(on_progress)

    def canceller():
        if started.wait(10.0):
            L.grrt_cancel(R.ctx)

    th = threading.Thread(target=canceller)
    th.start()
    fb = _fb(R)
    t0 = time.perf_counter()
    rc = L.grrt_render_cb(R.ctx, _ptr(fb), cb, None)
    dt = time.perf_counter() - t0
    th.join()
    return rc, dt, seen


@pytest.mark.parametrize("form", ["fp64", "mixed"])
def test_cancel_from_another_thread(grrt, need_gpu, form):
    # 2048x2048 at 4 spp: ~0.16 s in the FP64 form, ~0.07 s mixed, so the
    # cancel lands while the kernels run
    vals = grrt.config_params(2, width=2048, height=2048)
    R = grrt.Renderer(vals)
    if form == "mixed":
        R.set_precision(grrt.FORM_MIXED)
    L = grrt.lib()
    R.render()  # warm-up: device tables, kernels loaded
    t0 = time.perf_counter()
    full = R.render()
    t_full = time.perf_counter() - t0
    rc, dt, seen = _render_cancelled_from_thread(grrt, R)
    print(f"\n  [{form}] full render {t_full * 1e3:.1f} ms; cancelled render returned after {dt * 1e3:.1f} ms "
          f"(progress reports before the cancel: {seen[:3]})")
    assert rc != 0, "the render was not cancelled"
    assert b"render cancelled" in L.grrt_error(R.ctx)
    assert seen and 0.0 < seen[0] < 1.0
    assert dt < 0.8 * t_full + 0.02, f"cancelled render took {dt:.3f} s against {t_full:.3f} s for a full one"
    # the context renders normally afterwards, bit for bit as a fresh one
    again = R.render()
    assert np.array_equal(again.view(np.uint32), full.view(np.uint32))
    F = grrt.Renderer(vals)
    if form == "mixed":
        F.set_precision(grrt.FORM_MIXED)
    assert np.array_equal(F.render().view(np.uint32), full.view(np.uint32))
    assert L.grrt_progress(R.ctx) == 1.0


def test_cancel_volumetric_spectral(grrt, need_gpu):
    """The spectral path polls the same flag (a 256x256 frame, 32 bins)."""
    freqs = grrt.log_bins(1e14, 1e18, 32)
    R = grrt.Renderer(grrt.config_params(3, width=256, height=256), freqs=freqs)
    L = grrt.lib()
    want = R.render_spectral()
    started = threading.Event()

    def on_progress(f, user):
        started.set()

    cb = grrt.PROGRESS_FN(on_progress)

    def canceller():
        if started.wait(10.0):
            L.grrt_cancel(R.ctx)

    th = threading.Thread(target=canceller)
    th.start()
    out = np.empty((256, 256, 32))
    rc = L.grrt_render_spectral_cb(R.ctx, out.ctypes.data_as(C.POINTER(C.c_double)), 256, 256, cb, None)
    th.join()
    assert rc != 0 and b"render cancelled" in L.grrt_error(R.ctx)
    assert np.array_equal(R.render_spectral(), want)


def test_progress_reports(grrt, need_gpu):
    """Progress values are monotone on the calling thread, end at 1.0, and
    grrt_progress reads 1.0 after a finished render (0.0 before any)."""
    R = grrt.Renderer(grrt.config_params(2, width=1024, height=1024))  # 4 spp
    L = grrt.lib()
    assert L.grrt_progress(R.ctx) == 0.0
    seen, threads = [], set()

    def on_progress(f, user):
        seen.append(float(f))
        threads.add(threading.get_ident())

    cb = grrt.PROGRESS_FN(on_progress)
    fb = _fb(R)
    assert L.grrt_render_cb(R.ctx, _ptr(fb), cb, None) == 0
    assert seen and seen[-1] == 1.0
    assert all(b >= a for a, b in zip(seen, seen[1:])), seen
    assert threads == {threading.get_ident()}, "progress must fire on the calling thread"
    assert L.grrt_progress(R.ctx) == 1.0
    # the callback's render equals the plain one
    assert np.array_equal(fb, R.render())
    # spectral renders report progress the same way
    freqs = grrt.log_bins(1e14, 1e18, 8)
    V = grrt.Renderer(grrt.config_params(3, width=128, height=128), freqs=freqs)
    seen.clear()
    out = np.empty((128, 128, 8))
    assert L.grrt_render_spectral_cb(V.ctx, out.ctypes.data_as(C.POINTER(C.c_double)), 128, 128, cb, None) == 0
    assert seen and seen[-1] == 1.0 and all(b >= a for a, b in zip(seen, seen[1:]))
    assert L.grrt_progress(V.ctx) == 1.0
