"""Host-buffer renders (grrt_render, grrt_render_spectral) against the same
frame rendered into device memory. Results of 4 MB or more reach the caller's
buffer through the library's pinned staging buffer, in chunks copied on the
host threads; the caller must get exactly the device result, also for sizes
that do not split evenly into the chunks, and on repeated calls (the staging
buffer is kept and grown)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,h", [(512, 512), (601, 499), (256, 128)], ids=["4MiB", "odd", "small"])
def test_host_render_equals_device_render(grrt, need_gpu, w, h):
    import torch
    R = grrt.Renderer(grrt.config_params(2, width=w, height=h, spp=1))
    R.set_precision(grrt.FORM_MIXED)
    dev = torch.full((h, w, 4), float("nan"), dtype=torch.float32, device="cuda")
    R.render_device(dev)
    torch.cuda.synchronize()
    want = dev.cpu().numpy()
    for _ in range(2):
        got = R.render()
        np.testing.assert_array_equal(got, want)


def test_host_spectral_render_equals_device_render(grrt, need_gpu):
    import torch
    freqs = grrt.log_bins(1e14, 1e18, 32)
    w, h = 160, 120  # 4.9 MB of doubles
    R = grrt.Renderer(grrt.config_params(3, width=w, height=h), freqs=freqs)
    dev = torch.full((h, w, len(freqs)), float("nan"), dtype=torch.float64, device="cuda")
    R.render_spectral_device(dev, w, h)
    torch.cuda.synchronize()
    want = dev.cpu().numpy()
    got = R.render_spectral()
    np.testing.assert_array_equal(got.reshape(want.shape), want)


def test_host_render_into_page_locked_buffer(grrt, need_gpu):
    """A page-locked framebuffer (here torch's pinned memory) takes one direct
    copy instead of the staging path; the caller still gets exactly the
    device result."""
    import ctypes as C
    import torch
    w, h = 601, 499
    R = grrt.Renderer(grrt.config_params(2, width=w, height=h, spp=1))
    R.set_precision(grrt.FORM_MIXED)
    dev = torch.full((h, w, 4), float("nan"), dtype=torch.float32, device="cuda")
    R.render_device(dev)
    torch.cuda.synchronize()
    want = dev.cpu().numpy()
    fb = torch.full((h, w, 4), float("nan"), dtype=torch.float32).pin_memory()
    L = grrt.lib()
    for _ in range(2):
        fb.fill_(float("nan"))
        rc = L.grrt_render(R.ctx, C.cast(fb.data_ptr(), C.POINTER(C.c_float)))
        assert rc == 0, L.grrt_error(R.ctx)
        np.testing.assert_array_equal(fb.numpy(), want)
