"""grrt_render_spectral_device_noalloc: the spectral render for callers that
may not allocate device memory while rendering (a host with a fixed device
memory budget that forbids driver allocations during a frame, or a process
near the memory limit). Its scratch is a fixed array inside libgrrt.so
instead of cudaMalloc'd memory.

Checked through the C ABI against grrt_render_spectral_device, the entry
point that allocates its scratch, on two calls in a row (the shared array
keeps the previous call's contents, so the second call also shows that the
entry point resets what must start at zero). Tolerance: the parity tests'
1e-9 relative (both run the same kernel, so the values are expected equal).
This file runs last in the suite and needs nothing the other tests set up.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-9


def test_noalloc_spectral_matches_allocating_entry_point(grrt, need_gpu):
    import torch

    freqs = grrt.log_bins(1e14, 1e18, 32)
    W, H = 64, 48
    R = grrt.Renderer(grrt.config_params(3, width=W, height=H), freqs=freqs)
    nb = len(freqs)
    # existing entry point (it also moves the scene to the device)
    want = torch.full((H, W, nb), float("nan"), dtype=torch.float64, device="cuda")
    R.render_spectral_device(want, W, H)
    torch.cuda.synchronize()
    want = want.cpu().numpy()
    assert np.isfinite(want).all() and (want > 0).any()

    d_freqs = torch.tensor(freqs, dtype=torch.float64, device="cuda")
    for call in range(2):
        got = torch.full((H, W, nb), float("nan"), dtype=torch.float64, device="cuda")
        R.render_spectral_device_noalloc(d_freqs, nb, got, W, H)
        torch.cuda.synchronize()
        got = got.cpu().numpy()
        err = np.abs(got - want) / np.maximum(np.abs(want), 1e-300)
        assert np.all(err <= TOL), f"call {call}: max relative difference {err.max():.3e}"


def test_noalloc_rejects_beyond_its_limits(grrt, need_gpu):
    import torch

    freqs = grrt.log_bins(1e14, 1e18, 33)
    R = grrt.Renderer(grrt.config_params(3, width=16, height=16), freqs=freqs)
    L = grrt.lib()
    d_freqs = torch.tensor(freqs, dtype=torch.float64, device="cuda")
    out = torch.zeros((16, 16, 33), dtype=torch.float64, device="cuda")
    # the scene is not on the device before the first render of this context
    rc = L.grrt_render_spectral_device_noalloc(R.ctx, d_freqs.data_ptr(), 32, out.data_ptr(), 16, 16, None)
    assert rc == -1 and b"not on the device" in L.grrt_error(R.ctx)
    R.render_spectral_device(out, 16, 16)
    torch.cuda.synchronize()
    rc = L.grrt_render_spectral_device_noalloc(R.ctx, d_freqs.data_ptr(), 33, out.data_ptr(), 16, 16, None)
    assert rc == -1 and b"num_bins must be 1..32" in L.grrt_error(R.ctx)


@pytest.mark.parametrize("case", ["no_bins", "null_freqs", "null_spec", "zero_width", "negative_height"])
def test_noalloc_rejects_bad_arguments(grrt, need_gpu, case):
    import torch

    freqs = grrt.log_bins(1e14, 1e18, 8)
    R = grrt.Renderer(grrt.config_params(3, width=16, height=16), freqs=freqs)
    L = grrt.lib()
    d_freqs = torch.tensor(freqs, dtype=torch.float64, device="cuda")
    out = torch.zeros((16, 16, 8), dtype=torch.float64, device="cuda")
    R.render_spectral_device(out, 16, 16)
    torch.cuda.synchronize()
    args = dict(f=d_freqs.data_ptr(), nb=8, s=out.data_ptr(), w=16, h=16)
    want = b"bad buffer or size"
    if case == "no_bins":
        args["nb"], want = 0, b"num_bins must be 1..32"
    elif case == "null_freqs":
        args["f"] = None
    elif case == "null_spec":
        args["s"] = None
    elif case == "zero_width":
        args["w"] = 0
    else:
        args["h"] = -3
    rc = L.grrt_render_spectral_device_noalloc(R.ctx, args["f"], args["nb"], args["s"], args["w"], args["h"], None)
    assert rc == -1 and want in L.grrt_error(R.ctx)


def test_noalloc_without_volumetric_disk_gives_zeros(grrt, need_gpu):
    """As grrt_render_spectral_device (and the reference) does for a thin-disk scene."""
    import torch

    freqs = grrt.log_bins(1e14, 1e18, 4)
    R = grrt.Renderer(grrt.config_params(2, width=32, height=16), freqs=freqs)
    L = grrt.lib()
    d_freqs = torch.tensor(freqs, dtype=torch.float64, device="cuda")
    out = torch.full((16, 32, 4), float("nan"), dtype=torch.float64, device="cuda")
    R.render_spectral_device(out, 32, 16)  # uploads the scene; all zeros
    torch.cuda.synchronize()
    assert torch.all(out == 0.0)
    out.fill_(float("nan"))
    rc = L.grrt_render_spectral_device_noalloc(R.ctx, d_freqs.data_ptr(), 4, out.data_ptr(), 32, 16, None)
    torch.cuda.synchronize()
    assert rc == 0 and torch.all(out == 0.0)
