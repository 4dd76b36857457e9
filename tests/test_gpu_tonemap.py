"""grrt_tonemap_device against the host grrt_tonemap (the reference's
ToneMapper::apply_all, src/tonemapper.cpp:7-71) on a rendered frame: the log
sum is grouped by blocks on the device and the functions are CUDA's, so the
two agree to a few float ulp; an all-black frame is left as it is."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_device_tonemap_matches_host(grrt, need_gpu):
    import torch
    R = grrt.Renderer(grrt.config_params(2, width=96, height=80))
    frame = R.render()
    host = np.ascontiguousarray(frame.copy())
    grrt.lib().grrt_tonemap(host.ctypes.data_as(C.POINTER(C.c_float)), 96, 80)
    d = torch.from_numpy(np.ascontiguousarray(frame)).cuda()
    grrt.tonemap_device(d, 96, 80)
    torch.cuda.synchronize()
    got = d.cpu().numpy()
    assert not np.array_equal(host, frame)  # the host map changed the frame
    np.testing.assert_array_equal(got[..., 3], frame[..., 3])
    diff = np.abs(got - host)
    print(f"\n  max |device - host| {diff.max():.2e}; values differing {int(np.sum(diff > 0))} of {diff.size}")
    assert diff.max() <= 4e-7


def test_device_tonemap_leaves_black_frame(grrt, need_gpu):
    import torch
    d = torch.zeros((16, 16, 4), dtype=torch.float32, device="cuda")
    d[..., 3] = 1.0
    grrt.tonemap_device(d, 16, 16)
    torch.cuda.synchronize()
    assert torch.equal(d[..., :3], torch.zeros((16, 16, 3), device="cuda"))
