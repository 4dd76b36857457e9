"""grrt_render_rows_device: a rank's interleaved rows of a frame must equal
those rows of the full render bit for bit, in both precision forms and for a
volumetric scene, so a frame split across GPUs is the single-GPU frame."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg,form_name", [(2, "FORM_FP64"), (2, "FORM_MIXED"), (3, "FORM_FP64")])
def test_rows_equal_full_render(grrt, need_gpu, cfg, form_name):
    import torch
    W, H = 96, 80
    R = grrt.Renderer(grrt.config_params(cfg, width=W, height=H))
    R.set_precision(getattr(grrt, form_name))
    full = torch.full((H, W, 4), float("nan"), dtype=torch.float32, device="cuda")
    R.render_device(full)
    torch.cuda.synchronize()
    full = full.cpu().numpy()
    for world in (2, 3):
        for rank in range(world):
            row0, step, n = grrt.multi.shard_rows(H, world, rank)
            part = torch.full((n, W, 4), float("nan"), dtype=torch.float32, device="cuda")
            R.render_rows_device(row0, step, n, part)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(part.cpu().numpy(), full[row0::step], err_msg=f"rank {rank}/{world}")


def test_rows_outside_image_rejected(grrt, need_gpu):
    import torch
    R = grrt.Renderer(grrt.config_params(1, width=16, height=16))
    buf = torch.empty((16, 16, 4), dtype=torch.float32, device="cuda")
    with pytest.raises(RuntimeError, match="outside the image"):
        R.render_rows_device(1, 2, 9, buf)


@pytest.mark.parametrize("form_name", ["FORM_FP64", "FORM_MIXED"])
def test_spectral_rows_and_tiles_equal_full_render(grrt, need_gpu, form_name):
    """grrt_render_spectral_rows_device / _tile_device: a volumetric spectral
    frame split by interleaved rows (2 and 3 ranks) or cut into tiles equals
    the full render bit for bit, with the same per-sample fates."""
    import torch
    W, H, nb = 64, 48, 16
    freqs = grrt.log_bins(1e14, 1e18, nb)
    R = grrt.Renderer(grrt.config_params(3, width=W, height=H), freqs=freqs)
    R.set_precision(getattr(grrt, form_name))
    full = torch.full((H, W, nb), float("nan"), dtype=torch.float64, device="cuda")
    ffate = torch.full((H * W,), -1, dtype=torch.int32, device="cuda")
    R.render_spectral_device(full, W, H, ffate)
    torch.cuda.synchronize()
    full, ffate = full.cpu().numpy(), ffate.cpu().numpy().reshape(H, W)
    assert (full > 0).any()
    for world in (2, 3):
        for rank in range(world):
            row0, step, n = grrt.multi.shard_rows(H, world, rank)
            part = torch.full((n, W, nb), float("nan"), dtype=torch.float64, device="cuda")
            pf = torch.full((n * W,), -1, dtype=torch.int32, device="cuda")
            R.render_spectral_rows_device(row0, step, n, part, pf)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(part.cpu().numpy(), full[row0::step], err_msg=f"rank {rank}/{world}")
            np.testing.assert_array_equal(pf.cpu().numpy().reshape(n, W), ffate[row0::step])
    for (x, y, w, h) in [(0, 0, W, H), (5, 7, 17, 9), (W - 1, H - 1, 1, 1), (30, 20, 1, 1)]:
        t = torch.full((h, w, nb), float("nan"), dtype=torch.float64, device="cuda")
        R.render_spectral_tile_device(x, y, w, h, t)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(t.cpu().numpy(), full[y:y + h, x:x + w], err_msg=f"tile {x},{y},{w},{h}")
    buf = torch.empty((4, W, nb), dtype=torch.float64, device="cuda")
    with pytest.raises(RuntimeError, match="outside the image"):
        R.render_spectral_rows_device(1, 16, 4, buf)
    with pytest.raises(RuntimeError, match="outside the image"):
        R.render_spectral_tile_device(60, 0, 5, 1, buf)
