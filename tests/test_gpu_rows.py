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
