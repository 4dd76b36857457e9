"""Analytic cross-checks that do not go through the oracle.

Schwarzschild shadow (README.md:215 of the reference): a static observer at
radius r sees the hole's shadow as a disc of angular radius psi_c with
sin(psi_c) = 3*sqrt(3)*M/r * sqrt(1 - 2M/r) (Synge's formula; the README's
arcsin(3*sqrt(3)*M/r) is its large-r limit). The camera's ray for image-plane
angles (alpha, beta) (src/camera.cpp:69-96) makes the angle psi with the
direction to the hole, cos(psi) = cos(alpha) * cos(beta), so a sample must
fall into the horizon exactly when psi < psi_c.
"""
import math

import numpy as np
import pytest

import oracle_bind

pytestmark = pytest.mark.gpu


def test_schwarzschild_shadow_edge(grrt, need_gpu):
    import torch

    W = H = 256
    vals = grrt.config_params(1, width=W, height=H, disk_enabled=0)  # C1 geometry, no disk, black sky
    R = grrt.Renderer(vals)
    fate = torch.full((W * H,), -1, dtype=torch.int32, device="cuda")
    R.render_device(None, None, fate)
    torch.cuda.synchronize()
    term = (fate.cpu().numpy().view(np.uint32) & 3).astype(np.int64)
    px, py = oracle_bind.jittered_samples(W, H, 1, np.arange(W * H))
    fov, r_obs, M = vals["fov"], vals["observer_r"], vals["mass"]
    alpha = (px - W / 2.0) * fov / W
    beta = (py - H / 2.0) * fov / W
    psi = np.arccos(np.clip(np.cos(alpha) * np.cos(beta), -1.0, 1.0))
    psi_c = math.asin(3.0 * math.sqrt(3.0) * M / r_obs * math.sqrt(1.0 - 2.0 * M / r_obs))
    pix = fov / W  # one pixel, in radians
    inside, outside = psi[term == 0], psi[term == 1]
    assert len(inside) > 3000 and len(outside) > 3000
    assert np.count_nonzero(term == 2) < 10, "rays near the photon sphere hit the step budget"
    edge_in, edge_out = inside.max(), outside.min()
    edge = 0.5 * (edge_in + edge_out)
    print(f"\n  shadow edge: captured up to {edge_in:.7f}, escaping from {edge_out:.7f} rad; Synge "
          f"{psi_c:.7f} rad (edge - Synge = {(edge - psi_c) / pix:+.4f} px); README's large-r form "
          f"{math.asin(3 * math.sqrt(3) * M / r_obs):.7f} rad")
    # the captured and escaping samples are separated at psi_c, to a small
    # fraction of a pixel (the samples are jittered, so the gap is narrow)
    assert edge_in < psi_c < edge_out
    assert edge_out - edge_in < 0.2 * pix
    # the README's formula lies within one pixel
    assert abs(math.asin(3 * math.sqrt(3) * M / r_obs) - psi_c) < pix
