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
    assert len(inside) > 500 and len(outside) > 3000  # the shadow covers ~pi * 17^2 pixels
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


def hamiltonian_np(M, a, fin):
    """H = 1/2 g^{mu nu} p_mu p_nu of Boyer-Lindquist states (t, r, theta,
    phi, p_t, p_r, p_theta, p_phi), in the separable Kerr form."""
    r, th = fin[:, 1], fin[:, 2]
    pt, pr, pth, pph = fin[:, 4], fin[:, 5], fin[:, 6], fin[:, 7]
    s, c = np.sin(th), np.cos(th)
    s = np.where(np.abs(s) < 1e-10, np.where(s >= 0, 1e-10, -1e-10), s)
    sig = r * r + a * a * c * c
    dlt = r * r - 2 * M * r + a * a
    P = (r * r + a * a) * pt + a * pph
    Q = a * s * pt + pph / s
    return (dlt * pr * pr - P * P / dlt + pth * pth + Q * Q) / (2 * sig)


def test_hamiltonian_constraint(grrt, need_gpu):
    """|H| / p_t^2 at the final state of every sample that does not end at
    the horizon stays below 1e-7 (README.md:213; the reference's CUDA tests
    hold |H| < 1e-7 along a geodesic, cuda/tests/test_cuda.cu:385-402). The
    device reports the maximum over the frame (GRRTStats.hamiltonian_max,
    measured by the FP64 form's diagnostic instantiation, GRRT_DIAG_HAMILTONIAN,
    which renders the same image); the
    oracle's final states of the same samples give the same value. At the
    horizon stop (r_h + 0.01) Delta -> 0 and the P^2 / Delta term cancels, so
    the evaluation itself loses digits there (measured up to ~5e-4) and those
    samples are left out. Camera rays start null to 1e-10 (the reference's
    camera test)."""
    import torch
    from parity_util import OracleRGB

    W = H = 128
    R = grrt.Renderer(grrt.config_params(2, width=W, height=H, spp=1))  # Kerr a=0.998, stars
    rgb = torch.empty((H, W, 3), dtype=torch.float64, device="cuda")
    R.render_device(None, rgb, None)
    torch.cuda.synchronize()
    assert R.stats()["hamiltonian_max"] == 0.0  # measured by the diagnostic instantiation only
    plain = rgb.cpu().numpy()
    R.set_diagnostics(grrt.DIAG_HAMILTONIAN)
    R.render_device(None, rgb, None)
    torch.cuda.synchronize()
    h_dev = R.stats()["hamiltonian_max"]
    np.testing.assert_array_equal(rgb.cpu().numpy(), plain)  # the render itself is unchanged
    orc = OracleRGB(R, np.arange(W * H), 1e-9, band=False)
    M, a = R.table("scalars")[:2]
    h_orc = (np.abs(hamiltonian_np(M, a, orc.fin)) / orc.fin[:, 4] ** 2)[orc.term != 0]
    print(f"\n  max |H|/p_t^2 at the final states (not at the horizon): device {h_dev:.3e}, oracle "
          f"{h_orc.max():.3e} (oracle median {np.median(h_orc):.3e})")
    assert 0.0 < h_dev < 1e-7
    assert 0.5 * h_orc.max() <= h_dev <= 2.0 * h_orc.max()
    # camera rays are null
    px, py = oracle_bind.jittered_samples(W, H, 1, np.arange(0, W * H, 97))
    cam = np.array([R.camera_ray(x, y) for x, y in zip(px, py)])
    h_cam = np.abs(hamiltonian_np(M, a, cam)) / cam[:, 4] ** 2
    assert h_cam.max() < 1e-10, h_cam.max()
