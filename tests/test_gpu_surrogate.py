"""The learned surrogate on the GPU: its training kernels against the float64
CPU restatement (tests/mlp_ref.py), its training set against the oracle, and
what the trained network gains over the method without it.

Bars:
  * gradients: every parameter block within 1e-2 relative L2 of the
    restatement (which rounds to BF16 where the GPU stores BF16; the rest is
    FP32-accumulation rounding), cosine > 0.9999, loss within 1e-4;
  * forward (the fused inference kernel): outputs within 2e-3 (absolute +
    relative) of the restatement;
  * training set: every sample's termination equals the oracle's trace;
  * training: the loss falls by 10x;
  * render: sample fates equal the FP64 form's, every pixel within the
    colour budget (1e-3 relative), and the trained network integrates far less
    (DP45 attempts) than an untrained one with the same bands (the gain is the
    network's, not the fallback's).
"""
import math

import numpy as np
import pytest

import mlp_ref
from oracle_bind import Oracle, jittered_samples

pytestmark = pytest.mark.gpu


def test_gradients_match_float64_restatement(grrt, need_gpu):
    S = grrt.Surrogate(1)
    p = mlp_ref.random_params(7).astype(np.float32)
    S.set_params(p)
    X, Y = mlp_ref.random_batch(8, 256)
    X = X.astype(np.float32)
    Y = Y.astype(np.float32)
    loss, g = S.gradients(X, Y)
    want_loss, want = mlp_ref.loss_and_grads(p.astype(np.float64), X, Y, bf=True)
    assert abs(loss - want_loss) <= 1e-4 * abs(want_loss)
    bounds = np.cumsum([0, 256 * 4, 256, 65536, 256, 65536, 256, 65536, 256, 16 * 256, 16])
    names = ["W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4", "W5", "b5"]
    for k, name in enumerate(names):
        a, b = g[bounds[k]:bounds[k + 1]].astype(np.float64), want[bounds[k]:bounds[k + 1]]
        nb = np.linalg.norm(b)
        if nb == 0:
            assert np.linalg.norm(a) == 0
            continue
        rel = np.linalg.norm(a - b) / nb
        cos = float(a @ b / (np.linalg.norm(a) * nb))
        print(f"  {name}: rel L2 {rel:.2e} cos {cos:.8f}")
        assert rel < 1e-2 and cos > 0.9999, name


def test_forward_matches_float64_restatement(grrt, need_gpu):
    import torch
    S = grrt.Surrogate(2)
    p = mlp_ref.random_params(9).astype(np.float32)
    S.set_params(p)
    X, _ = mlp_ref.random_batch(10, 1000)  # 8 tiles of 128 rows, the last one partial
    X = X.astype(np.float32)
    xin = torch.from_numpy(X).cuda()
    out = torch.full((1000, 16), float("nan"), device="cuda")
    S.forward(xin, out, 1000)
    got = out.cpu().numpy().astype(np.float64)
    want, _, _ = mlp_ref.forward(p.astype(np.float64), X, bf=True)
    err = np.abs(got - want)
    assert np.all(err <= 2e-3 + 2e-3 * np.abs(want)), float(err.max())


def sweep(grrt, n_spin=2, n_incl=3):
    return grrt.sweep_cameras(width=64, height=64, spins=(0.998, 0.0, 0.5, 0.9)[:n_spin], n_incl=n_incl,
                              incl_lo_deg=30.0, incl_hi_deg=85.0)


def test_training_set_matches_oracle(grrt, need_gpu):
    cams = [dict(c, background_type=0) for c in sweep(grrt, 2, 2)]
    S = grrt.Surrogate(3)
    n_side = 48
    S.generate(cams, n_side)
    X, Y = S.dataset()
    assert len(X) == len(cams) * n_side * n_side
    for c, cam in enumerate(cams):
        R = grrt.Renderer(dict(cam, width=n_side, height=n_side, samples_per_pixel=1))
        px, py = jittered_samples(n_side, n_side, 1, np.arange(n_side * n_side))
        _, term, _, _, _ = Oracle(R).trace_rgb(px, py)
        got = Y[c * n_side * n_side:(c + 1) * n_side * n_side]
        assert np.array_equal(got[:, 6].astype(int), term), f"camera {c}"
        esc = term == 1
        nrm = got[esc, 3] ** 2 + got[esc, 4] ** 2
        assert np.allclose(nrm, 1.0, atol=1e-5)
        assert np.all(np.abs(got[esc, 2]) <= 1.0)
        # crossing u in [0, u_cut]: 0 = escaped first, u_cut = fell in first (or crossed inside 0.9 r_in)
        u_cut = np.float32(1.0 / (0.9 * R.table("flux_meta")[1]))
        for k in (0, 1):
            assert np.all((got[:, k] >= 0) & (got[:, k] <= u_cut * (1 + 1e-6)))
        assert np.all(got[term == 0, 1] > 0)  # a captured ray's second slot is never "escaped"


def test_training_reduces_loss(grrt, need_gpu):
    S = grrt.Surrogate(4)
    S.generate(sweep(grrt, 2, 3), 96)
    hist = S.train(600, batch=4096, lr=2e-3)
    first, last = float(np.mean(hist[:10])), float(np.mean(hist[-10:]))
    print(f"\n  loss {first:.4e} -> {last:.4e}")
    assert np.all(np.isfinite(hist))
    assert last < 0.1 * first


def render_pair(grrt, S, params):
    import torch
    R = grrt.Renderer(params)
    W, H = params["width"], params["height"]
    g2 = max(1, int(math.sqrt(params.get("samples_per_pixel", 1)))) ** 2
    ref = torch.empty((H, W, 3), dtype=torch.float64, device="cuda")
    rfate = torch.empty((H * W * g2,), dtype=torch.int32, device="cuda")
    R.set_precision(grrt.FORM_FP64)
    R.render_device(None, ref, rfate)
    torch.cuda.synchronize()
    ref_st = R.stats()
    out = torch.empty_like(ref)
    fate = torch.empty_like(rfate)
    S.render_device(R, None, out, fate)
    torch.cuda.synchronize()
    st = R.stats()
    exact, n = S.last_exact()
    render_pair.counts = S.last_counts()
    return (ref.cpu().numpy(), rfate.cpu().numpy(), ref_st), (out.cpu().numpy(), fate.cpu().numpy(), st), exact / n


def test_surrogate_render_and_ablation(grrt, need_gpu):
    """The surrogate render against the FP64 form, with a trained network and
    with an untrained one (the method without the network: its outputs rule
    nothing out, so its samples fall to the speculation or the exact re-trace).

    Black sky: the closed-form gate settles every sample whose smallest radius
    lies outside the disk before the network runs (76% of this frame), so the
    network only meets the samples near the disk. Star sky: no gate; the
    network's direction head decides which escapes can reach a star."""
    cams = [dict(c, background_type=0) for c in grrt.sweep_cameras(width=64, height=64, spins=(0.998, 0.9),
                                                                    n_incl=4, incl_lo_deg=60.0, incl_hi_deg=90.0)]
    trained = grrt.Surrogate(5)
    trained.generate(cams, 160)
    trained.train(3000, batch=8192, lr=2e-3)
    cal = trained.calibrate(cams, 96)
    fresh = grrt.Surrogate(6)  # the method without a trained network
    fresh.set_bands(**trained.bands())
    print(f"\n  calibration {cal}")
    for sky, bg in (("black", 0), ("stars", 1)):
        frame = grrt.config_params(2, width=160, height=160, spp=1, background_type=bg)  # a=0.998, 80 deg
        (ref, rfate, rst), (out, fate, st), frac = render_pair(grrt, trained, frame)
        c = render_pair.counts
        _, (out0, fate0, st0), frac0 = render_pair(grrt, fresh, frame)
        c0 = render_pair.counts
        scale = float(ref.max())
        rel = np.abs(out - ref) / np.maximum(np.abs(ref), 1e-6 * scale)
        rel0 = np.abs(out0 - ref) / np.maximum(np.abs(ref), 1e-6 * scale)
        print(f"  [{sky}] trained {c}, attempts {st['attempts']}; untrained {c0}, attempts {st0['attempts']}; "
              f"fp64 attempts {rst['attempts']}; max rel err {rel.max():.3e} (untrained {rel0.max():.3e}); "
              f"fate differences {int(np.sum(fate != rfate))}")
        for o, f, s in ((out, fate, st), (out0, fate0, st0)):
            r = np.abs(o - ref) / np.maximum(np.abs(ref), 1e-6 * scale)
            assert s["rays"] == rst["rays"] == 160 * 160
            assert np.mean(f != rfate) <= 1e-3
            assert np.mean(r.max(axis=2) > 1e-3) <= 1e-3
        # what the trained network gains over the method without it
        if sky == "black":
            assert c["network"] < 0.4 * c["samples"]  # the gate settled the rest
            assert st["attempts"] < 0.95 * st0["attempts"]
            assert st["attempts"] < 0.3 * rst["attempts"]
        else:
            assert c["network"] == c["samples"]
            assert st["attempts"] < 0.9 * st0["attempts"]
            assert c["exact"] < 0.6 * c0["exact"]
            assert st["attempts"] < 0.7 * rst["attempts"]
