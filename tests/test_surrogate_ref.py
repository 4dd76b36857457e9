"""The float64 restatement of the surrogate network (tests/mlp_ref.py) that
checks the GPU training kernels: its backward pass against central finite
differences of its own forward pass. CPU only."""
import numpy as np

import mlp_ref


def test_restatement_gradients_match_finite_differences(monkeypatch):
    # with the head weight zero the loss is the plain masked squared error, a
    # function of the parameters alone (the heads' gradient is checked below)
    monkeypatch.setitem(mlp_ref.WEIGHTS, "sig", 0.0)
    p = mlp_ref.random_params(3)
    X, Y = mlp_ref.random_batch(4, 24)
    _, g = mlp_ref.loss_and_grads(p, X, Y, bf=False)
    rng = np.random.default_rng(5)
    # parameters from every block, weights and biases (rows 6..15 of W5 have zero gradient)
    layout = np.cumsum([0, 256 * 4, 256, 65536, 256, 65536, 256, 65536, 256, 16 * 256, 16])
    idx = []
    for b in range(10):
        idx += list(rng.integers(layout[b], layout[b + 1], 6))
    worst = 0.0
    for i in idx:
        h = 1e-6 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mlp_ref.loss_only(pp, X, Y) - mlp_ref.loss_only(pm, X, Y)) / (2 * h)
        scale = max(abs(fd), abs(g[i]))
        if scale > 1e-9:
            worst = max(worst, abs(fd - g[i]) / scale)
    assert worst < 1e-5, worst


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7, 1.0 + 3 * 2 ** -8, -2.5, 3.14159])
    got = mlp_ref.bf16(x)
    assert got[0] == 1.0
    assert got[1] == 1.0  # tie -> even mantissa
    assert got[2] == 1.0 + 2 ** -7
    assert got[3] == 1.0 + 2 ** -6  # tie -> even
    assert got[4] == -2.5
    assert abs(got[5] - 3.140625) < 1e-12


def test_sigma_head_gradient_matches_finite_differences():
    """The log-sigma heads (rows 6-8 of W5 and b5) see their residuals as
    constants: their own parameters' gradients are finite differences of the loss."""
    p = mlp_ref.random_params(11)
    X, Y = mlp_ref.random_batch(12, 32)
    _, g = mlp_ref.loss_and_grads(p, X, Y, bf=False)
    w5 = 256 * 4 + 256 + 3 * (65536 + 256)
    b5 = w5 + 16 * 256
    idx = ([w5 + 6 * 256 + k for k in (0, 17, 255)] + [w5 + 7 * 256 + k for k in (3, 100)] +
           [w5 + 8 * 256 + k for k in (5, 200)] + [b5 + 6, b5 + 7, b5 + 8])
    for i in idx:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mlp_ref.loss_only(pp, X, Y) - mlp_ref.loss_only(pm, X, Y)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(abs(fd), 1e-6), (i, fd, g[i])
