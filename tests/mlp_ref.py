"""Float64 CPU restatement of the surrogate's network, loss and gradients
(grrt_b200/csrc/surrogate.cpp, device/surrogate.cu), used only as the checker
of the GPU kernels.

With ``bf16=True`` it rounds to BF16 exactly where the GPU path stores BF16:
the hidden activations, the weights of layers 2-5, the output gradient and the
hidden-layer gradients; all arithmetic in between is float64. The GPU
accumulates in FP32, so the two agree to FP32 accumulation rounding plus rare
one-ulp BF16 flips. With ``bf16=False`` it is the plain float64 network, whose
gradients are checked against finite differences.
"""
import numpy as np

HID = 256
OUT_PAD = 16
USED = 6      # fitted targets
HEADS = 9     # outputs used: targets + log-sigma heads of u1, u2, direction
WEIGHTS = {"u": 16.0, "dir": 0.5, "cth": 0.25, "sig": 0.1}  # surr::LossWeights
FIT_CAPTURE, FIT_GRAZE = 0.05, 0.02  # surr::kFitCapture, kFitGraze


def bf16(x):
    """Round float64/float32 values to the nearest BF16 (ties to even)."""
    a = np.asarray(x, dtype=np.float32).astype(np.float32).view(np.uint32).astype(np.uint64)
    a = (a + 0x7FFF + ((a >> 16) & 1)) & 0xFFFF0000
    return a.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    out = {}
    for name, shape in [("W1", (HID, 4)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID, HID)),
                        ("b3", (HID,)), ("W4", (HID, HID)), ("b4", (HID,)), ("W5", (OUT_PAD, HID)), ("b5", (OUT_PAD,))]:
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    assert o == len(p)
    return out


def pack(d):
    return np.concatenate([d[k].ravel() for k in ["W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4", "W5", "b5"]])


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, X, bf=True):
    P = unpack(p)
    r = bf16 if bf else (lambda v: np.asarray(v, dtype=np.float64))
    X = np.asarray(X, dtype=np.float64)
    zs, hs = [], []
    z = X @ P["W1"].T + P["b1"]
    zs.append(z)
    h = r(silu(z))
    hs.append(h)
    for l in (2, 3, 4):
        z = h @ r(P[f"W{l}"]).T + P[f"b{l}"]
        zs.append(z)
        h = r(silu(z))
        hs.append(h)
    o = h @ r(P["W5"]).T + P["b5"]
    return o, zs, hs


def row_weights(Y):
    Y = np.asarray(Y, dtype=np.float64)
    term = Y[:, 6].astype(int)
    w = np.zeros((len(Y), OUT_PAD))
    fit = (np.abs(Y[:, 8]) >= FIT_CAPTURE) & (Y[:, 9] >= FIT_GRAZE) & (Y[:, 7] == 0)
    u_ok = fit & ((term == 0) | (term == 1))
    esc = fit & (term == 1)
    w[:, 0] = w[:, 1] = np.where(u_ok, WEIGHTS["u"], 0.0)
    w[:, 2] = w[:, 3] = w[:, 4] = np.where(esc, WEIGHTS["dir"], 0.0)
    w[:, 5] = np.where(esc, WEIGHTS["cth"], 0.0)
    return w


def loss_terms(o, Y):
    """Loss and d(loss)/d(output) (the log-sigma heads get the likelihood
    gradient with the u residual held fixed, as the GPU loss kernel)."""
    B = len(o)
    w = row_weights(Y)
    d = np.zeros_like(o)
    d[:, :USED] = o[:, :USED] - Y[:, :USED]
    loss = np.sum(w * d * d)
    g = 2.0 * w * d
    u_ok = w[:, 0] > 0
    esc = w[:, 2] > 0
    for j in (6, 7):
        s = np.clip(o[:, j], -12.0, 4.0)
        e = np.exp(-2.0 * s)
        dj = d[:, j - 6]
        loss += np.sum(np.where(u_ok, WEIGHTS["sig"] * 0.5 * (dj * dj * e + 2.0 * s), 0.0))
        g[:, j] = np.where(u_ok, WEIGHTS["sig"] * (1.0 - dj * dj * e), 0.0)
    s = np.clip(o[:, 8], -12.0, 4.0)
    e = np.exp(-2.0 * s)
    d2 = np.sum(d[:, 2:5] ** 2, axis=1)
    loss += np.sum(np.where(esc, WEIGHTS["sig"] * 0.5 * (d2 * e + 6.0 * s), 0.0))
    g[:, 8] = np.where(esc, WEIGHTS["sig"] * (3.0 - d2 * e), 0.0)
    return float(loss / B), g / B


def loss_and_grads(p, X, Y, bf=True):
    P = unpack(p)
    r = bf16 if bf else (lambda v: np.asarray(v, dtype=np.float64))
    X = np.asarray(X, dtype=np.float64)
    Y = np.asarray(Y, dtype=np.float64)
    o, zs, hs = forward(p, X, bf)
    loss, g_o = loss_terms(o, Y)
    dO = r(g_o)
    g = {}
    g["W5"] = dO.T @ hs[3]
    g["b5"] = dO.sum(0)
    dz = r((dO @ r(P["W5"])) * dsilu(zs[3]))
    for l in (4, 3, 2):
        g[f"W{l}"] = dz.T @ hs[l - 2]
        g[f"b{l}"] = dz.sum(0)
        dz = r((dz @ r(P[f"W{l}"])) * dsilu(zs[l - 2]))
    g["W1"] = dz.T @ X
    g["b1"] = dz.sum(0)
    return loss, pack(g)


def loss_only(p, X, Y):
    """The loss as a function of the parameters. The log-sigma heads see the u
    residual as a constant, so finite differences of this function match the
    training gradient only for the parameters the heads alone use (their rows
    of W5 and b5) or with the head weight set to zero."""
    o, _, _ = forward(p, X, bf=False)
    return loss_terms(o, np.asarray(Y, dtype=np.float64))[0]


def random_params(seed, scale=1.0):
    rng = np.random.default_rng(seed)
    d = {"W1": rng.uniform(-1, 1, (HID, 4)) * np.sqrt(3 / 4) * scale, "b1": rng.normal(0, 0.1, HID)}
    for l in (2, 3, 4):
        d[f"W{l}"] = rng.uniform(-1, 1, (HID, HID)) * np.sqrt(3 / HID) * scale
        d[f"b{l}"] = rng.normal(0, 0.1, HID)
    W5 = np.zeros((OUT_PAD, HID))
    W5[:HEADS] = rng.uniform(-1, 1, (HEADS, HID)) * np.sqrt(3 / HID) * scale
    b5 = np.zeros(OUT_PAD)
    b5[:HEADS] = rng.normal(0, 0.1, HEADS)
    d["W5"], d["b5"] = W5, b5
    return pack(d)


def random_batch(seed, n):
    rng = np.random.default_rng(seed)
    X = rng.uniform(-1, 1, (n, 4))
    Y = np.zeros((n, 10))
    Y[:, :USED] = rng.normal(0, 0.5, (n, USED))
    Y[:, 6] = rng.choice([0, 1, 1, 1, 2], n)  # mostly escapes, some captures, a few masked
    Y[:, 7] = rng.choice([0, 1], n, p=[0.95, 0.05])  # relevant crossings after the second
    Y[:, 8] = rng.uniform(-1, 1, n)  # capture margin (a few inside the fit cut)
    Y[:, 9] = rng.uniform(0, 1, n)   # graze margin
    return X, Y
