"""CPU restatement of the learned predictor network, for checking the GPU kernels.

Test infrastructure only: the tests compare the engine's forward pass and gradients
(nedy_predictor_forward / nedy_predictor_loss_grad) with these functions.  The network
has no counterpart in the reference (its predictor is the polynomial extrapolation of
dyson::Extrapolate, src/dyson.cpp:47-117).

Parameter layout (FP32): W1 [256 x 12], b1 [256], W2 [256 x 256], b2 [256], W3 [2 x 256], b3 [2].
Forward: h1 = bf(tanh(bf(x) bf(W1)^T + b1)), h2 = bf(tanh(h1 bf(W2)^T + b2)), y = h2 bf(W3)^T + b3,
with bf() the round-to-nearest-even BF16 rounding of every matrix-product operand (the
GPU accumulates in FP32, here in FP64).  Loss 0.5 sum |y - t|^2 / n.
"""
import numpy as np

IN, W = 12, 256
SHAPES = [("W1", (W, IN)), ("b1", (W,)), ("W2", (W, W)), ("b2", (W,)), ("W3", (2, W)), ("b3", (2,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p):
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = np.asarray(p[o:o + n], np.float64).reshape(shp)
        o += n
    return out


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(p, x, rounding=True):
    r = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    q = unpack(p)
    x = np.asarray(x, np.float64)
    h1 = r(np.tanh(r(x) @ r(q["W1"]).T + q["b1"]))
    h2 = r(np.tanh(r(h1) @ r(q["W2"]).T + q["b2"]))
    y = r(h2) @ r(q["W3"]).T + q["b3"]
    return y, (x, h1, h2)


def loss_grad(p, x, t, rounding=True):
    """Loss and gradient (same layout as the parameters)."""
    r = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    q = unpack(p)
    y, (x, h1, h2) = forward(p, x, rounding)
    n = x.shape[0]
    d = y - np.asarray(t, np.float64)
    loss = 0.5 * np.sum(d * d) / n
    dy = d / n
    g = {}
    g["W3"] = r(dy).T @ r(h2)
    g["b3"] = dy.sum(0)
    dh2 = (r(dy) @ r(q["W3"])) * (1.0 - h2 * h2)
    g["W2"] = r(dh2).T @ r(h1)
    g["b2"] = dh2.sum(0)
    dh1 = (r(dh2) @ r(q["W2"])) * (1.0 - h1 * h1)
    g["W1"] = r(dh1).T @ r(x)
    g["b1"] = dh1.sum(0)
    return loss, np.concatenate([g[name].ravel() for name, _ in SHAPES])
