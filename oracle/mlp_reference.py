"""FP64 CPU reference of the learned return map's network (test infrastructure:
the checker of the GPU training kernels, never on the product path).

MLP 4 -> 64 -> 64 -> 3 with SiLU, parameters in the flat layout of
icempm_2d_sp_b200/csrc/surrogate.cu (row-major W[out][in]):
W1[64][4] b1[64] W2[64][64] b2[64] W3[3][64] b3[3].  Loss: mean over samples
of sum over outputs of the squared error; gradients by hand-written
backpropagation in float64.
"""
import numpy as np

IN, HID, OUT = 4, 64, 3
SIZES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (OUT, HID)), ("b3", (OUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p):
    out, k = {}, 0
    for name, shape in SIZES:
        m = int(np.prod(shape))
        out[name] = np.asarray(p[k:k + m], np.float64).reshape(shape)
        k += m
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).reshape(-1) for name, _ in SIZES])


def silu(z):
    return z / (1.0 + np.exp(-z))


def forward(p, x):
    w = unpack(p)
    z1 = x @ w["W1"].T + w["b1"]
    h1 = silu(z1)
    z2 = h1 @ w["W2"].T + w["b2"]
    h2 = silu(z2)
    return h2 @ w["W3"].T + w["b3"]


def loss_and_grad(p, x, y):
    """Mean over samples of sum_o (f(x)_o - y_o)^2 and its gradient (flat)."""
    w = unpack(p)
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    n = len(x)
    z1 = x @ w["W1"].T + w["b1"]
    s1 = 1.0 / (1.0 + np.exp(-z1))
    h1 = z1 * s1
    z2 = h1 @ w["W2"].T + w["b2"]
    s2 = 1.0 / (1.0 + np.exp(-z2))
    h2 = z2 * s2
    out = h2 @ w["W3"].T + w["b3"]
    d = out - y
    loss = (d * d).sum() / n
    dy = 2.0 * d / n
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    dz2 = (dy @ w["W3"]) * (s2 * (1.0 + z2 * (1.0 - s2)))
    g["W2"] = dz2.T @ h1
    g["b2"] = dz2.sum(0)
    dz1 = (dz2 @ w["W2"]) * (s1 * (1.0 + z1 * (1.0 - s1)))
    g["W1"] = dz1.T @ x
    g["b1"] = dz1.sum(0)
    return loss, pack(g)
