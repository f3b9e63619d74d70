"""CPU oracle of the dispatch cost model -- TEST INFRASTRUCTURE ONLY.

numpy restatement of the 6 -> 32 -> 32 -> 4 ReLU MLP the library trains on
the GPU (parameter layout W1[32][6] b1[32] W2[32][32] b2[32] W3[4][32] b3[4])
and of the gradient of sum_k 0.5 (y_k[variant_k] - target_k)^2, in float64,
to check the library's hand-written backward kernel.
"""
import numpy as np

IN, H, OUT = 6, 32, 4
SIZES = [("W1", (H, IN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (OUT, H)), ("b3", (OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(P):
    out, o = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = np.asarray(P[o:o + k], dtype=np.float64).reshape(shape)
        o += k
    return out


def pack(d):
    return np.concatenate([d[name].reshape(-1) for name, _ in SIZES]).astype(np.float32)


def forward(P, X):
    p = unpack(P)
    X = np.asarray(X, dtype=np.float64)
    z1 = X @ p["W1"].T + p["b1"]
    h1 = np.maximum(z1, 0)
    z2 = h1 @ p["W2"].T + p["b2"]
    h2 = np.maximum(z2, 0)
    y = h2 @ p["W3"].T + p["b3"]
    return y, (X, z1, h1, z2, h2)


def gradient(P, X, variant, target):
    p = unpack(P)
    y, (X, z1, h1, z2, h2) = forward(P, X)
    n = len(X)
    e = y[np.arange(n), variant] - np.asarray(target, np.float64)
    loss = 0.5 * float(np.sum(e * e))
    dy = np.zeros_like(y)
    dy[np.arange(n), variant] = e
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    dh2 = (dy @ p["W3"]) * (z2 > 0)
    g["W2"] = dh2.T @ h1
    g["b2"] = dh2.sum(0)
    dh1 = (dh2 @ p["W2"]) * (z1 > 0)
    g["W1"] = dh1.T @ X
    g["b1"] = dh1.sum(0)
    return pack(g).astype(np.float64), loss
