"""CPU oracle for the learned kNN radius network (FP64 numpy).

TEST INFRASTRUCTURE ONLY: checks the device training kernels
(gts_b200/csrc/mlp.cu) -- same parameter layout, same standardisation, same
mean-squared-error loss -- and is never used by the product path.

Layout: W1[128][33] b1[128] W2[128][128] b2[128] W3[128] b3.
"""
import numpy as np

N_IN, N_H = 33, 128
SIZES = [("W1", N_H * N_IN), ("b1", N_H), ("W2", N_H * N_H), ("b2", N_H), ("W3", N_H), ("b3", 1)]
N_PARAMS = sum(n for _, n in SIZES)


def unpack(P):
    out, o = {}, 0
    for name, n in SIZES:
        out[name] = np.asarray(P[o:o + n], np.float64)
        o += n
    out["W1"] = out["W1"].reshape(N_H, N_IN)
    out["W2"] = out["W2"].reshape(N_H, N_H)
    return out


def loss_and_grad(X, t, P, norm):
    """Mean squared error of the standardised prediction and its gradient."""
    p = unpack(P)
    mu, sig = np.asarray(norm[:N_IN], np.float64), np.asarray(norm[N_IN:], np.float64)
    x = (np.asarray(X, np.float64) - mu) / sig
    z1 = x @ p["W1"].T + p["b1"]
    h1 = np.maximum(z1, 0)
    z2 = h1 @ p["W2"].T + p["b2"]
    h2 = np.maximum(z2, 0)
    y = h2 @ p["W3"] + p["b3"][0]
    B = len(t)
    e = y - np.asarray(t, np.float64)
    loss = float((e * e).mean())
    dy = 2 * e / B
    g3 = h2.T @ dy
    gb3 = dy.sum(keepdims=True)
    dz2 = np.outer(dy, p["W3"]) * (z2 > 0)
    g2 = dz2.T @ h1
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ p["W2"]) * (z1 > 0)
    g1 = dz1.T @ x
    gb1 = dz1.sum(0)
    grad = np.concatenate([g1.ravel(), gb1, g2.ravel(), gb2, g3, gb3])
    return loss, grad


def predict(X, P, norm):
    p = unpack(P)
    mu, sig = np.asarray(norm[:N_IN], np.float64), np.asarray(norm[N_IN:], np.float64)
    x = (np.asarray(X, np.float64) - mu) / sig
    h1 = np.maximum(x @ p["W1"].T + p["b1"], 0)
    h2 = np.maximum(h1 @ p["W2"].T + p["b2"], 0)
    return h2 @ p["W3"] + p["b3"][0]
