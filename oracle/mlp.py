"""Oracle for the surrogate network's training kernels (test infrastructure
only): the 8 -> 64 -> 64 -> 2 SiLU perceptron of psphray_b200/csrc/psg_mlp.cu
in float64 numpy, its loss (mean over samples of the summed squared error)
and the gradient of that loss by hand-written backpropagation.

The reference has no counterpart: it integrates every particle with LSODA
(src/solve.c:170-224); this network stands in for that step.
"""
from __future__ import annotations

import numpy as np

NIN, H, NOUT = 8, 64, 2
SIZES = [("W1", (H, NIN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (NOUT, H)), ("b3", (NOUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + n], np.float64).reshape(shape)
        o += n
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SIZES])


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def forward(p: np.ndarray, x: np.ndarray) -> np.ndarray:
    w = unpack(p)
    z1 = x @ w["W1"].T + w["b1"]
    h1 = z1 * _sig(z1)
    z2 = h1 @ w["W2"].T + w["b2"]
    h2 = z2 * _sig(z2)
    return h2 @ w["W3"].T + w["b3"]


def loss_and_grad(p: np.ndarray, x: np.ndarray, t: np.ndarray):
    """Summed squared error and the gradient of its mean over samples."""
    w = unpack(p)
    n = len(x)
    z1 = x @ w["W1"].T + w["b1"]
    s1 = _sig(z1)
    h1 = z1 * s1
    z2 = h1 @ w["W2"].T + w["b2"]
    s2 = _sig(z2)
    h2 = z2 * s2
    y = h2 @ w["W3"].T + w["b3"]
    d = y - t
    sse = float((d * d).sum())
    dy = 2.0 * d / n
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    dz2 = (dy @ w["W3"]) * s2 * (1.0 + z2 * (1.0 - s2))
    g["W2"] = dz2.T @ h1
    g["b2"] = dz2.sum(0)
    dz1 = (dz2 @ w["W2"]) * s1 * (1.0 + z1 * (1.0 - s1))
    g["W1"] = dz1.T @ x
    g["b1"] = dz1.sum(0)
    return sse, pack(g)


def init_params(seed: int) -> np.ndarray:
    """He-style initialisation (the same generator as the training driver)."""
    rng = np.random.default_rng(seed)
    d = {"W1": rng.normal(0, np.sqrt(2.0 / 5), (H, NIN)), "b1": np.zeros(H),
         "W2": rng.normal(0, np.sqrt(2.0 / H), (H, H)), "b2": np.zeros(H),
         "W3": rng.normal(0, np.sqrt(1.0 / H), (NOUT, H)), "b3": np.zeros(NOUT)}
    d["W1"][:, 5:] = 0.0
    return pack(d)
