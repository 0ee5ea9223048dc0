"""CPU oracle of the warm-start surrogate (test infrastructure only).

The network: x (inputs, zero-padded to a multiple of 8) -> `depth` layers
z = x W + b, h = GELU(z) -> coefficients c = h W_out + b_out -> field
y = c B + mean.  Loss: mean of (y - t)^2 over the finite targets, scaled as
the GPU kernels scale it (1 / number of elements).

Forward and backward in float64 numpy.  `bf16_points=True` rounds to BF16 at
the same points as the GPU implementation (inputs and weights of every GEMM,
the activations h, the coefficients c, the output gradient, the coefficient
gradient and the pre-activation gradients), so that the GPU gradients must
agree with these to FP32-accumulation accuracy; `bf16_points=False` is the
exact network, checked by finite differences in the tests.
"""
import math

import numpy as np


def bf16(x):
    """Round float values to the nearest BF16 (ties to even), as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    nan = np.isnan(f)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    out[nan] = np.nan
    return out


def gelu(z):
    return 0.5 * z * (1.0 + np.vectorize(math.erf)(z / math.sqrt(2.0)))


def gelu_grad(z):
    return (0.5 * (1.0 + np.vectorize(math.erf)(z / math.sqrt(2.0)))
            + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi))


def forward(params, x, bf16_points=True):
    """params: dict with 'W' (list), 'b' (list), 'Wout', 'bout', 'B', 'mean'.
    Returns (y, cache)."""
    r = bf16 if bf16_points else (lambda a: np.asarray(a, np.float64))
    h = r(x)
    cache = {"x": [], "z": []}
    for W, b in zip(params["W"], params["b"]):
        cache["x"].append(h)
        z = h @ r(W) + b
        cache["z"].append(z)
        h = r(gelu(z))
    cache["h"] = h
    c = h @ r(params["Wout"]) + params["bout"]
    cache["c"] = r(c)
    y = cache["c"] @ r(params["B"]) + params["mean"]
    return y, cache


def loss_and_grads(params, x, t, bf16_points=True):
    r = bf16 if bf16_points else (lambda a: np.asarray(a, np.float64))
    y, cache = forward(params, x, bf16_points)
    valid = np.isfinite(t)
    e = np.where(valid, y - np.where(valid, t, 0.0), 0.0)
    n = y.size
    loss = float(np.sum(e * e))
    dy = 2.0 * e / n
    dyr = r(dy)
    g = {}
    g["B"] = cache["c"].T @ dyr
    g["mean"] = dy.sum(axis=0)
    dc = dyr @ r(params["B"]).T
    dcr = r(dc)
    g["Wout"] = cache["h"].T @ dcr
    g["bout"] = dc.sum(axis=0)
    dh = dcr @ r(params["Wout"]).T
    gW, gb = [None] * len(params["W"]), [None] * len(params["W"])
    for l in range(len(params["W"]) - 1, -1, -1):
        dz = dh * gelu_grad(cache["z"][l])
        dzr = r(dz)
        gW[l] = cache["x"][l].T @ dzr
        gb[l] = dz.sum(axis=0)
        if l > 0:
            dh = dzr @ r(params["W"][l]).T
    g["W"], g["b"] = gW, gb
    return loss, g, y
