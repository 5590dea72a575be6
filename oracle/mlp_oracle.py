"""CPU restatement of the control-variate network (TEST INFRASTRUCTURE ONLY).

NumPy forward and backward passes of the network the library trains on the
tensor cores (include/cubature/mlp.cuh): 7 -> 128 -> 128 -> 128 -> 1, SiLU,
inputs 2x - 1 padded to 16, targets scaled by 1 / max|y|, mean squared
error.  Values are rounded to bf16 (round to nearest even) at the points
where the kernels store bf16 -- inputs, weights, Z, H, dZ -- and products
are accumulated in FP64, so the CUDA gradients differ only by FP32
summation order and the occasional bf16 rounding that order flips.  Used
only by tests as the checker of the tensor-core kernels.
"""
from __future__ import annotations

import numpy as np

PARAMS = 35336
W0, B0 = 0, 128 * 16
W1, B1 = B0 + 128, B0 + 128 + 128 * 128
W2 = B1 + 128
B2 = W2 + 128 * 128
W3 = B2 + 128
B3 = W3 + 128


def bf16(a) -> np.ndarray:
    """float32 -> nearest bf16 value (ties to even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


# precision of the parameters as the kernels hold them (FP32 master copy)
PARAM_DTYPE = np.float32


def unpack(p):
    p = np.asarray(p, dtype=PARAM_DTYPE)
    return {"W0": p[W0:B0].reshape(128, 16), "b0": p[B0:W1], "W1": p[W1:B1].reshape(128, 128),
            "b1": p[B1:W2], "W2": p[W2:B2].reshape(128, 128), "b2": p[B2:W3],
            "w3": p[W3:B3], "b3": p[B3]}


def inputs(x) -> np.ndarray:
    x = np.asarray(x, dtype=np.float64)
    X = np.zeros((x.shape[0], 16), dtype=np.float32)
    X[:, :7] = (2.0 * x - 1.0).astype(np.float32)
    return bf16(X)


def forward(p, x):
    q = unpack(p)
    X = inputs(x).astype(np.float64)
    acts = {"X": X}
    h = X
    for l, (w, b) in enumerate([("W0", "b0"), ("W1", "b1"), ("W2", "b2")], start=1):
        z = h @ bf16(q[w]).astype(np.float64).T + q[b]
        Z = bf16(z).astype(np.float64)
        H = bf16(silu(Z)).astype(np.float64)
        acts[f"Z{l}"], acts[f"H{l}"] = Z, H
        h = H
    g = h @ q["w3"].astype(np.float64) + float(q["b3"])
    return g, acts


def grad(p, x, y_scaled):
    """Loss (mean squared error) and gradient vector of one minibatch."""
    q = unpack(p)
    g, a = forward(p, x)
    B = len(g)
    err = g - np.asarray(y_scaled, dtype=np.float64)
    e = 2.0 * err / B
    G = np.zeros(PARAMS, dtype=np.float64)
    G[W3:B3] = e @ a["H3"]
    G[B3] = e.sum()
    w3 = q["w3"].astype(np.float64)
    dZ = bf16(e[:, None] * w3[None, :] * silu_grad(a["Z3"])).astype(np.float64)
    Ws = {1: bf16(q["W1"]).astype(np.float64), 2: bf16(q["W2"]).astype(np.float64)}
    for l in (3, 2, 1):
        prev = a["X"] if l == 1 else a[f"H{l - 1}"]
        wo, bo = [(W0, B0), (W1, B1), (W2, B2)][l - 1]
        dW = dZ.T @ prev
        G[wo:bo] = dW.ravel()
        G[bo:bo + 128] = dZ.sum(axis=0)
        if l == 1:
            break
        dH = dZ @ Ws[l - 1]
        dZ = bf16(dH * silu_grad(a[f"Z{l - 1}"])).astype(np.float64)
    return float(np.mean(err ** 2)), G
