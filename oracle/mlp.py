"""Learned reconstructor (3-layer MLP) forward and backward in float64 (oracle).

Restates the device numerics of the project's MLP with its linear skip path
(there is no counterpart in the reference): inputs, hidden activations, loss gradients and hidden-layer
gradients are rounded to bfloat16 where the GPU stores them in bfloat16;
products and sums are exact here (float64) where the GPU accumulates in
float32.  GELU is the exact erf form.
"""

import math

import numpy as np

_ERF = np.vectorize(math.erf)


def bf16(x):
    """Round float32 values to bfloat16 (round to nearest even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64).reshape(a.shape)


def gelu(x):
    return 0.5 * x * (1.0 + _ERF(x / math.sqrt(2.0)))


def gelu_grad(x):
    cdf = 0.5 * (1.0 + _ERF(x / math.sqrt(2.0)))
    return cdf + x * np.exp(-0.5 * x * x) / math.sqrt(2 * math.pi)


def forward(params, x, in_scale=1.0):
    """params: [(W1, b1), (W2, b2), (W3, b3)] and optionally (Ws, None), the linear
    skip path; W [out][in].  Returns y and the cache."""
    (W1, b1), (W2, b2), (W3, b3) = params[:3]
    xb = bf16(np.asarray(x, np.float32) * np.float32(in_scale))
    z1 = xb @ bf16(W1).T + b1
    h1 = bf16(gelu(z1))
    z2 = h1 @ bf16(W2).T + b2
    h2 = bf16(gelu(z2))
    y = h2 @ bf16(W3).T + b3
    if len(params) > 3:
        y = y + xb @ bf16(params[3][0]).T
    return y, dict(xb=xb, z1=z1, h1=h1, z2=z2, h2=h2)


def backward(params, x, t, in_scale=1.0, out_scale=1.0):
    """Loss (mean squared error on y vs t / out_scale) and the gradients."""
    (W1, _), (W2, _), (W3, _) = params[:3]
    y, c = forward(params, x, in_scale)
    B, nout = y.shape
    d = y - np.asarray(t, np.float64) / out_scale
    loss = float(np.mean(d * d))
    dy = bf16(2.0 * d / (B * nout))
    g = {"dW3": dy.T @ c["h2"], "db3": dy.sum(axis=0), "dWs": dy.T @ c["xb"]}
    dz2 = bf16((dy @ bf16(W3)) * gelu_grad(c["z2"]))
    g["dW2"], g["db2"] = dz2.T @ c["h1"], dz2.sum(axis=0)
    dz1 = bf16((dz2 @ bf16(W2)) * gelu_grad(c["z1"]))
    g["dW1"], g["db1"] = dz1.T @ c["xb"], dz1.sum(axis=0)
    return loss, g
