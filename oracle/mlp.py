"""CPU restatement of the learned-radius network (float64 arithmetic on the BF16-rounded weights
the device uses).  TEST INFRASTRUCTURE ONLY: the checker for the device forward and backward
kernels; the library never calls it.

Layout of the 4801 parameters: W1 [64][8], b1 [64], W2 [64][64] (row = output unit), b2 [64],
W3 [64], b3.  Inputs are standardised with the model's (mean, 1/scale).  The output is the raw
feature 7 (the previous step's log K-th distance) plus the network, y = f7 + net(x); loss is the
mean over all rows of the pinball loss of the 0.99 quantile, tau (t - y) for t > y and
(1 - tau)(y - t) otherwise, with t = log(sqrt(kth_d2)/R_0) and rows with kth_d2 <= 0 contributing
zero.
"""

from __future__ import annotations

import math

import numpy as np

F, H = 8, 64
TAU = np.float64(np.float32(0.99))  # the quantile of the pinball loss (a float32 constant on the device)
OW1, OB1 = 0, 512
OW2, OB2 = 576, 576 + 4096
OW3, OB3 = OB2 + 64, OB2 + 128


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def _erf(x):
    return np.vectorize(math.erf)(x)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def unpack(params):
    p = np.asarray(params, np.float32)
    q = bf16_round(p).astype(np.float64)
    W1 = q[OW1:OB1].reshape(H, F)
    b1 = p[OB1:OW2].astype(np.float64)
    W2 = q[OW2:OB2].reshape(H, H)
    b2 = p[OB2:OW3].astype(np.float64)
    W3 = q[OW3:OB3].astype(np.float64)
    b3 = float(p[OB3])
    return W1, b1, W2, b2, W3, b3


def loss_and_grad(params, norm, features, kth_d2, R_0):
    W1, b1, W2, b2, W3, b3 = unpack(params)
    mean, inv = norm[:F].astype(np.float64), norm[F:2 * F].astype(np.float64)
    x = (features.astype(np.float64) - mean) * inv
    valid = kth_d2 > 0
    x[~valid] = 0.0
    t = np.where(valid, 0.5 * np.log(np.where(valid, kth_d2, 1.0).astype(np.float64)) - math.log(R_0), 0.0)
    n = len(x)
    a1 = x @ W1.T + b1
    h1 = gelu(a1)
    a2 = h1 @ W2.T + b2
    h2 = gelu(a2)
    base = np.where(valid, features[:, F - 1].astype(np.float64), 0.0)
    y = h2 @ W3 + b3 + base
    err = np.where(valid, y - t, 0.0)
    above = err >= 0.0
    loss = float(np.where(above, (1.0 - TAU) * err, -TAU * err).sum() / n)
    dy = np.where(valid, np.where(above, 1.0 - TAU, -TAU), 0.0) / n
    g = np.zeros(len(params))
    g[OW3:OB3] = h2.T @ dy
    g[OB3] = dy.sum()
    d2 = (dy[:, None] * W3[None, :]) * gelu_grad(a2)
    g[OW2:OB2] = (d2.T @ h1).ravel()
    g[OB2:OW3] = d2.sum(0)
    d1 = (d2 @ W2) * gelu_grad(a1)
    g[OW1:OB1] = (d1.T @ x).ravel()
    g[OB1:OW2] = d1.sum(0)
    return loss, g


def predict_log(params, norm, features):
    W1, b1, W2, b2, W3, b3 = unpack(params)
    x = (features.astype(np.float64) - norm[:F]) * norm[F:2 * F]
    return gelu(gelu(x @ W1.T + b1) @ W2.T + b2) @ W3 + b3 + features[:, F - 1].astype(np.float64)
