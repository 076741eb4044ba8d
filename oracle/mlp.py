"""CPU oracle of the learned planner's network (test infrastructure only).

The same 3-layer perceptron as merle_b200/csrc/mlp.cu - in -> H -> H -> out,
ReLU between, parameters in one array laid out W1 [H x in], b1, W2 [H x H],
b2, W3 [out x H], b3 (row-major) - with its forward pass in float64 and in
bfloat16 rounding, and the gradient of the masked mean squared error by
backpropagation.  Used by tests/ to pin the GPU forward and backward kernels.
There is no counterpart in the reference; the arithmetic is the textbook
chain rule for a ReLU multilayer perceptron.
"""
from __future__ import annotations

import numpy as np


def split(p: np.ndarray, nin: int, nh: int, nout: int):
    p = np.asarray(p, np.float64)
    o = 0
    out = []
    for shape in [(nh, nin), (nh,), (nh, nh), (nh,), (nout, nh), (nout,)]:
        k = int(np.prod(shape))
        out.append(p[o:o + k].reshape(shape))
        o += k
    assert o == len(p)
    return out


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (round to nearest even) and back."""
    a = np.asarray(x, np.float32).copy()
    u = a.view(np.uint32)
    lsb = (u >> 16) & 1
    u = (u + 0x7FFF + lsb) & 0xFFFF0000
    return u.view(np.float32).astype(np.float64)


def forward(p, x, nin, nh, nout, bf=False):
    W1, b1, W2, b2, W3, b3 = split(p, nin, nh, nout)
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    x = np.asarray(x, np.float64)
    h1 = np.maximum(r(x) @ r(W1).T + r(b1), 0)
    if bf:
        h1 = bf16(h1)
    h2 = np.maximum(h1 @ r(W2).T + r(b2), 0)
    if bf:
        h2 = bf16(h2)
    y = h2 @ r(W3).T + r(b3)
    if bf:
        y = bf16(y)
    return y, (x, h1, h2)


def loss_and_grad(p, x, t, mask, nin, nh, nout):
    """mean((y - t)^2 over mask != 0) and its gradient (the parameter layout)."""
    W1, b1, W2, b2, W3, b3 = split(p, nin, nh, nout)
    y, (x, h1, h2) = forward(p, x, nin, nh, nout)
    mask = np.asarray(mask, np.float64)
    cnt = max(1.0, float((mask != 0).sum()))
    d = (y - np.asarray(t, np.float64)) * mask
    loss = float((d * d).sum() / cnt)
    dy = 2.0 * d / cnt
    gW3 = dy.T @ h2
    gb3 = dy.sum(0)
    d2 = (dy @ W3) * (h2 > 0)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (h1 > 0)
    gW1 = d1.T @ x
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g
