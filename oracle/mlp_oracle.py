"""ORACLE - test infrastructure only: the join-order MLP in numpy.

Same model as the CUDA kernels (16 -> 64 -> 64 -> 1, ReLU), parameter
layout W1[64][16] b1[64] W2[64][64] b2[64] W3[64] b3. The forward pass uses
weights rounded to bfloat16 (round to nearest, ties to even, on the fp32
bit pattern) and biases in fp32, with float64 arithmetic here; the loss is
mean squared error / 2 and gradients are taken with respect to the rounded
weights, as the kernels do.
"""
import numpy as np

F, H = 16, 64
W1, B1 = 0, H * F
W2 = B1 + H
B2 = W2 + H * H
W3 = B2 + H
B3 = W3 + H
P = B3 + 1


def to_bf16(w):
    """fp32 -> nearest bfloat16 (ties to even), returned as fp32 values."""
    b = np.asarray(w, np.float32).view(np.uint32).astype(np.uint64)
    lsb = (b >> 16) & 1
    r = ((b + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(params, bf16=True):
    p = np.asarray(params, np.float32)
    q = to_bf16(p) if bf16 else p
    w1 = q[W1:B1].reshape(H, F).astype(np.float64)
    w2 = q[W2:B2].reshape(H, H).astype(np.float64)
    w3 = q[W3:B3].astype(np.float64)
    b1 = p[B1:W2].astype(np.float64)
    b2 = p[B2:W3].astype(np.float64)
    b3 = float(p[B3])
    return w1, b1, w2, b2, w3, b3


def forward(params, x):
    w1, b1, w2, b2, w3, b3 = unpack(params)
    x = np.asarray(x, np.float64)
    a1 = x @ w1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ w2.T + b2
    h2 = np.maximum(a2, 0)
    return h2 @ w3 + b3, (x, h1, h2)


def loss_and_grad(params, x, y):
    w1, b1, w2, b2, w3, b3 = unpack(params)
    o, (x, h1, h2) = forward(params, x)
    n = len(y)
    d = (o - np.asarray(y, np.float64)) / n
    loss = 0.5 * float(np.sum((o - y) ** 2)) / n
    g = np.zeros(P)
    g[W3:B3] = d @ h2
    g[B3] = d.sum()
    dh2 = np.outer(d, w3) * (h2 > 0)
    g[W2:B2] = (dh2.T @ h1).reshape(-1)
    g[B2:W3] = dh2.sum(0)
    dh1 = (dh2 @ w2) * (h1 > 0)
    g[W1:B1] = (dh1.T @ x).reshape(-1)
    g[B1:W2] = dh1.sum(0)
    return loss, g
