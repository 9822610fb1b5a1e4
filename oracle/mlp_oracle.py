"""FP64 restatement of the warm-start MLP (test infrastructure only: the gradient, Adam and
initialisation checks of the library's network kernels compare against it).

The network has no reference counterpart. Its definition is the C ABI's (dfsph_c.h, "learned
warm-start network"): x' = x * in_scale; h1 = relu(W1 x' + b1); h2 = relu(W2 h1 + b2);
y = W3 h2 + b3; loss = mean over samples of sum over outputs of (y - t)^2. Parameters are one flat
FP32 vector, row-major [out][in]: W1[64][8] b1[64] W2[64][64] b2[64] W3[2][64] b3[2].
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT = 8, 64, 2
W1 = 0
B1 = W1 + N_HID * N_IN
W2 = B1 + N_HID
B2 = W2 + N_HID * N_HID
W3 = B2 + N_HID
B3 = W3 + N_OUT * N_HID
N_PARAMS = B3 + N_OUT  # 4866


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[W1:B1].reshape(N_HID, N_IN), p[B1:W2], p[W2:B2].reshape(N_HID, N_HID), p[B2:W3],
            p[W3:B3].reshape(N_OUT, N_HID), p[B3:N_PARAMS])


def forward(p, in_scale, x):
    """Network outputs (n, 2) in FP64."""
    w1, b1, w2, b2, w3, b3 = unpack(p)
    xs = np.asarray(x, dtype=np.float64) * np.asarray(in_scale, dtype=np.float64)
    h1 = np.maximum(xs @ w1.T + b1, 0.0)
    h2 = np.maximum(h1 @ w2.T + b2, 0.0)
    return h2 @ w3.T + b3


def _bf16(a):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward_bf16(p, in_scale, x):
    """The inference arithmetic of the tensor-core path: inputs, weights and hidden activations
    rounded to BF16, biases and accumulation in FP32 (here FP64)."""
    w1, b1, w2, b2, w3, b3 = unpack(p)
    xs = _bf16(np.asarray(x, dtype=np.float32) * np.asarray(in_scale, dtype=np.float32))
    h1 = _bf16(np.maximum(xs @ _bf16(w1).T + b1, 0.0))
    h2 = _bf16(np.maximum(h1 @ _bf16(w2).T + b2, 0.0))
    return h2 @ _bf16(w3).T + b3


def loss_and_grad(p, in_scale, x, t):
    """(loss, gradient (N_PARAMS,)) in FP64 by reverse-mode differentiation."""
    w1, b1, w2, b2, w3, b3 = unpack(p)
    xs = np.asarray(x, dtype=np.float64) * np.asarray(in_scale, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    n = xs.shape[0]
    a1 = xs @ w1.T + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ w2.T + b2
    h2 = np.maximum(a2, 0.0)
    y = h2 @ w3.T + b3
    r = y - t
    loss = float((r * r).sum() / n)
    dy = 2.0 * r / n
    g = np.zeros(N_PARAMS)
    g[W3:B3] = (dy.T @ h2).ravel()
    g[B3:N_PARAMS] = dy.sum(0)
    d2 = (dy @ w3) * (a2 > 0)
    g[W2:B2] = (d2.T @ h1).ravel()
    g[B2:W3] = d2.sum(0)
    d1 = (d2 @ w2) * (a1 > 0)
    g[W1:B1] = (d1.T @ xs).ravel()
    g[B1:W2] = d1.sum(0)
    return loss, g


def adam(p, m, v, g, lr, step, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam update with bias correction; returns (p, m, v)."""
    m = beta1 * m + (1.0 - beta1) * g
    v = beta2 * v + (1.0 - beta2) * g * g
    mh = m / (1.0 - beta1 ** step)
    vh = v / (1.0 - beta2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v


def _splitmix_uniform(seed: int, idx: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser of (seed << 32) + idx + golden-ratio increment, top 24 bits to [-1, 1)."""
    with np.errstate(over="ignore"):
        z = (np.uint64(seed) << np.uint64(32)) + idx.astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(40)).astype(np.float64) * (1.0 / 16777216.0)
    return u.astype(np.float32) * np.float32(2.0) - np.float32(1.0)


def init_params(seed: int) -> np.ndarray:
    """The library's deterministic initialisation: He-uniform W1 over the 5 real inputs (the 3 pad
    columns zero), He-uniform W2, zero W3 and biases. FP32."""
    p = np.zeros(N_PARAMS, dtype=np.float32)
    idx = np.arange(N_PARAMS)
    u = _splitmix_uniform(seed, idx)
    w1 = (idx < B1) & ((idx % N_IN) < 5)
    p[w1] = u[w1] * np.sqrt(np.float32(6.0 / 5.0))
    w2 = (idx >= W2) & (idx < B2)
    p[w2] = u[w2] * np.sqrt(np.float32(6.0 / N_HID))
    return p
