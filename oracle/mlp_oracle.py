"""CPU restatement of the step-controller MLP -- TEST INFRASTRUCTURE ONLY.

The checker for the CUDA forward / backward / Adam kernels of
``reapers_b200/csrc/rp_mlp.cu``: only tests/ import it.  The reference has no
learned component, so this is a plain numpy statement of the same network
(in -> 64 -> 64 -> out, tanh hidden layers, linear output, loss = mean of
1/2 squared error) with the same flat parameter layout
[W1 (64 x in), b1, W2 (64 x 64), b2, W3 (out x 64), b3], row-major, plus
central finite differences and Adam (Kingma & Ba 2015, Algorithm 1) for the
gradient and optimiser checks.  Parity: the analytic backprop here is pinned
against finite differences in float64 (tests/test_oracle_cpu.py).
"""
from __future__ import annotations

import numpy as np

HID = 64


def num_params(n_in, n_out):
    return HID * n_in + HID + HID * HID + HID + n_out * HID + n_out


def unpack(p, n_in, n_out):
    p = np.asarray(p)
    o = 0
    W1 = p[o:o + HID * n_in].reshape(HID, n_in); o += HID * n_in
    b1 = p[o:o + HID]; o += HID
    W2 = p[o:o + HID * HID].reshape(HID, HID); o += HID * HID
    b2 = p[o:o + HID]; o += HID
    W3 = p[o:o + n_out * HID].reshape(n_out, HID); o += n_out * HID
    b3 = p[o:o + n_out]; o += n_out
    assert o == p.size
    return W1, b1, W2, b2, W3, b3


def forward(p, X, n_in, n_out):
    W1, b1, W2, b2, W3, b3 = unpack(p, n_in, n_out)
    h1 = np.tanh(X @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h2 @ W3.T + b3


def loss(p, X, Y, n_in, n_out):
    e = forward(p, X, n_in, n_out) - Y
    return 0.5 * float(np.mean(np.sum(e * e, axis=1)))


def grad(p, X, Y, n_in, n_out):
    """(loss, gradient) by backpropagation, in the dtype of p."""
    W1, b1, W2, b2, W3, b3 = unpack(p, n_in, n_out)
    n = X.shape[0]
    h1 = np.tanh(X @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    y = h2 @ W3.T + b3
    e = y - Y
    L = 0.5 * float(np.mean(np.sum(e * e, axis=1)))
    dy = e / n
    gW3 = dy.T @ h2
    gb3 = dy.sum(0)
    dh2 = (dy @ W3) * (1 - h2 * h2)
    gW2 = dh2.T @ h1
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2) * (1 - h1 * h1)
    gW1 = dh1.T @ X
    gb1 = dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return L, g


def finite_diff(p, X, Y, n_in, n_out, idx, h=1e-6):
    """Central differences of the loss (float64) at parameter indices idx."""
    p = np.array(p, dtype=np.float64)
    X = np.asarray(X, dtype=np.float64)
    Y = np.asarray(Y, dtype=np.float64)
    out = np.empty(len(idx))
    for k, i in enumerate(idx):
        q = p.copy()
        q[i] += h
        lp = loss(q, X, Y, n_in, n_out)
        q[i] -= 2 * h
        lm = loss(q, X, Y, n_in, n_out)
        out[k] = (lp - lm) / (2 * h)
    return out


def adam_step(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (returns new p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v
