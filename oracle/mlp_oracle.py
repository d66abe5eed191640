"""FP64 numpy restatement of the learned chooser's network.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA forward/backward kernels
(tapas-reduce_b200/csrc/mlp.cu).  Same parameter layout (per layer W out x in
row-major, then b), tanh hidden layers, linear output, loss = mean over
samples and outputs of the squared error.  The network has no counterpart in
the reference; its correctness is pinned by finite differences
(tests/test_mlp_oracle.py).
"""
from __future__ import annotations

import numpy as np


def layout(dims):
    off = []
    o = 0
    for a, b in zip(dims[:-1], dims[1:]):
        off.append((o, o + a * b))
        o += a * b + b
    return off, o


def unpack(params, dims):
    offs, _ = layout(dims)
    Ws, bs = [], []
    for (wo, bo), a, b in zip(offs, dims[:-1], dims[1:]):
        Ws.append(np.asarray(params[wo:wo + a * b], np.float64).reshape(b, a))
        bs.append(np.asarray(params[bo:bo + b], np.float64))
    return Ws, bs


def forward(params, dims, X):
    Ws, bs = unpack(params, dims)
    a = np.asarray(X, np.float64)
    acts = [a]
    for i, (W, b) in enumerate(zip(Ws, bs)):
        z = a @ W.T + b
        a = np.tanh(z) if i + 1 < len(Ws) else z
        acts.append(a)
    return a, acts


def loss_and_grad(params, dims, X, Y):
    Ws, bs = unpack(params, dims)
    y, acts = forward(params, dims, X)
    Y = np.asarray(Y, np.float64)
    n, nout = Y.shape
    loss = float(np.mean((y - Y) ** 2))
    delta = 2.0 * (y - Y) / (n * nout)
    offs, total = layout(dims)
    g = np.zeros(total)
    for layer in range(len(Ws) - 1, -1, -1):
        aprev = acts[layer]
        gW = delta.T @ aprev
        gb = delta.sum(axis=0)
        wo, bo = offs[layer]
        g[wo:wo + gW.size] = gW.ravel()
        g[bo:bo + gb.size] = gb
        if layer > 0:
            delta = (delta @ Ws[layer]) * (1.0 - aprev ** 2)
    return loss, g


def init_params(dims, seed=0):
    rng = np.random.default_rng(seed)
    offs, total = layout(dims)
    p = np.zeros(total)
    for (wo, bo), a, b in zip(offs, dims[:-1], dims[1:]):
        lim = np.sqrt(6.0 / (a + b))
        p[wo:wo + a * b] = rng.uniform(-lim, lim, a * b)
    return p
