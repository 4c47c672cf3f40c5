"""ORACLE (test infrastructure only): a float64 numpy restatement of the
warm-start MLP's forward pass and mean-squared-error gradients, used to check
the CUDA training kernels (libhdc hdc_mlp_*).  The layout matches the
library: per layer W [out][in] then b [out]; hidden layers ReLU, linear
output, optional residual slice of the input added to the output."""

from __future__ import annotations

import numpy as np


def unpack(params, dims):
    out, off = [], 0
    for l in range(len(dims) - 1):
        w = params[off: off + dims[l] * dims[l + 1]].reshape(dims[l + 1], dims[l])
        off += dims[l] * dims[l + 1]
        b = params[off: off + dims[l + 1]]
        off += dims[l + 1]
        out.append((w.astype(np.float64), b.astype(np.float64)))
    return out


def forward(params, dims, x, residual_offset=-1):
    layers = unpack(params, dims)
    acts = [x.astype(np.float64)]
    for l, (w, b) in enumerate(layers):
        z = acts[-1] @ w.T + b
        if l < len(layers) - 1:
            z = np.maximum(z, 0.0)
        acts.append(z)
    y = acts[-1]
    if residual_offset >= 0:
        y = y + acts[0][:, residual_offset: residual_offset + dims[-1]]
    return y, acts


def gradients(params, dims, x, target, residual_offset=-1):
    """Loss = mean over all output elements of (y - t)^2 and its gradient."""
    layers = unpack(params, dims)
    y, acts = forward(params, dims, x, residual_offset)
    n = y.size
    loss = float(np.mean((y - target) ** 2))
    delta = 2.0 * (y - target) / n
    grads = []
    for l in range(len(layers) - 1, -1, -1):
        w, _ = layers[l]
        gw = delta.T @ acts[l]
        gb = delta.sum(axis=0)
        grads.append((gw, gb))
        if l > 0:
            delta = (delta @ w) * (acts[l] > 0)
    grads.reverse()
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, flat
