"""Test infrastructure, not product code: a NumPy restatement of the chemistry
surrogate's network (12 -> 4 x 256 GELU -> 9), its features and its loss, for
checking the tensor-core forward and backward kernels.

It follows the device arithmetic where it matters for a tight comparison:
BF16 rounding (round to nearest even) of the network inputs, the weights, the
hidden activations and the output gradients fed to the matrix products; FP32
biases and gradients of the pre-activations; GELU in its tanh form.  Products are
accumulated in float64 (the device accumulates in FP32).
"""
from __future__ import annotations

import numpy as np
from math import sqrt, pi

DIMS = [16, 256, 256, 256, 256, 16]
N_IN, N_OUT = 12, 9


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (nearest, ties to even), returned as float64."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


_C = sqrt(2.0 / pi)


def gelu(x):
    """GELU in its tanh form."""
    return 0.5 * x * (1.0 + np.tanh(_C * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(_C * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * _C * (1.0 + 3 * 0.044715 * x * x)


def unflatten(flat: np.ndarray):
    """(W_l [out x in], b_l [out]) per layer from the flat parameter vector."""
    out, off = [], 0
    for l in range(5):
        din, dout = DIMS[l], DIMS[l + 1]
        w = flat[off:off + din * dout].reshape(dout, din)
        off += din * dout
        b = flat[off:off + dout]
        off += dout
        out.append((w.astype(np.float64), b.astype(np.float64)))
    return out


def features(states: np.ndarray, mu: np.ndarray, sig: np.ndarray) -> np.ndarray:
    """Normalised, BF16-rounded network inputs (n x 16) of states (T, p, Y[9], dt)."""
    f = np.empty((states.shape[0], N_IN), dtype=np.float32)
    f[:, 0] = states[:, 0]
    f[:, 1] = np.log10(states[:, 1])
    f[:, 2:11] = states[:, 2:11]
    f[:, 11] = np.log10(states[:, 11])
    x = np.zeros((states.shape[0], 16))
    x[:, :N_IN] = bf16((f - mu.astype(np.float32)) / sig.astype(np.float32))
    return x


def loss_and_grads(flat: np.ndarray, x: np.ndarray, target: np.ndarray):
    """Mean-squared loss over the 9 outputs and the gradient of every
    parameter, flattened like the device's parameter vector."""
    layers = unflatten(flat)
    acts, pre = [x], []
    a = x
    for l, (w, b) in enumerate(layers):
        z = (a @ bf16(w).T).astype(np.float32).astype(np.float64) + b
        pre.append(z)
        if l < 4:
            a = bf16(gelu(z))
            acts.append(a)
    pred = pre[-1][:, :N_OUT]
    n = x.shape[0]
    err = pred - target[:, :N_OUT]
    loss = float(np.mean(err ** 2))
    dz = np.zeros((n, 16))
    dz[:, :N_OUT] = 2.0 * err / (n * N_OUT)
    grads = [None] * 5
    for l in range(4, -1, -1):
        w, b = layers[l]
        dzb = bf16(dz)
        gw = dzb.T @ acts[l]
        gb = dz.sum(axis=0)
        grads[l] = (gw, gb)
        if l > 0:
            da = dzb @ bf16(w)
            dz = da * gelu_grad(pre[l - 1])
    flat_g = np.concatenate([np.concatenate([g.ravel(), gb]) for g, gb in grads])
    return loss, flat_g
