"""CPU oracle of the MLP surrogate (test infrastructure only: tests and smoke() use it
to check the tensor-core kernels; nothing in the product calls it).

Restates the network of the surrogate in numpy FP64: n_in -> GELU hidden layers ->
linear output, with the same input/output scaling and the loss 0.5 mean((y' - t')^2)
over samples and outputs.  With ``bf16=True`` it rounds the values the GPU keeps in
BF16 (scaled inputs, weights, pre-activations, activations and the output gradient)
to BF16 (round to nearest even) so the comparison isolates summation order.

The surrogate has no counterpart in the reference; the oracle is pinned by central
finite differences of its own loss (tests/test_mlp_oracle.py).
"""
import math

import numpy as np

_erf = np.vectorize(math.erf, otypes=[np.float64])


def bf16_round(x):
    """Round float values to the nearest BF16 (ties to even), returned as float64."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def unflatten(p, dims):
    out, k = [], 0
    for l in range(len(dims) - 1):
        o, i = dims[l + 1], dims[l]
        W = np.asarray(p[k:k + o * i], dtype=np.float64).reshape(o, i)
        k += o * i
        b = np.asarray(p[k:k + o], dtype=np.float64)
        k += o
        out.append((W, b))
    return out


def forward_backward(p, dims, X, T, x_mean, x_sd, y_mean, y_sd, bf16=False, need_grad=True):
    """(loss, flat gradient or None, scaled outputs)."""
    rd = bf16_round if bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    layers = unflatten(p, dims)
    X = np.asarray(X, dtype=np.float64)
    a = rd((X - x_mean) / x_sd)
    acts, zs = [a], []
    for l, (W, b) in enumerate(layers):
        Wr = rd(W)
        y = a @ Wr.T + b
        if l < len(layers) - 1:
            z = rd(y)
            zs.append(z)
            a = rd(gelu(z))
            acts.append(a)
        else:
            out = y
    t = (np.asarray(T, dtype=np.float64) - y_mean) / y_sd
    B, n_out = out.shape
    d = out - t
    loss = 0.5 * np.mean(d * d)
    if not need_grad:
        return loss, None, out
    g = rd(d / (B * n_out))
    grads = []
    for l in range(len(layers) - 1, -1, -1):
        W, b = layers[l]
        dW = g.T @ acts[l]
        db = g.sum(0)
        grads.append((dW, db))
        if l > 0:
            g = rd((g @ rd(W)) * gelu_grad(zs[l - 1]))
    grads.reverse()
    flat = np.concatenate([np.concatenate([dW.ravel(), db]) for dW, db in grads])
    return loss, flat, out
