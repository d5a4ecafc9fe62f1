"""Pins the CPU MLP oracle (oracle/mlp_oracle.py) by central finite differences of its
own FP64 loss; the GPU surrogate's gradients are later compared with this oracle."""
import numpy as np

import mlp_oracle as mo


def test_oracle_gradient_vs_fd():
    rng = np.random.default_rng(7)
    dims = [5, 8, 8, 3]
    n_par = sum(dims[l + 1] * dims[l] + dims[l + 1] for l in range(len(dims) - 1))
    p = rng.normal(0, 0.5, n_par)
    X = rng.normal(0, 1, (6, 5))
    T = rng.normal(0, 1, (6, 3))
    args = (np.zeros(5), np.ones(5), np.zeros(3), np.ones(3))
    loss, g, _ = mo.forward_backward(p, dims, X, T, *args)
    h = 1e-6
    fd = np.empty(n_par)
    for k in range(n_par):
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd[k] = (mo.forward_backward(pp, dims, X, T, *args, need_grad=False)[0] -
                 mo.forward_backward(pm, dims, X, T, *args, need_grad=False)[0]) / (2 * h)
    assert np.max(np.abs(g - fd)) < 1e-8 * max(1.0, np.max(np.abs(fd)))


def test_bf16_round():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.1415926, 1e-40, 65504.0])
    r = mo.bf16_round(v)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12
    assert r[5] == 65536.0
