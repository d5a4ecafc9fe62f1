"""Pins the CPU optimal-estimation oracle: on a linear forward model y = K x the MAP
solution is closed-form, x = xa + (Sa^-1 + K^T Se^-1 K)^-1 K^T Se^-1 (y - K xa), and a
Gauss-Newton step from xa lands on it (Rodgers 2000, eq. 4.5)."""
import numpy as np

import oe_oracle


def test_linear_model_map():
    rng = np.random.default_rng(1)
    n, m = 7, 40
    K = rng.normal(0, 1, (m, n))
    xa = rng.normal(0, 1, n)
    A = rng.normal(0, 1, (n, n))
    Sa = A @ A.T + n * np.eye(n)
    se = rng.uniform(0.1, 0.5, m)
    y = K @ rng.normal(0, 2, n)
    Sa_inv = np.linalg.inv(Sa)
    x_map = xa + np.linalg.solve(Sa_inv + K.T @ (K / se[:, None]), K.T @ ((y - K @ xa) / se))
    for method in ("gauss_newton", "levenberg_marquardt"):
        r = oe_oracle.optimal_estimation(y, lambda x: K @ x, lambda x: (K @ x, K), xa, Sa, se, method=method,
                                         max_iter=50, conv_factor=1e-12)
        assert np.allclose(r["x"], x_map, rtol=0, atol=1e-8 * np.max(np.abs(x_map)))
    r = oe_oracle.optimal_estimation(y, lambda x: K @ x, lambda x: (K @ x, K), xa, Sa, se, method="gauss_newton")
    assert r["n_iter"] <= 2 and np.allclose(r["x"], x_map, atol=1e-8 * np.max(np.abs(x_map)))


def test_linear_model_map_full_se():
    """The same closed form with a full (banded) Se and a channel mask: Se restricted to
    the kept channels, as optimal_estimation.jl:166-176 does."""
    rng = np.random.default_rng(2)
    n, m = 6, 30
    K = rng.normal(0, 1, (m, n))
    xa = np.zeros(n)
    Sa = np.eye(n) * 2.0
    i = np.arange(m)
    Se = 0.04 * np.where(np.abs(i[:, None] - i[None, :]) <= 2, 0.6 ** np.abs(i[:, None] - i[None, :]), 0.0)
    keep = np.ones(m, bool)
    keep[[3, 17]] = False
    y = K @ rng.normal(0, 1, n)
    k = np.flatnonzero(keep)
    W = np.linalg.inv(Se[np.ix_(k, k)])
    Kk = K[k]
    x_map = np.linalg.solve(np.linalg.inv(Sa) + Kk.T @ W @ Kk, Kk.T @ W @ y[k])
    r = oe_oracle.optimal_estimation(y, lambda x: K @ x, lambda x: (K @ x, K), xa, Sa, Se, method="gauss_newton",
                                     max_iter=5, conv_factor=1e-14, keep=keep)
    assert np.allclose(r["x"], x_map, rtol=0, atol=1e-9 * np.max(np.abs(x_map)))
