"""The robust (Huber-IRLS) retrieval oracle on a linear forward model (CPU only): one
outer iteration is plain optimal estimation; outlier channels are down-weighted within
[1/max_inflation^2, 1) and inliers keep w = 1, so sigma_eff >= sigma_floor; the robust
state is closer to the truth than the plain one when a few channels carry gross errors;
the global scale never drops below 1 (robust_estimation.jl:13-60, 186-241)."""
import numpy as np

import robust_oracle as ro
from oe_oracle import optimal_estimation


def problem(seed=3, n_y=60, n=8):
    g = np.random.default_rng(seed)
    K = g.standard_normal((n_y, n))
    c = g.standard_normal(n_y)
    xa = np.zeros(n)
    Sa = np.eye(n) * 4.0
    xt = g.standard_normal(n)
    se = np.full(n_y, 0.04)
    y = K @ xt + c + 0.2 * g.standard_normal(n_y)
    y[[5, 17, 40]] += np.array([6.0, -8.0, 10.0])  # gross errors
    fwd = lambda x: K @ x + c
    fwd_jac = lambda x: (K @ x + c, K)
    return y, fwd, fwd_jac, xa, Sa, se, xt


def test_one_outer_is_plain_oe():
    y, fwd, fj, xa, Sa, se, _ = problem()
    r = ro.robust_estimation(y, fwd, fj, xa, Sa, se, max_outer=1)
    p = optimal_estimation(y, fwd, fj, xa, Sa, se)
    assert np.array_equal(r["x"], p["x"])
    assert r["n_outer"] == 1


def test_weights_and_improvement():
    y, fwd, fj, xa, Sa, se, xt = problem()
    r = ro.robust_estimation(y, fwd, fj, xa, Sa, se, huber_c=1.5, max_inflation=10.0, max_outer=8,
                             weight_tol=0.01)
    w = r["weights"]
    assert np.all(w <= 1.0) and np.all(w >= 1.0 / 100.0 - 1e-15)
    assert np.all(w[[5, 17, 40]] < 0.2)
    assert np.all(r["sigma_eff"] >= np.sqrt(se) - 1e-15)
    p = optimal_estimation(y, fwd, fj, xa, Sa, se)
    assert np.linalg.norm(r["x"] - xt) < 0.5 * np.linalg.norm(p["x"] - xt)
    assert r["outer_converged"]


def test_global_scale_and_mask():
    y, fwd, fj, xa, Sa, se, _ = problem()
    keep = np.ones(len(y), bool)
    keep[40] = False
    r = ro.robust_estimation(y, fwd, fj, xa, Sa, se, keep=keep, global_scale=True, max_outer=6)
    assert r["s_global"] >= 1.0
    assert r["weights"][40] == 1.0  # blacklisted channels are not reweighted
