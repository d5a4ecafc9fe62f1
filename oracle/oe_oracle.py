"""CPU oracle of optimal_estimation (test infrastructure only).

Restates the Levenberg-Marquardt / Gauss-Newton iteration of
src/Estimation/optimal_estimation.jl:142-253 in numpy FP64 with a diagonal or full Se, for a
forward model given as callbacks:  fwd(x) -> F and fwd_jac(x) -> (F, K).  Pinned by
the closed-form MAP solution of a linear model (tests/test_oe_oracle.py).
"""
import numpy as np


def optimal_estimation(y, fwd, fwd_jac, xa, Sa, se, x0=None, method="levenberg_marquardt", max_iter=15,
                       max_linesearch=8, gamma0=1.0, gamma_factor=3.0, gamma_min=1e-4, conv_factor=1e-1,
                       keep=None):
    """-> dict(x, converged, n_iter, cost, F, K).  se: per-channel variances, or a full
    covariance matrix (inverted on the kept channels, optimal_estimation.jl:166-176)."""
    y = np.asarray(y, dtype=np.float64)
    keep = np.ones(len(y), bool) if keep is None else np.asarray(keep, bool)
    se = np.asarray(se, dtype=np.float64)
    if se.ndim == 2:
        k = np.flatnonzero(keep)
        Wm = np.zeros((len(y), len(y)))
        Wm[np.ix_(k, k)] = np.linalg.inv(se[np.ix_(k, k)])
        return _oe(y, fwd, fwd_jac, xa, Sa, Wm, x0, method, max_iter, max_linesearch, gamma0, gamma_factor,
                   gamma_min, conv_factor)
    w = np.where(keep, 1.0 / se, 0.0)
    return _oe(y, fwd, fwd_jac, xa, Sa, w, x0, method, max_iter, max_linesearch, gamma0, gamma_factor, gamma_min,
               conv_factor)


def _oe(y, fwd, fwd_jac, xa, Sa, w, x0, method, max_iter, max_linesearch, gamma0, gamma_factor, gamma_min,
        conv_factor):
    dense = w.ndim == 2
    Wop = (lambda v: w @ v) if dense else (lambda v: w * v)
    n = len(xa)
    Sa_inv = np.linalg.inv(Sa)
    xa = np.asarray(xa, dtype=np.float64)
    x = xa.copy() if x0 is None else np.asarray(x0, dtype=np.float64).copy()

    def cost(r, dx):  # optimal_estimation.jl:88-92
        return float(r @ Wop(r) + dx @ (Sa_inv @ dx))

    F, K = fwd_jac(x)
    r = y - F
    J = cost(r, x - xa)
    costs = [J]
    gamma = 0.0 if method == "gauss_newton" else gamma0
    converged = False
    it = 0
    while it < max_iter:
        it += 1
        KtWK = K.T @ (w @ K) if dense else K.T @ (K * w[:, None])
        g = K.T @ Wop(r) - Sa_inv @ (x - xa)
        accepted = False
        for _ in range(max_linesearch):
            H = (1.0 + gamma) * Sa_inv + KtWK
            L = np.linalg.cholesky(H)
            dx = np.linalg.solve(L.T, np.linalg.solve(L, g))
            xt = x + dx
            Ft = fwd(xt)
            rt = y - Ft
            Jt = cost(rt, xt - xa)
            if Jt < J:
                d2 = dx @ (Sa_inv @ dx + KtWK @ dx)
                x = xt
                F, K = fwd_jac(x)
                r = y - F
                J = Jt
                costs.append(J)
                if method != "gauss_newton":
                    gamma = max(gamma / gamma_factor, gamma_min)
                accepted = True
                if d2 / n < conv_factor:
                    converged = True
                break
            if method == "gauss_newton":
                break
            gamma *= gamma_factor
        if converged or not accepted:
            break
    return dict(x=x, converged=converged, n_iter=it, cost=costs, F=F, K=K,
                M=K.T @ (w @ K) if dense else K.T @ (K * w[:, None]))
