"""CPU oracle of robust_estimation (test infrastructure only).

Restates the outer Huber-IRLS loop of src/Estimation/robust_estimation.jl:145-241
around the numpy optimal-estimation oracle (oe_oracle.py), for a diagonal Se floor and a
forward model given as callbacks fwd(x) -> F, fwd_jac(x) -> (F, K).  The degrees of
freedom of each inner solve are tr A with A = (Sa^-1 + M)^-1 M and M = K^T Se_eff^-1 K at
the solution (optimal_estimation.jl:257-270)."""
import numpy as np

from oe_oracle import optimal_estimation


def robust_estimation(y, fwd, fwd_jac, xa, Sa, se_floor, keep=None, huber_c=1.5, max_inflation=10.0,
                      max_outer=5, weight_tol=0.1, global_scale=False, x0=None, **oe_kw):
    y = np.asarray(y, dtype=np.float64)
    se_floor = np.asarray(se_floor, dtype=np.float64)
    n_y = len(y)
    keep = np.ones(n_y, bool) if keep is None else np.asarray(keep, bool)
    kidx = np.flatnonzero(keep)
    m = len(kidx)
    w_min = 1.0 / max_inflation ** 2
    sigma_floor = np.sqrt(se_floor)
    Sa_inv = np.linalg.inv(Sa)
    w = np.ones(n_y)
    s = 1.0
    shat = []
    x_warm = np.asarray(xa if x0 is None else x0, dtype=np.float64).copy()
    converged = False
    n_outer = 0
    res = None
    for outer in range(1, max_outer + 1):
        n_outer = outer
        res = optimal_estimation(y, fwd, fwd_jac, xa, Sa, s * se_floor / w, x0=x_warm, keep=keep, **oe_kw)
        x_warm = res["x"]
        M = res["M"]
        dof = float(np.trace(np.linalg.solve(Sa_inv + M, M)))
        r = res["F"] - y
        shat_floor = float(np.sum(r[kidx] ** 2 / se_floor[kidx])) / (m - dof)
        shat.append(shat_floor)
        z = r / (np.sqrt(s) * sigma_floor)
        w_new = w.copy()
        for i in kidx:
            az = abs(z[i])
            w_new[i] = 1.0 if az <= huber_c else max(huber_c / az, w_min)
        dw = float(np.max(np.abs(w_new - w)))
        w = w_new
        if global_scale:
            s = max(shat_floor, 1.0)
        if dw < weight_tol:
            converged = True
            res = optimal_estimation(y, fwd, fwd_jac, xa, Sa, s * se_floor / w, x0=x_warm, keep=keep, **oe_kw)
            break
    return dict(x=res["x"], weights=w, sigma_eff=np.sqrt(s * se_floor / w), n_outer=n_outer,
                outer_converged=converged, shat_history=shat, s_global=s, F=res["F"])
