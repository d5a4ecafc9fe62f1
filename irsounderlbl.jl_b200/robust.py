"""Robust (Huber-IRLS, adaptive Se) retrieval around optimal estimation
(src/Estimation/robust_estimation.jl:86-241).

Host logic over the GPU retrieval: each outer iteration solves the MAP problem with
the effective covariance Se_eff = s W^-1 Se_floor (W = diag(w), diagonal Se), forms the
normalized departures z = r / (sqrt(s) sigma_floor) on the kept channels and updates
the Huber weights w = 1 for |z| <= c, else max(c/|z|, 1/max_inflation^2); with
global_scale, s <- max(chi2_floor/(m - tr A), 1).  The weights are frozen inside each
inner solve; the loop stops when max|dw| < weight_tol (then solves once more with the
final weights) or after max_outer iterations.  robust_estimation_batch runs the scenes
that are still iterating as one batched GPU retrieval per outer step.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from ._lib import IRSError


@dataclass
class RobustRetrievalResult:
    """RobustRetrievalResult (robust_estimation.jl:70-80)."""
    result: object              # the final inner RetrievalResult (single scene) or batch entry
    weights: np.ndarray
    sigma_floor: np.ndarray
    sigma_eff: np.ndarray
    z: np.ndarray
    n_outer: int
    outer_converged: bool
    shat_history: List[float]
    s_global: float


def _floor_variances(Se, n_y):
    Se = np.asarray(Se, dtype=np.float64)
    if Se.ndim == 2:
        if Se.shape != (n_y, n_y):
            raise IRSError(f"Se must be n_y×n_y with n_y = length(y) = {n_y}")
        if np.any(Se - np.diag(np.diag(Se))):
            raise IRSError("a dense Se floor is not supported on this path: pass its diagonal")
        return np.diag(Se).copy()
    if Se.shape != (n_y,):
        raise IRSError(f"Se must be n_y×n_y with n_y = length(y) = {n_y}")
    return Se.copy()


def _check(huber_c, max_inflation, max_outer):
    if not huber_c > 0:
        raise IRSError(f"huber_c must be > 0, got {huber_c}")
    if not max_inflation >= 1:
        raise IRSError(f"max_inflation must be ≥ 1, got {max_inflation}")
    if not max_outer >= 1:
        raise IRSError(f"max_outer must be ≥ 1, got {max_outer}")


def _huber(z, kidx, w, huber_c, w_min):  # robust_estimation.jl:202-207
    w_new = w.copy()
    az = np.abs(z[kidx])
    w_new[kidx] = np.where(az <= huber_c, 1.0, np.maximum(huber_c / np.where(az > 0, az, 1.0), w_min))
    return w_new


def robust_estimation(y, spec, base_prof, linelists, *, xa, Sa, Se, channel_mask=None, huber_c: float = 1.5,
                      max_inflation: float = 10.0, max_outer: int = 5, weight_tol: float = 0.1,
                      global_scale: bool = False, x0=None, verbose: bool = False, **kwargs) -> RobustRetrievalResult:
    """robust_estimation (robust_estimation.jl:145-241) for one scene; kwargs go to
    optimal_estimation."""
    from .estimation import optimal_estimation
    _check(huber_c, max_inflation, max_outer)
    y = np.asarray(y, dtype=np.float64)
    n_y = len(y)
    se_floor = _floor_variances(Se, n_y)
    keep = np.ones(n_y, bool) if channel_mask is None else np.asarray(channel_mask, bool)
    kidx = np.flatnonzero(keep)
    w_min = 1.0 / max_inflation ** 2
    sigma_floor = np.sqrt(se_floor)
    w = np.ones(n_y)
    s = 1.0
    shat = []
    x_warm = np.asarray(xa if x0 is None else x0, dtype=np.float64).copy()
    converged = False
    n_outer = 0
    res = None
    for outer in range(1, max_outer + 1):
        n_outer = outer
        res = optimal_estimation(y, spec, base_prof, linelists, xa=xa, Sa=Sa, Se=s * se_floor / w,
                                 channel_mask=channel_mask, x0=x_warm, **kwargs)
        x_warm = res.x
        r = res.y_fit - y
        m = len(kidx)
        shat_floor = float(np.sum(r[kidx] ** 2 / se_floor[kidx])) / (m - res.dof)
        shat.append(shat_floor)
        z = r / (np.sqrt(s) * sigma_floor)
        w_new = _huber(z, kidx, w, huber_c, w_min)
        dw = float(np.max(np.abs(w_new - w)))
        if verbose:
            print(f"  outer {outer}: ŝ_floor={shat_floor:.3g} χ²/m={res.chi2 / m:.3g} DOF={res.dof:.2f} "
                  f"inflated={int(np.sum(w_new[kidx] < 1 - 1e-9))}/{m} s={s:.3g} Δw={dw:.3g}")
        w = w_new
        if global_scale:
            s = max(shat_floor, 1.0)
        if dw < weight_tol:
            converged = True
            res = optimal_estimation(y, spec, base_prof, linelists, xa=xa, Sa=Sa, Se=s * se_floor / w,
                                     channel_mask=channel_mask, x0=x_warm, **kwargs)
            break
    return RobustRetrievalResult(result=res, weights=w, sigma_floor=sigma_floor, sigma_eff=np.sqrt(s * se_floor / w),
                                 z=(res.y_fit - y) / (np.sqrt(s) * sigma_floor), n_outer=n_outer,
                                 outer_converged=converged, shat_history=shat, s_global=s)


def robust_estimation_batch(ys, spec, base_profs, linelists, *, xa, Sa, Se, channel_mask=None,
                            huber_c: float = 1.5, max_inflation: float = 10.0, max_outer: int = 5,
                            weight_tol: float = 0.1, global_scale: bool = False, x0=None,
                            **kwargs) -> List[RobustRetrievalResult]:
    """robust_estimation for a batch of scenes: every outer step is one batched GPU
    retrieval (optimal_estimation_batch) over the scenes still iterating.  Se: per-scene
    floor variances [n_scene, n_ch] (or one [n_ch] vector).  Each entry's `result` is a
    dict(x, y_fit, M, n_iter, converged, cost, dof)."""
    from .estimation import oe_diagnostics, optimal_estimation_batch
    _check(huber_c, max_inflation, max_outer)
    ys = np.atleast_2d(np.asarray(ys, dtype=np.float64))
    ns, n_y = ys.shape
    se = np.asarray(Se, dtype=np.float64)
    se = np.broadcast_to(se, (ns, n_y)).copy() if se.ndim == 1 else se.copy()
    if se.shape != (ns, n_y):
        raise IRSError("Se must be [n_scene, n_ch] floor variances or one [n_ch] vector")
    xa = np.asarray(xa, dtype=np.float64)
    xa = np.broadcast_to(xa, (ns, xa.shape[-1])).copy() if xa.ndim == 1 else xa
    keep = np.ones(n_y, bool) if channel_mask is None else np.asarray(channel_mask, bool)
    kidx = np.flatnonzero(keep)
    m = len(kidx)
    w_min = 1.0 / max_inflation ** 2
    Sa = np.asarray(Sa, dtype=np.float64)
    Sa_inv = np.linalg.inv(Sa)
    w = np.ones((ns, n_y))
    s = np.ones(ns)
    x_warm = (xa if x0 is None else np.broadcast_to(np.asarray(x0, np.float64), xa.shape)).copy()
    shat = [[] for _ in range(ns)]
    n_outer = np.zeros(ns, int)
    done = np.zeros(ns, bool)
    conv = np.zeros(ns, bool)
    final = [None] * ns

    def solve(idx):
        r = optimal_estimation_batch(ys[idx], spec, [base_profs[i] for i in idx], linelists, xa=xa[idx], Sa=Sa,
                                     Se=s[idx, None] * se[idx] / w[idx], x0=x_warm[idx], channel_mask=channel_mask,
                                     **kwargs)
        out = []
        for j, i in enumerate(idx):
            dof = oe_diagnostics(r["M"][j], Sa, Sa_inv)[2]
            out.append(dict(x=r["x"][j], y_fit=r["y_fit"][j], M=r["M"][j], n_iter=int(r["n_iter"][j]),
                            converged=bool(r["converged"][j]), cost=float(r["cost"][j]), dof=dof))
        return out

    for outer in range(1, max_outer + 1):
        idx = np.flatnonzero(~done)
        if len(idx) == 0:
            break
        finishing = []
        for i, res in zip(idx, solve(idx)):
            n_outer[i] = outer
            x_warm[i] = res["x"]
            final[i] = res
            r = res["y_fit"] - ys[i]
            shat_floor = float(np.sum(r[kidx] ** 2 / se[i, kidx])) / (m - res["dof"])
            shat[i].append(shat_floor)
            z = r / (np.sqrt(s[i]) * np.sqrt(se[i]))
            w_new = _huber(z, kidx, w[i], huber_c, w_min)
            dw = float(np.max(np.abs(w_new - w[i])))
            w[i] = w_new
            if global_scale:
                s[i] = max(shat_floor, 1.0)
            if dw < weight_tol:
                conv[i] = True
                finishing.append(i)
            elif outer == max_outer:
                done[i] = True
        if finishing:  # one more solve with the final weights
            for i, res in zip(finishing, solve(np.array(finishing))):
                final[i] = res
                x_warm[i] = res["x"]
                done[i] = True
    out = []
    for i in range(ns):
        sf = np.sqrt(se[i])
        out.append(RobustRetrievalResult(result=final[i], weights=w[i], sigma_floor=sf,
                                         sigma_eff=np.sqrt(s[i] * se[i] / w[i]),
                                         z=(final[i]["y_fit"] - ys[i]) / (np.sqrt(s[i]) * sf),
                                         n_outer=int(n_outer[i]), outer_converged=bool(conv[i]),
                                         shat_history=shat[i], s_global=float(s[i])))
    return out
