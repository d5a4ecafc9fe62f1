"""The reference's array-level operators (voigt.jl, ils.jl, schwarzschild.jl,
transmittance.jl, planck.jl), for use outside forward_model.

The evaluators, the ILS taps and convolution and the RTE run on the GPU through the
C ABI (irs_voigt_profile, irs_faddeeva, irs_ils_kernel, irs_apply_ils,
irs_schwarzschild_rte); the closed-form Planck helpers and the transmittance product
are array expressions on the host, as in the reference.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional

import numpy as np

from ._lib import IRSError, check, dptr

C1, C2 = 1.191042953e-5, 1.4387769      # planck.jl:11-14
ILS_HALFWIDTH_CM = 16.0                 # ils.jl:20


def _ctx(backend):
    if backend is not None:
        return backend
    from . import default_context
    return default_context()


def _arr(a):
    return np.ascontiguousarray(np.atleast_1d(np.asarray(a, dtype=np.float64)))


def voigt_profile(nu, nu0: float, gamma_l: float, gamma_d: float, method=None, backend=None):
    """voigt_profile(ν, ν₀, γ_L, γ_D[, method]) (voigt.jl:177-200), cm; ν scalar or array."""
    from . import FullFaddeeva
    method = FullFaddeeva if method is None else method
    ctx = _ctx(backend)
    x = _arr(nu)
    out = np.empty(len(x))
    check(ctx.lib.irs_voigt_profile(ctx.h, dptr(x), len(x), float(nu0), float(gamma_l), float(gamma_d), int(method),
                                    dptr(out)))
    return out if np.ndim(nu) else float(out[0])


def faddeeva(x, y, backend=None):
    """w(x + iy) = erfcx(y - ix), y >= 0, elementwise (complex)."""
    ctx = _ctx(backend)
    xa, ya = np.broadcast_arrays(_arr(x), _arr(y))
    xa, ya = np.ascontiguousarray(xa), np.ascontiguousarray(ya)
    re, im = np.empty(len(xa)), np.empty(len(xa))
    check(ctx.lib.irs_faddeeva(ctx.h, dptr(xa), dptr(ya), len(xa), dptr(re), dptr(im)))
    w = re + 1j * im
    return w if (np.ndim(x) or np.ndim(y)) else complex(w[0])


def faddeeva_voigt(x, y, backend=None):
    """faddeeva_voigt(x, y) = Re w(x + iy) (voigt.jl:152-160)."""
    w = faddeeva(x, y, backend)
    return np.real(w) if np.ndim(w) else w.real


def ils_kernel(dnu: float, opd_max: float, fwhm_gauss: float, apodization: str = "gaussian", backend=None):
    """ils_kernel(Δν, opd_max, fwhm; apodization) (ils.jl:80-115) -> (δν, taps)."""
    from . import APODIZATION
    if apodization not in APODIZATION:
        raise IRSError(f"Unknown apodization {apodization}; expected :gaussian or one of "
                       f"{[k for k in APODIZATION if k != 'gaussian']}")
    ctx = _ctx(backend)
    n_half = math.ceil(ILS_HALFWIDTH_CM / dnu)
    k = np.empty(2 * n_half + 1)
    check(ctx.lib.irs_ils_kernel(ctx.h, float(dnu), float(opd_max), float(fwhm_gauss), APODIZATION[apodization],
                                 len(k), dptr(k)))
    return np.arange(-n_half, n_half + 1) * dnu, k


def apply_ils(nu_grid, spectrum, ils_dnu, ils_kern, backend=None):
    """apply_ils(ν_grid, spectrum, ils_δν, ils_kernel) (ils.jl:131-153): direct convolution."""
    ctx = _ctx(backend)
    g = np.asarray(getattr(nu_grid, "nu", nu_grid), dtype=np.float64)
    s = _arr(spectrum)
    if len(s) != len(g):
        raise IRSError("spectrum length mismatch")
    dnu = float(getattr(nu_grid, "dnu", (g[-1] - g[0]) / (len(g) - 1) if len(g) > 1 else 1.0))
    kern = _arr(ils_kern)
    out = np.empty(len(s))
    check(ctx.lib.irs_apply_ils(ctx.h, dptr(s), len(s), dnu, dptr(kern), len(kern), dptr(out)))
    return out


def schwarzschild_rte(nu_grid, tau_layers, T_levels, T_sfc: float, *, mu: float = 1.0, eps_sfc: float = 1.0,
                      source_function: str = "toon", T_ave=None, backend=None) -> np.ndarray:
    """schwarzschild_rte(ν_grid, τ_layers, T_levels, T_sfc; μ, ε_sfc, source_function, T_ave)
    (schwarzschild.jl:130-274); τ_layers is n_ν × n_layers as in the reference."""
    if source_function not in ("toon", "cim"):
        raise IRSError(f"source_function must be :toon or :cim, got :{source_function}")
    ctx = _ctx(backend)
    g = _arr(getattr(nu_grid, "nu", nu_grid))
    tau = np.asarray(tau_layers, dtype=np.float64)
    if tau.ndim != 2 or tau.shape[0] != len(g):
        raise IRSError(f"τ_layers rows {tau.shape[0] if tau.ndim == 2 else '?'} ≠ ν_grid.n {len(g)}")
    L = tau.shape[1]
    T_lev = _arr(T_levels)
    if len(T_lev) != L + 1:
        raise IRSError(f"T_levels must have n_layers+1 = {L + 1} entries")
    ta = None
    if T_ave is not None:
        ta = _arr(T_ave)
        if len(ta) != L:
            raise IRSError(f"T_ave must have n_layers = {L} entries, got {len(ta)}")
    tl = np.ascontiguousarray(tau.T)
    out = np.empty(len(g))
    check(ctx.lib.irs_schwarzschild_rte(ctx.h, dptr(g), len(g), L, dptr(tl), dptr(T_lev), float(T_sfc), float(mu),
                                        float(eps_sfc), 0 if source_function == "cim" else 1,
                                        dptr(ta) if ta is not None else None, dptr(out)))
    return out


def level_transmittances(tau_layers, mu: float = 1.0) -> np.ndarray:
    """level_transmittances(τ_layers, μ) (transmittance.jl:26-43): n_ν × (n_layers + 1), TOA = 1."""
    tau = np.asarray(tau_layers, dtype=np.float64)
    n_nu, L = tau.shape
    T = np.empty((n_nu, L + 1))
    T[:, L] = 1.0
    for k in range(L - 1, -1, -1):
        T[:, k] = T[:, k + 1] * np.exp(-tau[:, k] / mu)
    return T


def planck_radiance(nu, T):
    """planck_radiance (planck.jl:20-24), mW/(m^2 sr cm^-1)."""
    nu = np.asarray(nu, dtype=np.float64)
    return C1 * nu ** 3 / np.expm1(C2 * nu / np.asarray(T, dtype=np.float64))


def dB_dT(nu, T):
    """dB_dT (planck.jl:67-71)."""
    nu = np.asarray(nu, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    x = C2 * nu / T
    ex = np.exp(x)
    return C1 * C2 * nu ** 4 * ex / (T * T * (ex - 1.0) ** 2)
