"""Relaxation-matrix line mixing restated in numpy -- TEST INFRASTRUCTURE ONLY.

This is the oracle for the relmat line-mixing path (first-order VP_Y from the
relaxation matrix, and the full-matrix VP_W eigenmode sum).  It is imported by
tests/ only, as the checker; the product library never calls it.

It follows src/CrossSections/line_mixing.jl of IRSounderLBL.jl:
  RelmatLine / RelmatBand / W0B0Table / HITRANRelmatData   :35-118
  _build_coupling                                           :530-578
  _build_W_matrix                                           :607-700
  _calc_W_and_Y                                             :712-738
  isotopologue masses, abundances, _band_eff_strength       :743-811
  default_vpw_whitelist                                     :813-849
  band_modes                                                :892-955
  compute_vpw_band_xsec                                     :972-1020
  _diagonal_band_modes                                      :1030-1052
  compute_vpw_band_perturbation                             :1065-1075
  _vpw_perturbation                                         :1120-1154
  _append_dispersive_lines! / lm_dispersive_kernel!         :1166-1220
  compute_lm_dispersive_correction                          :1303-1337
  partition_function (TIPS-2024, linear at 1 K, clamped)    src/HITRAN/partition.jl:8-32

The eigendecomposition is numpy.linalg.eig (LAPACK zgeev, the routine behind Julia's
`eigen`), and w(z) is scipy.special.wofz (w(x + iy) = erfcx(y - ix), the identity the
reference evaluates).  Bands are the plain containers of irs_b200.relmat (the host
mirror of the data types); the oracle only reads their fields.
"""
from __future__ import annotations

import numpy as np
from scipy.special import wofz

from oracle import read_tips

T0_LM = 296.0                      # line_mixing.jl:30
CT_LM = 1.4388                     # line_mixing.jl:31
CTGAMD = 3.5812e-7                 # line_mixing.jl:755
SQRT_LN2 = float(np.sqrt(np.log(2.0)))
INV_SQRT_PI = float(1.0 / np.sqrt(np.pi))
X_FAR = 122.0                      # voigt.jl:13
T_REF = 296.0                      # partition.jl:6

MASS_AMU = {2: {1: 43.98983, 2: 44.99318, 3: 45.99398, 4: 44.99403, 5: 45.99706,
                6: 44.99706, 7: 47.99832, 8: 47.00134, 9: 48.00196, 10: 47.00427},
            6: {1: 16.031300, 2: 17.034655, 3: 17.037475, 4: 18.040830}}      # :743-753
ISO_ABUND = {2: {1: 0.984204, 2: 0.011057, 3: 0.003947, 4: 0.000734, 5: 4.434e-5,
                 6: 1.625e-5, 7: 3.957e-6, 8: 1.4717e-7, 9: 6.554e-8, 10: 0.0},
             6: {1: 0.988274, 2: 0.0111031, 3: 0.000615751, 4: 6.91785e-6}}   # :758-766
SUBS = ("pp", "pq", "pr", "qp", "qq", "qr", "rp", "rq", "rr")

_TIPS = None


def mass_amu(molecule, iso):      # _lm_mass_amu, :770
    return MASS_AMU.get(int(molecule), {}).get(int(iso), 44.0)


def iso_abund(molecule, iso):     # _lm_iso_abund, :771
    return ISO_ABUND.get(int(molecule), {}).get(int(iso), 1e-8)


def partition_function(mol, iso, T):
    """partition.jl:8-32: TIPS-2024 table, linear at 1 K with clamped indices; Q ~ T otherwise."""
    global _TIPS
    if _TIPS is None:
        _TIPS = read_tips()
    tmin, tabs = _TIPS
    q = tabs.get((int(mol), int(iso)))
    if q is None:
        return T / T_REF
    n = len(q)
    lo = int(np.floor(T)) - tmin + 1
    hi = lo + 1
    lo = min(max(lo, 1), n)
    hi = min(max(hi, 1), n)
    fr = T - np.floor(T)
    return q[lo - 1] * (1.0 - fr) + q[hi - 1] * fr


def _ratio_part(band, T):
    iso = 10 if band.isot == 10 else band.isot
    return partition_function(band.molecule, iso, T_REF) / partition_function(band.molecule, iso, T)


def _f64(a):
    return np.asarray(a, dtype=np.float64)


def build_coupling(band, wtfit):
    """_build_coupling (:530-578): ordered pairs (i, j), j != i, Ji_j <= Ji_i, the
    isotopologue-symmetry skip and a WTfit entry; CSR over the outer line i."""
    L = band.lines
    n = len(L)
    li, lf, isot = int(band.li), int(band.lf), int(band.isot)
    sym = isot > 2 and isot != 7 and isot != 10
    Ji = L["ji"].astype(int)
    br = L["branch"].astype(int)
    row_ptr = [0]
    col, w0, b0 = [], [], []
    for i in range(n):
        jji = Ji[i]
        jjf = jji + br[i]
        for j in range(n):
            if j == i:
                continue
            jjip = Ji[j]
            jjfp = jjip + br[j]
            if jjip > jji:
                continue
            if sym and abs(jji - jjip) % 2 != 0:
                continue
            if li <= lf:
                ji_e, jf_e, jip_e, jfp_e = jji, jjf, jjip, jjfp
            else:
                ji_e, jf_e, jip_e, jfp_e = jjf, jji, jjfp, jjip
            ti = "p" if ji_e > jf_e else ("q" if ji_e == jf_e else "r")
            tip = "p" if jip_e > jfp_e else ("q" if jip_e == jfp_e else "r")
            v = wtfit.get(ti + tip, {}).get((ji_e, jip_e))
            if v is None:
                continue
            col.append(j)
            w0.append(v[0])
            b0.append(v[1])
        row_ptr.append(len(col))
    return np.array(row_ptr), np.array(col, dtype=int), np.array(w0), np.array(b0)


def decoupled(band):
    li, lf = int(band.li), int(band.lf)
    return li > 8 or lf > 8 or abs(li - lf) > 1


def build_w_matrix(band, wtfit, T):
    """_build_W_matrix (:607-700) -> (W [n, n] with W[i, j] as the reference indexes it, PopuT)."""
    L = band.lines
    n = len(L)
    if n == 0:
        return np.zeros((0, 0)), np.zeros(0)
    rp = _ratio_part(band, T)
    popu = _f64(L["popu_t0"]) * rp * np.exp(-CT_LM * _f64(L["e_lower"]) * (1.0 / T - 1.0 / T0_LM))
    gam = _f64(L["gv_air"]) * (T0_LM / T) ** _f64(L["n_air"])
    if decoupled(band):
        return np.diag(gam), popu
    nu = _f64(L["nu"])
    dipo_t = _f64(L["dipo_t"])
    s_eff = nu * popu * dipo_t ** 2
    order = np.argsort(-s_eff, kind="stable")          # sortperm(rev=true), stable
    row_ptr, col, w0, b0 = build_coupling(band, wtfit)
    W = np.zeros((n, n))
    dlg = np.log(T0_LM / T)
    for i in order:
        for t in range(row_ptr[i], row_ptr[i + 1]):
            j = col[t]
            ycal = np.exp(w0[t] - b0[t] * dlg)
            W[j, i] = ycal
            W[i, j] = ycal * popu[i] / popu[j]
    off = ~np.eye(n, dtype=bool)
    W[off] = -np.abs(W[off])
    W[np.diag_indices(n)] = gam
    Ji = L["ji"].astype(int)
    dipo0 = np.abs(_f64(L["dipo0"]))
    isot = int(band.isot)
    sym = isot > 2 and isot != 7 and isot != 10
    for ir in range(n):
        i = order[ir]
        js = order
        ok = np.ones(n, dtype=bool) if not sym else (np.abs(Ji[i] - Ji[js]) % 2 == 0)
        terms = dipo0[js] * W[js, i]
        lw = np.arange(n) > ir
        sum_lw = float(np.sum(terms[ok & lw]))
        sum_up = float(np.sum(terms[ok & ~lw]))
        if sum_lw == 0.0:
            continue
        ratio = -sum_up / sum_lw
        for irp in range(ir + 1, n):
            j = order[irp]
            W[j, i] = W[j, i] * ratio
            W[i, j] = W[j, i] * popu[i] / popu[j]
    return W, popu


def calc_y(band, wtfit, T):
    """_calc_W_and_Y (:712-738): Y_i = 2 sum_{j != i} |D_j|/|D_i| W[j, i]/(nu_i - nu_j)."""
    n = len(band.lines)
    if n == 0:
        return np.zeros(0)
    if decoupled(band):
        return np.zeros(n)
    W, _ = build_w_matrix(band, wtfit, T)
    d = _f64(band.lines["dipo_t"])
    nu = _f64(band.lines["nu"])
    Y = np.zeros(n)
    for i in range(n):
        s = 0.0
        for j in range(n):
            if j == i:
                continue
            dn = nu[i] - nu[j]
            if abs(dn) < 1e-4:
                dn = (1.0 if dn >= 0.0 else -1.0) * 1e-4
            s += 2.0 * abs(d[j]) / abs(d[i]) * (1.0 / dn) * W[j, i]
        Y[i] = s
    return Y


def band_eff_strength(band):
    """_band_eff_strength (:804-811), at T_REF."""
    L = band.lines
    nu = _f64(L["nu"])
    stim = 1.0 - np.exp(-CT_LM * nu / T0_LM)
    return float(np.sum(_f64(L["dipo_t"]) ** 2 * _f64(L["popu_t0"]) * nu * stim))


def default_vpw_whitelist(bands, n_top=5, isotopes=None, nu_window=None):
    """default_vpw_whitelist (:813-849)."""
    def in_window(b):
        return nu_window is None or (b.nu_max >= nu_window[0] and b.nu_min <= nu_window[1])
    if isotopes is None:
        scored = [(b.name, band_eff_strength(b) * iso_abund(b.molecule, b.isot)) for b in bands if in_window(b)]
        scored.sort(key=lambda x: x[1], reverse=True)
        return {s[0] for s in scored[:n_top]}
    out = set()
    for iso in isotopes:
        scored = [(b.name, band_eff_strength(b)) for b in bands if int(b.isot) == iso and in_window(b)]
        scored.sort(key=lambda x: x[1], reverse=True)
        out |= {s[0] for s in scored[:n_top]}
    return out


def band_modes(band, wtfit, T, p_atm, keep_threshold=0.0):
    """band_modes (:892-955) -> (poles, amplitudes, f)."""
    n = len(band.lines)
    if n == 0:
        return np.zeros(0, complex), np.zeros(0, complex), 0.0
    W, rho = build_w_matrix(band, wtfit, T)
    nu = _f64(band.lines["nu"])
    dipo_t = _f64(band.lines["dipo_t"])
    d_eff = (dipo_t * np.sqrt(nu * (1.0 - np.exp(-CT_LM * nu / T)))).astype(complex)
    M = 1j * p_atm * W
    M[np.diag_indices(n)] = nu + 1j * p_atm * np.diag(W)
    lam, X = np.linalg.eig(M)
    a = X.T @ d_eff
    b = np.linalg.solve(X, rho * d_eff)
    A = a * b
    iso = 10 if band.isot == 10 else band.isot
    gD = CTGAMD * (np.sum(nu) / n) * np.sqrt(T / mass_amu(band.molecule, iso))
    f = SQRT_LN2 / max(gD, 1e-10)
    keep = lam.imag > 0
    if keep_threshold > 0 and keep.any():
        keep &= np.abs(A) >= keep_threshold * np.max(np.abs(A[keep]))
    return lam[keep], A[keep], f


def diagonal_band_modes(band, T, p_atm, f):
    """_diagonal_band_modes (:1030-1052): poles nu + i gamma_L, amplitudes S(T)."""
    L = band.lines
    nu = _f64(L["nu"])
    gam = _f64(L["gv_air"]) * (T0_LM / T) ** _f64(L["n_air"]) * p_atm
    rp = _ratio_part(band, T)
    popu = _f64(L["popu_t0"]) * rp * np.exp(-CT_LM * _f64(L["e_lower"]) * (1.0 / T - 1.0 / T0_LM))
    stim = 1.0 - np.exp(-CT_LM * nu / T)
    S = _f64(L["dipo_t"]) ** 2 * popu * nu * stim
    return nu + 1j * gam, S.astype(complex), f


def _w(x, y, x_far):
    """w(x + iy) with the far-wing limit (y + ix)/(sqrt(pi)(x^2 + y^2)) for |x| > x_far."""
    w = wofz(x + 1j * y)
    far = np.abs(x) > x_far
    if np.any(far):
        den = INV_SQRT_PI / (x[far] ** 2 + y[far] ** 2)
        w[far] = y[far] * den + 1j * x[far] * den
    return w


def vpw_band_xsec(grid, poles, amps, f, cutoff=25.0, x_far=X_FAR):
    """compute_vpw_band_xsec (:972-1020): (f/sqrt(pi)) Re sum_k conj(A_k) w(z_k)."""
    grid = _f64(grid)
    sig = np.zeros(len(grid))
    if len(poles) == 0:
        return sig
    for lam, A in zip(poles, amps):
        m = np.abs(grid - lam.real) <= cutoff
        if not m.any():
            continue
        x = (grid[m] - lam.real) * f
        y = np.full(x.shape, lam.imag * f)
        w = _w(x, y, x_far)
        sig[m] += A.real * w.real + A.imag * w.imag
    return sig * (f * INV_SQRT_PI)


def vpw_band_perturbation(grid, band, wtfit, T, p_atm, cutoff=25.0, keep_threshold=1e-4, x_far=X_FAR):
    """compute_vpw_band_perturbation (:1065-1075): full modes minus the no-coupling modes."""
    lam, A, f = band_modes(band, wtfit, T, p_atm, keep_threshold)
    full = vpw_band_xsec(grid, lam, A, f, cutoff, x_far)
    bl, bA, _ = diagonal_band_modes(band, T, p_atm, f)
    return full - vpw_band_xsec(grid, bl, bA, f, cutoff, x_far)


def _key(band):
    return (min(int(band.li), int(band.lf)), max(int(band.li), int(band.lf)))


def dispersive_lines(band, Y, T, p_atm):
    """_append_dispersive_lines! (:1193-1220) -> (nu0, f, y, YSn) of the active lines."""
    L = band.lines
    iso = 10 if band.isot == 10 else band.isot
    M = mass_amu(band.molecule, int(band.isot))
    qr = partition_function(band.molecule, iso, T_REF) / partition_function(band.molecule, iso, T)
    nu = _f64(L["nu"])
    nu0 = nu + _f64(L["shift"]) * p_atm
    gD = CTGAMD * nu * np.sqrt(T / M)
    gL = _f64(L["gv_air"]) * (T0_LM / T) ** _f64(L["n_air"]) * p_atm
    f = SQRT_LN2 / np.maximum(gD, 1e-10)
    st0 = 1.0 - np.exp(-CT_LM * nu / T0_LM)
    stT = 1.0 - np.exp(-CT_LM * nu / T)
    S0 = _f64(L["dipo_t"]) ** 2 * _f64(L["popu_t0"]) * nu * st0
    ST = S0 * qr * np.exp(-CT_LM * _f64(L["e_lower"]) * (1.0 / T - 1.0 / T0_LM)) * stT / st0
    keep = (Y != 0.0) & ~(ST <= 0.0)
    return nu0[keep], f[keep], (gL * f)[keep], (Y * p_atm * ST * f * INV_SQRT_PI)[keep]


def dispersive_eval(grid, nu0, f, y, ysn, cutoff=25.0, x_far=X_FAR):
    """lm_dispersive_kernel! (:1166-1186): sum YSn Im w over lines with |nu - nu0| <= cutoff."""
    grid = _f64(grid)
    out = np.zeros(len(grid))
    for c, fk, yk, wk in zip(nu0, f, y, ysn):
        m = np.abs(grid - c) <= cutoff
        if not m.any():
            continue
        x = (grid[m] - c) * fk
        out[m] += wk * _w(x, np.full(x.shape, yk), x_far).imag
    return out


def _band_active(band, wtfit_tables, isotopes, min_band_strength):
    if int(band.li) > 8:
        return None
    if isotopes is not None and int(band.isot) not in isotopes:
        return None
    if min_band_strength > 0.0 and band_eff_strength(band) < min_band_strength:
        return None
    return wtfit_tables.get(_key(band))


def lm_dispersive_correction(grid, bands, wtfit_tables, T, p_atm, cutoff=25.0, min_band_strength=0.0,
                             x_far=X_FAR, skip=None, isotopes=None):
    """compute_lm_dispersive_correction (:1303-1337)."""
    cols = [[], [], [], []]
    for b in bands:
        wt = _band_active(b, wtfit_tables, isotopes, min_band_strength)
        if wt is None or (skip is not None and b.name in skip):
            continue
        Y = calc_y(b, wt, T)
        for acc, v in zip(cols, dispersive_lines(b, Y, T, p_atm)):
            acc.append(v)
    if not cols[0]:
        return np.zeros(len(grid))
    return dispersive_eval(grid, *[np.concatenate(c) for c in cols], cutoff=cutoff, x_far=x_far)


def vpw_perturbation(grid, bands, wtfit_tables, T, p_atm, whitelist, cutoff=25.0, keep_threshold=1e-4,
                     min_band_strength=0.0, x_far=X_FAR, isotopes=None):
    """_vpw_perturbation (:1120-1154): VP_Y for the bands outside the whitelist plus the
    eigenmode perturbation of the whitelisted ones."""
    d = lm_dispersive_correction(grid, bands, wtfit_tables, T, p_atm, cutoff, min_band_strength, x_far,
                                 skip=whitelist, isotopes=isotopes)
    for b in bands:
        if b.name not in whitelist:
            continue
        wt = _band_active(b, wtfit_tables, isotopes, min_band_strength)
        if wt is None:
            continue
        d = d + vpw_band_perturbation(grid, b, wt, T, p_atm, cutoff, keep_threshold, x_far)
    return d
