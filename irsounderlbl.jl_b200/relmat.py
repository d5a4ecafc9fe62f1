"""Relaxation-matrix line mixing: the reference's data types, file readers and
operators (src/CrossSections/line_mixing.jl), over the C ABI of libirs_b200.

Host logic (readers, band selection, whitelist) is Python as in the reference; the
relaxation matrix W(T), Y(T) and the VP_W eigenmodes are built by the library's host
C++ (relmat.cpp) and the pole sums run on the GPU (lm_pert.cuh).
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field
from typing import Dict, Iterable, List, Optional, Set, Tuple

import numpy as np

from . import _lib
from ._lib import (IRS_LM_RELMAT_VPW, IRS_LM_RELMAT_VPY, RELMAT_LINE_DTYPE, IRSError, RelmatBandC,
                   WtfitEntryC, check, dptr)

T0_LM = 296.0        # line_mixing.jl:30
CT_LM = 1.4388       # line_mixing.jl:31
X_FAR = 122.0        # voigt.jl:13
SUBS = ("pp", "pq", "pr", "qp", "qq", "qr", "rp", "rq", "rr")
ISO_ABUND = {2: {1: 0.984204, 2: 0.011057, 3: 0.003947, 4: 0.000734, 5: 4.434e-5, 6: 1.625e-5,
                 7: 3.957e-6, 8: 1.4717e-7, 9: 6.554e-8, 10: 0.0},
             6: {1: 0.988274, 2: 0.0111031, 3: 0.000615751, 4: 6.91785e-6}}   # line_mixing.jl:758-766
MASS_AMU = {2: {1: 43.98983, 2: 44.99318, 3: 45.99398, 4: 44.99403, 5: 45.99706, 6: 44.99706,
                7: 47.99832, 8: 47.00134, 9: 48.00196, 10: 47.00427},
            6: {1: 16.031300, 2: 17.034655, 3: 17.037475, 4: 18.040830}}      # line_mixing.jl:743-753


def lm_mass_amu(molecule, iso) -> float:        # _lm_mass_amu, line_mixing.jl:770
    return MASS_AMU.get(int(molecule), {}).get(int(iso), 44.0)


def lm_iso_abund(molecule, iso) -> float:       # _lm_iso_abund, line_mixing.jl:771
    return ISO_ABUND.get(int(molecule), {}).get(int(iso), 1e-8)


def relmat_lines(rows: Iterable[tuple]) -> np.ndarray:
    """RelmatLine records (isot, ν, Ji, branch, gV_air, n_air, shift, E_lower, Dipo0, PopuT0, DipoT)."""
    return np.array(list(rows), dtype=RELMAT_LINE_DTYPE)


@dataclass
class RelmatBand:
    """RelmatBand (line_mixing.jl:72-86); molecule 2 = CO2 by default."""
    name: str
    li: int
    lf: int
    isot: int
    nu_min: float
    nu_max: float
    lines: np.ndarray
    molecule: int = 2

    def __post_init__(self):
        self.lines = np.ascontiguousarray(self.lines, dtype=RELMAT_LINE_DTYPE)


class W0B0Table:
    """W0B0Table (line_mixing.jl:92-104): nine dicts (Ji, Jip) -> (W0R, B0R) by branch pair."""

    def __init__(self):
        for s in SUBS:
            setattr(self, s, {})

    def get(self, sub, default=None):
        return getattr(self, sub, default)


@dataclass
class HITRANRelmatData:
    """HITRANRelmatData (line_mixing.jl:106-118): bands, W0B0 tables keyed (lli, llf), species."""
    bands: List[RelmatBand]
    wtfit: Dict[Tuple[int, int], W0B0Table]
    species: int = 2


def band_eff_strength(band: RelmatBand) -> float:
    """_band_eff_strength (line_mixing.jl:804-811): integrated intensity at T_REF."""
    L = band.lines
    nu = L["nu"].astype(np.float64)
    stim = 1.0 - np.exp(-CT_LM * nu / T0_LM)
    return float(np.sum(L["dipo_t"] ** 2 * L["popu_t0"] * nu * stim))


def default_vpw_whitelist(data: HITRANRelmatData, n_top: int = 5, isotopes: Optional[List[int]] = None,
                          nu_window: Optional[Tuple[float, float]] = None) -> Set[str]:
    """default_vpw_whitelist (line_mixing.jl:813-849)."""
    def in_window(b):
        return nu_window is None or (b.nu_max >= nu_window[0] and b.nu_min <= nu_window[1])
    if isotopes is None:
        scored = [(b.name, band_eff_strength(b) * lm_iso_abund(b.molecule, b.isot)) for b in data.bands
                  if in_window(b)]
        scored.sort(key=lambda x: x[1], reverse=True)
        return {n for n, _ in scored[:n_top]}
    out: Set[str] = set()
    for iso in isotopes:
        scored = [(b.name, band_eff_strength(b)) for b in data.bands if int(b.isot) == iso and in_window(b)]
        scored.sort(key=lambda x: x[1], reverse=True)
        out |= {n for n, _ in scored[:n_top]}
    return out


@dataclass
class VPYLineMixing:
    """VPYLineMixing (line_mixing.jl:144-149).

    With a HITRANRelmatData, Y(T) comes from the relaxation matrix (_calc_W_and_Y) and the
    dispersive lines are the S-file lines, as the reference does.  With a per-line array
    instead, each CO2 line of the HITRAN list carries y0 and Y(T) = y0 (296/T)^0.75 per
    atm (the synthetic stand-in for the relmat, aligned with the CO2 list order)."""
    data: object
    min_band_strength: float = 0.0

    def __post_init__(self):
        if not isinstance(self.data, HITRANRelmatData):
            self.data = np.ascontiguousarray(self.data, dtype=np.float64)

    @property
    def y0(self):
        return None if isinstance(self.data, HITRANRelmatData) else self.data

    @property
    def mode(self) -> int:
        return IRS_LM_RELMAT_VPY if isinstance(self.data, HITRANRelmatData) else _lib.IRS_LM_PER_LINE_Y


@dataclass
class VPWLineMixing:
    """VPWLineMixing (line_mixing.jl:177-200): bands in `whitelist` by their eigenmodes, the
    others by first-order VP_Y; the default whitelist is default_vpw_whitelist."""
    data: HITRANRelmatData
    whitelist: Set[str] = None
    min_band_strength: float = 0.0
    n_top: int = 5
    isotopes: Optional[List[int]] = None
    nu_window: Optional[Tuple[float, float]] = None

    def __post_init__(self):
        if self.whitelist is None:
            self.whitelist = default_vpw_whitelist(self.data, self.n_top, self.isotopes, self.nu_window)
        self.whitelist = set(self.whitelist)

    mode = IRS_LM_RELMAT_VPW
    y0 = None


@dataclass
class BandModes:
    """BandModes (line_mixing.jl:869-873)."""
    poles: np.ndarray
    amplitudes: np.ndarray
    f: float


# ------------------------------------------------------------------ readers
def _parse_fortran_d(s: str) -> float:                 # line_mixing.jl:305-307
    return float(s.strip().replace("D", "e").replace("d", "e"))


def _parse_int(s: str) -> int:
    return int(s.strip())


def parse_bandinfo(basedir: str, nu_min: float, nu_max: float, stot_min: float = 1e-28) -> List[dict]:
    """_parse_bandinfo (line_mixing.jl:338-391): BandInfo.dat entries overlapping [nu_min, nu_max]."""
    out = []
    with open(os.path.join(basedir, "BandInfo.dat")) as fh:
        for raw in fh:
            line = raw.rstrip("\r\n ")
            if len(line) < 71:
                continue
            try:
                isot = _parse_int(line[0:1])
                isot = 10 if isot == 0 else isot
                lf = _parse_int(line[3:4])
                li = _parse_int(line[8:9])
                stot = float(line[13:25])
                if stot < stot_min:
                    continue
                sg_min = float(line[26:38])
                sg_max = float(line[39:51])
                if sg_min > nu_max or sg_max < nu_min:
                    continue
                jmx_p, jmx_q, jmx_r = _parse_int(line[59:63]), _parse_int(line[63:67]), _parse_int(line[67:71])
                sfile = "S" + line[0:13].rstrip()
                li_eff = 55 if (jmx_p < 40 or jmx_r < 40 or (0 <= jmx_q < 40)) else li
                out.append(dict(sfile=sfile, li=li_eff, lf=lf, isot=isot, nu_min=sg_min, nu_max=sg_max,
                                Stot=stot, jmxP=jmx_p, jmxQ=jmx_q, jmxR=jmx_r))
            except ValueError:
                continue
    return out


def parse_sfile(path: str) -> np.ndarray:
    """_parse_sfile (line_mixing.jl:393-432): RelmatLine records of one S*.dat file."""
    rows = []
    with open(path) as fh:
        for raw in fh:
            line = raw.rstrip("\n")
            if len(line) < 215:
                continue
            try:
                c = line[2]
                isot = 10 if c == "0" else ord(c) - ord("0")
                if not -128 <= isot <= 127:
                    continue
                nu = float(line[3:15])
                S = float(line[15:25])
                gv = float(line[35:40])
                e_lower = float(line[63:73])
                n_air = np.float32(line[73:77].strip())
                shift = np.float32(line[81:89].strip())
                br = line[139]
                ji = _parse_int(line[140:143])
                dipo0 = _parse_fortran_d(line[183:199])
                popu0 = _parse_fortran_d(line[199:215])
            except ValueError:
                continue
            branch = -1 if br == "P" else (1 if br == "R" else 0)
            stim = 1.0 - math.exp(-CT_LM * nu / T0_LM)
            den = abs(popu0) * nu * stim
            dipo_t = math.sqrt(max(0.0, abs(S) / den)) if den != 0 else (math.inf if S != 0 else math.nan)
            rows.append((isot, nu, ji, branch, gv, n_air, shift, e_lower, dipo0, popu0, dipo_t))
    return relmat_lines(rows)


def load_wtfit(basedir: str, lli: int, llf: int) -> W0B0Table:
    """_load_wtfit (line_mixing.jl:434-472): WTfit{lli}{llf}.dat, empty when absent."""
    tbl = W0B0Table()
    fname = os.path.join(basedir, f"WTfit{lli}{llf}.dat")
    if not os.path.isfile(fname):
        return tbl
    with open(fname) as fh:
        for raw in fh:
            line = raw.rstrip("\r\n")
            if len(line) < 84:
                continue
            try:
                w0, b0 = _parse_fortran_d(line[0:20]), _parse_fortran_d(line[20:40])
                jic, jfc = _parse_int(line[68:72]), _parse_int(line[72:76])
                jipc, jfpc = _parse_int(line[76:80]), _parse_int(line[80:84])
            except ValueError:
                continue
            ti = "p" if jic > jfc else ("q" if jic == jfc else "r")
            tip = "p" if jipc > jfpc else ("q" if jipc == jfpc else "r")
            getattr(tbl, ti + tip)[(jic, jipc)] = (w0, b0)
    return tbl


def load_hitran_relmat(basedir: str, nu_min: float, nu_max: float, stot_min: float = 1e-28) -> HITRANRelmatData:
    """load_hitran_relmat (line_mixing.jl:480-523)."""
    bands, tables = [], {}
    for bi in parse_bandinfo(basedir, nu_min, nu_max, stot_min):
        li, lf = bi["li"], bi["lf"]
        if li > 8 or lf > 8 or abs(li - lf) > 1:
            continue
        sfile = os.path.join(basedir, bi["sfile"] + "  .dat")
        if not os.path.isfile(sfile):
            sfile = os.path.join(basedir, bi["sfile"] + ".dat")
        if not os.path.isfile(sfile):
            continue
        lines = parse_sfile(sfile)
        if len(lines) == 0:
            continue
        bands.append(RelmatBand(bi["sfile"], li, lf, bi["isot"], bi["nu_min"], bi["nu_max"], lines))
        key = (min(li, lf), max(li, lf))
        if key not in tables:
            tables[key] = load_wtfit(basedir, *key)
    return HITRANRelmatData(bands, tables)


# ------------------------------------------------------------------ C ABI marshalling
class _CRelmat:
    """irs_relmat_band / irs_wtfit_entry arrays (and the buffers they point into)."""

    def __init__(self, bands: List[RelmatBand], tables: Dict[Tuple[int, int], W0B0Table],
                 whitelist: Set[str] = frozenset()):
        self.keep = []
        self.bands = (RelmatBandC * max(len(bands), 1))()
        for k, b in enumerate(bands):
            L = np.ascontiguousarray(b.lines, dtype=RELMAT_LINE_DTYPE)
            self.keep.append(L)
            c = self.bands[k]
            c.lines = L.ctypes.data if len(L) else None
            c.n_lines = len(L)
            c.nu_min, c.nu_max = float(b.nu_min), float(b.nu_max)
            c.li, c.lf, c.isot, c.molecule = int(b.li), int(b.lf), int(b.isot), int(b.molecule)
            c.whitelisted = int(b.name in whitelist)
        rows = []
        for (lli, llf), t in tables.items():
            for si, sub in enumerate(SUBS):
                for (ji, jip), (w0, b0) in t.get(sub).items():
                    rows.append((int(lli), int(llf), si, int(ji), int(jip), 0, float(w0), float(b0)))
        self.n_wt = len(rows)
        self.wt = (WtfitEntryC * max(len(rows), 1))(*rows)
        self.n_bands = len(bands)


def _band_key(band) -> Tuple[int, int]:
    return (min(int(band.li), int(band.lf)), max(int(band.li), int(band.lf)))


_TIPS = None


def _q_ratio(band, T: float) -> float:
    """Q(296 K)/Q(T) of the band's isotopologue from the bundled TIPS-2024 tables."""
    global _TIPS
    if _TIPS is None:
        from . import _read_tips
        _TIPS = _read_tips()
    q = _TIPS.get((int(band.molecule), int(band.isot)))

    def Q(t):  # partition.jl:8-24
        if q is None:
            return t / 296.0
        n = len(q)
        lo = int(math.floor(t)) - 70 + 1
        hi = lo + 1
        lo, hi = min(max(lo, 1), n), min(max(hi, 1), n)
        fr = t - math.floor(t)
        return q[lo - 1] * (1.0 - fr) + q[hi - 1] * fr
    return Q(296.0) / Q(T)


def _single(band, wtfit):
    return _CRelmat([band], {_band_key(band): wtfit} if wtfit is not None else {})


def build_w_matrix(band: RelmatBand, wtfit: W0B0Table, T: float):
    """_build_W_matrix (line_mixing.jl:607-700) -> (W, PopuT); host C++ of the library."""
    c = _single(band, wtfit)
    n = len(band.lines)
    W = np.zeros((n, n))
    popu = np.zeros(n)
    check(_lib.load().irs_relmat_w_matrix(c.bands, c.wt, c.n_wt, float(T), _q_ratio(band, T),
                                          dptr(W), dptr(popu)))
    return W, popu


def calc_w_and_y(band: RelmatBand, wtfit: W0B0Table, T: float) -> np.ndarray:
    """_calc_W_and_Y (line_mixing.jl:712-738)."""
    c = _single(band, wtfit)
    Y = np.zeros(len(band.lines))
    check(_lib.load().irs_relmat_y(c.bands, c.wt, c.n_wt, float(T), _q_ratio(band, T), dptr(Y)))
    return Y


def band_modes(band: RelmatBand, wtfit: W0B0Table, T: float, p_atm: float,
               keep_threshold: float = 0.0) -> BandModes:
    """band_modes (line_mixing.jl:892-955): eigenmodes of diag(ν) + i p W(T)."""
    c = _single(band, wtfit)
    n = len(band.lines)
    poles = np.zeros(2 * max(n, 1))
    amps = np.zeros(2 * max(n, 1))
    f = C.c_double()
    nk = C.c_int64()
    check(_lib.load().irs_band_modes(c.bands, c.wt, c.n_wt, float(T), float(p_atm), _q_ratio(band, T),
                                     float(keep_threshold), dptr(poles), dptr(amps), C.byref(f), C.byref(nk)))
    k = nk.value
    return BandModes(poles[:2 * k].view(np.complex128).copy(), amps[:2 * k].view(np.complex128).copy(), f.value)


def _grid(nu_grid) -> np.ndarray:
    return np.ascontiguousarray(getattr(nu_grid, "nu", nu_grid), dtype=np.float64)


def _ctx(backend):
    if backend is not None:
        return backend
    from . import default_context
    return default_context()


def compute_vpw_band_xsec(nu_grid, modes: BandModes, cutoff: float = 25.0, x_far: float = X_FAR,
                          backend=None) -> np.ndarray:
    """compute_vpw_band_xsec (line_mixing.jl:972-1020) on the GPU."""
    ctx = _ctx(backend)
    g = _grid(nu_grid)
    p = np.ascontiguousarray(np.asarray(modes.poles, dtype=np.complex128)).view(np.float64)
    a = np.ascontiguousarray(np.asarray(modes.amplitudes, dtype=np.complex128)).view(np.float64)
    out = np.empty(len(g))
    check(ctx.lib.irs_vpw_band_xsec(ctx.h, dptr(g), len(g), dptr(p) if len(p) else None,
                                    dptr(a) if len(a) else None, len(p) // 2, float(modes.f), float(cutoff),
                                    float(x_far), dptr(out)))
    return out


def _iso_mask(isotopes) -> int:
    if isotopes is None:
        return 0
    m = 0
    for i in isotopes:
        if not 0 <= int(i) < 32:
            raise IRSError("isotopologue ids must be in 0..31")
        m |= 1 << int(i)
    return m if m else (1 << 31)  # an empty set keeps nothing (no band has isotopologue 31)


def _perturbation(ctx, data: HITRANRelmatData, mode, whitelist, nu_grid, T, p_atm, cutoff, x_far,
                  keep_threshold, min_band_strength, isotopes, bands=None) -> np.ndarray:
    ctx.upload_relmat(data, whitelist, min_band_strength, bands)
    g = _grid(nu_grid)
    out = np.empty(len(g))
    check(ctx.lib.irs_lm_perturbation(ctx.h, mode, dptr(g), len(g), float(T), float(p_atm), float(cutoff),
                                      float(x_far), float(keep_threshold), _iso_mask(isotopes), dptr(out)))
    return out


def compute_lm_dispersive_correction(nu_grid, relmat: HITRANRelmatData, T: float, p_atm: float, *,
                                     cutoff: float = 25.0, min_band_strength: float = 0.0, x_far: float = X_FAR,
                                     skip: Optional[Set[str]] = None, isotopes=None, backend=None) -> np.ndarray:
    """compute_lm_dispersive_correction (line_mixing.jl:1303-1337): first-order VP_Y perturbation."""
    bands = None if not skip else [b for b in relmat.bands if b.name not in skip]
    return _perturbation(_ctx(backend), relmat, IRS_LM_RELMAT_VPY, set(), nu_grid, T, p_atm, cutoff, x_far, 0.0,
                         min_band_strength, isotopes, bands)


def vpw_perturbation(nu_grid, relmat: HITRANRelmatData, T: float, p_atm: float, *, whitelist: Set[str],
                     cutoff: float = 25.0, keep_threshold: float = 1e-4, min_band_strength: float = 0.0,
                     x_far: float = X_FAR, isotopes=None, backend=None) -> np.ndarray:
    """_vpw_perturbation (line_mixing.jl:1120-1154)."""
    return _perturbation(_ctx(backend), relmat, IRS_LM_RELMAT_VPW, set(whitelist), nu_grid, T, p_atm, cutoff,
                         x_far, keep_threshold, min_band_strength, isotopes)


def compute_vpw_band_perturbation(nu_grid, band: RelmatBand, wtfit: W0B0Table, T: float, p_atm: float, *,
                                  cutoff: float = 25.0, keep_threshold: float = 1e-4, x_far: float = X_FAR,
                                  backend=None) -> np.ndarray:
    """compute_vpw_band_perturbation (line_mixing.jl:1065-1075): full minus no-coupling modes."""
    one = HITRANRelmatData([band], {_band_key(band): wtfit}, int(band.molecule))
    return vpw_perturbation(nu_grid, one, T, p_atm, whitelist={band.name}, cutoff=cutoff,
                            keep_threshold=keep_threshold, x_far=x_far, backend=backend)


def _voigt_plus(nu_grid, ll, T, p_atm, cutoff, x_far, backend, dsig):
    from . import compute_voigt_cross_sections
    sv = compute_voigt_cross_sections(nu_grid, ll, T, p_atm, cutoff=cutoff, x_far=x_far, backend=backend)
    return np.maximum(sv + dsig, 0.0)


def _linelist_isotopes(ll) -> Set[int]:                 # line_mixing.jl:202-203
    return {10 if int(i) == 0 else int(i) for i in np.unique(ll.lines["iso_id"])}


def compute_voigt_lm_cross_sections(nu_grid, ll_co2, relmat: HITRANRelmatData, T: float, p_atm: float, *,
                                    cutoff: float = 25.0, lm_cutoff: Optional[float] = None,
                                    min_band_strength: float = 0.0, isotopes=None, x_far: float = X_FAR,
                                    backend=None) -> np.ndarray:
    """compute_voigt_lm_cross_sections (line_mixing.jl:1351-1369): max(σ_Voigt + σ_disp, 0)."""
    ctx = _ctx(backend)
    d = compute_lm_dispersive_correction(nu_grid, relmat, T, p_atm, cutoff=cutoff if lm_cutoff is None else lm_cutoff,
                                         min_band_strength=min_band_strength, x_far=x_far, isotopes=isotopes,
                                         backend=ctx)
    return _voigt_plus(nu_grid, ll_co2, T, p_atm, cutoff, x_far, ctx, d)


def compute_voigt_vpw_cross_sections(nu_grid, ll_co2, relmat: HITRANRelmatData, T: float, p_atm: float, *,
                                     whitelist: Set[str], cutoff: float = 25.0, lm_cutoff: Optional[float] = None,
                                     keep_threshold: float = 1e-4, min_band_strength: float = 0.0, isotopes=None,
                                     x_far: float = X_FAR, backend=None) -> np.ndarray:
    """compute_voigt_vpw_cross_sections (line_mixing.jl:1093-1110): max(σ_Voigt + Δσ_VPW, 0)."""
    ctx = _ctx(backend)
    d = vpw_perturbation(nu_grid, relmat, T, p_atm, whitelist=whitelist,
                         cutoff=cutoff if lm_cutoff is None else lm_cutoff, keep_threshold=keep_threshold,
                         min_band_strength=min_band_strength, x_far=x_far, isotopes=isotopes, backend=ctx)
    return _voigt_plus(nu_grid, ll_co2, T, p_atm, cutoff, x_far, ctx, d)
