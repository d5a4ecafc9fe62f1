"""Seeded synthetic inputs with the shapes and distributions of the benchmark cases.

HITRAN line lists are not redistributable, so every case uses synthetic lines
(numpy PCG64 streams with fixed seeds) drawn from these distributions:
  nu0 ~ U(nu_lo, nu_hi), S = 10^U(-25, -19), gamma_air ~ U(0.06, 0.09),
  gamma_self ~ U(0.08, 0.11), n_air ~ U(0.6, 0.8), E'' ~ U(0, 3000),
  delta_air ~ U(-0.005, 0), A = 0, iso = 1.
Profiles are the six bundled AFGL 50-level atmospheres (AFGL-TR-86-0110) and
perturbations of them.

  case "5k-co2"     5,000 CO2 lines in 645-700 cm^-1 (seed 1000), US standard
  case "iasi-400k"  400,000 lines over H2O, CO2, O3, N2O, CO, CH4 in 645-2760 cm^-1
                    (seed 1001 + species index), the 6 AFGL profiles
  perturbed profiles: AFGL base + T noise N(0, C), C_ij = 9 exp(-|i-j|/3)
                    (K^2, level units), H2O and O3 scaled by exp(N(0, 0.2^2)),
                    scan angle U(0, 48 deg)
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from ._lib import LINE_DTYPE

DATA = Path(__file__).resolve().parent / "data"
AFGL = ("us_standard", "tropical", "midlatitude_summer", "midlatitude_winter",
        "subarctic_summer", "subarctic_winter")
SPECIES6 = (1, 2, 3, 4, 5, 6)  # H2O CO2 O3 N2O CO CH4


def synthetic_linelist(n: int, mol: int, seed: int, nu_lo: float = 645.0, nu_hi: float = 700.0):
    """n lines of molecule `mol` with the distributions above, sorted by nu0."""
    from . import HITRANLinelist
    g = np.random.Generator(np.random.PCG64(seed))
    L = np.zeros(n, dtype=LINE_DTYPE)
    L["mol_id"] = mol
    L["iso_id"] = 1
    L["wavenumber"] = g.uniform(nu_lo, nu_hi, n)
    L["intensity"] = 10.0 ** g.uniform(-25.0, -19.0, n)
    L["a_coeff"] = 0.0
    L["air_broad"] = g.uniform(0.06, 0.09, n).astype(np.float32)
    L["self_broad"] = g.uniform(0.08, 0.11, n).astype(np.float32)
    L["temp_depend"] = g.uniform(0.6, 0.8, n).astype(np.float32)
    L["lower_energy"] = g.uniform(0.0, 3000.0, n)
    L["pressure_shift"] = g.uniform(-0.005, 0.0, n).astype(np.float32)
    return HITRANLinelist(L)


def lists_5k_co2():
    """{CO2: 5,000 lines in 645-700 cm^-1}, seed 1000."""
    return {2: synthetic_linelist(5000, 2, 1000, 645.0, 700.0)}


def lists_iasi_400k(n_total: int = 400_000, nu_lo: float = 645.0, nu_hi: float = 2760.0):
    """400,000 lines over six species (66,667 x 4 + 66,666 x 2), seeds 1001 + k."""
    base, extra = divmod(n_total, len(SPECIES6))
    out = {}
    for k, mol in enumerate(SPECIES6):
        out[mol] = synthetic_linelist(base + (1 if k < extra else 0), mol, 1001 + k, nu_lo, nu_hi)
    return out


def vpy_y0(n: int, seed: int = 1002) -> np.ndarray:
    """Per-line first-order mixing coefficients y0 ~ N(0, 0.01) per atm."""
    return np.random.Generator(np.random.PCG64(seed)).normal(0.0, 0.01, n)


def afgl_atmosphere(name: str = "us_standard"):
    """afgl_atmosphere (src/Atmosphere/standard_atm.jl:265-276) from the bundled CSV."""
    from . import AtmosphericProfile, IRSError
    name = name.replace("-", "_")
    if name not in AFGL:
        raise IRSError(f"Unknown AFGL atmosphere :{name}. Choose one of {AFGL}.")
    rows = [l.strip().split(",") for l in open(DATA / f"afgl_{name}_50lev.csv").readlines()[1:] if l.strip()]
    a = np.array(rows, dtype=np.float64)
    vmr = {1: a[:, 3].copy(), 2: a[:, 4].copy(), 3: a[:, 5].copy(), 4: a[:, 6].copy(),
           6: a[:, 7].copy(), 5: a[:, 8].copy()}
    return AtmosphericProfile(a[:, 0].copy(), a[:, 1].copy(), a[:, 2].copy(), vmr)


def perturbed_profiles(n: int, seed: int = 1002):
    """n perturbed AFGL profiles and their scan angles (degrees)."""
    from . import AtmosphericProfile
    g = np.random.Generator(np.random.PCG64(seed))
    bases = [afgl_atmosphere(a) for a in AFGL]
    nl = len(bases[0].pressure)
    idx = np.arange(nl)
    Ccov = 9.0 * np.exp(-np.abs(idx[:, None] - idx[None, :]) / 3.0)
    Lc = np.linalg.cholesky(Ccov)
    out, scans = [], []
    for k in range(n):
        b = bases[k % len(bases)]
        T = b.temperature + Lc @ g.standard_normal(nl)
        vmr = {s: v.copy() for s, v in b.vmr.items()}
        vmr[1] = vmr[1] * np.exp(0.2 * g.standard_normal(nl))
        vmr[3] = vmr[3] * np.exp(0.2 * g.standard_normal(nl))
        out.append(AtmosphericProfile(b.pressure.copy(), T, b.altitude.copy(), vmr))
        scans.append(g.uniform(0.0, 48.0))
    return out, np.array(scans)


def synthetic_relmat(n_bands: int = 6, j_max: int = 60, seed: int = 1003, nu_lo: float = 650.0,
                     nu_hi: float = 760.0, molecule: int = 2):
    """CO2-like relaxation-matrix data (HITRANRelmatData) for the VP_Y/VP_W paths.

    Band b: isotopologue 1 (2 for b % 3 == 2), l_i = b % 3, l_f = l_i + (b + 1) % 2;
    centre ~ U(nu_lo + 30, nu_hi - 30).  P and R branches at 2B spacing (B = 0.39 cm^-1),
    plus a Q branch packed near the centre (nu_c - 8e-4 J(J+1)) when l_i != l_f; even J
    only for isotopologue 1.  Lower-state populations (2J+1) exp(-c2 B J(J+1)/296)/527,
    band strengths 10^U(-20, -18), DipoT = Dipo0 from S = Dipo^2 PopuT0 nu stim;
    gamma_air = 0.075 - 3e-4 J (>= 0.05), n_air 0.72, shift -0.0025 cm^-1/atm.  Each
    (l_i, l_f) W0B0 table couples every branch pair and J pair with
    exp(W0) = 0.025 exp(-|J - J'|/8) cm^-1/atm and B0 = 0.75."""
    from .relmat import HITRANRelmatData, RelmatBand, W0B0Table, relmat_lines
    g = np.random.Generator(np.random.PCG64(seed))
    c2, B = 1.4388, 0.39
    bands, tables = [], {}
    for b in range(n_bands):
        isot = 2 if b % 3 == 2 else 1
        li = b % 3
        lf = li + (b + 1) % 2
        nu_c = g.uniform(nu_lo + 30.0, nu_hi - 30.0)
        s_band = 10.0 ** g.uniform(-20.0, -18.0)
        js = list(range(0, j_max + 1, 2 if isot == 1 else 1))
        rows = []
        for br in ((-1, 0, 1) if li != lf else (-1, 1)):
            for J in js:
                if br != 1 and J == 0:
                    continue
                nu = (nu_c - 2 * B * J if br == -1 else (nu_c + 2 * B * (J + 1) if br == 1 else nu_c - 8e-4 * J * (J + 1)))
                nu += g.uniform(-0.01, 0.01)
                E = B * J * (J + 1)
                pop = (2 * J + 1) * np.exp(-c2 * E / 296.0) / 527.0
                stim = 1.0 - np.exp(-c2 * nu / 296.0)
                dip = np.sqrt(s_band * pop / (pop * nu * stim))
                gam = max(0.075 - 3e-4 * J, 0.05) + g.uniform(-0.002, 0.002)
                rows.append((isot, nu, J, br, gam, 0.72, -0.0025, E, dip, pop, dip))
        rows.sort(key=lambda r: r[1])
        L = relmat_lines(rows)
        bands.append(RelmatBand(f"SB{b:02d}", li, lf, isot, float(L["nu"].min()), float(L["nu"].max()), L,
                                molecule))
        key = (min(li, lf), max(li, lf))
        if key not in tables:
            t = W0B0Table()
            for sub in ("pp", "pq", "pr", "qp", "qq", "qr", "rp", "rq", "rr"):
                d = t.get(sub)
                for J in range(0, j_max + 2):
                    for Jp in range(0, J + 1):
                        d[(J, Jp)] = (float(np.log(0.025 * np.exp(-(J - Jp) / 8.0))), 0.75)
                        d[(Jp, J)] = d[(J, Jp)]
            tables[key] = t
    return HITRANRelmatData(bands, tables, molecule)
