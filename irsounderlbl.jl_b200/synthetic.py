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
