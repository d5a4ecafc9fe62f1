"""Write the golden fixtures in this folder (run: python tests/golden/make_golden.py).

The reference (IRSounderLBL.jl) is Julia and cannot run in this image, and its
test suite stores no golden spectra.  Its Faddeeva function comes from
SpecialFunctions.jl 2.7.2 -> OpenSpecFun_jll 0.5.6 (erfcx of a complex argument,
src/CrossSections/voigt.jl:158-160); scipy.special.wofz implements the same
function, so the fixtures below are generated with scipy:

* ``wofz_grid.npz``: w(x + i y) on a grid covering the line-core region the
  kernels evaluate (|x| <= 130, 1e-6 <= y <= 300).
* ``xsec_fixtures.npz``: cross sections of the synthetic line lists that
  test/runtests.jl builds in memory (the 4-line CO2 fixture of :252-297 and the
  H2O self-broadened fixture of :1318-1343), computed by a direct numpy
  restatement of compute_voigt_cross_sections (voigt.jl:375-462) whose H(x, y)
  is scipy's wofz -- i.e. the reference's algorithm with the reference's
  Faddeeva implementation.  TIPS Q(T) comes from the bundled table.
"""
from pathlib import Path

import numpy as np
import scipy.special as sp

HERE = Path(__file__).resolve().parent
DATA = HERE.parents[1] / "irsounderlbl.jl_b200" / "data"

LINE_DTYPE = np.dtype({
    "names": ["mol_id", "iso_id", "wavenumber", "intensity", "a_coeff", "air_broad",
              "self_broad", "lower_energy", "temp_depend", "pressure_shift"],
    "formats": ["i1", "i1", "f8", "f8", "f8", "f4", "f4", "f8", "f4", "f4"],
    "offsets": [0, 1, 8, 16, 24, 32, 36, 40, 48, 52], "itemsize": 56})
MASS = [18.010, 44.010, 47.998, 44.013, 28.010, 16.043, 31.999, 34.015, 64.065, 36.461, 17.031]


def tips(mol, iso):
    for line in open(DATA / "tips2024_q.csv"):
        if line.startswith("#"):
            continue
        p = line.strip().split(",")
        if int(p[0]) == mol and int(p[1]) == iso:
            return np.array([float(v) for v in p[2:]])
    raise KeyError((mol, iso))


def tips_lookup(q, T):  # partition.jl:10-18
    i_lo = int(np.floor(T)) - 70 + 1
    i_hi = i_lo + 1
    i_lo = min(max(i_lo, 1), len(q))
    i_hi = min(max(i_hi, 1), len(q))
    fr = T - np.floor(T)
    return q[i_lo - 1] * (1 - fr) + q[i_hi - 1] * fr


def mk(mol, nu, S, gair, gself, E, n, delta):
    return (mol, 1, nu, S, 1.0, np.float32(gair), np.float32(gself), E, np.float32(n),
            np.float32(delta))


def xsec(lines, grid, T, p, vs, cutoff, x_far):
    """voigt.jl:375-462 with H = Re wofz (FullFaddeeva)."""
    nsf = {1: 0.95, 2: 0.75}
    dsf = {1: 0.002, 2: -0.003}
    nu0, f, y, Sn = [], [], [], []
    for l in lines:
        mol = int(l["mol_id"])
        n_air = float(l["temp_depend"])
        tr = 296.0 / T
        gl = tr ** n_air * float(l["air_broad"]) * (1 - vs) * p + \
            tr ** nsf.get(mol, n_air) * float(l["self_broad"]) * vs * p
        gd = max(l["wavenumber"] * 3.58126e-7 * np.sqrt(T / MASS[mol - 1]), 1e-10)
        q = tips(mol, int(l["iso_id"]))
        c2 = 1.4387752
        S = l["intensity"] * (tips_lookup(q, 296.0) / tips_lookup(q, T)) * \
            np.exp(-c2 * l["lower_energy"] * (1 / T - 1 / 296.0)) * \
            (1 - np.exp(-c2 * l["wavenumber"] / T)) / (1 - np.exp(-c2 * l["wavenumber"] / 296.0))
        fj = np.sqrt(np.log(2.0)) / gd
        nu0.append(l["wavenumber"] + (float(l["pressure_shift"]) * (1 - vs) + dsf.get(mol, 0.0) * vs) * p)
        f.append(fj)
        y.append(gl * fj)
        Sn.append(S * fj / np.sqrt(np.pi))
    nu0, f, y, Sn = map(np.array, (nu0, f, y, Sn))
    isp = 1 / np.sqrt(np.pi)

    def H(x, yy):
        far = np.abs(x) > x_far
        out = np.where(far, yy * isp / (x * x + yy * yy), 0.0)
        core = ~far
        out[core] = sp.wofz(x[core] + 1j * yy[core]).real
        return out

    xc = cutoff * f
    Hc = H(xc, y)
    sig = np.zeros(len(grid))
    for j in range(len(nu0)):
        d = grid - nu0[j]
        win = np.abs(d) <= cutoff
        x = d[win] * f[j]
        zr = d[win] / cutoff
        sig[win] += Sn[j] * (H(x, np.full_like(x, y[j])) - (2 - zr * zr) * Hc[j])
    return np.maximum(sig, 0.0)


def main():
    x = np.concatenate([np.linspace(0, 12, 161), np.linspace(12.5, 130, 48)])
    x = np.concatenate([-x[::-1][:-1], x])
    y = np.concatenate([[1e-6, 1e-4], np.logspace(-3, np.log10(300), 24)])
    X, Y = np.meshgrid(x, y)
    W = sp.wofz(X + 1j * Y)
    np.savez_compressed(HERE / "wofz_grid.npz", x=X.ravel(), y=Y.ravel(), re=W.real.ravel(),
                        im=W.imag.ravel())

    co2 = np.array([mk(2, 2348.0, 1e-19, 0.07, 0.09, 250.0, 0.75, 0.0),
                    mk(2, 2350.0, 5e-20, 0.07, 0.09, 250.0, 0.75, 0.0),
                    mk(2, 2351.2, 8e-20, 0.07, 0.09, 250.0, 0.75, 0.0),
                    mk(2, 2352.5, 2e-19, 0.07, 0.09, 250.0, 0.75, 0.0)], dtype=LINE_DTYPE)
    g1 = np.array([(2345000 + i) / 1000 for i in range(10001)])  # 2345:0.001:2355
    h2o = np.array([mk(1, 700.6, 3.0e-21, 0.09, 0.45, 200.0, 0.70, 0.005),
                    mk(1, 702.3, 1.2e-21, 0.09, 0.45, 450.0, 0.70, 0.005)], dtype=LINE_DTYPE)
    g2 = np.array([(349000 + i) / 500 for i in range(3501)])  # 698:0.002:705
    np.savez_compressed(
        HERE / "xsec_fixtures.npz",
        co2_lines=co2.view(np.uint8), co2_grid=g1,
        co2_sigma=xsec(co2, g1, 230.0, 0.2, 0.0, 25.0, 122.0),
        co2_sigma_exact=xsec(co2, g1, 230.0, 0.2, 0.0, 25.0, np.inf),
        h2o_lines=h2o.view(np.uint8), h2o_grid=g2,
        h2o_sigma=xsec(h2o, g2, 285.0, 0.9, 0.03, 25.0, 122.0))
    print("wrote", HERE / "wofz_grid.npz", HERE / "xsec_fixtures.npz")


if __name__ == "__main__":
    main()
