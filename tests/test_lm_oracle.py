"""Pins the relmat line-mixing oracle (oracle/lm_oracle.py) on the reference's own
known-answer tests (test/runtests.jl:714-944 of IRSounderLBL.jl): the no-coupling limit
of band_modes, the VP_W pole sum against the band-uniform Voigt sum, the far-wing
shortcut, the band-strength cutoff and the CH4 plumbing.  CPU only."""
import math

import numpy as np
import pytest

import lm_oracle as lo
from conftest import load_package


@pytest.fixture(scope="module")
def pkg():
    return load_package()


def band(pkg, name, rows, li=1, lf=1, isot=1, molecule=2):
    L = pkg.relmat_lines(rows)
    return pkg.RelmatBand(name, li, lf, isot, float(L["nu"].min()), float(L["nu"].max()), L, molecule)


def grid(a, b, d):  # wavenumber_grid(a, b, d)
    return a + d * np.arange(int(round((b - a) / d)) + 1)


def test_no_coupling_limit(pkg):  # runtests.jl:714-759
    b = band(pkg, "TEST01", [(1, 700.0, 0, 0, 0.07, 0.7, 0.0, 200.0, 1.0, 0.5, 1.0),
                             (1, 710.0, 2, 0, 0.07, 0.7, 0.0, 220.0, 1.0, 0.45, 1.0)])
    T, p = 296.0, 0.5
    lam, A, f = lo.band_modes(b, pkg.W0B0Table(), T, p)
    assert len(lam) == 2 and len(A) == 2
    k = np.argsort(lam.real)
    lam, A = lam[k], A[k]
    assert abs(lam[0].real - 700.0) < 1e-10 and abs(lam[1].real - 710.0) < 1e-10
    assert abs(lam[0].imag - p * 0.07) < 1e-10 and abs(lam[1].imag - p * 0.07) < 1e-10
    for a, (nu, pop) in zip(A, ((700.0, 0.5), (710.0, 0.45))):
        S = 1.0 * pop * nu * (1 - math.exp(-1.4388 * nu / T))
        assert abs(a.real - S) <= 1e-12 * S
        assert abs(a.imag) < 1e-12 * abs(a.real)
    gD = 3.5812e-7 * 705.0 * math.sqrt(T / 43.98983)
    assert abs(f - math.sqrt(math.log(2.0)) / gD) <= 1e-12 * f


def test_vpw_xsec_matches_voigt_without_coupling(pkg):  # runtests.jl:760-806
    from scipy.special import wofz
    b = band(pkg, "TEST02", [(1, 700.00, 0, 0, 0.07, 0.7, 0.0, 200.0, 1.0, 0.5, 1.0),
                             (1, 700.05, 2, 0, 0.07, 0.7, 0.0, 220.0, 1.0, 0.45, 1.0)])
    T, p = 296.0, 0.5
    lam, A, f = lo.band_modes(b, pkg.W0B0Table(), T, p)
    g = grid(699.5, 700.5, 0.005)
    sig = lo.vpw_band_xsec(g, lam, A, f, cutoff=10.0, x_far=np.inf)
    ref = np.zeros(len(g))
    for nu, pop in ((700.00, 0.5), (700.05, 0.45)):
        S = pop * nu * (1 - math.exp(-1.4388 * nu / T))
        ref += S * f / math.sqrt(math.pi) * wofz((g - nu) * f + 1j * 0.07 * p * f).real
    assert np.max(np.abs(sig - ref)) / np.max(np.abs(ref)) < 1e-12
    assert np.all(lo.vpw_band_xsec(grid(800.0, 800.5, 0.005), lam, A, f, cutoff=10.0) == 0.0)


def test_far_wing_shortcut(pkg):  # runtests.jl:808-853
    b = band(pkg, "TESTQ", [(1, 667.00, 20, 0, 0.03, 0.7, 0.0, 300.0, 1.0, 1.0, 1.0),
                            (1, 667.05, 18, 0, 0.03, 0.7, 0.0, 260.0, 1.0, 0.8, 1.0)])
    wt = pkg.W0B0Table()
    wt.qq[(20, 18)] = (math.log(0.03), 0.5)
    T, p, cut = 250.0, 0.1, 25.0
    g = grid(665.0, 669.0, 0.002)
    lam, A, f = lo.band_modes(b, wt, T, p)
    assert np.any(A.imag != 0.0)
    ex = lo.vpw_band_xsec(g, lam, A, f, cut, np.inf)
    fa = lo.vpw_band_xsec(g, lam, A, f, cut, lo.X_FAR)
    lz = lo.vpw_band_xsec(g, lam, A, f, cut, 0.0)
    pk = np.max(np.abs(ex))
    assert np.max(np.abs(fa - ex)) < 1e-5 * pk
    assert np.max(np.abs(lz - ex)) > 1e-3 * pk
    Y = lo.calc_y(b, wt, T)
    lines = lo.dispersive_lines(b, Y, T, p)
    ey = lo.dispersive_eval(g, *lines, cutoff=cut, x_far=np.inf)
    fy = lo.dispersive_eval(g, *lines, cutoff=cut, x_far=lo.X_FAR)
    ly = lo.dispersive_eval(g, *lines, cutoff=cut, x_far=0.0)
    pky = np.max(np.abs(ey))
    assert pky > 0
    assert np.max(np.abs(fy - ey)) < 1e-5 * pky
    assert np.max(np.abs(ly - ey)) > 1e-3 * pky


def _two_bands(pkg):
    s = band(pkg, "STRONG", [(1, 700.00, 20, 0, 0.03, 0.7, 0.0, 300.0, 1.0, 1.0, 1.0),
                             (1, 700.05, 18, 0, 0.03, 0.7, 0.0, 260.0, 1.0, 0.8, 1.0)])
    w = band(pkg, "WEAK", [(1, 720.00, 4, 0, 0.03, 0.7, 0.0, 300.0, 1.0e-3, 1.0, 1.0e-3),
                           (1, 720.05, 2, 0, 0.03, 0.7, 0.0, 260.0, 1.0e-3, 0.8, 1.0e-3)])
    wt = pkg.W0B0Table()
    wt.qq[(20, 18)] = (math.log(0.03), 0.5)
    wt.qq[(4, 2)] = (math.log(0.03), 0.5)
    return s, w, {(1, 1): wt}


def test_band_strength_cutoff(pkg):  # runtests.jl:855-906
    s, w, tabs = _two_bands(pkg)
    sS, sW = lo.band_eff_strength(s), lo.band_eff_strength(w)
    assert sS > sW
    thr = math.sqrt(sS * sW)
    T, p = 250.0, 0.5
    g = grid(695.0, 725.0, 0.01)
    full = lo.lm_dispersive_correction(g, [s, w], tabs, T, p, min_band_strength=0.0)
    cut = lo.lm_dispersive_correction(g, [s, w], tabs, T, p, min_band_strength=thr)
    strong = lo.lm_dispersive_correction(g, [s], tabs, T, p, min_band_strength=0.0)
    assert np.array_equal(cut, strong)
    assert np.max(np.abs(full - cut)) > 0.0
    w2 = pkg.RelmatBand("WEAK2", 1, 1, 2, 720.0, 720.05, w.lines)
    assert lo.band_eff_strength(w2) == sW


def test_ch4_plumbing(pkg):  # runtests.jl:908-944
    assert lo.mass_amu(6, 1) == 16.031300 and lo.iso_abund(6, 1) == 0.988274
    assert lo.mass_amu(2, 1) == 43.98983 and lo.mass_amu(99, 1) == 44.0
    b = band(pkg, "CH4Q", [(1, 1306.00, 6, 0, 0.05, 0.75, 0.0, 220.0, 1.0, 1.0, 1.0),
                           (1, 1306.05, 5, 0, 0.05, 0.75, 0.0, 200.0, 1.0, 0.9, 1.0)], molecule=6)
    wt = pkg.W0B0Table()
    wt.qq[(6, 5)] = (math.log(0.04), 0.5)
    sig = lo.lm_dispersive_correction(grid(1304.0, 1308.0, 0.01), [b], {(1, 1): wt}, 250.0, 0.5)
    assert np.all(np.isfinite(sig)) and np.max(np.abs(sig)) > 0.0


def test_perturbation_vanishes_without_coupling(pkg):
    """compute_vpw_band_perturbation -> 0 in the no-coupling limit (line_mixing.jl:1055-1063)."""
    b = band(pkg, "TEST02", [(1, 700.00, 0, 0, 0.07, 0.7, 0.0, 200.0, 1.0, 0.5, 1.0),
                             (1, 700.05, 2, 0, 0.07, 0.7, 0.0, 220.0, 1.0, 0.45, 1.0)])
    g = grid(699.5, 700.5, 0.005)
    lam, A, f = lo.band_modes(b, pkg.W0B0Table(), 250.0, 0.5)
    full = lo.vpw_band_xsec(g, lam, A, f)
    d = lo.vpw_band_perturbation(g, b, pkg.W0B0Table(), 250.0, 0.5, keep_threshold=0.0)
    assert np.max(np.abs(d)) < 1e-12 * np.max(np.abs(full))
