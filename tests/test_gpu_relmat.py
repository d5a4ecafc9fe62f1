"""Relaxation-matrix line mixing on the GPU against the numpy oracle (oracle/lm_oracle.py).

Tolerances: the device pole sums are FP64 (faddeeva64 against scipy's wofz, ~1e-13
relative), so perturbations agree to 1e-10 of their peak; with VP_W eigenmodes from the
library's own eigensolver against LAPACK, to 1e-9.  Forward models: FP64 path within
1e-6 K of the oracle, the mixed path within the usual 0.01 K RMS / 0.05 K max.
"""
import math

import numpy as np
import pytest

import lm_oracle as lo
from conftest import load_package

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    return load_package()


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.B200Context()
    yield c
    c.close()


@pytest.fixture(scope="module")
def relmat(pkg):
    return pkg.synthetic.synthetic_relmat(n_bands=6, j_max=40)


def band(pkg, name, rows, li=1, lf=1, isot=1):
    L = pkg.relmat_lines(rows)
    return pkg.RelmatBand(name, li, lf, isot, float(L["nu"].min()), float(L["nu"].max()), L)


def grid(a, b, d):
    return a + d * np.arange(int(round((b - a) / d)) + 1)


def test_vpw_band_xsec_reference_cases(pkg, ctx):
    """runtests.jl:760-853 on the device: the no-coupling Voigt limit, the cutoff, the
    far-wing switch (x_far = 122, inf and 0) with coupled Q lines."""
    b = band(pkg, "TEST02", [(1, 700.00, 0, 0, 0.07, 0.7, 0.0, 200.0, 1.0, 0.5, 1.0),
                             (1, 700.05, 2, 0, 0.07, 0.7, 0.0, 220.0, 1.0, 0.45, 1.0)])
    m = pkg.band_modes(b, pkg.W0B0Table(), 296.0, 0.5)
    g = grid(699.5, 700.5, 0.005)
    got = pkg.compute_vpw_band_xsec(g, m, cutoff=10.0, x_far=np.inf, backend=ctx)
    ref = lo.vpw_band_xsec(g, m.poles, m.amplitudes, m.f, 10.0, np.inf)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert np.all(pkg.compute_vpw_band_xsec(grid(800.0, 800.5, 0.005), m, cutoff=10.0, backend=ctx) == 0.0)
    q = band(pkg, "TESTQ", [(1, 667.00, 20, 0, 0.03, 0.7, 0.0, 300.0, 1.0, 1.0, 1.0),
                            (1, 667.05, 18, 0, 0.03, 0.7, 0.0, 260.0, 1.0, 0.8, 1.0)])
    wt = pkg.W0B0Table()
    wt.qq[(20, 18)] = (math.log(0.03), 0.5)
    m = pkg.band_modes(q, wt, 250.0, 0.1)
    g = grid(665.0, 669.0, 0.002)
    out = {}
    for xf in (np.inf, 122.0, 0.0):
        out[xf] = pkg.compute_vpw_band_xsec(g, m, cutoff=25.0, x_far=xf, backend=ctx)
        ref = lo.vpw_band_xsec(g, m.poles, m.amplitudes, m.f, 25.0, xf)
        assert np.max(np.abs(out[xf] - ref)) <= 1e-12 * np.max(np.abs(ref)), xf
    pk = np.max(np.abs(out[np.inf]))
    assert np.max(np.abs(out[122.0] - out[np.inf])) < 1e-5 * pk
    assert np.max(np.abs(out[0.0] - out[np.inf])) > 1e-3 * pk


@pytest.mark.parametrize("T,p", [(296.0, 1.0), (250.0, 0.4), (215.0, 0.02)])
def test_dispersive_correction(pkg, ctx, relmat, T, p):
    g = grid(640.0, 770.0, 0.01)
    for kw in (dict(), dict(isotopes={1}), dict(min_band_strength=1e-19)):
        got = pkg.compute_lm_dispersive_correction(g, relmat, T, p, backend=ctx, **kw)
        ref = lo.lm_dispersive_correction(g, relmat.bands, relmat.wtfit, T, p, **kw)
        assert np.max(np.abs(ref)) > 0
        assert np.max(np.abs(got - ref)) <= 1e-10 * np.max(np.abs(ref)), kw


@pytest.mark.parametrize("T,p", [(296.0, 1.0), (240.0, 0.3)])
def test_vpw_perturbation(pkg, ctx, relmat, T, p):
    g = grid(640.0, 770.0, 0.01)
    wl = pkg.default_vpw_whitelist(relmat, n_top=3)
    got = pkg.vpw_perturbation(g, relmat, T, p, whitelist=wl, backend=ctx)
    ref = lo.vpw_perturbation(g, relmat.bands, relmat.wtfit, T, p, wl)
    assert np.max(np.abs(got - ref)) <= 1e-9 * np.max(np.abs(ref))
    one = relmat.bands[1]
    k = (min(one.li, one.lf), max(one.li, one.lf))
    got = pkg.compute_vpw_band_perturbation(g, one, relmat.wtfit[k], T, p, backend=ctx)
    ref = lo.vpw_band_perturbation(g, one, relmat.wtfit[k], T, p)
    # one band's perturbation is a difference of two sums that agree to ~1e-4: compare
    # against the scale of the sums
    lam, A, f = lo.band_modes(one, relmat.wtfit[k], T, p, 1e-4)
    scale = np.max(np.abs(lo.vpw_band_xsec(g, lam, A, f)))
    assert np.max(np.abs(ref)) > 1e-6 * scale
    assert np.max(np.abs(got - ref)) <= 1e-9 * scale  # as the modes themselves (test_relmat_host)


def test_voigt_lm_and_vpw_cross_sections(pkg, ctx, oracle, relmat):
    ll = pkg.synthetic.synthetic_linelist(3000, 2, 77, 640.0, 770.0)
    g = grid(660.0, 740.0, 0.005)
    T, p = 260.0, 0.6
    sv = oracle.voigt_xsec(ll.lines, g, T, p)
    iso = {1}
    wl = pkg.default_vpw_whitelist(relmat, n_top=2)
    d_vpy = lo.lm_dispersive_correction(g, relmat.bands, relmat.wtfit, T, p, isotopes=iso)
    d_vpw = lo.vpw_perturbation(g, relmat.bands, relmat.wtfit, T, p, wl, isotopes=iso)
    got = pkg.compute_voigt_lm_cross_sections(g, ll, relmat, T, p, isotopes=iso, backend=ctx)
    ref = np.maximum(sv + d_vpy, 0.0)
    assert np.max(np.abs(got - ref)) <= 1e-10 * np.max(ref)
    got = pkg.compute_voigt_vpw_cross_sections(g, ll, relmat, T, p, whitelist=wl, isotopes=iso, backend=ctx)
    ref = np.maximum(sv + d_vpw, 0.0)
    assert np.max(np.abs(got - ref)) <= 1e-9 * np.max(ref)


def _fm_case(pkg):
    relmat = pkg.synthetic.synthetic_relmat(n_bands=4, j_max=24, seed=1005, nu_lo=670.0, nu_hi=735.0)
    lists = {2: pkg.synthetic.synthetic_linelist(2000, 2, 78, 660.0, 745.0),
             1: pkg.synthetic.synthetic_linelist(500, 1, 79, 660.0, 745.0)}
    prof = pkg.afgl_atmosphere("midlatitude_summer")
    snd = pkg.Sounder.make(695.0, 710.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    return relmat, lists, prof, snd


@pytest.mark.parametrize("vpw", [False, True])
def test_forward_model_relmat(pkg, ctx, oracle, orc_mod, vpw):
    """forward_model with VPYLineMixing(relmat) / VPWLineMixing(relmat) against the oracle
    forward model, whose per-layer perturbation comes from lm_oracle at the layer's
    Curtis-Godson (T, p) of CO2; the isotope filter keeps the bands the CO2 list has."""
    relmat, lists, prof, snd = _fm_case(pkg)
    lm = pkg.VPWLineMixing(relmat, n_top=2) if vpw else pkg.VPYLineMixing(relmat)
    iso = {1}
    kw = dict(internal_dnu=0.01, apply_continuum=True, continua=("h2o", "co2"))

    def pert(T, p, g):
        if vpw:
            return lo.vpw_perturbation(g, relmat.bands, relmat.wtfit, T, p, lm.whitelist, isotopes=iso)
        return lo.lm_dispersive_correction(g, relmat.bands, relmat.wtfit, T, p, isotopes=iso)

    opt = orc_mod.fm_options(line_mixing=3 if vpw else 2, **kw)
    R0, BT0 = oracle.forward_model(dict(p=prof.pressure, T=prof.temperature, vmr=prof.vmr),
                                   {s: l.lines for s, l in lists.items()},
                                   orc_mod.sounder(snd.nu_min, snd.nu_max, snd.dnu, opd_max=snd.opd_max,
                                                   fwhm_gauss=snd.fwhm_gauss), opt, lm=(2, pert))
    _, Rn, BTn = pkg.forward_model(prof, lists, sounder=snd, backend=ctx, precision="fp64", **kw)
    assert np.max(np.abs(BTn - BT0)) > 1e-3  # line mixing changes the spectrum
    _, R, BT = pkg.forward_model(prof, lists, sounder=snd, backend=ctx, precision="fp64", line_mixing=lm, **kw)
    assert np.max(np.abs(BT - BT0)) < 1e-6
    _, Rm, BTm = pkg.forward_model(prof, lists, sounder=snd, backend=ctx, precision="mixed", line_mixing=lm, **kw)
    assert np.sqrt(np.mean((BTm - BT0) ** 2)) < 0.01 and np.max(np.abs(BTm - BT0)) < 0.05


@pytest.mark.parametrize("vpw", [False, True])
def test_jacobian_relmat_vs_fd(pkg, ctx, oracle, orc_mod, vpw):  # runtests.jl:1426-1478
    """The analytic Jacobian with VPYLineMixing(relmat) / VPWLineMixing(relmat) against
    central differences of the oracle forward model (whose perturbation comes from
    lm_oracle), on the reference suite's coupled CO2 Q branch and 6-level profile."""
    dipo = 1.7e-13
    L = pkg.relmat_lines([(1, 700.40, 20, 0, 0.09, 0.75, -0.004, 250.0, dipo, 0.10, dipo),
                          (1, 700.55, 18, 0, 0.09, 0.75, -0.004, 240.0, dipo, 0.09, dipo),
                          (1, 701.30, 16, 0, 0.085, 0.75, -0.004, 300.0, 0.9 * dipo, 0.08, 0.9 * dipo)])
    b = pkg.RelmatBand("CO2Q", 1, 1, 1, 700.4, 701.3, L)
    wt = pkg.W0B0Table()
    wt.qq[(20, 18)] = (math.log(0.035), 0.5)
    wt.qq[(20, 16)] = (math.log(0.025), 0.5)
    wt.qq[(18, 16)] = (math.log(0.030), 0.5)
    relmat = pkg.HITRANRelmatData([b], {(1, 1): wt})
    lines = np.zeros(4, dtype=orc_mod.LINE_DTYPE)
    for k, (nu, S, E) in enumerate([(700.40, 2.0e-24, 250.0), (700.55, 1.8e-24, 240.0),
                                    (700.95, 9.0e-25, 500.0), (701.30, 1.4e-24, 300.0)]):
        lines[k] = (2, 1, nu, S, 1.0, 0.09, 0.08, E, 0.75, -0.004)
    ll = {2: pkg.HITRANLinelist(lines)}
    p = np.linspace(1000.0, 200.0, 6)
    T = 288.0 + (225.0 - 288.0) * (1000.0 - p) / 800.0
    prof = pkg.AtmosphericProfile(p, T, (1000.0 - p) / 66.0, {2: np.full(6, 4.0e-4)})
    spec = pkg.StateVectorSpec(6, [pkg.CO2], include_temperature=True, include_tsfc=True,
                               include_emissivity=True)
    snd_kw = dict(nu_min=699.0, nu_max=703.0, dnu=0.5, opd_max=2.0, fwhm_gauss=0.5)
    kw = dict(apply_continuum=False, with_ils=True, internal_dnu=0.005)
    lm = pkg.VPWLineMixing(relmat, whitelist={"CO2Q"}) if vpw else pkg.VPYLineMixing(relmat)

    def pert(Tl, pl, g):
        if vpw:
            return lo.vpw_perturbation(g, relmat.bands, relmat.wtfit, Tl, pl, {"CO2Q"}, isotopes={1})
        return lo.lm_dispersive_correction(g, relmat.bands, relmat.wtfit, Tl, pl, isotopes={1})

    steps = np.array([0.1] * 6 + [1e-3] * 6 + [0.1, 1e-3])
    Kf, yf, _ = oracle.fd_jacobian(dict(p=p, T=T, vmr={2: np.full(6, 4.0e-4)}), {2: lines},
                                   orc_mod.sounder(**snd_kw), dict(line_mixing=3 if vpw else 2, **kw),
                                   retrieved=[2], T_sfc=290.0, eps_sfc=0.98, steps=steps, lm=(2, pert))
    jac = pkg.analytic_jacobian(prof, ll, spec, sounder=pkg.Sounder.make(**snd_kw), T_sfc=290.0, eps_sfc=0.98,
                                backend=ctx, line_mixing=lm, **kw)
    rel = lambda c: np.max(np.abs(jac.K[:, c] - Kf[:, c])) / (np.max(np.abs(Kf[:, c])) + 1e-30)
    assert np.max(np.abs(jac.y0 - yf)) < 0.01
    assert rel(slice(6, 12)) < 1e-3     # CO2 column: FP32 line sum against FP64 differences
    assert rel(slice(0, 6)) < 2e-3      # temperature
    assert np.max(np.abs(jac.K[:, 12] - Kf[:, 12])) < 1e-3
    assert np.max(np.abs(jac.K[:, 13] - Kf[:, 13])) < 1e-2
    # and the line mixing is visible in the Jacobian
    jn = pkg.analytic_jacobian(prof, ll, spec, sounder=pkg.Sounder.make(**snd_kw), T_sfc=290.0, eps_sfc=0.98,
                               backend=ctx, **kw)
    assert np.max(np.abs(jn.K[:, 6:12] - Kf[:, 6:12])) > 3 * np.max(np.abs(jac.K[:, 6:12] - Kf[:, 6:12]))


def test_relmat_errors(pkg, ctx):
    c = pkg.B200Context()
    try:
        g = grid(700.0, 701.0, 0.01)
        with pytest.raises(pkg.IRSError):  # no relmat uploaded
            pkg._lib.check(c.lib.irs_lm_perturbation(c.h, 2, pkg.dptr(g), len(g), 250.0, 0.5, 25.0, 122.0, 1e-4,
                                                     0, pkg.dptr(np.empty(len(g)))))
        with pytest.raises(pkg.IRSError):  # bad mode
            pkg._lib.check(c.lib.irs_lm_perturbation(c.h, 7, pkg.dptr(g), len(g), 250.0, 0.5, 25.0, 122.0, 1e-4,
                                                     0, pkg.dptr(np.empty(len(g)))))
        with pytest.raises(pkg.IRSError):  # relmat line mixing with another Voigt method
            relmat, lists, prof, snd = _fm_case(pkg)
            pkg.forward_model(prof, lists, sounder=snd, backend=c, internal_dnu=0.01,
                              method=pkg.VoigtMethod.Weideman, line_mixing=pkg.VPYLineMixing(relmat))
    finally:
        c.close()
