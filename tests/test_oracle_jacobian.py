"""The oracle's analytic Jacobian against its own central finite differences, on the
synthetic fixtures and with the tolerances of the reference's Jacobian test suite
(test/runtests.jl:1221-1478).  This pins the Jacobian oracle the GPU Jacobian is
later compared with."""
import numpy as np
import pytest

IASI_SUB = dict(nu_min=699.0, nu_max=705.0, dnu=0.5, opd_max=2.0, fwhm_gauss=0.5)


def mk(orc_mod, mol, lines):
    a = np.zeros(len(lines), dtype=orc_mod.LINE_DTYPE)
    for k, (nu, S, gair, gself, E, n, d) in enumerate(lines):
        a[k] = (mol, 1, nu, S, 1.0, gair, gself, E, n, d)
    return a


def profile(nlev, species):
    p = np.linspace(1000.0, 200.0, nlev)
    T = 288.0 + (225.0 - 288.0) * (1000.0 - p) / 800.0
    return dict(p=p, T=T, vmr=species(p))


def rel(a, b, cols):
    return np.max(np.abs(a[:, cols] - b[:, cols])) / (np.max(np.abs(b[:, cols])) + 1e-30)


def steps_for(nlev, n_vmr, include_T=True):
    s = []
    if include_T:
        s += [0.1] * nlev
    s += [1e-3] * (nlev * n_vmr)
    return s + [0.1, 1e-3]


@pytest.mark.parametrize("nlev", [6, 11])
def test_vmr_jacobian_vs_fd(oracle, orc_mod, nlev):  # runtests.jl:1221-1282
    ll = {2: mk(orc_mod, 2, [(700.5, 3.0e-23, 0.08, 0.10, 250.0, 0.75, 0.0),
                             (702.0, 1.0e-23, 0.08, 0.10, 250.0, 0.75, 0.0)])}
    prof = profile(nlev, lambda p: {2: np.full(len(p), 4.0e-4)})
    snd = orc_mod.sounder(**IASI_SUB)
    opt = orc_mod.fm_options(apply_continuum=False, with_ils=True, T_sfc=290.0, eps_sfc=0.98, dptmn=0.0,
                             internal_dnu=0.005)
    K, y = oracle.analytic_jacobian(prof, ll, snd, opt, retrieved=[2], include_T=False)
    Kf, yf, _ = oracle.fd_jacobian(prof, ll, snd, dict(apply_continuum=False, with_ils=True, internal_dnu=0.005),
                                   retrieved=[2], include_T=False, T_sfc=290.0, eps_sfc=0.98,
                                   steps=[1e-3] * nlev + [0.5, 1e-3])
    assert K.shape == (13, nlev + 2)
    assert np.max(np.abs(y - yf)) < 1e-9
    assert rel(K, Kf, slice(0, nlev)) < 1e-5
    assert np.max(np.abs(K[:, nlev] - Kf[:, nlev])) < 1e-4
    assert np.max(np.abs(K[:, nlev + 1] - Kf[:, nlev + 1])) < 1e-4
    i_line = np.argmin(y)
    assert np.sum(K[i_line, :nlev]) < 0.0


def test_temperature_jacobian_vs_fd(oracle, orc_mod):  # runtests.jl:1345-1380
    ll = {2: mk(orc_mod, 2, [(700.5, 2.0e-21, 0.07, 0.08, 250.0, 0.75, -0.003),
                             (702.0, 8.0e-22, 0.07, 0.08, 600.0, 0.75, -0.003)])}
    prof = profile(6, lambda p: {2: np.full(len(p), 4.0e-4)})
    snd = orc_mod.sounder(**IASI_SUB)
    opt = orc_mod.fm_options(apply_continuum=False, with_ils=True, T_sfc=290.0, eps_sfc=0.98, dptmn=0.0,
                             internal_dnu=0.005)
    K, y = oracle.analytic_jacobian(prof, ll, snd, opt, retrieved=[2])
    Kf, yf, _ = oracle.fd_jacobian(prof, ll, snd, dict(apply_continuum=False, with_ils=True, internal_dnu=0.005),
                                   retrieved=[2], T_sfc=290.0, eps_sfc=0.98, steps=steps_for(6, 1))
    assert np.max(np.abs(y - yf)) < 1e-9
    assert rel(K, Kf, slice(0, 6)) < 1e-3
    assert np.max(np.abs(K[:, 12] - Kf[:, 12])) < 1e-4
    assert np.max(np.abs(K[:, 13] - Kf[:, 13])) < 1e-4
    assert K[np.argmin(y), 0] > 0.0


@pytest.mark.parametrize("species", ["h2o", "co2"])
def test_continuum_coupling_vs_fd(oracle, orc_mod, species):  # runtests.jl:1383-1424
    if species == "h2o":
        ll = {1: mk(orc_mod, 1, [(700.6, 3.0e-21, 0.09, 0.45, 200.0, 0.70, 0.005),
                                 (702.3, 1.2e-21, 0.09, 0.45, 450.0, 0.70, 0.005)])}
        prof = profile(6, lambda p: {1: 0.01 * np.exp(-3.0 * (1000.0 - p) / 800.0)})
        sp, conts = 1, ("h2o",)
    else:
        ll = {2: mk(orc_mod, 2, [(700.5, 2.0e-21, 0.07, 0.08, 250.0, 0.75, -0.006),
                                 (702.0, 8.0e-22, 0.07, 0.08, 600.0, 0.75, -0.006)])}
        prof = profile(6, lambda p: {2: np.full(len(p), 4.0e-4)})
        sp, conts = 2, ("co2",)
    snd = orc_mod.sounder(**IASI_SUB)
    kw = dict(apply_continuum=True, continua=conts, with_ils=True, internal_dnu=0.005)
    opt = orc_mod.fm_options(T_sfc=290.0, eps_sfc=0.98, dptmn=0.0, **kw)
    K, y = oracle.analytic_jacobian(prof, ll, snd, opt, retrieved=[sp])
    Kf, yf, _ = oracle.fd_jacobian(prof, ll, snd, kw, retrieved=[sp], T_sfc=290.0, eps_sfc=0.98,
                                   steps=steps_for(6, 1))
    Koff, _ = oracle.analytic_jacobian(prof, ll, snd, opt, retrieved=[sp], vmr_coupling=False)
    assert np.max(np.abs(y - yf)) < 1e-9
    assert rel(K, Kf, slice(6, 12)) < 1e-5
    assert rel(K, Kf, slice(0, 6)) < 1e-5
    assert np.max(np.abs(K[:, 12] - Kf[:, 12])) < 1e-4
    assert np.max(np.abs(K[:, 13] - Kf[:, 13])) < 1e-4
    assert rel(Koff, Kf, slice(6, 12)) > 10 * rel(K, Kf, slice(6, 12))


def test_line_mixing_jacobian_vs_fd(oracle, orc_mod):  # runtests.jl:1427-1478 (per-line Y)
    ll = {2: mk(orc_mod, 2, [(700.40, 2.0e-24, 0.09, 0.08, 250.0, 0.75, -0.004),
                             (700.55, 1.8e-24, 0.09, 0.08, 240.0, 0.75, -0.004),
                             (701.30, 1.4e-24, 0.09, 0.08, 300.0, 0.75, -0.004),
                             (700.95, 9.0e-25, 0.09, 0.08, 500.0, 0.75, -0.004)])}
    y0 = {2: np.array([0.03, -0.02, 0.025, 0.01])}
    prof = profile(6, lambda p: {2: np.full(len(p), 4.0e-4)})
    snd = orc_mod.sounder(699.0, 703.0, 0.5, opd_max=2.0, fwhm_gauss=0.5)
    kw = dict(apply_continuum=False, with_ils=True, line_mixing=True, internal_dnu=0.005)
    opt = orc_mod.fm_options(T_sfc=290.0, eps_sfc=0.98, dptmn=0.0, **kw)
    K, y = oracle.analytic_jacobian(prof, ll, snd, opt, retrieved=[2], y0=y0)
    Kf, yf, _ = oracle.fd_jacobian(prof, ll, snd, kw, retrieved=[2], T_sfc=290.0, eps_sfc=0.98,
                                   steps=steps_for(6, 1), y0=y0)
    # the dispersive term is live in this fixture
    _, BT0 = oracle.forward_model(prof, ll, snd, orc_mod.fm_options(T_sfc=290.0, eps_sfc=0.98, dptmn=0.0, internal_dnu=0.005,
                                                                    apply_continuum=False))
    assert np.max(np.abs(BT0 - y)) > 1e-3
    assert np.max(np.abs(y - yf)) < 1e-9
    assert rel(K, Kf, slice(6, 12)) < 1e-5
    assert rel(K, Kf, slice(0, 6)) < 5e-5
    assert np.max(np.abs(K[:, 12] - Kf[:, 12])) < 1e-4
    assert np.max(np.abs(K[:, 13] - Kf[:, 13])) < 1e-4
