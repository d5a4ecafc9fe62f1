"""Properties of the oracle's forward_model that the GPU parity tests rely on."""
import numpy as np
import pytest

from conftest import load_package


@pytest.fixture(scope="module")
def pkg():
    return load_package()


@pytest.fixture(scope="module")
def small_case(pkg):
    lists = {2: pkg.synthetic.synthetic_linelist(800, 2, 7, 690.0, 712.0),
             1: pkg.synthetic.synthetic_linelist(400, 1, 8, 690.0, 712.0)}
    prof = pkg.afgl_atmosphere("midlatitude_summer")
    return lists, dict(p=prof.pressure, T=prof.temperature, vmr=prof.vmr)


def test_channel_window_equals_full_run(oracle, orc_mod, small_case):
    lists, prof = small_case
    snd = orc_mod.sounder(698.0, 704.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    opt = orc_mod.fm_options(internal_dnu=0.0025, continua=("h2o", "co2"))
    ll = {s: l.lines for s, l in lists.items()}
    R, BT = oracle.forward_model(prof, ll, snd, opt)
    Rw, BTw = oracle.forward_model(prof, ll, snd, opt, channels=(7, 15))
    assert np.array_equal(Rw, R[7:15]) and np.array_equal(BTw, BT[7:15])


def test_forward_physical_ranges(oracle, orc_mod, small_case):
    lists, prof = small_case
    snd = orc_mod.sounder(698.0, 704.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    ll = {s: l.lines for s, l in lists.items()}
    _, BT = oracle.forward_model(prof, ll, snd, orc_mod.fm_options(internal_dnu=0.0025))
    assert np.all(np.isfinite(BT)) and np.all((BT > 180.0) & (BT < 320.0))
    # 10x stronger lines move the emission to the warm stratosphere: the band warms
    lines2 = {s: l.lines.copy() for s, l in lists.items()}
    lines2[2]["intensity"] *= 10.0
    _, BT2 = oracle.forward_model(prof, lines2, snd, orc_mod.fm_options(internal_dnu=0.0025))
    assert np.mean(BT2) > np.mean(BT) + 1.0
    # DPTMIN at 1e-6 is a sub-mK perturbation of the spectrum
    _, BT0 = oracle.forward_model(prof, ll, snd, orc_mod.fm_options(internal_dnu=0.0025, dptmn=0.0))
    assert np.max(np.abs(BT0 - BT)) < 5e-3


def test_transparent_atmosphere_sees_surface(oracle, orc_mod, small_case, pkg):
    _, prof = small_case
    snd = orc_mod.sounder(698.0, 704.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    opt = orc_mod.fm_options(internal_dnu=0.0025, apply_continuum=False, T_sfc=300.0)
    empty = pkg.HITRANLinelist(np.zeros(0, dtype=orc_mod.LINE_DTYPE)).lines
    _, BT = oracle.forward_model(prof, {2: empty}, snd, opt)
    # the ILS of a Planck spectrum at 300 K is ~300 K in brightness temperature
    np.testing.assert_allclose(BT, 300.0, atol=0.05)
