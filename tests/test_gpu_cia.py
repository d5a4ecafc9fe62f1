"""CIA on the GPU (inside the RTE kernels) against the FP64 oracle: forward model and
analytic Jacobian (whose continuum derivatives central-difference the CIA terms too,
vmr_jacobian.jl:287-344)."""
import numpy as np
import pytest

from cia_tables import blocks_co2, blocks_n2, blocks_o2
from conftest import load_package

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    return load_package()


@pytest.fixture(scope="module")
def tables():
    return {1: blocks_co2(), 2: blocks_n2(), 3: blocks_o2()}


@pytest.fixture(scope="module")
def ctx(pkg, tables):
    c = pkg.B200Context()
    for pair, b in tables.items():
        c.set_cia(pair, b)
    yield c
    c.close()


@pytest.fixture
def oracle_cia(oracle, tables):
    for pair, b in tables.items():
        oracle.set_cia(pair, b)
    yield oracle
    for pair in tables:
        oracle.set_cia(pair, None)


def _case(pkg):
    lists = {2: pkg.synthetic.synthetic_linelist(400, 2, 7, 690.0, 712.0),
             1: pkg.synthetic.synthetic_linelist(200, 1, 8, 690.0, 712.0)}
    snd = pkg.Sounder.make(697.0, 710.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    return lists, snd


@pytest.mark.parametrize("atm", ["us_standard", "tropical"])
def test_forward_with_cia(pkg, ctx, oracle_cia, orc_mod, atm):
    lists, snd = _case(pkg)
    prof = pkg.afgl_atmosphere(atm)
    kw = dict(internal_dnu=0.0025, continua=("h2o", "co2", "co2_cia", "n2", "o2"))
    R0, BT0 = oracle_cia.forward_model(dict(p=prof.pressure, T=prof.temperature, vmr=prof.vmr),
                                       {s: l.lines for s, l in lists.items()},
                                       orc_mod.sounder(697.0, 710.0, 0.25, opd_max=2.0, fwhm_gauss=0.5),
                                       orc_mod.fm_options(**kw))
    _, _, BTn = pkg.forward_model(prof, lists, sounder=snd, backend=ctx, precision="fp64",
                                  internal_dnu=0.0025, continua=("h2o", "co2"))
    assert np.max(np.abs(BTn - BT0)) > 0.05  # the CIA terms change the spectrum
    _, R, BT = pkg.forward_model(prof, lists, sounder=snd, backend=ctx, precision="fp64", **kw)
    assert np.max(np.abs(BT - BT0)) < 1e-6
    _, Rm, BTm = pkg.forward_model(prof, lists, sounder=snd, backend=ctx, precision="mixed", **kw)
    assert np.sqrt(np.mean((BTm - BT0) ** 2)) < 0.01


def test_jacobian_with_cia(pkg, ctx, oracle_cia, orc_mod):
    lists, snd = _case(pkg)
    prof = pkg.afgl_atmosphere("midlatitude_summer")
    spec = pkg.StateVectorSpec(len(prof.pressure), [pkg.H2O, pkg.CO2], include_emissivity=False)
    kw = dict(internal_dnu=0.005, continua=("h2o", "co2", "co2_cia", "n2", "o2"))
    jac = pkg.analytic_jacobian(prof, lists, spec, sounder=snd, backend=ctx, **kw)
    o = orc_mod.fm_options(dptmn=0.0, **kw)
    Kr, yr = oracle_cia.analytic_jacobian(dict(p=prof.pressure, T=prof.temperature, vmr=prof.vmr),
                                          {s: l.lines for s, l in lists.items()},
                                          orc_mod.sounder(697.0, 710.0, 0.25, opd_max=2.0, fwhm_gauss=0.5), o,
                                          retrieved=[1, 2], include_eps=False)
    assert np.max(np.abs(jac.y0 - yr)) < 0.01
    n = len(prof.pressure)
    for blk in (slice(0, n), slice(n, 2 * n), slice(2 * n, 3 * n), slice(3 * n, 3 * n + 1)):
        rel = np.max(np.abs(jac.K[:, blk] - Kr[:, blk])) / np.max(np.abs(Kr[:, blk]))
        assert rel < 2e-4, (blk, rel)
    jn = pkg.analytic_jacobian(prof, lists, spec, sounder=snd, backend=ctx, internal_dnu=0.005,
                               continua=("h2o", "co2"))
    assert np.max(np.abs(jn.K[:, :n] - Kr[:, :n])) > 3 * np.max(np.abs(jac.K[:, :n] - Kr[:, :n]))


def test_cia_table_errors(pkg, ctx):
    with pytest.raises(pkg.IRSError):
        ctx.set_cia(4, blocks_n2())
    with pytest.raises(pkg.IRSError):  # knots must increase
        ctx.set_cia(2, [(250.0, np.array([700.0, 699.0]), np.array([1e-45, 1e-45]))])
    ctx.set_cia(2, blocks_n2())
