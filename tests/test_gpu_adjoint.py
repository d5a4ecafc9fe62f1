"""The reverse-mode pullback (irs_vjp_batch) against the forward-mode Jacobian.

The pullback never forms K: it takes dy dBT/dR back through the channel resampling
and the ILS to the grid and contracts every RTE derivative term with it in one adjoint
sweep.  It must equal K^T dy from irs_jacobian_batch, whose K passes through FP32 (the
monochromatic columns D and the ILS sums) while the pullback sums in FP64: the
tolerance is 1e-5 of sum |K| |dy| per state element (FP32 rounding of the terms,
not of the cancelling sum).  It must also match a central difference of dy . BT along
a direction of the state (GPU forward model, mixed precision, frozen line set) within
2 %, the truncation and FP32 noise of that difference.  Cases: the 5 k CO2 list with
continua (BT and radiance observables, a reflecting surface with emissivity in the
state, no ILS), and the 400 k six-species list with VP_Y on CO2 (config 2) on a
window, two perturbed profiles with scan angles.
"""
import numpy as np
import pytest

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


def _check_vjp(pkg, ctx, profs, lists, spec, snd, geoms, dy, observable="bt", eps=None, **kw):
    n = len(profs)
    _, K, y = pkg.analytic_jacobian_batch(profs, lists, spec, sounder=snd, geoms=geoms, eps_sfcs=eps,
                                          observable=observable, backend=ctx, **kw)
    y2, dx = pkg.vjp_batch(profs, lists, spec, dy, sounder=snd, geoms=geoms, eps_sfcs=eps, observable=observable,
                           backend=ctx, **kw)
    assert np.allclose(y2, y, rtol=1e-12, atol=0)
    for p in range(n):
        ref = K[p].T @ dy[p]
        scale = np.abs(K[p]).T @ np.abs(dy[p])
        err = np.abs(dx[p] - ref)
        assert np.all(err <= 1e-5 * scale + 1e-30), (p, float(np.max(err / np.maximum(scale, 1e-300))))
    return dx


def test_pullback_equals_KT_dy_5k(pkg, ctx):
    lists = pkg.synthetic.lists_5k_co2()
    profs, ang = pkg.synthetic.perturbed_profiles(3, seed=21)
    base = pkg.afgl_atmosphere("us_standard")
    profs = [pkg.AtmosphericProfile(base.pressure, p.temperature, base.altitude, {**base.vmr, 1: p.vmr[1]})
             for p in profs]
    geoms = [pkg.ViewingGeometry(pkg.scan_angle_to_local_zenith(a)) for a in ang]
    snd = pkg.Sounder.make(650.0, 690.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    rng = np.random.default_rng(4)
    dy = rng.standard_normal((3, 161))
    kw = dict(internal_dnu=0.0025, apply_continuum=True, continua=("h2o", "co2"))
    spec = pkg.StateVectorSpec(50, [pkg.H2O, pkg.CO2], include_emissivity=False)
    _check_vjp(pkg, ctx, profs, lists, spec, snd, geoms, dy, **kw)
    _check_vjp(pkg, ctx, profs, lists, spec, snd, geoms, dy * 1e-3, observable="radiance", **kw)
    spec_e = pkg.StateVectorSpec(50, [pkg.H2O], include_emissivity=True)
    _check_vjp(pkg, ctx, profs, lists, spec_e, snd, geoms, dy, eps=[0.93, 0.97, 0.9], source_function="toon", **kw)
    _check_vjp(pkg, ctx, profs, lists, spec, snd, geoms, dy, with_ils=False, **kw)


def test_pullback_central_difference(pkg, ctx):
    lists = pkg.synthetic.lists_5k_co2()
    base = pkg.afgl_atmosphere("us_standard")
    snd = pkg.Sounder.make(660.0, 680.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    kw = dict(internal_dnu=0.0025, apply_continuum=True, continua=("h2o", "co2"))
    spec = pkg.StateVectorSpec(50, [pkg.H2O], include_emissivity=False)
    rng = np.random.default_rng(8)
    dy = rng.standard_normal(81)
    y, dx = pkg.vjp_batch([base], lists, spec, dy[None, :], sounder=snd, backend=ctx, **kw)
    x0 = pkg.pack_state(spec, base)
    v = np.zeros(spec.n)
    v[spec.temp_range.start:spec.temp_range.stop] = rng.standard_normal(50)
    v[spec.vmr_blocks[0].range.start:spec.vmr_blocks[0].range.stop] = 0.01 * rng.standard_normal(50)
    v[spec.tsfc_index] = 1.0
    h = 0.05

    def F(x):
        p, Ts, _ = pkg.unpack_state(spec, x, base)
        _, _, bt = pkg.forward_model_batch([p], lists, sounder=snd, T_sfcs=[Ts], backend=ctx, precision="mixed",
                                           dptmn=0.0, **kw)
        return bt[0] @ dy

    fd = (F(x0 + h * v) - F(x0 - h * v)) / (2 * h)
    assert abs(fd - dx[0] @ v) <= 0.02 * abs(fd), (fd, dx[0] @ v)


def test_pullback_400k_vpy_window(pkg, ctx):
    lists = pkg.synthetic.lists_iasi_400k()
    lm = pkg.VPYLineMixing(pkg.synthetic.vpy_y0(len(lists[2])))
    profs, ang = pkg.synthetic.perturbed_profiles(2, seed=1002)
    geoms = [pkg.ViewingGeometry(pkg.scan_angle_to_local_zenith(a)) for a in ang]
    snd = pkg.Sounder.make(700.0, 712.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    spec = pkg.StateVectorSpec(50, [pkg.H2O, pkg.O3], include_emissivity=False)
    dy = np.random.default_rng(2).standard_normal((2, 49))
    _check_vjp(pkg, ctx, profs, lists, spec, snd, geoms, dy, line_mixing=lm, internal_dnu=0.0025,
               apply_continuum=True, continua=("h2o", "co2"))
