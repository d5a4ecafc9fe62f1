"""The GPU analytic Jacobian (irs_jacobian_batch / irs_vjp_batch through the package API)
against the FP64 oracle's analytic Jacobian and against central finite differences of the
GPU FP64 forward model, on the fixtures of the reference's Jacobian suite
(test/runtests.jl:1221-1478) and on the 5,000-line CO2 list.

Tolerances: the GPU line sum and its derivatives are FP32 (Kahan-compensated tile sums)
and the channel contraction is FP32, so each column block (T levels, VMR levels, T_sfc,
eps) is compared relative to its largest entry: 2e-4 against the oracle's analytic
Jacobian.  The observable itself (FP32 tau, FP64 RTE) is within 0.01 K of the oracle's
FP64 forward model, the bound the mixed forward path meets."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

IASI_SUB = dict(nu_min=699.0, nu_max=705.0, dnu=0.5, opd_max=2.0, fwhm_gauss=0.5)


@pytest.fixture(scope="module")
def pkg():
    return load_package()


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.B200Context()
    yield c
    c.close()


def mk(orc_mod, mol, lines):
    a = np.zeros(len(lines), dtype=orc_mod.LINE_DTYPE)
    for k, (nu, S, gair, gself, E, n, d) in enumerate(lines):
        a[k] = (mol, 1, nu, S, 1.0, gair, gself, E, n, d)
    return a


def profile(pkg, nlev, species):
    p = np.linspace(1000.0, 200.0, nlev)
    T = 288.0 + (225.0 - 288.0) * (1000.0 - p) / 800.0
    return pkg.AtmosphericProfile(p, T, np.zeros(nlev), species(p))


def as_oracle(prof):
    return dict(p=prof.pressure, T=prof.temperature, vmr=prof.vmr)


def block_rel(K, Kr, cols):
    return np.max(np.abs(K[:, cols] - Kr[:, cols])) / (np.max(np.abs(Kr[:, cols])) + 1e-30)


def blocks(spec):
    out = []
    if spec.include_temperature:
        out.append(slice(spec.temp_range.start, spec.temp_range.stop))
    out += [slice(b.range.start, b.range.stop) for b in spec.vmr_blocks]
    for k in (spec.tsfc_index, spec.emis_index):
        if k >= 0:
            out.append(slice(k, k + 1))
    return out


def check_vs_oracle(pkg, ctx, oracle, orc_mod, prof, lls, spec, snd_kw, kw, y0=None, T_sfc=290.0, eps=0.98,
                    tol=2e-4, channels=None):
    snd = pkg.Sounder.make(**snd_kw)
    lm = pkg.VPYLineMixing(y0[2]) if y0 is not None else None
    ll_pkg = {s: pkg.HITRANLinelist(v) for s, v in lls.items()}
    jac = pkg.analytic_jacobian(prof, ll_pkg, spec, sounder=snd, T_sfc=T_sfc, eps_sfc=eps, backend=ctx,
                                line_mixing=lm, **kw)
    o = orc_mod.fm_options(T_sfc=T_sfc, eps_sfc=eps, dptmn=0.0, line_mixing=y0 is not None, **kw)
    Kr, yr = oracle.analytic_jacobian(as_oracle(prof), lls, orc_mod.sounder(**snd_kw), o,
                                      retrieved=spec.species, include_T=spec.include_temperature,
                                      include_tsfc=spec.include_tsfc, include_eps=spec.include_emissivity,
                                      log_vmr=spec.log_vmr, channels=channels, y0=y0)
    K, y = jac.K, jac.y0
    if channels is not None:
        K, y = K[channels[0]:channels[1]], y[channels[0]:channels[1]]
    assert K.shape == Kr.shape
    assert np.max(np.abs(y - yr)) < 0.01
    errs = [block_rel(K, Kr, b) for b in blocks(spec)]
    print("block rel errors", ["%.2e" % e for e in errs])
    assert max(errs) < tol, errs
    return jac, Kr


@pytest.mark.parametrize("nlev", [6, 11])
def test_vmr_jacobian_vs_oracle(pkg, ctx, oracle, orc_mod, nlev):  # runtests.jl:1221-1282
    ll = {2: mk(orc_mod, 2, [(700.5, 3.0e-23, 0.08, 0.10, 250.0, 0.75, 0.0),
                             (702.0, 1.0e-23, 0.08, 0.10, 250.0, 0.75, 0.0)])}
    prof = profile(pkg, nlev, lambda p: {2: np.full(len(p), 4.0e-4)})
    spec = pkg.StateVectorSpec(nlev, [pkg.CO2], include_temperature=False)
    jac, _ = check_vs_oracle(pkg, ctx, oracle, orc_mod, prof, ll, spec, IASI_SUB,
                             dict(apply_continuum=False, with_ils=True, internal_dnu=0.005))
    assert jac.K.shape == (13, nlev + 2)
    i_line = np.argmin(jac.y0)
    assert np.sum(jac.K[i_line, :nlev]) < 0.0


def test_temperature_jacobian_vs_oracle(pkg, ctx, oracle, orc_mod):  # runtests.jl:1345-1380
    ll = {2: mk(orc_mod, 2, [(700.5, 2.0e-21, 0.07, 0.08, 250.0, 0.75, -0.003),
                             (702.0, 8.0e-22, 0.07, 0.08, 600.0, 0.75, -0.003)])}
    prof = profile(pkg, 6, lambda p: {2: np.full(len(p), 4.0e-4)})
    spec = pkg.StateVectorSpec(6, [pkg.CO2])
    jac, _ = check_vs_oracle(pkg, ctx, oracle, orc_mod, prof, ll, spec, IASI_SUB,
                             dict(apply_continuum=False, with_ils=True, internal_dnu=0.005))
    assert jac.K[np.argmin(jac.y0), 0] > 0.0


@pytest.mark.parametrize("species", ["h2o", "co2"])
def test_continuum_coupling_vs_oracle(pkg, ctx, oracle, orc_mod, species):  # runtests.jl:1383-1424
    if species == "h2o":
        ll = {1: mk(orc_mod, 1, [(700.6, 3.0e-21, 0.09, 0.45, 200.0, 0.70, 0.005),
                                 (702.3, 1.2e-21, 0.09, 0.45, 450.0, 0.70, 0.005)])}
        prof = profile(pkg, 6, lambda p: {1: 0.01 * np.exp(-3.0 * (1000.0 - p) / 800.0)})
        sp, conts = 1, ("h2o",)
    else:
        ll = {2: mk(orc_mod, 2, [(700.5, 2.0e-21, 0.07, 0.08, 250.0, 0.75, -0.006),
                                 (702.0, 8.0e-22, 0.07, 0.08, 600.0, 0.75, -0.006)])}
        prof = profile(pkg, 6, lambda p: {2: np.full(len(p), 4.0e-4)})
        sp, conts = 2, ("co2",)
    spec = pkg.StateVectorSpec(6, [sp])
    check_vs_oracle(pkg, ctx, oracle, orc_mod, prof, ll, spec, IASI_SUB,
                    dict(apply_continuum=True, continua=conts, with_ils=True, internal_dnu=0.005))


def test_line_mixing_jacobian_vs_oracle(pkg, ctx, oracle, orc_mod):  # runtests.jl:1427-1478
    # sorted by wavenumber so that y0 stays aligned with HITRANLinelist's order
    ll = {2: mk(orc_mod, 2, [(700.40, 2.0e-24, 0.09, 0.08, 250.0, 0.75, -0.004),
                             (700.55, 1.8e-24, 0.09, 0.08, 240.0, 0.75, -0.004),
                             (700.95, 9.0e-25, 0.09, 0.08, 500.0, 0.75, -0.004),
                             (701.30, 1.4e-24, 0.09, 0.08, 300.0, 0.75, -0.004)])}
    y0 = {2: np.array([0.03, -0.02, 0.01, 0.025])}
    prof = profile(pkg, 6, lambda p: {2: np.full(len(p), 4.0e-4)})
    spec = pkg.StateVectorSpec(6, [pkg.CO2])
    check_vs_oracle(pkg, ctx, oracle, orc_mod, prof, ll, spec,
                    dict(nu_min=699.0, nu_max=703.0, dnu=0.5, opd_max=2.0, fwhm_gauss=0.5),
                    dict(apply_continuum=False, with_ils=True, internal_dnu=0.005), y0=y0)


def test_two_species_radiance_linear_vmr(pkg, ctx, oracle, orc_mod):
    ll = {1: mk(orc_mod, 1, [(700.6, 3.0e-21, 0.09, 0.45, 200.0, 0.70, 0.005),
                             (703.3, 1.2e-21, 0.09, 0.45, 450.0, 0.70, 0.005)]),
          2: mk(orc_mod, 2, [(700.5, 2.0e-21, 0.07, 0.08, 250.0, 0.75, -0.006),
                             (702.0, 8.0e-22, 0.07, 0.08, 600.0, 0.75, -0.006)])}
    prof = profile(pkg, 8, lambda p: {1: 0.01 * np.exp(-3.0 * (1000.0 - p) / 800.0),
                                      2: np.full(len(p), 4.0e-4)})
    spec = pkg.StateVectorSpec(8, [pkg.H2O, pkg.CO2], log_vmr=False)
    snd = pkg.Sounder.make(**IASI_SUB)
    kw = dict(apply_continuum=True, continua=("h2o", "co2"), with_ils=True, internal_dnu=0.005)
    jac = pkg.analytic_jacobian(prof, {s: pkg.HITRANLinelist(v) for s, v in ll.items()}, spec, sounder=snd,
                                T_sfc=291.0, eps_sfc=0.97, observable="radiance", backend=ctx, **kw)
    o = orc_mod.fm_options(T_sfc=291.0, eps_sfc=0.97, dptmn=0.0, **kw)
    Kr, yr = oracle.analytic_jacobian(as_oracle(prof), ll, orc_mod.sounder(**IASI_SUB), o, retrieved=[1, 2],
                                      log_vmr=False, observable="radiance")
    assert np.max(np.abs(jac.y0 - yr)) < 1e-4 * np.max(np.abs(yr))
    errs = [block_rel(jac.K, Kr, b) for b in blocks(spec)]
    print("block rel errors", ["%.2e" % e for e in errs])
    assert max(errs) < 2e-4


def test_jacobian_5k_lines_vs_oracle_window(pkg, ctx, oracle, orc_mod):
    """The 5,000-line CO2 list on the 50-level AFGL profile (645-700 cm-1), T + log CO2
    + T_sfc + eps, against the oracle on a window of channels."""
    ll = pkg.synthetic.lists_5k_co2()
    prof = pkg.afgl_atmosphere("us_standard")
    snd_kw = dict(nu_min=645.0, nu_max=700.0, dnu=0.25, opd_max=2.0, fwhm_gauss=0.5)
    spec = pkg.StateVectorSpec(len(prof.pressure), [pkg.CO2])
    check_vs_oracle(pkg, ctx, oracle, orc_mod, prof, {2: ll[2].lines}, spec, snd_kw,
                    dict(apply_continuum=False, with_ils=True, internal_dnu=0.01), T_sfc=None, eps=1.0,
                    channels=(100, 108))


def test_analytic_vs_gpu_finite_differences(pkg, ctx, orc_mod):
    """Central differences of the GPU FP64 forward model (all perturbed states in one
    batch) against the GPU analytic Jacobian, with the reference suite's steps."""
    ll = {2: pkg.HITRANLinelist(mk(orc_mod, 2, [(700.5, 2.0e-21, 0.07, 0.08, 250.0, 0.75, -0.003),
                                                (702.0, 8.0e-22, 0.07, 0.08, 600.0, 0.75, -0.003)]))}
    prof = profile(pkg, 6, lambda p: {2: np.full(len(p), 4.0e-4)})
    spec = pkg.StateVectorSpec(6, [pkg.CO2])
    snd = pkg.Sounder.make(**IASI_SUB)
    kw = dict(apply_continuum=False, with_ils=True, internal_dnu=0.005)
    jac = pkg.analytic_jacobian(prof, ll, spec, sounder=snd, T_sfc=290.0, eps_sfc=0.98, backend=ctx, **kw)
    steps = np.array([0.1] * 6 + [1e-3] * 6 + [0.1, 1e-3])
    fd = pkg.finite_difference_jacobian(prof, ll, spec, T_sfc=290.0, eps_sfc=0.98, steps=steps,
                                        fm_kwargs=dict(sounder=snd, **kw), backend=ctx)
    assert np.max(np.abs(jac.y0 - fd.y0)) < 0.01
    assert block_rel(jac.K, fd.K, slice(0, 6)) < 1e-3
    assert block_rel(jac.K, fd.K, slice(6, 12)) < 1e-4
    assert np.max(np.abs(jac.K[:, 12] - fd.K[:, 12])) < 1e-4
    assert np.max(np.abs(jac.K[:, 13] - fd.K[:, 13])) < 1e-4


def test_batch_and_vjp(pkg, ctx, orc_mod):
    """A batch of profiles gives each profile's own Jacobian; the pullback is K^T dy
    (within FP32 rounding: it is computed without K);
    reduced VMR bases are the full log-VMR columns times the basis."""
    ll = {2: pkg.HITRANLinelist(mk(orc_mod, 2, [(700.5, 2.0e-21, 0.07, 0.08, 250.0, 0.75, -0.003),
                                                (702.0, 8.0e-22, 0.07, 0.08, 600.0, 0.75, -0.003)])),
          1: pkg.HITRANLinelist(mk(orc_mod, 1, [(701.1, 3.0e-21, 0.09, 0.45, 200.0, 0.70, 0.005)]))}
    snd = pkg.Sounder.make(**IASI_SUB)
    kw = dict(apply_continuum=True, with_ils=True, internal_dnu=0.005)
    profs = [profile(pkg, 7, lambda p, k=k: {1: (0.008 + 0.002 * k) * np.exp(-3.0 * (1000.0 - p) / 800.0),
                                            2: np.full(len(p), 4.0e-4 + 2e-5 * k)}) for k in range(3)]
    for k, p in enumerate(profs):
        p.temperature = p.temperature + 2.0 * k
    spec = pkg.StateVectorSpec(7, [pkg.H2O, pkg.CO2])
    nu, Kb, yb = pkg.analytic_jacobian_batch(profs, ll, spec, sounder=snd, backend=ctx, **kw)
    for k, p in enumerate(profs):
        j = pkg.analytic_jacobian(p, ll, spec, sounder=snd, backend=ctx, **kw)
        assert np.array_equal(j.K, Kb[k])
        assert np.array_equal(j.y0, yb[k])
    y, pb = pkg.forward_model_rrule(profs[1], ll, spec, sounder=snd, backend=ctx, **kw)
    assert np.array_equal(y, yb[1])
    dy = np.random.default_rng(5).standard_normal(len(nu))
    dx = pb(dy)
    # the pullback runs in reverse mode (FP64 sums) while K passes through FP32: agreement
    # to 1e-5 of sum |K| |dy| per element
    assert np.all(np.abs(dx - Kb[1].T @ dy) <= 1e-5 * (np.abs(Kb[1]).T @ np.abs(dy)))
    # ColumnScale for H2O and a 2-block PartialColumns for CO2
    B = pkg.partial_column_basis(7, [range(0, 3), range(3, 7)])
    spec_r = pkg.StateVectorSpec(7, [pkg.ColumnScale(pkg.H2O), pkg.PartialColumns(pkg.CO2, B)])
    _, Kr, yr = pkg.analytic_jacobian_batch(profs, ll, spec_r, sounder=snd, backend=ctx, **kw)
    assert np.allclose(yr, yb, rtol=0, atol=1e-9)
    full_h2o = Kb[:, :, 7:14].sum(axis=2)
    full_co2 = Kb[:, :, 14:21] @ B
    scale = np.max(np.abs(Kb))
    assert np.max(np.abs(Kr[:, :, 7] - full_h2o)) < 1e-4 * scale
    assert np.max(np.abs(Kr[:, :, 8:10] - full_co2)) < 1e-4 * scale
    assert np.allclose(Kr[:, :, :7], Kb[:, :, :7], rtol=1e-12, atol=1e-12 * scale)


def test_jacobian_errors(pkg, ctx, orc_mod):
    ll = {2: pkg.HITRANLinelist(mk(orc_mod, 2, [(700.5, 2.0e-21, 0.07, 0.08, 250.0, 0.75, -0.003)]))}
    prof = profile(pkg, 6, lambda p: {2: np.full(len(p), 4.0e-4)})
    snd = pkg.Sounder.make(**IASI_SUB)
    with pytest.raises(pkg.IRSError):
        pkg.analytic_jacobian(prof, ll, pkg.StateVectorSpec(6, [pkg.CO2]), sounder=snd, observable="tb",
                              backend=ctx)
    with pytest.raises(pkg.IRSError):
        pkg.analytic_jacobian(prof, ll, pkg.StateVectorSpec(6, [pkg.O3]), sounder=snd, backend=ctx)
    with pytest.raises(pkg.IRSError):
        pkg.analytic_jacobian(prof, ll, pkg.StateVectorSpec(7, [pkg.CO2]), sounder=snd, backend=ctx)
