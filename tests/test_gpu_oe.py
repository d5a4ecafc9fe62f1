"""Batched optimal estimation on the GPU (irs_oe_batch) against the numpy oracle of
optimal_estimation.jl driven by the FP64 oracle's forward model and analytic Jacobian.

Tolerances: the GPU retrieval uses the mixed forward model and the FP32 line-sum
Jacobian, the oracle FP64 throughout, so retrieved states are compared in units of
the posterior standard deviation: |x_gpu - x_oracle| <= 0.02 sigma_post for a single
Gauss-Newton step and <= 0.1 sigma_post at convergence."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

IASI_SUB = dict(nu_min=699.0, nu_max=705.0, dnu=0.5, opd_max=2.0, fwhm_gauss=0.5)
KW = dict(apply_continuum=False, with_ils=True, internal_dnu=0.005)


@pytest.fixture(scope="module")
def pkg():
    return load_package()


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.B200Context()
    yield c
    c.close()


def lines(orc_mod):
    a = np.zeros(3, dtype=orc_mod.LINE_DTYPE)
    for k, (nu, S, gair, gself, E, n, d) in enumerate([(700.5, 2.0e-21, 0.07, 0.08, 250.0, 0.75, -0.003),
                                                       (702.0, 8.0e-22, 0.07, 0.08, 600.0, 0.75, -0.003),
                                                       (703.6, 1.5e-21, 0.07, 0.08, 400.0, 0.75, -0.003)]):
        a[k] = (2, 1, nu, S, 1.0, gair, gself, E, n, d)
    return a


def base_profile(pkg, nlev=6):
    p = np.linspace(1000.0, 200.0, nlev)
    T = 288.0 + (225.0 - 288.0) * (1000.0 - p) / 800.0
    return pkg.AtmosphericProfile(p, T, np.zeros(nlev), {2: np.full(nlev, 4.0e-4)})


def oracle_fns(pkg, oracle, orc_mod, spec, base, ll):
    snd = orc_mod.sounder(**IASI_SUB)

    def opt(x):
        prof, Ts, es = pkg.unpack_state(spec, x, base)
        return dict(p=prof.pressure, T=prof.temperature, vmr=prof.vmr), orc_mod.fm_options(
            T_sfc=Ts, eps_sfc=es, dptmn=0.0, **KW)

    def fwd(x):
        pr, o = opt(x)
        return oracle.forward_model(pr, ll, snd, o)[1]

    def fwd_jac(x):
        pr, o = opt(x)
        K, y = oracle.analytic_jacobian(pr, ll, snd, o, retrieved=spec.species, include_T=spec.include_temperature,
                                        include_tsfc=spec.include_tsfc, include_eps=spec.include_emissivity)
        return y, K

    return fwd, fwd_jac


def setup(pkg, ctx, orc_mod, dT=1.5, dv=0.05):
    ll = {2: lines(orc_mod)}
    base = base_profile(pkg)
    spec = pkg.StateVectorSpec(6, [pkg.CO2], include_emissivity=False)
    xa = pkg.pack_state(spec, base)
    Sa = pkg.build_sa(spec, base, sigma_T=2.0, sigma_vmr=0.2)
    xt = xa.copy()
    xt[:6] += dT * np.linspace(1.0, 0.3, 6)
    xt[6:12] += dv
    xt[12] += 1.0
    snd = pkg.Sounder.make(**IASI_SUB)
    prof, Ts, _ = pkg.unpack_state(spec, xt, base)
    llp = {2: pkg.HITRANLinelist(ll[2])}
    y = pkg.forward_model(prof, llp, sounder=snd, T_sfc=Ts, backend=ctx, dptmn=0.0, **KW)[2]
    se = np.full(len(y), 0.2 ** 2)
    return ll, llp, base, spec, xa, Sa, y, se, snd


def test_single_gauss_newton_step(pkg, ctx, oracle, orc_mod):
    import oe_oracle
    ll, llp, base, spec, xa, Sa, y, se, snd = setup(pkg, ctx, orc_mod)
    r = pkg.optimal_estimation_batch(y[None], spec, [base], llp, xa=xa, Sa=Sa, Se=se, method="gauss_newton",
                                     max_iter=1, sounder=snd, backend=ctx, fm_kwargs=KW)
    fwd, fwd_jac = oracle_fns(pkg, oracle, orc_mod, spec, base, ll)
    ro = oe_oracle.optimal_estimation(y, fwd, fwd_jac, xa, Sa, se, method="gauss_newton", max_iter=1)
    S_hat = np.linalg.inv(np.linalg.inv(Sa) + ro["M"])
    sd = np.sqrt(np.diag(S_hat))
    assert r["n_iter"][0] == ro["n_iter"] == 1
    assert np.max(np.abs(r["x"][0] - ro["x"]) / sd) < 0.02
    assert np.allclose(r["M"][0], ro["M"], rtol=1e-3, atol=1e-4 * np.max(np.abs(ro["M"])))


def test_lm_retrieval_vs_oracle(pkg, ctx, oracle, orc_mod):
    import oe_oracle
    ll, llp, base, spec, xa, Sa, y, se, snd = setup(pkg, ctx, orc_mod, dT=3.0, dv=0.15)
    res = pkg.optimal_estimation(y, spec, base, llp, xa=xa, Sa=Sa, Se=se, sounder=snd, backend=ctx, fm_kwargs=KW)
    fwd, fwd_jac = oracle_fns(pkg, oracle, orc_mod, spec, base, ll)
    ro = oe_oracle.optimal_estimation(y, fwd, fwd_jac, xa, Sa, se)
    sd = np.sqrt(np.diag(res.S_hat))
    print("n_iter gpu", res.n_iter, "oracle", ro["n_iter"], "max dx/sd", np.max(np.abs(res.x - ro["x"]) / sd))
    assert res.converged and ro["converged"]
    assert np.max(np.abs(res.x - ro["x"]) / sd) < 0.1
    assert res.cost <= ro["cost"][0] and res.cost < 0.5 * ro["cost"][0]
    assert 0.0 < res.dof < spec.n and np.isfinite(res.H) and res.H > 0
    assert np.allclose(res.A, res.S_hat @ (res.K.T @ (res.K / se[:, None])), atol=1e-3)


def test_batch_matches_single_scenes(pkg, ctx, orc_mod):
    ll, llp, base, spec, xa, Sa, y, se, snd = setup(pkg, ctx, orc_mod)
    ys = [y]
    for dT in (-2.0, 4.0):
        ys.append(setup(pkg, ctx, orc_mod, dT=dT, dv=-0.1)[6])
    ys = np.stack(ys)
    rb = pkg.optimal_estimation_batch(ys, spec, [base] * 3, llp, xa=xa, Sa=Sa, Se=se, sounder=snd, backend=ctx,
                                      fm_kwargs=KW)
    for k in range(3):
        r1 = pkg.optimal_estimation_batch(ys[k:k + 1], spec, [base], llp, xa=xa, Sa=Sa, Se=se, sounder=snd,
                                          backend=ctx, fm_kwargs=KW)
        assert r1["n_iter"][0] == rb["n_iter"][k]
        assert np.allclose(r1["x"][0], rb["x"][k], rtol=0, atol=1e-9)
    assert rb["converged"].all()


def test_closed_loop_5k_lines(pkg, ctx):
    """T + log H2O + T_sfc (101 elements) on the 5,000-line CO2 list with MT-CKD
    continua, noise from scene_nedt(0.2 K at 280 K): the retrieval moves the
    temperature towards the truth where the averaging kernel is informative."""
    lists = pkg.synthetic.lists_5k_co2()
    snd = pkg.Sounder.make(645.0, 700.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    kw = dict(internal_dnu=0.0025, apply_continuum=True, continua=("h2o", "co2"))
    base = pkg.afgl_atmosphere("us_standard")
    spec = pkg.StateVectorSpec(50, [pkg.H2O], include_emissivity=False)
    xa = pkg.pack_state(spec, base)
    Sa = pkg.build_sa(spec, base, sigma_T=2.0, L_T=1.0, sigma_vmr=0.3)
    rng = np.random.default_rng(1004)
    xt = xa + np.linalg.cholesky(Sa) @ rng.standard_normal(spec.n)
    prof, Ts, _ = pkg.unpack_state(spec, xt, base)
    nu, _, bt = pkg.forward_model(prof, lists, sounder=snd, T_sfc=Ts, backend=ctx, dptmn=0.0, **kw)
    sig = pkg.scene_nedt(nu, bt, nedt_280K=0.2)
    y = bt + sig * rng.standard_normal(len(bt))
    res = pkg.optimal_estimation(y, spec, base, lists, xa=xa, Sa=Sa, Se=sig ** 2, sounder=snd, backend=ctx,
                                 fm_kwargs=kw)
    assert res.converged
    wT = np.diag(res.A)[:50]  # per-level information on temperature
    assert wT.sum() > 1.0
    err_prior = np.sqrt(np.sum(wT * (xa[:50] - xt[:50]) ** 2) / wT.sum())
    err_post = np.sqrt(np.sum(wT * (res.x[:50] - xt[:50]) ** 2) / wT.sum())
    print(f"A-weighted T error: prior {err_prior:.2f} K -> retrieved {err_post:.2f} K, dof {res.dof:.1f}")
    assert err_post < err_prior
    assert res.chi2 < 3.0 * int(res.channel_mask.sum())


@pytest.mark.parametrize("masked", [False, True])
def test_apodized_se_vs_oracle(pkg, ctx, oracle, orc_mod, masked):
    """The retrieval with the apodised (banded, non-diagonal) Se of IASI L1C through the
    banded entry point, against the oracle with the same full Se inverted on the kept
    channels; and the cost is r^T Se^-1 r (not its diagonal part)."""
    import oe_oracle
    ll, llp, base, spec, xa, Sa, y, se, snd = setup(pkg, ctx, orc_mod, dT=3.0, dv=0.15)
    nu = pkg.sounder_grid(snd)
    Se = pkg.scene_measurement_covariance(nu, y, nedt_280K=0.2, dnu_sample=0.5)
    keep = np.ones(len(y), bool)
    if masked:
        keep[[1, 6]] = False
    res = pkg.optimal_estimation(y, spec, base, llp, xa=xa, Sa=Sa, Se=Se, channel_mask=keep, sounder=snd,
                                 backend=ctx, fm_kwargs=KW)
    fwd, fwd_jac = oracle_fns(pkg, oracle, orc_mod, spec, base, ll)
    ro = oe_oracle.optimal_estimation(y, fwd, fwd_jac, xa, Sa, Se, keep=keep)
    sd = np.sqrt(np.diag(res.S_hat))
    assert res.converged and ro["converged"]
    assert np.max(np.abs(res.x - ro["x"]) / sd) < 0.1
    k = np.flatnonzero(keep)
    W = np.linalg.inv(Se[np.ix_(k, k)])
    r = (y - res.y_fit)[k]
    assert abs(res.chi2 - r @ W @ r) <= 1e-8 * max(1.0, res.chi2)
    # the diagonal of the same Se gives a different retrieval
    rd = pkg.optimal_estimation(y, spec, base, llp, xa=xa, Sa=Sa, Se=np.diag(Se), channel_mask=keep, sounder=snd,
                                backend=ctx, fm_kwargs=KW)
    assert np.max(np.abs(rd.x - res.x) / sd) > 0.01


def test_gauss_newton_step_151_elements(pkg, ctx, oracle, orc_mod):
    """Config 2's state (T + log H2O + log O3 + T_sfc on 50 levels = 151 elements, above
    the 127 that one 256-thread block of the normal equations covers): one Gauss-Newton
    step against the oracle, within 0.02 posterior sigma."""
    import oe_oracle
    a = np.zeros(7, dtype=orc_mod.LINE_DTYPE)
    spec_lines = [(2, 700.5, 2.0e-21, 250.0), (2, 702.0, 8.0e-22, 600.0), (2, 703.6, 1.5e-21, 400.0),
                  (1, 701.1, 3.0e-21, 200.0), (1, 704.2, 1.0e-21, 900.0),
                  (3, 699.8, 4.0e-21, 300.0), (3, 702.9, 2.0e-21, 150.0)]
    for k, (mol, nu, S, E) in enumerate(spec_lines):
        a[k] = (mol, 1, nu, S, 1.0, 0.07, 0.09, E, 0.75, -0.003)
    ll = {m: a[a["mol_id"] == m] for m in (1, 2, 3)}
    llp = {m: pkg.HITRANLinelist(v) for m, v in ll.items()}
    base = pkg.afgl_atmosphere("midlatitude_summer")
    spec = pkg.StateVectorSpec(50, [pkg.H2O, pkg.O3], include_emissivity=False)
    assert spec.n == 151
    xa = pkg.pack_state(spec, base)
    Sa = pkg.build_sa(spec, base, sigma_T=2.0, sigma_vmr=0.2)
    rng = np.random.default_rng(151)
    xt = xa + np.linalg.cholesky(Sa) @ rng.standard_normal(spec.n)
    snd = pkg.Sounder.make(**IASI_SUB)
    prof, Ts, _ = pkg.unpack_state(spec, xt, base)
    y = pkg.forward_model(prof, llp, sounder=snd, T_sfc=Ts, backend=ctx, dptmn=0.0, **KW)[2]
    se = np.full(len(y), 0.2 ** 2)
    r = pkg.optimal_estimation_batch(y[None], spec, [base], llp, xa=xa, Sa=Sa, Se=se, method="gauss_newton",
                                     max_iter=1, sounder=snd, backend=ctx, fm_kwargs=KW)
    fwd, fwd_jac = oracle_fns(pkg, oracle, orc_mod, spec, base, ll)
    ro = oe_oracle.optimal_estimation(y, fwd, fwd_jac, xa, Sa, se, method="gauss_newton", max_iter=1)
    sd = np.sqrt(np.diag(np.linalg.inv(np.linalg.inv(Sa) + ro["M"])))
    assert r["n_iter"][0] == ro["n_iter"] == 1
    assert np.max(np.abs(r["x"][0] - ro["x"]) / sd) < 0.02
    assert np.allclose(r["M"][0], ro["M"], rtol=1e-3, atol=1e-4 * np.max(np.abs(ro["M"])))
