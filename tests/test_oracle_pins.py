"""Pins the FP64 oracle before anything is checked against it.

Two sources pin it: the golden fixtures of tests/golden (scipy.special.wofz, the
same Faddeeva function the reference's SpecialFunctions.jl/OpenSpecFun reaches),
and the known-answer and limit tests of the reference's own test/runtests.jl,
restated here with the reference's tolerances (file:line given per test).
"""
import numpy as np
import pytest


def _lines(orc_mod, raw):
    return raw.view(orc_mod.LINE_DTYPE)


# ---------------------------------------------------------------- Faddeeva
def test_faddeeva_matches_wofz(oracle, golden):
    d = golden["wofz"]
    w = oracle.faddeeva(d["x"], d["y"])
    ref = d["re"] + 1j * d["im"]
    assert np.max(np.abs(w - ref) / np.abs(ref)) < 5e-14
    m = d["y"] >= 1e-3
    assert np.max(np.abs(w.real - ref.real)[m] / np.abs(ref.real)[m]) < 1e-11


def test_xsec_matches_scipy_restatement(oracle, orc_mod, golden):
    g = golden["xsec"]
    co2 = _lines(orc_mod, g["co2_lines"])
    s = oracle.voigt_xsec(co2, g["co2_grid"], 230.0, 0.2, cutoff=25.0)
    assert np.max(np.abs(s - g["co2_sigma"])) < 1e-13 * g["co2_sigma"].max()
    s = oracle.voigt_xsec(co2, g["co2_grid"], 230.0, 0.2, cutoff=25.0, x_far=np.inf)
    assert np.max(np.abs(s - g["co2_sigma_exact"])) < 1e-13 * g["co2_sigma_exact"].max()
    h2o = _lines(orc_mod, g["h2o_lines"])
    s = oracle.voigt_xsec(h2o, g["h2o_grid"], 285.0, 0.9, vmr_self=0.03)
    assert np.max(np.abs(s - g["h2o_sigma"])) < 1e-13 * g["h2o_sigma"].max()


# -------------------------------------------- test/runtests.jl restatements
def test_wavenumber_grid(oracle, orc_mod):  # runtests.jl:123-136, :517-526
    snd = orc_mod.sounder(645.0, 2760.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    assert snd.n_channels == 8461
    g, dhi = oracle.internal_grid(snd, orc_mod.fm_options(internal_dnu=None, high_res_factor=1,
                                                          with_ils=False))
    assert len(g) == 8461 and g[0] == 645.0 and g[-1] == 2760.0 and dhi == 0.25
    g, dhi = oracle.internal_grid(snd, orc_mod.fm_options(internal_dnu=0.0025))
    assert dhi == 0.0025 and len(g) == 858801 and g[0] == 629.0 and g[-1] == 2776.0


def test_planck_round_trip(oracle):  # runtests.jl:192-213
    B = oracle.lib.orc_planck(1000.0, 300.0)
    assert B > 0
    assert oracle.lib.orc_bt(1000.0, B) == pytest.approx(300.0, rel=1e-8)
    assert oracle.lib.orc_planck(1000.0, 300.0) > oracle.lib.orc_planck(1000.0, 250.0)
    nu = 645.0 + 0.25 * np.arange(8461)
    bt = np.array([oracle.lib.orc_bt(v, oracle.lib.orc_planck(v, 280.0)) for v in nu])
    np.testing.assert_allclose(bt, 280.0, rtol=1e-7)
    assert oracle.lib.orc_bt(1000.0, 0.0) == 0.0


def test_voigt_profile_properties(oracle):  # runtests.jl:216-244
    nu0, gl, gd, d = 1000.0, 0.05, 0.02, 0.001
    nus = np.array([(995000 + i) / 1000 for i in range(10001)])
    V = np.array([oracle.lib.orc_voigt_profile(v, nu0, gl, gd, 3) for v in nus])
    assert V.sum() * d == pytest.approx(1.0, rel=3e-2)
    assert nus[np.argmax(V)] == pytest.approx(nu0, abs=d)
    mid = (len(nus) + 1) // 2 - 1
    for k in range(1, 11):
        assert V[mid - k] == pytest.approx(V[mid + k], rel=1e-10)
    VL = oracle.lib.orc_voigt_profile(nu0 + gl, nu0, gl, 1e-6, 3)
    assert VL == pytest.approx(1.0 / (np.pi * gl) / 2.0, rel=0.02)


def _four_line(orc_mod, golden):
    g = golden["xsec"]
    return _lines(orc_mod, g["co2_lines"]), g["co2_grid"]


def test_x_far_shortcut(oracle, orc_mod, golden):  # runtests.jl:247-273
    ll, g = _four_line(orc_mod, golden)
    ex = oracle.voigt_xsec(ll, g, 230.0, 0.2, x_far=np.inf)
    fa = oracle.voigt_xsec(ll, g, 230.0, 0.2, x_far=122.0)
    peak = ex.max()
    assert np.max(np.abs(fa - ex)) < 1e-5 * peak
    m = ex > 1e-6 * peak
    assert np.max(np.abs((fa[m] - ex[m]) / ex[m])) < 3e-4
    assert np.max(np.abs(oracle.voigt_xsec(ll, g, 230.0, 0.2, x_far=0.0) - ex)) > 1e-3 * peak


def test_voigt_methods_agree(oracle, orc_mod, golden):  # runtests.jl:276-297
    ll, g = _four_line(orc_mod, golden)
    F = oracle.voigt_xsec(ll, g, 230.0, 0.2, method="FullFaddeeva")
    W = oracle.voigt_xsec(ll, g, 230.0, 0.2, method="Weideman")
    P = oracle.voigt_xsec(ll, g, 230.0, 0.2, method="PseudoVoigt")
    for s in (F, W, P):
        assert np.all(np.isfinite(s)) and np.all(s >= 0)
    m = F > 1e-3 * F.max()
    assert np.max(np.abs((W[m] - F[m]) / F[m])) < 2e-3
    assert np.max(np.abs((P[m] - F[m]) / F[m])) < 5e-2


def test_partition_and_broadening(oracle, orc_mod):  # runtests.jl:321-349
    assert oracle.lib.orc_Q_ratio(1, 1, 296.0) == pytest.approx(1.0)
    assert oracle.lib.orc_Q_ratio(1, 1, 350.0) < 1.0
    assert oracle.lib.orc_Q_ratio(1, 1, 250.0) > 1.0
    line = np.array([(1, 1, 667.0, 1e-19, 1e-3, 0.060, 0.450, 0.0, 0.76, 0.0)],
                    dtype=orc_mod.LINE_DTYPE)
    _, S, gl, gd = oracle.line_params(line, 296.0, 1.0)
    assert gl == pytest.approx(0.060, rel=1e-6) and gd > 0
    _, _, gl2, _ = oracle.line_params(line, 296.0, 0.5)
    assert gl2 < gl
    _, _, gl3, gd3 = oracle.line_params(line, 400.0, 1.0)
    assert gl3 < gl and gd3 > gd
    assert S == pytest.approx(1e-19, rel=1e-6)


def test_rte_limits_toon(oracle):  # runtests.jl:352-378
    nu = 645.0 + 0.25 * np.arange(8461)
    L = 5
    T_lev = np.full(L + 1, 280.0)
    planck = np.vectorize(oracle.lib.orc_planck)
    I = oracle.rte(nu, np.full((L, len(nu)), 100.0), T_lev, 300.0)
    np.testing.assert_allclose(I, planck(nu, 280.0), rtol=1e-3)
    I = oracle.rte(nu, np.full((L, len(nu)), 1e-10), T_lev, 300.0)
    np.testing.assert_allclose(I, planck(nu, 300.0), rtol=1e-4)
    I = oracle.rte(nu, np.full((L, len(nu)), 2.0), T_lev, 280.0)
    np.testing.assert_allclose(I, planck(nu, 280.0), rtol=1e-6)


def test_cim_correction_and_canonical_form(oracle):  # runtests.jl:387-466
    cim, lit = oracle.lib.orc_cim_correction, oracle.lib.orc_lit_correction
    assert cim(0.03) == pytest.approx(0.03 / 6.0)
    assert cim(1e-9) == pytest.approx(1e-9 / 6.0, rel=1e-6)
    assert cim(1.0) == pytest.approx(0.16395341373865302, rel=1e-12)
    assert cim(1.0) != pytest.approx(lit(1.0), rel=1e-3)
    assert cim(1000.0) == pytest.approx(1.0 - 2.0 / 1000.0, rel=1e-3)
    assert cim(1e7) == pytest.approx(1.0, rel=1e-6)
    assert cim(0.06 - 1e-9) == pytest.approx(cim(0.06 + 1e-9), rel=1e-3)

    nu = 645.0 + 10.0 * np.arange(17)
    L = 5
    T_lev = np.array([300.0, 290.0, 280.0, 270.0, 260.0, 250.0])
    T_ave = np.array([296.0, 285.0, 274.0, 263.0, 252.0])
    tau = np.full((L, len(nu)), 0.7)
    planck = np.vectorize(oracle.lib.orc_planck)
    # the canonical LBLRTM EMIN form (runtests.jl:412-429), assembled independently
    Tr = np.ones((L + 1, len(nu)))
    for k in range(L - 1, -1, -1):
        Tr[k] = Tr[k + 1] * np.exp(-tau[k])
    Iref = planck(nu, 305.0) * Tr[0]
    for k in range(L):
        tr = np.exp(-tau[k])
        Ba, Bt = planck(nu, T_ave[k]), planck(nu, T_lev[k + 1])
        em = (1 - tr) * (Ba + (Bt - Ba) * np.vectorize(cim)(tau[k]))
        Iref += em * Tr[k + 1]
    I = oracle.rte(nu, tau, T_lev, 305.0, source_function="cim", T_ave=T_ave)
    np.testing.assert_allclose(I, Iref, rtol=1e-12)
    It = oracle.rte(nu, tau, T_lev, 305.0, source_function="toon")
    assert not np.allclose(I, It, rtol=1e-3)
    I = oracle.rte(nu, np.full((L, len(nu)), 100.0), T_lev, 305.0, source_function="cim", T_ave=T_ave)
    np.testing.assert_allclose(I, planck(nu, 250.0), rtol=1e-3)
    I = oracle.rte(nu, np.full((L, len(nu)), 1e-10), T_lev, 305.0, source_function="cim", T_ave=T_ave)
    np.testing.assert_allclose(I, planck(nu, 305.0), rtol=1e-4)
    I = oracle.rte(nu, np.full((L, len(nu)), 2.0), np.full(L + 1, 280.0), 280.0,
                   source_function="cim", T_ave=np.full(L, 280.0))
    np.testing.assert_allclose(I, planck(nu, 280.0), rtol=1e-6)
    with pytest.raises(RuntimeError):
        oracle.rte(nu, tau, T_lev, 305.0, source_function="cim")


def test_ils_kernel(oracle):  # runtests.jl:469-503
    dv, k = oracle.ils_kernel(0.25, 2.0, 0.5)
    assert k.sum() * 0.25 == pytest.approx(1.0, rel=1e-2)
    np.testing.assert_allclose(k, k[::-1], rtol=1e-6)
    assert np.argmax(k) == (len(k) + 1) // 2 - 1
    _, kh = oracle.ils_kernel(0.0625, 2.0, 0.5)
    assert kh.sum() * 0.0625 == pytest.approx(1.0, rel=1e-2)
    for style in ("norton_beer_weak", "norton_beer_medium", "norton_beer_strong"):
        _, kn = oracle.ils_kernel(0.25, 2.0, 0.5, apodization=style)
        assert kn.sum() * 0.25 == pytest.approx(1.0, rel=1e-2)
        np.testing.assert_allclose(kn, kn[::-1], rtol=1e-6)
        assert np.argmax(kn) == (len(kn) + 1) // 2 - 1
        assert not np.allclose(kn, k)


def test_cg_layers(oracle):  # layers.jl:36-106 limits
    import ctypes as C
    vc, pc = C.c_double(), C.c_double()
    oracle.lib.orc_layer_cg(4e-4, 4e-4, 1000.0, 600.0, C.byref(vc), C.byref(pc))
    assert vc.value == 4e-4 and pc.value == 800.0
    oracle.lib.orc_layer_cg(1e-2, 3e-3, 1000.0, 600.0, C.byref(vc), C.byref(pc))
    assert 3e-3 < vc.value < 1e-2 and 600.0 < pc.value < 1000.0
    assert oracle.lib.orc_cg_temperature_mass(280.0, 280.0, 1000.0, 600.0) == 280.0
    t = oracle.lib.orc_cg_temperature_mass(288.0, 255.0, 1000.0, 600.0)
    assert 255.0 < t < 288.0


def test_scan_angle(oracle):  # geometry.jl:92-101
    z = oracle.lib.orc_scan_angle_to_local_zenith(48.33)
    assert z == pytest.approx(57.5, abs=0.3)
    assert oracle.lib.orc_scan_angle_to_local_zenith(0.0) == 0.0
