"""Parity of the CUDA path (through the C ABI) against the FP64 oracle.

Tolerances:
  * FP64 kernels against the FP64 oracle: cross sections to 1e-12 of the peak,
    brightness temperatures to 1e-6 K (both sides are FP64; only the order of
    the ILS and radiance sums differs).
  * mixed (FP32 Faddeeva, Kahan FP32 line sum) against the FP64 oracle: BT RMS
    <= 0.01 K and max <= 0.05 K -- the accuracy target the path is specified to.
At the 400,000-line size the oracle runs on channel windows (the window result is
identical to the full run, which tests/test_oracle_forward.py checks), and the
mixed kernel is checked against the FP64 kernel over the whole spectrum.
"""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    m = load_package()
    return m


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.B200Context()
    yield c
    c.close()


def oracle_profile(p):
    return dict(p=p.pressure, T=p.temperature, vmr=p.vmr)


def oracle_sounder(orc_mod, s):
    return orc_mod.sounder(s.nu_min, s.nu_max, s.dnu, opd_max=s.opd_max, fwhm_gauss=s.fwhm_gauss)


# ------------------------------------------------------------ cross sections
@pytest.mark.parametrize("method", ["FullFaddeeva", "Weideman", "PseudoVoigt"])
def test_cross_sections_fp64_fixture(pkg, ctx, oracle, orc_mod, golden, method):
    g = golden["xsec"]
    lines = g["co2_lines"].view(orc_mod.LINE_DTYPE)
    ll = pkg.HITRANLinelist(lines)
    grid = g["co2_grid"]
    ref = oracle.voigt_xsec(lines, grid, 230.0, 0.2, method=method)
    got = pkg.compute_voigt_cross_sections(grid, ll, 230.0, 0.2, method=pkg.VoigtMethod[method],
                                           backend=ctx)
    assert np.max(np.abs(got - ref)) <= 1e-12 * ref.max()
    if method == "FullFaddeeva":
        assert np.max(np.abs(got - g["co2_sigma"])) <= 1e-12 * ref.max()


def test_cross_sections_fp64_self_broadened(pkg, ctx, oracle, orc_mod, golden):
    g = golden["xsec"]
    lines = g["h2o_lines"].view(orc_mod.LINE_DTYPE)
    got = pkg.compute_voigt_cross_sections(g["h2o_grid"], pkg.HITRANLinelist(lines), 285.0, 0.9,
                                           vmr_self=0.03, backend=ctx)
    assert np.max(np.abs(got - g["h2o_sigma"])) <= 1e-12 * g["h2o_sigma"].max()


@pytest.mark.parametrize("T,p", [(296.0, 1.0), (230.0, 0.2), (200.0, 1e-3), (250.0, 1e-6)])
def test_cross_sections_5k(pkg, ctx, oracle, T, p):
    ll = pkg.synthetic.lists_5k_co2()[2]
    grid = np.array([(251600 + i) / 400 for i in range(34801)])
    ref = oracle.voigt_xsec(ll.lines, grid, T, p)
    f64 = pkg.compute_voigt_cross_sections(grid, ll, T, p, backend=ctx)
    assert np.max(np.abs(f64 - ref)) <= 1e-12 * ref.max()
    for prec in ("mixed", "mixed_direct"):
        mx = pkg.compute_voigt_cross_sections(grid, ll, T, p, backend=ctx, precision=prec)
        # FP32 parameters and an FP32 Faddeeva accurate to ~4e-7 of each line's peak:
        # ~1e-6 relative near the cores, ~1e-5 of the peak everywhere
        m = ref > 1e-2 * ref.max()
        assert np.max(np.abs(mx[m] - ref[m]) / ref[m]) < 2e-4, prec
        assert np.max(np.abs(mx - ref)) < 2e-5 * ref.max(), prec


def test_cross_sections_mixed_weideman_pv(pkg, ctx, oracle, orc_mod, golden):
    g = golden["xsec"]
    lines = g["co2_lines"].view(orc_mod.LINE_DTYPE)
    ll = pkg.HITRANLinelist(lines)
    for method, tol in (("Weideman", 5e-5), ("PseudoVoigt", 5e-5)):
        ref = oracle.voigt_xsec(lines, g["co2_grid"], 230.0, 0.2, method=method)
        got = pkg.compute_voigt_cross_sections(g["co2_grid"], ll, 230.0, 0.2, backend=ctx,
                                               method=pkg.VoigtMethod[method], precision="mixed")
        assert np.max(np.abs(got - ref)) <= tol * ref.max(), method


@pytest.mark.parametrize("method", ["Weideman", "FullFaddeeva"])
def test_cross_sections_5k_far_field(pkg, ctx, oracle, method):
    """The 5,000-line list on its 34,801-point grid, where most lines reach a block only
    through the interpolated far field, the mid and cutoff-edge classes: mixed (far
    field) and mixed_direct against the FP64 oracle, for both Voigt evaluators that have
    a far-wing switch."""
    ll = pkg.synthetic.lists_5k_co2()[2]
    grid = np.array([(251600 + i) / 400 for i in range(34801)])
    for T, p in ((296.0, 1.0), (220.0, 0.05)):
        ref = oracle.voigt_xsec(ll.lines, grid, T, p, method=method)
        m = ref > 1e-2 * ref.max()
        for prec in ("mixed", "mixed_direct"):
            got = pkg.compute_voigt_cross_sections(grid, ll, T, p, backend=ctx, precision=prec,
                                                   method=pkg.VoigtMethod[method])
            if method == "FullFaddeeva":
                assert np.max(np.abs(got[m] - ref[m]) / ref[m]) < 2e-4, (method, prec, T)
                assert np.max(np.abs(got - ref)) < 2e-5 * ref.max(), (method, prec, T)
            else:  # FP32 Weideman-24, as the golden-fixture test
                assert np.max(np.abs(got - ref)) < 5e-5 * ref.max(), (method, prec, T)


# ------------------------------------------------------------ forward model
def _run(pkg, ctx, oracle, orc_mod, prof, lists, snd, channels=None, y0=None, geom=None, T_sfc=None,
         eps=1.0, method="FullFaddeeva", **kw):
    """Oracle and both GPU precisions on the same inputs; `method` is a VoigtMethod name."""
    opt = orc_mod.fm_options(mu=(geom.mu if geom else 1.0), eps_sfc=eps, T_sfc=T_sfc,
                             line_mixing=y0 is not None, method=method, **kw)
    ref = oracle.forward_model(oracle_profile(prof), {s: l.lines for s, l in lists.items()},
                               oracle_sounder(orc_mod, snd), opt, channels=channels,
                               y0=None if y0 is None else {2: y0})
    lm = pkg.VPYLineMixing(y0) if y0 is not None else None
    out = {}
    for prec in ("fp64", "mixed", "mixed_direct"):
        _, R, BT = pkg.forward_model(prof, lists, sounder=snd, geom=geom, T_sfc=T_sfc, eps_sfc=eps,
                                     backend=ctx, precision=prec, line_mixing=lm,
                                     method=pkg.VoigtMethod[method], **kw)
        if channels:
            R, BT = R[channels[0]:channels[1]], BT[channels[0]:channels[1]]
        out[prec] = (R, BT)
    return ref, out


def _check(ref, out, fp64_tol=1e-6, rms=0.01, mx=0.05):
    (R0, BT0) = ref
    R, BT = out["fp64"]
    assert np.max(np.abs(BT - BT0)) < fp64_tol
    assert np.max(np.abs(R - R0) / np.abs(R0)) < 1e-9
    for prec in ("mixed", "mixed_direct"):
        Rm, BTm = out[prec]
        d = BTm - BT0
        assert np.sqrt(np.mean(d * d)) <= rms and np.max(np.abs(d)) <= mx, prec


def test_forward_5k_co2(pkg, ctx, oracle, orc_mod):
    lists = pkg.synthetic.lists_5k_co2()
    prof = pkg.afgl_atmosphere("us_standard")
    snd = pkg.Sounder.make(645.0, 700.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    ref, out = _run(pkg, ctx, oracle, orc_mod, prof, lists, snd, internal_dnu=0.0025,
                    apply_continuum=False)
    _check(ref, out)


def test_forward_5k_co2_with_continua(pkg, ctx, oracle, orc_mod):
    lists = pkg.synthetic.lists_5k_co2()
    prof = pkg.afgl_atmosphere("tropical")
    snd = pkg.Sounder.make(645.0, 700.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    ref, out = _run(pkg, ctx, oracle, orc_mod, prof, lists, snd, internal_dnu=0.0025,
                    apply_continuum=True, continua=("h2o", "co2"))
    _check(ref, out)


@pytest.mark.parametrize("variant", ["toon", "slant_reflecting", "mass_weighted", "norton_beer",
                                     "no_ils", "weideman", "pseudovoigt", "no_dptmin"])
def test_forward_options(pkg, ctx, oracle, orc_mod, variant):
    lists = {2: pkg.synthetic.synthetic_linelist(800, 2, 7, 690.0, 712.0),
             1: pkg.synthetic.synthetic_linelist(400, 1, 8, 690.0, 712.0)}
    prof = pkg.afgl_atmosphere("midlatitude_summer")
    snd = pkg.Sounder.make(699.0, 703.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    kw = dict(internal_dnu=0.0025, apply_continuum=True, continua=("h2o", "co2"))
    geom, eps, T_sfc = None, 1.0, None
    if variant == "toon":
        kw["source_function"] = "toon"
    elif variant == "slant_reflecting":
        geom, eps, T_sfc = pkg.ViewingGeometry(50.0), 0.93, 301.5
    elif variant == "mass_weighted":
        kw["T_method"] = "mass_weighted"
    elif variant == "norton_beer":
        kw["apodization"] = "norton_beer_medium"
    elif variant == "no_ils":
        kw["with_ils"] = False
    elif variant == "weideman":
        kw["method"] = "Weideman"
    elif variant == "pseudovoigt":
        kw["method"] = "PseudoVoigt"
    elif variant == "no_dptmin":
        kw["dptmn"] = 0.0
    ref, out = _run(pkg, ctx, oracle, orc_mod, prof, lists, snd, geom=geom, eps=eps, T_sfc=T_sfc, **kw)
    _check(ref, out)


def test_forward_line_mixing(pkg, ctx, oracle, orc_mod):
    ll = pkg.synthetic.synthetic_linelist(1500, 2, 11, 680.0, 720.0)
    y0 = pkg.synthetic.vpy_y0(len(ll), seed=12)
    prof = pkg.afgl_atmosphere("us_standard")
    snd = pkg.Sounder.make(695.0, 705.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    ref, out = _run(pkg, ctx, oracle, orc_mod, prof, {2: ll}, snd, y0=y0, internal_dnu=0.0025,
                    apply_continuum=False)
    _check(ref, out)
    # the dispersive term is live: switching it off changes the spectrum
    _, _, BT0 = pkg.forward_model(prof, {2: ll}, sounder=snd, backend=ctx, internal_dnu=0.0025,
                                  apply_continuum=False)
    assert np.max(np.abs(BT0 - out["fp64"][1])) > 1e-3


def test_batch_and_device_entry_points_agree(pkg, ctx):
    lists = pkg.synthetic.lists_5k_co2()
    profs, scans = pkg.synthetic.perturbed_profiles(3, seed=5)
    snd = pkg.Sounder.make(645.0, 700.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    geoms = [pkg.ViewingGeometry(pkg.scan_angle_to_local_zenith(s)) for s in scans]
    _, R, BT = pkg.forward_model_batch(profs, lists, sounder=snd, geoms=geoms, backend=ctx,
                                       internal_dnu=0.0025, precision="mixed")
    for k in range(3):
        _, R1, BT1 = pkg.forward_model(profs[k], lists, sounder=snd, geom=geoms[k], backend=ctx,
                                       internal_dnu=0.0025, precision="mixed")
        assert np.array_equal(BT1, BT[k])
    # deterministic: a second batch call is bit-identical
    _, R2, BT2 = pkg.forward_model_batch(profs, lists, sounder=snd, geoms=geoms, backend=ctx,
                                         internal_dnu=0.0025, precision="mixed")
    assert np.array_equal(BT2, BT)


def test_errors_raise(pkg, ctx):
    lists = pkg.synthetic.lists_5k_co2()
    prof = pkg.afgl_atmosphere()
    snd = pkg.Sounder.make(645.0, 650.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    bad = pkg.AtmosphericProfile(prof.pressure, -prof.temperature, prof.altitude, prof.vmr)
    with pytest.raises(pkg.IRSError, match="positive"):
        pkg.forward_model(bad, lists, sounder=snd, backend=ctx)
    with pytest.raises(pkg.IRSError, match="lm_cutoff"):
        pkg.forward_model(prof, lists, sounder=snd, backend=ctx, lm_cutoff=10.0,
                          line_mixing=pkg.VPYLineMixing(np.zeros(5000)))
    with pytest.raises(pkg.IRSError, match="uniform"):
        pkg.compute_voigt_cross_sections(np.array([700.0, 700.1, 700.3]), lists[2], 250.0, 0.5,
                                         backend=ctx, precision="mixed")


# ------------------------------------------------------- 400,000-line scale
@pytest.fixture(scope="module")
def iasi_lists(pkg):
    return pkg.synthetic.lists_iasi_400k()


@pytest.mark.parametrize("window", [(100, 104), (6600, 6604)])
def test_iasi_400k_windows_vs_oracle(pkg, ctx, oracle, orc_mod, iasi_lists, window):
    prof = pkg.afgl_atmosphere("midlatitude_winter")
    snd = pkg.IASIInstrument()
    ref, out = _run(pkg, ctx, oracle, orc_mod, prof, iasi_lists, snd, channels=window,
                    internal_dnu=0.0025, apply_continuum=True, continua=("h2o", "co2"))
    _check(ref, out)


def test_iasi_400k_mixed_vs_fp64_full_spectrum(pkg, ctx, iasi_lists):
    prof = pkg.afgl_atmosphere("us_standard")
    _, _, BT64 = pkg.forward_model(prof, iasi_lists, backend=ctx, internal_dnu=0.0025,
                                   precision="fp64")
    _, _, BTm = pkg.forward_model(prof, iasi_lists, backend=ctx, internal_dnu=0.0025,
                                  precision="mixed")
    assert BT64.shape == (8461,) and np.all(np.isfinite(BT64)) and np.all(BT64 > 150)
    d = BTm - BT64
    assert np.sqrt(np.mean(d * d)) <= 0.01 and np.max(np.abs(d)) <= 0.05


def test_iasi_400k_far_field_vs_direct(pkg, ctx, iasi_lists):
    """The far-field interpolation (IRS_MIXED) against the direct FP32 sum
    (IRS_MIXED_DIRECT) over the whole IASI spectrum, with line mixing on CO2: BT
    within 1e-3 K (the interpolation error is ~1e-7 of each far line's term), while
    the line-sum kernel evaluates a fraction of the pairs."""
    prof = pkg.afgl_atmosphere("tropical")
    lm = pkg.VPYLineMixing(pkg.synthetic.vpy_y0(len(iasi_lists[2])))
    out = {}
    for prec in ("mixed_direct", "mixed"):
        _, _, out[prec] = pkg.forward_model(prof, iasi_lists, backend=ctx, internal_dnu=0.0025, precision=prec,
                                            line_mixing=lm)
        st = ctx.stage_times()
        if prec == "mixed":
            print("pairs", st.pairs, "evaluated", st.evaluated_pairs)
            assert st.evaluated_pairs < 0.3 * st.pairs
    d = out["mixed"] - out["mixed_direct"]
    assert np.max(np.abs(d)) < 1e-3


def test_far_field_fine_grid_core_reach(pkg, ctx):
    """A grid fine enough (and x_far large enough) that the Faddeeva cores reach
    thousands of points: the strip far field starts beyond every line's core reach, and
    IRS_MIXED still agrees with the direct FP32 sum (IRS_MIXED_DIRECT) to 1e-3 K."""
    lists = pkg.synthetic.lists_5k_co2()
    snd = pkg.Sounder.make(660.0, 664.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    prof = pkg.afgl_atmosphere("us_standard")
    out = {}
    for prec in ("mixed_direct", "mixed"):
        _, _, out[prec] = pkg.forward_model(prof, lists, sounder=snd, backend=ctx, internal_dnu=5e-5,
                                            x_far=400.0, precision=prec)
    assert np.all(np.isfinite(out["mixed"])) and np.all(out["mixed"] > 150)
    assert np.max(np.abs(out["mixed"] - out["mixed_direct"])) < 1e-3


def test_strip_far_field_batch_groups(pkg, ctx, monkeypatch):
    """The strip far field keeps its node values in a buffer of bounded size
    (IRS_STRIP_BUFFER_BYTES at context creation); a batch whose (segment, strip) cells
    exceed it runs the line sum in groups of profile-layers, with the same brightness
    temperatures as one launch.  A buffer too small for one profile-layer leaves the
    strip far field out (the warps take their whole windows): within 1e-3 K."""
    lists = pkg.synthetic.lists_5k_co2()
    snd = pkg.Sounder.make(660.0, 680.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    profs, _ = pkg.synthetic.perturbed_profiles(3)
    kw = dict(sounder=snd, internal_dnu=0.0025, precision="mixed")
    _, _, bt1 = pkg.forward_model_batch(profs, lists, backend=ctx, **kw)
    out = {}
    for limit in (5 * 30 * 528, 100):  # a few profile-layers of at most 30 strips; less than one
        monkeypatch.setenv("IRS_STRIP_BUFFER_BYTES", str(limit))
        c2 = pkg.B200Context()
        try:
            _, _, out[limit] = pkg.forward_model_batch(profs, lists, backend=c2, **kw)
        finally:
            c2.close()
    assert np.array_equal(out[5 * 30 * 528], bt1)
    assert np.max(np.abs(out[100] - bt1)) < 1e-3
