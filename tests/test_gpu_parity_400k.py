"""Parity at the shipped scale: the 400,000-line six-species list (
and config 2 with VP_Y on CO2) against the FP64 oracle, across the IASI range.

The synthetic lines are uniform in 645-2760 cm^-1, so "band" windows are placed where
the real species' strongest bands lie (CO2 nu2 667, O3 nu3 1042, N2O nu1 1285, CH4
nu4 1306, H2O nu2 1595, CO 2143, N2O nu3 2224, CO2 nu3 2349) plus both ends of the range.
The oracle runs each window on its own (the window result equals the full run).  The
monochromatic path (with_ils = false: no +-16 cm^-1 ILS halo, so each window is ~200
grid points) is checked for all six AFGL profiles; the full path with the ILS on
windows at both ends.

Tolerances (the same as tests/test_gpu_parity.py): FP64 kernels within 1e-6 K of the
FP64 oracle; mixed (FP32 + Kahan) BT RMS <= 0.01 K and max <= 0.05 K over every
(profile, channel) sample.  The Jacobian of config 2 (state T + log H2O + log O3 +
T_sfc = 151): each column block within 2e-4 of its largest entry against the oracle's
analytic Jacobian, and against GPU central differences with the reference's steps
(default_fd_steps: 0.5 K, 1e-3 in log VMR) within 2 % of each column's largest entry
(the FD truncation of those steps) for the two most sensitive columns of each block.
The synthetic 400k atmosphere is opaque near the surface at every channel, so its T_sfc
and lowest-level columns are zero, in the oracle as here."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

BAND_NU = (645.0, 667.5, 1042.0, 1285.0, 1306.0, 1595.0, 2143.0, 2224.0, 2349.0, 2759.5)
N_WIN = 3  # channels per window


def windows():
    out = []
    for nu in BAND_NU:
        c0 = min(int(round((nu - 645.0) / 0.25)), 8461 - N_WIN)
        out.append((c0, c0 + N_WIN))
    return out


@pytest.fixture(scope="module")
def pkg():
    return load_package()


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.B200Context()
    yield c
    c.close()


@pytest.fixture(scope="module")
def lists(pkg):
    return pkg.synthetic.lists_iasi_400k()


def _oracle_windows(oracle, orc_mod, prof, lists, opt, y0=None):
    snd = orc_mod.sounder(645.0, 2760.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    out = []
    for c0, c1 in windows():
        _, bt = oracle.forward_model(dict(p=prof.pressure, T=prof.temperature, vmr=prof.vmr),
                                     {s: l.lines for s, l in lists.items()}, snd, opt, channels=(c0, c1),
                                     y0=None if y0 is None else {2: y0})
        out.append(bt)
    return np.concatenate(out)


def _gpu_windows(BT):
    return np.concatenate([BT[:, c0:c1] for c0, c1 in windows()], axis=1)


def _stats(d):
    return float(np.sqrt(np.mean(d * d))), float(np.max(np.abs(d)))


def test_all_afgl_profiles_band_windows(pkg, ctx, oracle, orc_mod, lists):
    """Six AFGL profiles x ten windows (bands and both ends), monochromatic path."""
    profs = [pkg.afgl_atmosphere(a) for a in pkg.synthetic.AFGL]
    kw = dict(internal_dnu=0.0025, apply_continuum=True, continua=("h2o", "co2"), with_ils=False)
    opt = orc_mod.fm_options(**kw)
    ref = np.stack([_oracle_windows(oracle, orc_mod, p, lists, opt) for p in profs])
    got = {}
    for prec in ("fp64", "mixed"):
        _, _, BT = pkg.forward_model_batch(profs, lists, sounder=pkg.IASIInstrument(), backend=ctx, precision=prec,
                                           **kw)
        got[prec] = _gpu_windows(BT)
    d64 = got["fp64"] - ref
    rms_m, max_m = _stats(got["mixed"] - ref)
    print(f"400k x 6 AFGL x {len(windows())} windows: FP64 max {np.max(np.abs(d64)):.2e} K, "
          f"mixed RMS {rms_m:.2e} K max {max_m:.2e} K")
    assert np.all(ref > 150.0) and np.all(np.isfinite(ref))
    assert np.max(np.abs(d64)) < 1e-6, np.max(np.abs(d64))
    assert rms_m <= 0.01 and max_m <= 0.05, (rms_m, max_m)
    # each profile's own spectrum is checked (not an average over profiles)
    for k in range(len(profs)):
        r, m = _stats(got["mixed"][k] - ref[k])
        assert r <= 0.01 and m <= 0.05, (k, r, m)


def test_vpy_perturbed_profiles_band_windows(pkg, ctx, oracle, orc_mod, lists):
    """Config 2 forward: VP_Y on the CO2 lines, two perturbed profiles with scan angles."""
    y0 = pkg.synthetic.vpy_y0(len(lists[2]))
    lm = pkg.VPYLineMixing(y0)
    profs, ang = pkg.synthetic.perturbed_profiles(2, seed=1002)
    geoms = [pkg.ViewingGeometry(pkg.scan_angle_to_local_zenith(a)) for a in ang]
    kw = dict(internal_dnu=0.0025, apply_continuum=True, continua=("h2o", "co2"), with_ils=False)
    ref = np.stack([_oracle_windows(oracle, orc_mod, p, lists,
                                    orc_mod.fm_options(mu=g.mu, line_mixing=True, **kw), y0=y0)
                    for p, g in zip(profs, geoms)])
    for prec in ("fp64", "mixed"):
        _, _, BT = pkg.forward_model_batch(profs, lists, sounder=pkg.IASIInstrument(), geoms=geoms, backend=ctx,
                                           precision=prec, line_mixing=lm, **kw)
        d = _gpu_windows(BT) - ref
        if prec == "fp64":
            assert np.max(np.abs(d)) < 1e-6, np.max(np.abs(d))
        else:
            r, m = _stats(d)
            assert r <= 0.01 and m <= 0.05, (r, m)


@pytest.mark.parametrize("name,window", [("tropical", (0, 3)), ("subarctic_winter", (8458, 8461))])
def test_ils_windows_at_both_ends(pkg, ctx, oracle, orc_mod, lists, name, window):
    """The full path with the ILS at the first and last channels (the ILS halo reaches
    past the line list there)."""
    prof = pkg.afgl_atmosphere(name)
    kw = dict(internal_dnu=0.0025, apply_continuum=True, continua=("h2o", "co2"))
    snd = orc_mod.sounder(645.0, 2760.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    R0, BT0 = oracle.forward_model(dict(p=prof.pressure, T=prof.temperature, vmr=prof.vmr),
                                   {s: l.lines for s, l in lists.items()}, snd, orc_mod.fm_options(**kw),
                                   channels=window)
    for prec in ("fp64", "mixed"):
        _, R, BT = pkg.forward_model(prof, lists, backend=ctx, precision=prec, **kw)
        d = BT[window[0]:window[1]] - BT0
        if prec == "fp64":
            assert np.max(np.abs(d)) < 1e-6 and np.max(np.abs(R[window[0]:window[1]] - R0) / R0) < 1e-9
        else:
            assert np.max(np.abs(d)) <= 0.05 and np.sqrt(np.mean(d * d)) <= 0.01


def _blocks(spec):
    out = [slice(spec.temp_range.start, spec.temp_range.stop)]
    out += [slice(b.range.start, b.range.stop) for b in spec.vmr_blocks]
    out.append(slice(spec.tsfc_index, spec.tsfc_index + 1))
    return out


def test_config2_jacobian_windows(pkg, ctx, oracle, orc_mod, lists):
    """Config 2: 400k lines + VP_Y, state T + log H2O + log O3 + T_sfc on two perturbed
    profiles with scan angles, against the oracle's analytic Jacobian on band windows
    (monochromatic path) and against GPU central differences of selected columns."""
    y0 = pkg.synthetic.vpy_y0(len(lists[2]))
    lm = pkg.VPYLineMixing(y0)
    profs, ang = pkg.synthetic.perturbed_profiles(2, seed=1002)
    geoms = [pkg.ViewingGeometry(pkg.scan_angle_to_local_zenith(a)) for a in ang]
    spec = pkg.StateVectorSpec(50, [pkg.H2O, pkg.O3], include_emissivity=False)
    kw = dict(internal_dnu=0.0025, apply_continuum=True, continua=("h2o", "co2"), with_ils=False)
    snd = pkg.IASIInstrument()
    _, K, y = pkg.analytic_jacobian_batch(profs, lists, spec, sounder=snd, geoms=geoms, backend=ctx,
                                          line_mixing=lm, **kw)
    osnd = orc_mod.sounder(645.0, 2760.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    wins = [windows()[k] for k in (1, 2, 5, 8)]  # CO2 nu2 (VP_Y), O3, H2O, CO2 nu3 (VP_Y)
    for p, (prof, g) in enumerate(zip(profs, geoms)):
        o = orc_mod.fm_options(mu=g.mu, dptmn=0.0, line_mixing=True, **kw)
        for c0, c1 in wins:
            Kr, yr = oracle.analytic_jacobian(dict(p=prof.pressure, T=prof.temperature, vmr=prof.vmr),
                                              {s: l.lines for s, l in lists.items()}, osnd, o,
                                              retrieved=[1, 3], include_eps=False, channels=(c0, c1),
                                              y0={2: y0})
            Kg = K[p, c0:c1]
            assert np.max(np.abs(y[p, c0:c1] - yr)) < 0.01
            for b in _blocks(spec):
                rel = np.max(np.abs(Kg[:, b] - Kr[:, b])) / (np.max(np.abs(Kr[:, b])) + 1e-30)
                assert rel < 2e-4, (p, c0, b, rel)
    # central differences of the two most sensitive columns of each block (the 400k
    # synthetic atmosphere is opaque near the surface at every channel: the T_sfc and
    # lowest-level columns are zero there, and so must their differences be)
    steps = pkg.default_fd_steps(spec)
    for p, (prof, g) in enumerate(zip(profs, geoms)):
        cols = []
        for b in _blocks(spec)[:3]:
            sc = np.max(np.abs(K[p][:, b]), axis=0)
            cols += [b.start + int(k) for k in np.argsort(sc)[-2:]]
        cols.append(spec.tsfc_index)
        x0 = pkg.pack_state(spec, prof)
        xs = []
        for j in cols:
            for sgn in (1.0, -1.0):
                x = x0.copy()
                x[j] += sgn * steps[j]
                xs.append(x)
        states = [pkg.unpack_state(spec, x, prof) for x in xs]
        _, _, BT = pkg.forward_model_batch([s[0] for s in states], lists, sounder=snd, geoms=[g] * len(xs),
                                           T_sfcs=[s[1] for s in states], backend=ctx, precision="mixed",
                                           line_mixing=lm, dptmn=0.0, **kw)
        for k, j in enumerate(cols):
            fd = (BT[2 * k] - BT[2 * k + 1]) / (2 * steps[j])
            scale = np.max(np.abs(K[p, :, j]))
            if scale == 0.0:
                assert np.max(np.abs(fd)) < 1e-5, (p, j)
            else:
                err = np.max(np.abs(fd - K[p, :, j])) / scale
                assert err <= 0.02, (p, j, err)
