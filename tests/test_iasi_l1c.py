"""IASI L1C EPS-native reader (CPU only) on a synthetic granule written in the format's
framing, as the reference suite's round trip (runtests.jl:528-607), plus the noise
covariance helpers (noise_covariance.jl:113-152)."""
import math

import numpy as np
import pytest

from conftest import load_package
from l1c_synth import write_nat


@pytest.fixture(scope="module")
def pkg():
    return load_package()


@pytest.fixture(scope="module")
def l1c(pkg):
    from importlib import import_module
    return import_module("irs_b200.iasi_l1c")


def test_round_trip(pkg, l1c, tmp_path):
    path = tmp_path / "g.nat"
    write_nat(path, l1c)
    g = pkg.read_iasi_l1c(str(path))
    assert pkg.nfov(g) == 120
    assert g.mph["INSTRUMENT_ID"] == "IASI"
    assert len(g.wno) == 8461 and g.wno[0] == 645.0 and g.wno[-1] == 2760.0
    assert np.allclose(g.spc, 70.0, rtol=1e-12)
    i = int(np.flatnonzero((g.step == 1) & (g.pix == 1))[0])
    assert abs(g.lat[i] - 30.0) < 1e-6 and abs(g.lon[i] + 120.0) < 1e-6
    assert abs(g.zen[i] - 5.0) < 1e-6 and abs(g.sza[i] - 40.0) < 1e-6
    assert abs(g.azi[i] - 100.0) < 1e-6 and abs(g.saa[i] - 160.0) < 1e-6
    d = math.radians
    phi = math.degrees(math.acos(math.cos(d(g.sza[i])) * math.cos(d(g.zen[i]))
                                 - math.sin(d(g.sza[i])) * math.sin(d(g.zen[i])) * math.cos(d(g.saa[i] - g.azi[i]))))
    assert abs(g.sra[i] - phi) < 1e-6
    assert abs(l1c._solar_reflection_angle(30.0, 200.0, 30.0, 20.0)) < 1e-3      # specular: glint
    assert abs(l1c._solar_reflection_angle(30.0, 20.0, 30.0, 20.0) - 60.0) < 1e-9  # anti-specular: 2 theta
    assert pkg.solar_reflection_angle(g) is g.sra
    gc = pkg.read_iasi_l1c(str(path), cldlim=(0, 20))
    assert 0 < pkg.nfov(gc) < pkg.nfov(g) and np.all((gc.cld >= 0) & (gc.cld <= 20))
    lo, hi = g.sra.min(), g.sra.max()
    mid = 0.5 * (lo + hi)
    gg = pkg.read_iasi_l1c(str(path), sralim=(0, mid))
    assert 0 < pkg.nfov(gg) < pkg.nfov(g) and np.all(gg.sra <= mid)
    gw = pkg.read_iasi_l1c(str(path), wnolim=(700.0, 710.0), bright=True)
    assert gw.wno[0] == 700.0 and gw.wno[-1] == 710.0
    assert gw.is_bt and np.all((gw.spc > 100) & (gw.spc < 400))
    nu, R = pkg.measurement(g, i)
    assert len(nu) == len(R) == 8461


def test_filters_and_guards(pkg, l1c, tmp_path):
    path = tmp_path / "g2.nat"
    write_nat(path, l1c, n_mdr=2)
    g = pkg.read_iasi_l1c(str(path))
    assert pkg.nfov(g) == 240 and set(g.line) == {1, 2}
    assert pkg.nfov(pkg.read_iasi_l1c(str(path), max_fov=50)) == 50
    gl = pkg.read_iasi_l1c(str(path), latlim=(30.0, 30.1))
    assert np.all((gl.lat >= 30.0) & (gl.lat <= 30.1)) and pkg.nfov(gl) < 240
    with pytest.raises(pkg.IRSError):
        pkg.read_iasi_l1c(str(path), wnolim=(600.0, 700.0))
    bad = tmp_path / "bad.nat"
    write_nat(bad, l1c, geo=lambda q, s, p, m: (-120.0, 95.0, 5.0, 0.0, 40.0, 0.0, 0, 0))
    with pytest.raises(pkg.IRSError, match="lat/lon"):
        pkg.read_iasi_l1c(str(bad))
    assert pkg.nfov(pkg.read_iasi_l1c(str(bad), validate=False)) == 120
    raw = np.full((1, 120, 8700), 7000, np.int16)
    write_nat(bad, l1c, raw=raw, exponent=2)  # 700 W -> an impossible BT
    with pytest.raises(pkg.IRSError, match="BT"):
        pkg.read_iasi_l1c(str(bad))


def test_noise_covariance_helpers(pkg):
    nu = 645.0 + 0.25 * np.arange(20)
    A = np.random.default_rng(0).standard_normal((20, 20))
    nc = pkg.SounderNoiseCovariance(nu, A @ A.T * 1e-6, "radiance")
    sub = pkg.subset_channels(nc, nu[[3, 7, 11]] + 1e-4)
    assert np.array_equal(sub.cov, nc.cov[np.ix_([3, 7, 11], [3, 7, 11])])
    with pytest.raises(pkg.IRSError):
        pkg.subset_channels(nc, [700.0])
    Tb = np.full(20, 260.0)
    bt = pkg.to_bt(nc, Tb)
    from importlib import import_module
    est = import_module("irs_b200.estimation")
    D = 1.0 / est._dB_dT(nu, Tb)
    assert np.allclose(bt.cov, D[:, None] * nc.cov * D[None, :], rtol=1e-14) and bt.space == "bt"
    assert pkg.to_bt(bt, Tb) is bt
    with pytest.raises(pkg.IRSError):
        pkg.to_bt(nc, Tb[:-1])
    assert np.array_equal(pkg.measurement_covariance(nc), 0.5 * (nc.cov + nc.cov.T))
    with pytest.raises(pkg.IRSError):
        pkg.load_noise_covariance("x.nc", format="other")
