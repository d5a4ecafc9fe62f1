"""CPU-only checks of the product side: the C ABI library loads and exports every
symbol include/irs_b200.h declares, host-side argument validation, presets and the
seeded synthetic inputs.  No compute call needs a GPU here."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, load_package


@pytest.fixture(scope="module")
def pkg():
    m = load_package()
    from importlib import import_module
    build = import_module("irs_b200.build")
    build.build()
    return m


def header_symbols():
    text = (ROOT / "include" / "irs_b200.h").read_text()
    return sorted(set(re.findall(r"\b(irs_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(pkg):
    lib = C.CDLL(str(ROOT / "irsounderlbl.jl_b200" / "libirs_b200.so"))
    syms = header_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(lib, s), s
    # and the ctypes binding declares a signature for each of them
    from irs_b200 import _lib
    assert set(syms) <= set(_lib.SIGNATURES)


def test_abi_version_and_error_path(pkg):
    from irs_b200 import _lib
    lib = _lib.load()
    assert lib.irs_abi_version() == 1
    s = _lib.Sounder(645.0, 700.0, 0.25, 221, 2.0, 0.5)
    o = pkg.fm_options(internal_dnu=0.0025)
    n_nu, n_ch = C.c_int64(), C.c_int64()
    assert lib.irs_grid_size(C.byref(s), C.byref(o), C.byref(n_nu), C.byref(n_ch)) == 0
    assert (n_nu.value, n_ch.value) == (34801, 221)
    s2 = _lib.Sounder(645.0, 2760.0, 0.25, 8461, 2.0, 0.5)
    assert lib.irs_grid_size(C.byref(s2), C.byref(o), C.byref(n_nu), C.byref(n_ch)) == 0
    assert (n_nu.value, n_ch.value) == (858801, 8461)
    bad = _lib.Sounder(645.0, 700.0, -0.25, 0, 2.0, 0.5)
    assert lib.irs_grid_size(C.byref(bad), C.byref(o), C.byref(n_nu), C.byref(n_ch)) == -1
    assert b"invalid sounder grid" in lib.irs_last_error()


def test_presets_and_geometry(pkg):
    assert pkg.IASIInstrument().n_channels == 8461
    assert pkg.IASINGInstrument().n_channels == 16921
    assert pkg.CrISInstrument().nu_min == 650.0
    assert pkg.MTGIRSInstrument("lwir").nu_max == 1210.0
    with pytest.raises(pkg.IRSError):
        pkg.CrISInstrument("bogus")
    with pytest.raises(pkg.IRSError):
        pkg.ViewingGeometry(95.0)
    assert pkg.scan_angle_to_local_zenith(48.33) == pytest.approx(57.5, abs=0.3)
    with pytest.raises(pkg.IRSError):
        pkg.scan_angle_to_local_zenith(80.0)


def test_option_validation(pkg):
    with pytest.raises(pkg.IRSError):
        pkg.fm_options(apodization="bogus")
    with pytest.raises(pkg.IRSError):
        pkg.fm_options(source_function="bogus")
    with pytest.raises(pkg.IRSError):
        pkg.fm_options(T_method="bogus")
    o = pkg.fm_options(precision="mixed", line_mixing=pkg.VPYLineMixing(np.zeros(1)))
    assert o.precision == 1 and o.line_mixing == 1


def test_synthetic_inputs_are_seeded(pkg):
    a = pkg.synthetic.lists_5k_co2()[2].lines
    b = pkg.synthetic.lists_5k_co2()[2].lines
    assert a.dtype.itemsize == 56 and len(a) == 5000
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    assert np.all(np.diff(a["wavenumber"]) >= 0)
    assert 645.0 <= a["wavenumber"].min() and a["wavenumber"].max() <= 700.0
    big = pkg.synthetic.lists_iasi_400k(n_total=600, nu_lo=645.0, nu_hi=2760.0)
    assert sum(len(v) for v in big.values()) == 600 and sorted(big) == [1, 2, 3, 4, 5, 6]
    profs, scans = pkg.synthetic.perturbed_profiles(4)
    assert len(profs) == 4 and np.all((scans >= 0) & (scans <= 48))
    assert len(profs[0].pressure) == 50


def test_missing_library_fails_loudly(pkg, tmp_path):
    from irs_b200 import _lib
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.load(tmp_path / "libirs_b200.so")
