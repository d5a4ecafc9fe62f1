"""HITRAN .par ingest (CPU only): the fixed-width record parser, the parsed-list cache
(runtests.jl:946-993 of IRSounderLBL.jl, with a .npy blob where the reference writes
.jld2) and the list filters."""
import os
import time

import numpy as np
import pytest

from conftest import load_package


@pytest.fixture(scope="module")
def pkg():
    return load_package()


def mk(mol, iso, nu, S):  # the reference suite's 67-character records
    return (f"{mol:2d}{iso}{repr(nu):>12}{repr(S):>10}{'0.0':>10}{'0.05':>5}{'0.07':>5}{'0.0':>10}"
            f"{'0.75':>4}{'0.0':>8}")


def test_parse_full_record(pkg):
    # a 160-character HITRAN2004+ record: the first 67 columns carry the fields
    # I2 I1 F12.6 E10.3 E10.3 F5.4 F5.3 F10.4 F4.2 F8.6, then the quanta and references
    rec = (" 2" + "1" + "  667.661366" + " 2.867E-19" + " 1.544E+00" + ".0723" + "0.090" + "  413.9463"
           + "0.75" + "-.002300")
    rec = rec + " " * (160 - len(rec))
    assert len(rec) == 160
    f = pkg.parse_hitran_par(rec)
    assert f[0] == 2 and f[1] == 1
    assert f[2] == 667.661366 and f[3] == 2.867e-19 and f[4] == 1.544
    assert f[5] == np.float32(0.0723) and f[6] == np.float32(0.090)
    assert f[7] == 413.9463 and f[8] == np.float32(0.75) and f[9] == np.float32(-0.0023)
    with pytest.raises(ValueError):
        pkg.parse_hitran_par(" 2x" + rec[3:])


def test_load_hitran_par_and_filters(pkg, tmp_path):
    par = tmp_path / "mixed.par"
    par.write_text("\n".join([mk(2, 1, 720.0, 3.0e-21), "short", mk(2, 1, 700.0, 1.0e-21),
                              " 2x" + mk(2, 1, 705.0, 1.0e-21)[3:], mk(2, 0, 710.0, 2.0e-21), ""]) + "\n")
    ll = pkg.load_hitran_par(str(par))
    assert len(ll) == 3 and list(ll.lines["wavenumber"]) == [700.0, 710.0, 720.0]  # sorted, bad rows skipped
    assert list(ll.lines["iso_id"]) == [1, 0, 1]
    assert len(pkg.load_hitran_par(str(par), nu_min=705.0, nu_max=715.0)) == 1
    assert len(pkg.filter_linelist(ll, 700.0, 712.0)) == 2
    assert len(pkg.filter_linelist(ll, 2.0e-21)) == 2
    with pytest.raises(pkg.IRSError):
        pkg.load_hitran_par(str(tmp_path / "absent.par"))


def test_linelist_cache(pkg, tmp_path, monkeypatch):  # runtests.jl:946-993
    par = tmp_path / "synthetic.par"
    par.write_text("\n".join(mk(2, 1, nu, S) for nu, S in ((700.0, 1.0e-21), (710.0, 2.0e-21),
                                                              (720.0, 3.0e-21))) + "\n")
    cache = tmp_path / "cache"
    monkeypatch.setenv("IRSOUNDER_LINELIST_CACHE", str(cache))
    assert pkg.linelist_cache_dir() == str(cache)
    ll1 = pkg.load_linelist(str(par))
    assert len(ll1) == 3
    assert len(list(cache.glob("*.npy"))) == 1
    ll2 = pkg.load_linelist(str(par))
    assert ll2.lines.tobytes() == ll1.lines.tobytes()          # exact round trip
    w = pkg.load_linelist(str(par), nu_min=705.0, nu_max=715.0)
    assert len(w) == 1 and w.lines["wavenumber"][0] == 710.0
    assert pkg.load_linelist(str(par), cache=False).lines.tobytes() == ll1.lines.tobytes()
    assert pkg.load_linelist(str(par), rebuild=True).lines.tobytes() == ll1.lines.tobytes()
    time.sleep(0.01)
    with open(par, "a") as f:
        f.write(mk(2, 1, 730.0, 4.0e-21) + "\n")
    assert len(pkg.load_linelist(str(par))) == 4
    assert len(list(cache.glob("*.npy"))) == 2
    assert pkg.clear_linelist_cache() == 2
    assert len(list(cache.glob("*.npy"))) == 0


def test_load_linelist_isotopologues(pkg, tmp_path):
    base = tmp_path / "co2"
    (tmp_path / "co2.par").write_text(mk(2, 1, 700.0, 1.0e-21) + "\n")
    (tmp_path / "co2_iso2.par").write_text(mk(2, 2, 701.0, 1.0e-22) + "\n")
    ll = pkg.load_linelist(str(base), [1, 2], cache=False)
    assert len(ll) == 2 and sorted(ll.lines["iso_id"]) == [1, 2]
    with pytest.raises(pkg.IRSError, match="iso3"):
        pkg.load_linelist(str(base), [1, 3], cache=False)
    with pytest.raises(pkg.IRSError, match="No lines"):
        pkg.load_linelist(str(base), [1], nu_min=800.0, cache=False)
