"""Relaxation-matrix line mixing, host side (CPU only): the library's C++ W(T), Y(T)
and VP_W eigenmodes (relmat.cpp through the C ABI; no device work) against the numpy
oracle, the relmat file readers on files written in the reference's fixed-width
formats, and the whitelist logic."""
import math

import numpy as np
import pytest

import lm_oracle as lo
from conftest import load_package


@pytest.fixture(scope="module")
def pkg():
    m = load_package()
    from importlib import import_module
    import_module("irs_b200.build").build()
    return m


@pytest.fixture(scope="module")
def relmat(pkg):
    return pkg.synthetic.synthetic_relmat(n_bands=6, j_max=40)


def key(b):
    return (min(b.li, b.lf), max(b.li, b.lf))


@pytest.mark.parametrize("T", [200.0, 250.0, 296.0, 312.5])
def test_w_and_y_match_oracle(pkg, relmat, T):
    for b in relmat.bands:
        wt = relmat.wtfit[key(b)]
        W, pop = pkg.build_w_matrix(b, wt, T)
        Wr, popr = lo.build_w_matrix(b, wt, T)
        assert np.max(np.abs(W - Wr)) <= 1e-12 * np.max(np.abs(Wr)), b.name
        assert np.max(np.abs(pop - popr)) <= 1e-13 * np.max(popr)
        Y = pkg.calc_w_and_y(b, wt, T)
        Yr = lo.calc_y(b, wt, T)
        assert np.max(np.abs(Y - Yr)) <= 1e-11 * np.max(np.abs(Yr)), b.name


def test_w_structure(pkg, relmat):
    """Decoupled bands give a diagonal W and Y = 0; symmetric-top isotopologues
    (isot > 2, not 7 or 10) couple only even J differences; li > lf swaps the J roles."""
    b0 = relmat.bands[1]
    wt = relmat.wtfit[key(b0)]
    dec = pkg.RelmatBand("DEC", 1, 3, 1, b0.nu_min, b0.nu_max, b0.lines)
    W, _ = pkg.build_w_matrix(dec, wt, 250.0)
    assert np.count_nonzero(W - np.diag(np.diag(W))) == 0
    assert np.all(pkg.calc_w_and_y(dec, wt, 250.0) == 0.0)
    L = b0.lines.copy()
    L["isot"] = 3
    sym = pkg.RelmatBand("SYM", b0.li, b0.lf, 3, b0.nu_min, b0.nu_max, L)
    W, _ = pkg.build_w_matrix(sym, wt, 250.0)
    Wr, _ = lo.build_w_matrix(sym, wt, 250.0)
    J = L["ji"].astype(int)
    odd = (np.abs(J[:, None] - J[None, :]) % 2) == 1
    assert np.all(W[odd] == 0.0)
    assert np.max(np.abs(W - Wr)) <= 1e-12 * np.max(np.abs(Wr))
    swap = pkg.RelmatBand("SWAP", 2, 1, 1, b0.nu_min, b0.nu_max, b0.lines)
    W, _ = pkg.build_w_matrix(swap, relmat.wtfit[(1, 2)] if (1, 2) in relmat.wtfit else wt, 250.0)
    Wr, _ = lo.build_w_matrix(swap, relmat.wtfit[(1, 2)] if (1, 2) in relmat.wtfit else wt, 250.0)
    assert np.max(np.abs(W - Wr)) <= 1e-12 * np.max(np.abs(Wr))


@pytest.mark.parametrize("T,p", [(296.0, 1.0), (250.0, 0.5), (220.0, 0.05)])
def test_band_modes_match_oracle(pkg, relmat, T, p):
    for b in relmat.bands:
        wt = relmat.wtfit[key(b)]
        m = pkg.band_modes(b, wt, T, p, keep_threshold=0.0)
        lam, A, f = lo.band_modes(b, wt, T, p, keep_threshold=0.0)
        assert len(m.poles) == len(lam) == len(b.lines)
        assert abs(m.f - f) <= 1e-14 * f
        # invariants: trace of M and sum of amplitudes (= sum of S(T) = d^T rho d)
        assert abs(np.sum(m.poles) - np.sum(lam)) <= 1e-11 * np.sum(np.abs(lam))
        assert abs(np.sum(m.amplitudes) - np.sum(A)) <= 1e-10 * np.sum(np.abs(A))
        # each pole has a partner within 1e-9 cm^-1
        d = np.abs(m.poles[:, None] - lam[None, :])
        assert np.max(np.min(d, axis=1)) < 1e-9
        # the cross section the modes produce
        g = np.linspace(b.nu_min - 2.0, b.nu_max + 2.0, 4001)
        s = lo.vpw_band_xsec(g, m.poles, m.amplitudes, m.f)
        sr = lo.vpw_band_xsec(g, lam, A, f)
        assert np.max(np.abs(s - sr)) <= 1e-9 * np.max(np.abs(sr)), b.name


def test_band_modes_keep_threshold(pkg, relmat):
    b = relmat.bands[2]
    wt = relmat.wtfit[key(b)]
    m = pkg.band_modes(b, wt, 250.0, 0.3, keep_threshold=0.2)
    lam, A, f = lo.band_modes(b, wt, 250.0, 0.3, keep_threshold=0.2)
    assert 0 < len(m.poles) < len(b.lines)
    assert abs(len(m.poles) - len(lam)) <= 1  # a mode within rounding of the threshold may differ
    assert np.all(np.abs(m.amplitudes) >= 0.2 * np.max(np.abs(m.amplitudes)) * (1 - 1e-9))


def test_whitelist_matches_oracle(pkg, relmat):
    for kw in (dict(), dict(n_top=2), dict(isotopes=[1]), dict(isotopes=[1, 2], n_top=1),
               dict(nu_window=(700.0, 710.0), n_top=3)):
        assert pkg.default_vpw_whitelist(relmat, **kw) == lo.default_vpw_whitelist(relmat.bands, **kw)
    for b in relmat.bands:
        assert pkg.band_eff_strength(b) == pytest.approx(lo.band_eff_strength(b), rel=1e-14)
    vpw = pkg.VPWLineMixing(relmat, n_top=2)
    assert vpw.whitelist == lo.default_vpw_whitelist(relmat.bands, n_top=2)
    assert pkg.VPYLineMixing(relmat).mode == 2 and vpw.mode == 3
    assert pkg.VPYLineMixing(np.zeros(4)).mode == 1


# --------------------------------------------------------------- file readers
def _fd(x, width, dec):  # Fortran D edit descriptor
    s = f"{x:.{dec}E}".replace("E", "D")
    return s.rjust(width)


def _put(buf, col, text):  # 1-based column
    buf[col - 1:col - 1 + len(text)] = list(text)


def write_relmat_files(d, relmat):
    bi = []
    for k, b in enumerate(relmat.bands):
        ident = f"{b.isot % 10}  {b.lf}    {b.li}    "  # I1, A2, i1, A2, A2, i1, A2, A2 (13 chars)
        ident = ident[:13].ljust(13)
        jmx = 50
        line = (ident + f"{1e-20 * (k + 1):12.4E}" + " " + f"{b.nu_min:12.6f}" + " " + f"{b.nu_max:12.6f}"
                + " " * 8 + f"{jmx:4d}{jmx:4d}{jmx:4d}")
        bi.append(line)
        rows = []
        for r in b.lines:
            buf = [" "] * 215
            _put(buf, 3, str(int(r["isot"]) % 10))
            _put(buf, 4, f"{r['nu']:12.6f}")
            stim = 1 - math.exp(-1.4388 * r["nu"] / 296.0)
            S = r["dipo_t"] ** 2 * r["popu_t0"] * r["nu"] * stim
            _put(buf, 16, f"{S:10.3E}")
            _put(buf, 36, f"{r['gv_air']:5.4f}"[-5:])
            _put(buf, 64, f"{r['e_lower']:10.4f}")
            _put(buf, 74, f"{r['n_air']:4.2f}")
            _put(buf, 82, f"{r['shift']:8.6f}"[:8])
            _put(buf, 140, {-1: "P", 0: "Q", 1: "R"}[int(r["branch"])])
            _put(buf, 141, f"{int(r['ji']):3d}")
            _put(buf, 184, _fd(r["dipo0"], 16, 8))
            _put(buf, 200, _fd(r["popu_t0"], 16, 8))
            rows.append("".join(buf))
        (d / ("S" + ident.rstrip() + ".dat")).write_text("\n".join(rows) + "\n")
    (d / "BandInfo.dat").write_text("\n".join(bi) + "\n")
    for (lli, llf), t in relmat.wtfit.items():
        out = []
        for sub in ("pp", "qq", "rr", "pr"):
            for (ji, jip), (w0, b0) in list(t.get(sub).items())[:200]:
                jf = ji + (1 if sub[0] == "p" else (0 if sub[0] == "q" else -1)) * -1
                jfp = jip + (1 if sub[1] == "p" else (0 if sub[1] == "q" else -1)) * -1
                out.append(_fd(w0, 20, 12) + _fd(b0, 20, 12) + f"{0.0:14.6f}{0.0:14.6f}"
                           + f"{ji:4d}{jf:4d}{jip:4d}{jfp:4d}")
        (d / f"WTfit{lli}{llf}.dat").write_text("\n".join(out) + "\n")


def test_readers_round_trip(pkg, relmat, tmp_path):
    sub = pkg.HITRANRelmatData([b for b in relmat.bands if b.li <= 8 and abs(b.li - b.lf) <= 1][:3], relmat.wtfit)
    write_relmat_files(tmp_path, sub)
    info = pkg.parse_bandinfo(str(tmp_path), 0.0, 5000.0)
    assert len(info) == 3
    assert [i["li"] for i in info] == [b.li for b in sub.bands]
    got = pkg.load_hitran_relmat(str(tmp_path), 0.0, 5000.0)
    assert len(got.bands) == 3
    for g, b in zip(got.bands, sub.bands):
        assert g.isot == b.isot and g.li == b.li and g.lf == b.lf
        assert np.allclose(g.lines["nu"], b.lines["nu"], atol=1e-6)
        assert np.array_equal(g.lines["ji"], b.lines["ji"])
        assert np.array_equal(g.lines["branch"], b.lines["branch"])
        assert np.allclose(g.lines["dipo0"], b.lines["dipo0"], rtol=1e-8)
        assert np.allclose(g.lines["popu_t0"], b.lines["popu_t0"], rtol=1e-8)
        assert np.allclose(g.lines["dipo_t"], b.lines["dipo_t"], rtol=5e-3)  # from the E10.3 intensity
    for k, t in got.wtfit.items():
        ref = sub.wtfit[k]
        for sname in ("pp", "qq", "rr", "pr"):
            for jj, v in t.get(sname).items():
                assert v == pytest.approx(ref.get(sname)[jj], rel=1e-11)
    # the window and intensity filters
    assert pkg.parse_bandinfo(str(tmp_path), 0.0, 1.0) == []
    assert len(pkg.parse_bandinfo(str(tmp_path), 0.0, 5000.0, stot_min=2.5e-20)) == 1
