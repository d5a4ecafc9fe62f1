"""HITRAN CIA (CPU only): the .cia reader, and the oracle's CIA optical depths pinned
on the closed form of continuum.jl:252-362 for an isothermal, dry, line-free
atmosphere (tau = sigma(nu, T) x pair density^2 x dz in each layer)."""
import numpy as np
import pytest

from cia_tables import blocks_co2, blocks_n2, blocks_o2, loaded, write_cia
from conftest import load_package


@pytest.fixture(scope="module")
def pkg():
    return load_package()


def test_reader(pkg, tmp_path):
    p = tmp_path / "N2-N2.cia"
    write_cia(p, "N2-N2", blocks_n2(), descending=(1,), negative=(1,))
    got = pkg.load_cia_table(str(p))
    ref = loaded(blocks_n2(), negative=(1,))
    assert len(got) == 3
    for (T, nu, sg), (Tr, nur, sgr) in zip(got, ref):
        assert T == Tr
        assert np.all(np.diff(nu) > 0)
        assert np.array_equal(nu, nur) and np.array_equal(sg, sgr)
    assert min(s.min() for _, _, s in got) == 0.0
    (tmp_path / "empty.cia").write_text("\n")
    assert pkg.load_cia_table(str(tmp_path / "empty.cia")) is None


def sigma_ref(blocks, nu, T):
    """continuum.jl:333-362 written out for the test."""
    lo = hi = None
    for bT, x, y in blocks:
        if nu < x[0] or nu > x[-1]:
            continue
        s = float(np.interp(nu, x, y))
        if bT <= T and (lo is None or bT > lo[0]):
            lo = (bT, s)
        if bT >= T and (hi is None or bT < hi[0]):
            hi = (bT, s)
    if lo is None and hi is None:
        return 0.0
    if lo is None:
        return hi[1]
    if hi is None or lo[0] == hi[0]:
        return lo[1]
    w = (T - lo[0]) / (hi[0] - lo[0])
    return (1 - w) * lo[1] + w * hi[1]


@pytest.mark.parametrize("T", [190.0, 237.5, 250.0, 320.0])
def test_oracle_cia_closed_form(pkg, oracle, orc_mod, T):
    tabs = {2: blocks_n2(), 3: blocks_o2(), 1: blocks_co2()}
    for pair, b in tabs.items():
        oracle.set_cia(pair, b)
    try:
        p = np.linspace(1000.0, 600.0, 5)
        prof = dict(p=p, T=np.full(5, T), vmr={2: np.full(5, 4.0e-4)})
        snd = orc_mod.sounder(697.0, 710.0, 0.5, opd_max=2.0, fwhm_gauss=0.5)
        lines = {2: np.zeros(0, dtype=orc_mod.LINE_DTYPE)}
        opt = orc_mod.fm_options(internal_dnu=0.01, continua=("co2_cia", "n2", "o2"), with_ils=True)
        _, _, tau = oracle.forward_model(prof, lines, snd, opt, return_tau=True)
        grid, _ = oracle.internal_grid(snd, opt)
        nw = tau.shape[1]
        g = grid[:nw] if len(grid) >= nw else grid
        kb = 1.380649e-23
        for k in range(4):
            pm, dp = 0.5 * (p[k] + p[k + 1]), p[k] - p[k + 1]
            dz = 8.314462 * T / (0.028964 * 9.80665) * dp / pm * 100.0
            nair = pm * 100.0 / (kb * T) * 1e-6
            for i in range(0, nw, 97):
                nu = g[i]
                want = (sigma_ref(tabs[1], nu, T) * 4.0e-4 * nair * nair
                        + sigma_ref(tabs[2], nu, T) * (0.78084 * nair) ** 2
                        + sigma_ref(tabs[3], nu, T) * (0.20946 * nair) ** 2) * dz
                assert tau[k, i] == pytest.approx(want, rel=1e-12, abs=1e-300)
    finally:
        for pair in tabs:
            oracle.set_cia(pair, None)
