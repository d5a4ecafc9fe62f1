"""IASI L1C granule -> batched optimal estimation on the GPU: spectra simulated by the
forward model for known states are written into a synthetic EPS-native granule (int16,
the format's scaling), read back as brightness temperatures and retrieved as one batch."""
import numpy as np
import pytest

from conftest import load_package
from l1c_synth import write_nat
from test_gpu_oe import KW, base_profile, lines

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    return load_package()


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.B200Context()
    yield c
    c.close()


def test_granule_retrieval(pkg, ctx, orc_mod, tmp_path):
    from importlib import import_module
    l1c = import_module("irs_b200.iasi_l1c")
    llp = {2: pkg.HITRANLinelist(lines(orc_mod))}
    base = base_profile(pkg)
    spec = pkg.StateVectorSpec(6, [pkg.CO2], include_emissivity=False)
    xa = pkg.pack_state(spec, base)
    Sa = pkg.build_sa(spec, base, sigma_T=2.0, sigma_vmr=0.2)
    snd = pkg.Sounder.make(699.0, 705.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    zen = [5.0, 20.0, 35.0, 45.0]
    truth, bts = [], []
    raw = np.full((1, 120, 8700), 7000, np.int16)
    n0 = int(round((699.0 - 645.0) / 0.25))
    for k, z in enumerate(zen):
        xt = xa.copy()
        xt[:6] += (1.0 + 0.5 * k) * np.linspace(1.0, 0.3, 6)
        xt[6:12] += 0.05 * (k - 1.5)
        xt[12] += 0.5 * k
        prof, Ts, _ = pkg.unpack_state(spec, xt, base)
        _, R, BT = pkg.forward_model(prof, llp, sounder=snd, geom=pkg.ViewingGeometry(z), T_sfc=Ts, backend=ctx,
                                     dptmn=0.0, **KW)
        bts.append(BT)
        raw[0, k, n0:n0 + len(R)] = np.round(R / (1e-7 * 1e5)).astype(np.int16)
        truth.append(xt)
    geo = lambda q, s, p, m: (10.0, 45.0, zen[q] if q < 4 else 10.0, 0.0, 60.0, 90.0, 0, 100)
    path = tmp_path / "sim.nat"
    write_nat(path, l1c, raw=raw, geo=geo)
    g = pkg.read_iasi_l1c(str(path), wnolim=(699.0, 705.0), bright=True, max_fov=4)
    assert pkg.nfov(g) == 4 and np.allclose(g.zen, zen)
    r = pkg.retrieve_granule(g, spec, base, llp, xa=xa, Sa=Sa, nedt_280K=0.2, backend=ctx, fm_kwargs=KW)
    assert r["converged"].all()
    # the same batch retrieved straight from the simulated brightness temperatures: the
    # granule path differs only by the int16 quantisation of the product (~0.005 K)
    nu = g.wno
    se = np.stack([pkg.scene_nedt(nu, b, nedt_280K=0.2) ** 2 for b in g.spc])
    d = pkg.optimal_estimation_batch(np.stack(bts), spec, [base] * 4, llp, xa=xa, Sa=Sa, Se=se, sounder=snd,
                                     geoms=[pkg.ViewingGeometry(z) for z in zen], backend=ctx, fm_kwargs=KW)
    assert np.max(np.abs(g.spc - np.stack(bts))) < 0.02
    for k in range(4):
        S_hat = np.linalg.inv(np.linalg.inv(Sa) + r["M"][k])
        sd = np.sqrt(np.diag(S_hat))
        assert np.max(np.abs(r["x"][k] - d["x"][k]) / sd) < 0.2
        assert np.max(np.abs(r["x"][k] - truth[k])[:6] / sd[:6]) < 3.0   # temperatures within 3 posterior sigma
