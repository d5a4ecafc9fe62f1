"""The array-level operators through the C ABI against the FP64 oracle: voigt_profile
for the three evaluators, w(z), ils_kernel for every apodisation, apply_ils against a
direct numpy convolution, and schwarzschild_rte for both source functions with and
without a reflecting surface."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    return load_package()


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.B200Context()
    yield c
    c.close()


@pytest.mark.parametrize("method,tol", [("FullFaddeeva", 1e-12), ("Weideman", 1e-12), ("PseudoVoigt", 1e-12)])
def test_voigt_profile(pkg, ctx, oracle, orc_mod, method, tol):
    nu = np.linspace(699.0, 701.0, 2001)
    for gl, gd in ((0.07, 1.0e-3), (1e-4, 1.2e-3), (0.5, 1e-3)):
        got = pkg.voigt_profile(nu, 700.0, gl, gd, pkg.VoigtMethod[method], backend=ctx)
        ref = np.array([oracle.lib.orc_voigt_profile(v, 700.0, gl, gd, orc_mod.METHOD[method]) for v in nu])
        assert np.max(np.abs(got - ref)) <= tol * np.max(ref), (gl, gd)
    assert isinstance(pkg.voigt_profile(700.1, 700.0, 0.07, 1e-3, backend=ctx), float)


def test_faddeeva(pkg, ctx, oracle):
    x = np.concatenate([np.linspace(-30, 30, 601), [0.0, 1e-3, 200.0]])
    for y in (1e-6, 0.1, 1.0, 7.5, 40.0):
        got = pkg.faddeeva(x, np.full(len(x), y), backend=ctx)
        ref = oracle.faddeeva(x, y)
        assert np.max(np.abs(got - ref) / np.abs(ref)) < 1e-12, y
    assert np.allclose(pkg.faddeeva_voigt(x, 0.5, backend=ctx), oracle.faddeeva(x, 0.5).real, rtol=1e-12, atol=0)
    with pytest.raises(pkg.IRSError):
        pkg.faddeeva(1.0, -1.0, backend=ctx)


def test_faddeeva32_against_wofz(pkg, ctx, golden):
    """The FP32 evaluator of the mixed line sums (rational continued fractions with one
    reciprocal, Weideman N = 16) against scipy's wofz on the golden grid: every point
    within 2e-6 of the line-centre value Re w(i y) (the FP32 accuracy the mixed path's
    0.01 K budget rests on; ~5e-7 expected), on each side of the region switches."""
    import ctypes as C
    d = golden["wofz"]
    x, y = np.ascontiguousarray(d["x"]), np.ascontiguousarray(d["y"])
    keep = (np.abs(x) <= 122.0) & (y <= 100.0)  # the Faddeeva core of the line sums
    x, y = np.ascontiguousarray(x[keep]), np.ascontiguousarray(y[keep])
    re, im = np.empty(len(x)), np.empty(len(x))
    pkg.check(ctx.lib.irs_faddeeva32(ctx.h, pkg._lib.dptr(x), pkg._lib.dptr(y), len(x), pkg._lib.dptr(re),
                                     pkg._lib.dptr(im)))
    from scipy.special import erfcx
    centre = erfcx(y)  # Re w(i y)
    err = np.maximum(np.abs(re - d["re"][keep]), np.abs(im - d["im"][keep])) / centre
    s = np.abs(x) + y
    for lo, hi in ((0, 8), (8, 15), (15, np.inf)):
        m = (s >= lo) & (s < hi)
        assert m.sum() > 100, (lo, hi)
        assert err[m].max() < 2e-6, (lo, hi, err[m].max())


@pytest.mark.parametrize("apod", ["gaussian", "norton_beer_weak", "norton_beer_medium", "norton_beer_strong"])
def test_ils_kernel_and_apply(pkg, ctx, oracle, apod):
    d, k = pkg.ils_kernel(0.01, 2.0, 0.5, apod, backend=ctx)
    dr, kr = oracle.ils_kernel(0.01, 2.0, 0.5, apod)
    assert np.array_equal(d, dr)
    assert np.max(np.abs(k - kr)) <= 1e-12 * np.max(np.abs(kr))
    g = 690.0 + 0.01 * np.arange(8000)
    s = 1.0 + np.sin(g * 3.0) + np.exp(-((g - 715.0) / 0.05) ** 2)
    got = pkg.apply_ils(g, s, d, k, backend=ctx)
    ref = np.convolve(s, kr[::-1], mode="same") * 0.01
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("src", ["toon", "cim"])
@pytest.mark.parametrize("eps", [1.0, 0.93])
def test_schwarzschild_rte(pkg, ctx, oracle, src, eps):
    rng = np.random.default_rng(4)
    g = 700.0 + 0.0025 * np.arange(5000)
    L = 12
    tau = rng.uniform(0.0, 0.8, (len(g), L)) * np.linspace(1.0, 0.1, L)[None]
    tau[:100] = 1e-7                               # the CIM/LIT small-s series branches
    T_lev = np.linspace(290.0, 215.0, L + 1)
    T_ave = 0.5 * (T_lev[:-1] + T_lev[1:]) + 0.3
    got = pkg.schwarzschild_rte(g, tau, T_lev, 292.0, mu=0.9, eps_sfc=eps, source_function=src,
                                T_ave=T_ave if src == "cim" else None, backend=ctx)
    ref = oracle.rte(g, np.ascontiguousarray(tau.T), T_lev, 292.0, mu=0.9, eps=eps, source_function=src,
                     T_ave=T_ave if src == "cim" else None)
    assert np.max(np.abs(got - ref) / ref) < 1e-12
    with pytest.raises(pkg.IRSError):
        pkg.schwarzschild_rte(g, tau, T_lev, 292.0, source_function="cim", backend=ctx)


def test_host_helpers(pkg, oracle):
    nu = np.linspace(650.0, 2700.0, 50)
    T = np.linspace(190.0, 320.0, 50)
    assert np.allclose(pkg.planck_radiance(nu, T), [oracle.lib.orc_planck(a, b) for a, b in zip(nu, T)],
                       rtol=1e-14, atol=0)
    assert np.allclose(pkg.dB_dT(nu, T), [oracle.lib.orc_dB_dT(a, b) for a, b in zip(nu, T)], rtol=1e-13, atol=0)
    tau = np.abs(np.random.default_rng(1).normal(0, 0.3, (10, 4)))
    Tr = pkg.level_transmittances(tau, 0.8)
    assert np.all(Tr[:, -1] == 1.0) and np.allclose(Tr[:, 0], np.exp(-tau.sum(1) / 0.8), rtol=1e-14)
