"""Robust (Huber-IRLS) retrieval on the GPU against the robust oracle driven by the FP64
oracle forward model (robust_estimation.jl:145-241), on the small OE case of
test_gpu_oe.py with gross errors planted in three channels."""
import numpy as np
import pytest

import robust_oracle
from conftest import load_package
from test_gpu_oe import KW, oracle_fns, setup

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    return load_package()


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.B200Context()
    yield c
    c.close()


def case(pkg, ctx, orc_mod, dT=2.0):
    ll, llp, base, spec, xa, Sa, y, se, snd = setup(pkg, ctx, orc_mod, dT=dT, dv=0.1)
    y = y.copy()
    y[[2, 5, 9]] += np.array([3.0, -4.0, 5.0])
    return ll, llp, base, spec, xa, Sa, y, se, snd


def test_robust_vs_oracle(pkg, ctx, oracle, orc_mod):
    ll, llp, base, spec, xa, Sa, y, se, snd = case(pkg, ctx, orc_mod)
    r = pkg.robust_estimation(y, spec, base, llp, xa=xa, Sa=Sa, Se=se, max_outer=6, sounder=snd, backend=ctx,
                              fm_kwargs=KW)
    fwd, fwd_jac = oracle_fns(pkg, oracle, orc_mod, spec, base, ll)
    ro = robust_oracle.robust_estimation(y, fwd, fwd_jac, xa, Sa, se, max_outer=6)
    sd = np.sqrt(np.diag(r.result.S_hat))
    print("outer", r.n_outer, ro["n_outer"], "weights", np.round(r.weights, 3), np.round(ro["weights"], 3))
    assert r.n_outer == ro["n_outer"] and r.outer_converged == ro["outer_converged"]
    assert np.max(np.abs(r.weights - ro["weights"])) < 0.05
    assert np.all(r.weights[[2, 5, 9]] < 1.0) and np.all(r.sigma_eff >= r.sigma_floor * (1 - 1e-12))
    assert np.max(np.abs(r.result.x - ro["x"]) / sd) < 0.1
    assert len(r.shat_history) == r.n_outer
    p1 = pkg.robust_estimation(y, spec, base, llp, xa=xa, Sa=Sa, Se=se, max_outer=1, sounder=snd, backend=ctx,
                               fm_kwargs=KW)
    plain = pkg.optimal_estimation(y, spec, base, llp, xa=xa, Sa=Sa, Se=se, sounder=snd, backend=ctx, fm_kwargs=KW)
    assert np.allclose(p1.result.x, plain.x, rtol=0, atol=1e-12)


def test_robust_batch_matches_single(pkg, ctx, orc_mod):
    scenes = [case(pkg, ctx, orc_mod, dT=d) for d in (2.0, -1.5, 3.0)]
    ll, llp, base, spec, xa, Sa, _, se, snd = scenes[0]
    ys = np.stack([c[6] for c in scenes])
    rb = pkg.robust_estimation_batch(ys, spec, [base] * 3, llp, xa=xa, Sa=Sa, Se=se, max_outer=6, sounder=snd,
                                     backend=ctx, fm_kwargs=KW)
    for k in range(3):
        r1 = pkg.robust_estimation(ys[k], spec, base, llp, xa=xa, Sa=Sa, Se=se, max_outer=6, sounder=snd,
                                   backend=ctx, fm_kwargs=KW)
        assert rb[k].n_outer == r1.n_outer
        assert np.allclose(rb[k].weights, r1.weights, rtol=0, atol=1e-9)
        assert np.allclose(rb[k].result["x"], r1.result.x, rtol=0, atol=1e-9)


def test_robust_errors(pkg, ctx, orc_mod):
    ll, llp, base, spec, xa, Sa, y, se, snd = case(pkg, ctx, orc_mod)
    for bad in (dict(huber_c=0.0), dict(max_inflation=0.5), dict(max_outer=0)):
        with pytest.raises(pkg.IRSError):
            pkg.robust_estimation(y, spec, base, llp, xa=xa, Sa=Sa, Se=se, sounder=snd, backend=ctx, **bad)
    with pytest.raises(pkg.IRSError):
        pkg.robust_estimation(y, spec, base, llp, xa=xa, Sa=Sa, Se=se[:-1], sounder=snd, backend=ctx)
