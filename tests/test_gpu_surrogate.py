"""The tensor-core GEMM and the MLP surrogate (irs_gemm_bf16, irs_surrogate_*).

* GEMM: BF16 inputs, FP32 accumulation, against numpy FP32 products of the same
  BF16 values (relative 1e-4 of the output scale: only the summation order differs).
* Gradients: against the numpy oracle of the same network (oracle/mlp_oracle.py) with
  the GPU's BF16 roundings replayed (relative Frobenius error 1e-2 per parameter block:
  FP32 vs FP64 sums can move a BF16 rounding by one unit).
* Training and OOD on a smooth synthetic map, then the surrogate trained on spectra of
  the GPU line-by-line path: its held-out error against LBL, what it gains over the
  climatological mean (the estimate without it), and the LBL fallback for OOD inputs.
"""
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


def to_bf16_bits(x):
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return (((a + 0x7FFF + ((a >> 16) & 1)) >> 16)).astype(np.uint16)


def from_bf16_bits(b):
    return (b.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (300, 520, 200), (1, 7, 5), (1024, 1024, 1024),
                                   (512, 8461, 1024), (8461, 192, 256), (4096, 8461, 192)])
def test_gemm_bf16(pkg, ctx, M, N, K):
    import ctypes as C
    rng = np.random.default_rng(M + N + K)
    A = to_bf16_bits(rng.standard_normal((M, K)))
    B = to_bf16_bits(rng.standard_normal((N, K)))
    out = np.empty((M, N), np.float32)
    pkg._lib.check(ctx.lib.irs_gemm_bf16(ctx.h, A.ctypes.data_as(C.c_void_p), B.ctypes.data_as(C.c_void_p), M, N, K,
                                         pkg._lib.fptr(out)))
    ref = from_bf16_bits(A).astype(np.float64) @ from_bf16_bits(B).astype(np.float64).T
    assert np.max(np.abs(out - ref)) <= 1e-4 * max(1.0, np.sqrt(K)) + 1e-5 * np.max(np.abs(ref))


def test_surrogate_gradients_vs_oracle(pkg, ctx):
    import mlp_oracle as mo
    n_in, hid, nl, n_out = 152, 64, 2, 101  # 101 outputs: rows of the output not 16-byte aligned
    s = pkg.Surrogate(ctx, n_in=n_in, n_hidden=hid, n_layers=nl, n_out=n_out, seed=11)
    rng = np.random.default_rng(3)
    X = rng.normal(0, 1, (96, n_in)).astype(np.float32)
    Y = rng.normal(0, 1, (96, n_out)).astype(np.float32)
    p = s.get_params()
    p = p + rng.normal(0, 0.05, p.shape).astype(np.float32)  # non-zero biases too
    s.set_params(p)
    assert np.array_equal(s.get_params(), p)
    g, loss = s.gradients(X, Y)
    dims = [n_in] + [hid] * nl + [n_out]
    z = np.zeros
    lo, go, out = mo.forward_backward(p, dims, X, Y, z(n_in), np.ones(n_in), z(n_out), np.ones(n_out), bf16=True)
    assert abs(loss - lo) <= 1e-3 * lo
    P, _ = s.predict(X)  # inference writes the unscaled outputs straight from the GEMM epilogue
    assert np.max(np.abs(P - out)) <= 5e-3 * np.max(np.abs(out))
    k = 0
    for o, i in [(dims[l + 1], dims[l]) for l in range(len(dims) - 1)]:
        for size in (o * i, o):
            a, b = g[k:k + size].astype(np.float64), go[k:k + size]
            assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(b), (k, size)
            k += size
    s.close()


@pytest.mark.parametrize("n_out,batch,hid", [(8461, 4200, 128), (1001, 700, 256)])
def test_predict_unaligned_rows_vs_oracle(pkg, ctx, n_out, batch, hid):
    """Inference rows that are not 16-byte aligned (n_out odd) leave the GEMM through
    the staged row-run epilogue with the output scale and shift per column: 8461 x 4200
    runs 128 x 256 tiles, several per CTA, with a ragged last row tile; 1001 x 700 runs
    ragged 128 x 128 tiles.  Against the oracle network with the GPU's BF16 roundings."""
    import mlp_oracle as mo
    n_in, nl = 152, 2
    s = pkg.Surrogate(ctx, n_in=n_in, n_hidden=hid, n_layers=nl, n_out=n_out, seed=5)
    rng = np.random.default_rng(7)
    s.fit_scaling(rng.normal(0.3, 2.0, (64, n_in)), rng.normal(250.0, 20.0, (64, n_out)) + rng.normal(0, 5, n_out))
    p = s.get_params()
    p = p + rng.normal(0, 0.05, p.shape).astype(np.float32)
    s.set_params(p)
    X = rng.normal(0, 1, (batch, n_in)).astype(np.float32)
    P, _ = s.predict(X)
    dims = [n_in] + [hid] * nl + [n_out]
    _, _, out = mo.forward_backward(p, dims, X, np.zeros((batch, n_out)), s.x_mean, s.x_sd, s.y_mean, s.y_sd,
                                    bf16=True, need_grad=False)
    assert P.shape == out.shape and np.isfinite(P).all()
    scaled = (P.astype(np.float64) - s.y_mean) / s.y_sd
    assert np.max(np.abs(scaled - out)) <= 5e-3 * np.max(np.abs(out))
    s.close()


def test_predict_into_caller_buffers(pkg, ctx):
    """predict(out=, ood=) fills the caller's arrays in place (the serving-loop form) with
    the values of a plain predict, and rejects arrays of the wrong shape or type."""
    s = pkg.Surrogate(ctx, n_in=152, n_hidden=64, n_layers=2, n_out=221, seed=2)
    X = np.random.default_rng(4).normal(0, 1, (300, 152)).astype(np.float32)
    P0, O0 = s.predict(X)
    P = np.full((300, 221), np.nan, np.float32)
    O = np.full(300, np.nan, np.float32)
    P1, O1 = s.predict(X, out=P, ood=O)
    assert P1 is P and O1 is O
    assert np.array_equal(P, P0)
    # the OOD score is a row sum of squares accumulated with FP32 atomics from several
    # warps and tiles, so its rounding order (not its value) varies between calls
    np.testing.assert_allclose(O, O0, rtol=1e-5, atol=1e-6)
    for bad in (np.empty((300, 220), np.float32), np.empty((300, 221), np.float64),
                np.empty((221, 300), np.float32).T):
        with pytest.raises(ValueError):
            s.predict(X, out=bad)
    s.close()


def test_training_and_ood(pkg, ctx):
    rng = np.random.default_rng(5)
    n_in, n_out = 152, 300
    A = rng.normal(0, 1 / np.sqrt(8), (8, 16))
    Bm = rng.normal(0, 1, (16, n_out))

    def f(X):  # a smooth map of 8 of the inputs
        return (np.tanh(X[:, :8] @ A) @ Bm * 3.0 + 250.0).astype(np.float32)

    X = rng.normal(0, 1, (4096, n_in)).astype(np.float32)
    Y = f(X)
    s = pkg.Surrogate(ctx, n_in=n_in, n_hidden=256, n_layers=3, n_out=n_out, seed=1)
    thr = s.fit_scaling(X, Y)
    losses = s.train(X, Y, epochs=120, batch=256, lr=2e-3, seed=2)
    assert losses[-1] < 0.1 * losses[0]
    Xt = rng.normal(0, 1, (512, n_in)).astype(np.float32)
    P, ood = s.predict(Xt)
    rms = np.sqrt(np.mean((P - f(Xt)) ** 2))
    assert rms < 0.25 * np.std(f(Xt))
    assert np.mean(ood > thr) < 0.01
    Xo = Xt[:16] + 12.0
    _, ood_o = s.predict(Xo)
    assert np.all(ood_o > thr)
    s.close()


def test_surrogate_on_lbl_spectra(pkg, ctx):
    """Trained only on spectra of the GPU LBL path (5,000-line CO2 list + MT-CKD
    continua, 221 channels); judged by LBL on held-out profiles."""
    lists = pkg.synthetic.lists_5k_co2()
    snd = pkg.Sounder.make(645.0, 700.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    kw = dict(precision="mixed", internal_dnu=0.0025, apply_continuum=True, continua=("h2o", "co2"))

    def lbl(profs, ang):
        geoms = [pkg.ViewingGeometry(pkg.scan_angle_to_local_zenith(a)) for a in ang]
        return pkg.forward_model_batch(profs, lists, sounder=snd, geoms=geoms, backend=ctx, **kw)[2]

    profs, ang = pkg.synthetic.perturbed_profiles(1024 + 128, seed=2024)
    BT = lbl(profs, ang)
    X = pkg.surrogate_features(profs, ang)
    tr, te = slice(0, 1024), slice(1024, None)
    s = pkg.Surrogate(ctx, n_in=X.shape[1], n_hidden=512, n_layers=3, n_out=BT.shape[1], seed=3)
    s.fit_scaling(X[tr], BT[tr])
    losses = s.train(X[tr], BT[tr].astype(np.float32), epochs=150, batch=128, lr=1e-3, seed=4)
    assert losses[-1] < 0.02 * losses[0]
    P, ood = s.predict(X[te])
    rms = float(np.sqrt(np.mean((P - BT[te]) ** 2)))
    clim = float(np.sqrt(np.mean((BT[tr].mean(0) - BT[te]) ** 2)))  # the estimate without the network
    print(f"surrogate held-out BT RMS {rms:.3f} K vs climatology {clim:.3f} K")
    assert rms < 0.2 * clim
    # OOD fallback: a profile 40 K warmer is computed by LBL, exactly
    hot = pkg.AtmosphericProfile(profs[1030].pressure, profs[1030].temperature + 40.0, profs[1030].altitude,
                                 profs[1030].vmr)
    batch = [profs[1024], hot, profs[1025]]
    res = pkg.surrogate_forward_batch(s, batch, [ang[1024], 10.0, ang[1025]], lists, sounder=snd, holdout=0.5,
                                      seed=1, backend=ctx, **kw)
    assert res["lbl_mask"].tolist() == [False, True, False]
    assert np.array_equal(res["BT"][1], lbl([hot], [10.0])[0])
    assert res["holdout_rms"] is not None and res["holdout_rms"] < 0.2 * clim
    # What the network gains a retrieval: optimal estimation of T + log H2O + T_sfc from
    # the surrogate's first guess against the same retrieval started at the a priori
    base = pkg.afgl_atmosphere("us_standard")
    spec = pkg.StateVectorSpec(50, [pkg.H2O], include_emissivity=False)
    xa = pkg.pack_state(spec, base)
    Sa = pkg.build_sa(spec, base, sigma_T=3.0, L_T=1.0, sigma_vmr=0.3)
    rng = np.random.default_rng(77)
    n_sc = 6
    xt = xa + (np.linalg.cholesky(Sa) @ rng.standard_normal((spec.n, n_sc))).T
    truth = [pkg.unpack_state(spec, x, base) for x in xt]
    ang_sc = rng.uniform(0.0, 48.0, n_sc)
    geoms = [pkg.ViewingGeometry(pkg.scan_angle_to_local_zenith(a)) for a in ang_sc]
    _, _, bt = pkg.forward_model_batch([t[0] for t in truth], lists, sounder=snd, geoms=geoms,
                                       T_sfcs=[t[1] for t in truth], backend=ctx, **kw)
    se = np.full(bt.shape[1], 0.2 ** 2)
    y = bt + 0.2 * rng.standard_normal(bt.shape)
    x0 = pkg.surrogate_first_guess(s, y, spec, [base] * n_sc, ang_sc, xa=xa, Sa=Sa, Se=se)

    def cost(xs):
        profs_x = [pkg.unpack_state(spec, x, base) for x in xs]
        F = pkg.forward_model_batch([p[0] for p in profs_x], lists, sounder=snd, geoms=geoms,
                                    T_sfcs=[p[1] for p in profs_x], backend=ctx, dptmn=0.0, **kw)[2]
        Si = np.linalg.inv(Sa)
        return np.array([np.sum((y[k] - F[k]) ** 2 / se) + (xs[k] - xa) @ Si @ (xs[k] - xa) for k in range(n_sc)])

    j_prior, j_first = cost(np.tile(xa, (n_sc, 1))), cost(x0)
    okw = dict(sounder=snd, geoms=geoms, backend=ctx, fm_kwargs={k: v for k, v in kw.items() if k != "precision"})
    r_prior = pkg.optimal_estimation_batch(y, spec, [base] * n_sc, lists, xa=xa, Sa=Sa, Se=se, **okw)
    r_first = pkg.optimal_estimation_batch(y, spec, [base] * n_sc, lists, xa=xa, Sa=Sa, Se=se, x0=x0, **okw)
    print(f"OE cost at start: a priori {np.median(j_prior):.1f}, surrogate first guess {np.median(j_first):.1f}; "
          f"LBL iterations {r_prior['n_iter'].sum()} -> {r_first['n_iter'].sum()}")
    # the network's first guess starts the retrieval well inside the a-priori cost, and
    # both starts converge to the same solutions (the iteration counts are reported)
    assert np.median(j_first) < 0.75 * np.median(j_prior)
    assert r_first["converged"].all() and r_prior["converged"].all()
    sd = np.sqrt(np.diag(Sa))
    assert np.max(np.abs(r_first["x"] - r_prior["x"]) / sd) < 0.5
    s.close()


def test_surrogate_accuracy_within_0p1K(pkg, ctx):
    """The surrogate's accuracy target (0.1 K RMS, judged by LBL) at a reduced size: the
    5,000-line CO2 list with MT-CKD continua (221 channels), 16,384 training spectra of the
    perturbed-AFGL sampler (scan angles 0-48 deg) from the GPU LBL path, 3 x 512 GELU,
    200 epochs; 512 held-out spectra.  Measured 0.063 K."""
    lists = pkg.synthetic.lists_5k_co2()
    snd = pkg.Sounder.make(645.0, 700.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    kw = dict(precision="mixed", internal_dnu=0.0025, apply_continuum=True, continua=("h2o", "co2"))
    n_tr, n_te = 16384, 512
    profs, ang = pkg.synthetic.perturbed_profiles(n_tr + n_te, seed=2024)
    geoms = [pkg.ViewingGeometry(pkg.scan_angle_to_local_zenith(a)) for a in ang]
    BT = pkg.forward_model_batch(profs, lists, sounder=snd, geoms=geoms, backend=ctx, **kw)[2]
    X = pkg.surrogate_features(profs, ang)
    tr, te = slice(0, n_tr), slice(n_tr, None)
    s = pkg.Surrogate(ctx, n_in=X.shape[1], n_hidden=512, n_layers=3, n_out=BT.shape[1], seed=3)
    s.fit_scaling(X[tr], BT[tr])
    s.train(X[tr], BT[tr].astype(np.float32), epochs=200, batch=256, lr=1e-3, seed=4)
    P, ood = s.predict(X[te])
    rms = float(np.sqrt(np.mean((P - BT[te]) ** 2)))
    print(f"surrogate held-out BT RMS {rms:.4f} K over {n_te} spectra")
    assert rms <= 0.1, rms
    assert np.sum(ood > s.ood_threshold) <= n_te // 100  # held-out inputs are in distribution
    s.close()
