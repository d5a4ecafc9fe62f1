"""Multi-device entry points on one GPU.

* irs_forward_model_batch_multi with two contexts (both on device 0: independent
  streams and workspaces, no kernel waits on another) gives the single-context
  spectra of the same batch, profile for profile, for even and odd splits.
* forward_model_batch_distributed without a process group is forward_model_batch.
* DataParallelSurrogate over a one-rank NCCL group: one full-batch step through
  irs_surrogate_grad_device + all-reduce + irs_surrogate_apply_device moves the
  parameters as irs_surrogate_train does for one epoch of one full batch.
"""
import os
import socket

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    return load_package()


def _case(pkg, n):
    lists = pkg.synthetic.lists_5k_co2()
    base = pkg.afgl_atmosphere("us_standard")
    profs = [pkg.AtmosphericProfile(base.pressure, base.temperature + 1.5 * k - 3.0, base.altitude, base.vmr)
             for k in range(n)]
    snd = pkg.Sounder.make(660.0, 680.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    return lists, profs, snd


def test_multi_context_batch_equals_single(pkg):
    lists, profs, snd = _case(pkg, 5)
    kw = dict(internal_dnu=0.0025, apply_continuum=True, continua=("h2o", "co2"), precision="mixed")
    a, b, c = pkg.B200Context(0), pkg.B200Context(0), pkg.B200Context(0)
    try:
        _, R1, BT1 = pkg.forward_model_batch(profs, lists, sounder=snd, backend=a, **kw)
        for ctxs in ([a, b], [a, b, c]):  # 3 + 2 and 2 + 2 + 1 profiles
            _, R, BT = pkg.forward_model_batch_multi(profs, lists, backends=ctxs, sounder=snd, **kw)
            assert np.array_equal(BT, BT1) and np.array_equal(R, R1), len(ctxs)
        with pytest.raises(pkg.IRSError, match="appear once"):  # one context is one host thread's
            pkg.forward_model_batch_multi(profs, lists, backends=[a, b, a], sounder=snd, **kw)
        _, R, BT = pkg.forward_model_batch_distributed(profs, lists, dist=None, backend=a, sounder=snd, **kw)
        assert np.array_equal(BT, BT1)
        assert len(np.unique(BT1[:, 10])) == len(profs)
    finally:
        a.close()
        b.close()
        c.close()


def test_data_parallel_step_one_rank(pkg):
    import torch
    import torch.distributed as dist
    from irs_b200.surrogate import DataParallelSurrogate
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    ctx = pkg.B200Context(0)
    try:
        rng = np.random.default_rng(5)
        n_in, n_out, n = 20, 37, 64
        X = rng.standard_normal((n, n_in)).astype(np.float32)
        Y = rng.standard_normal((n, n_out)).astype(np.float32)
        ref = pkg.Surrogate(ctx, n_in=n_in, n_hidden=64, n_layers=2, n_out=n_out, seed=9)
        dp_s = pkg.Surrogate(ctx, n_in=n_in, n_hidden=64, n_layers=2, n_out=n_out, seed=9)
        p0 = ref.get_params()
        assert np.array_equal(p0, dp_s.get_params())
        ref.train(X, Y, epochs=1, batch=n, lr=1e-2, seed=1)
        dp = DataParallelSurrogate(dp_s, dist)
        losses = dp.train(X, Y, epochs=1, batch=n, lr=1e-2, seed=1)
        torch.cuda.synchronize()
        p_ref, p_dp = ref.get_params(), dp_s.get_params()
        step_ref, step_dp = p_ref - p0, p_dp - p0
        # Adam's first step is lr * g / (|g| + eps) per weight: equal wherever the gradient
        # is not within summation-order noise of zero
        big = np.abs(step_ref) > 0.5e-2
        assert big.mean() > 0.5
        assert np.max(np.abs(step_dp[big] - step_ref[big])) < 1e-4
        assert np.isfinite(losses).all() and losses[0] > 0
        ref.close()
        dp_s.close()
    finally:
        ctx.close()
        dist.destroy_process_group()
