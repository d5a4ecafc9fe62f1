"""The multi-GPU host logic on CPU (gloo, world size 2), with the oracles as the compute.

* shard_range (irs_shard_range of the library, host only): contiguous, balanced shards
  that cover the batch exactly.
* distributed_batch: each rank computes its shard of profiles (the FP64 oracle's
  forward_model stands in for the GPU) and the all-gather returns exactly the
  single-rank spectra, in profile order.
* train_data_parallel: one gradient all-reduce + Adam step per mini-batch over two ranks
  equals the single-rank step on the concatenated batch (the MLP oracle as the model,
  Adam restated as the library's adam_kernel).
"""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import load_package

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _spawn(target, world, *args):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q) + args) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


def _init(rank, world, port):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    sys.path.insert(0, str(ROOT / "tests"))
    sys.path.insert(0, str(ROOT / "oracle"))
    return dist


def test_shard_range():
    pkg = load_package()
    for n in range(0, 40):
        for k in range(1, 10):
            shards = [pkg.shard_range(n, k, i) for i in range(k)]
            assert shards[0][0] == 0
            for (a, c), (b, _) in zip(shards, shards[1:]):
                assert a + c == b  # contiguous
            assert sum(c for _, c in shards) == n
            assert max(c for _, c in shards) - min(c for _, c in shards) <= 1
            assert [c for _, c in shards] == sorted((c for _, c in shards), reverse=True)
    with pytest.raises(pkg.IRSError):
        pkg.shard_range(5, 0, 0)
    with pytest.raises(pkg.IRSError):
        pkg.shard_range(5, 2, 2)


# ---------------------------------------------------------------- sharded forward
def _small_case():
    pkg = load_package()
    import oracle as orc
    lists = {2: pkg.synthetic.synthetic_linelist(300, 2, 7, 695.0, 705.0)}
    base = pkg.afgl_atmosphere("us_standard")
    profs = [pkg.AtmosphericProfile(base.pressure, base.temperature + dT, base.altitude, base.vmr)
             for dT in (-6.0, -3.0, 0.0, 2.0, 5.0)]
    snd = orc.sounder(699.0, 701.0, 0.25, opd_max=2.0, fwhm_gauss=0.5)
    opt = orc.fm_options(internal_dnu=0.005, apply_continuum=False)
    return pkg, orc, lists, profs, snd, opt


def _oracle_compute(orc, o, lists, profs, snd, opt):
    def compute(first, count):
        R, BT = [], []
        for p in profs[first:first + count]:
            r, bt = o.forward_model(dict(p=p.pressure, T=p.temperature, vmr=p.vmr),
                                    {s: l.lines for s, l in lists.items()}, snd, opt)
            R.append(r)
            BT.append(bt)
        return np.array(R), np.array(BT)
    return compute


def _forward_rank(rank, world, port, q):
    dist = _init(rank, world, port)
    pkg, orc, lists, profs, snd, opt = _small_case()
    o = orc.Oracle()
    R, BT = pkg.distributed_batch(_oracle_compute(orc, o, lists, profs, snd, opt), len(profs), dist)
    q.put((rank, R, BT, pkg.shard_range(len(profs), world, rank)))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_forward_gathers_single_rank_order(oracle):
    res = _spawn(_forward_rank, 2)
    pkg, orc, lists, profs, snd, opt = _small_case()
    R1, BT1 = pkg.distributed_batch(_oracle_compute(orc, oracle, lists, profs, snd, opt), len(profs), None)
    assert [r[3] for r in res] == [(0, 3), (3, 2)]
    for rank, R, BT, _ in res:  # every rank holds the whole batch, bit for bit
        assert np.array_equal(R, R1) and np.array_equal(BT, BT1), rank
    assert len(np.unique(BT1[:, 0])) == len(profs)  # the profiles differ, so the order is checked


# ---------------------------------------------------------------- data-parallel step
DIMS = [7, 16, 16, 5]


def _mlp_problem(n_total=24, seed=3):
    rng = np.random.default_rng(seed)
    n_par = sum(DIMS[l + 1] * DIMS[l] + DIMS[l + 1] for l in range(len(DIMS) - 1))
    p0 = 0.3 * rng.standard_normal(n_par)
    X = rng.standard_normal((n_total, DIMS[0]))
    Y = rng.standard_normal((n_total, DIMS[-1]))
    return p0, X, Y


class _Adam:
    """The library's adam_kernel (b1 0.9, b2 0.999, eps 1e-8, bias-corrected), FP64."""

    def __init__(self, p):
        self.p, self.m, self.v, self.t = p.copy(), np.zeros_like(p), np.zeros_like(p), 0

    def step(self, g, lr):
        self.t += 1
        self.m = 0.9 * self.m + 0.1 * g
        self.v = 0.999 * self.v + 0.001 * g * g
        c1, c2 = 1 - 0.9 ** self.t, 1 - 0.999 ** self.t
        self.p -= lr * (self.m / c1) / (np.sqrt(self.v / c2) + 1e-8)


def _dp_rank(rank, world, port, q, batch, epochs):
    dist = _init(rank, world, port)
    import torch
    import mlp_oracle as mo
    pkg = load_package()
    from irs_b200.surrogate import train_data_parallel
    p0, X, Y = _mlp_problem()
    first, count = pkg.shard_range(len(X), world, rank)
    Xl, Yl = X[first:first + count], Y[first:first + count]
    z = np.zeros(DIMS[0]), np.ones(DIMS[0]), np.zeros(DIMS[-1]), np.ones(DIMS[-1])
    opt = _Adam(p0)

    def grad_fn(rows):
        loss, g, _ = mo.forward_backward(opt.p, DIMS, Xl[rows], Yl[rows], *z)
        return torch.from_numpy(g), loss

    def apply_fn(g, lr):
        opt.step(g.numpy(), lr)

    losses = train_data_parallel(grad_fn, apply_fn, count, batch=batch, epochs=epochs, lr=1e-2, seed=11, rank=rank,
                                 world=world, all_reduce=dist.all_reduce)
    q.put((rank, opt.p, losses, first, count))
    dist.barrier()
    dist.destroy_process_group()


def test_data_parallel_step_equals_concatenated_batch():
    import mlp_oracle as mo
    pkg = load_package()
    from irs_b200.surrogate import cosine_lr, dp_rows
    batch, epochs, world = 4, 2, 2
    res = _spawn(_dp_rank, world, batch, epochs)
    p0, X, Y = _mlp_problem()
    z = np.zeros(DIMS[0]), np.ones(DIMS[0]), np.zeros(DIMS[-1]), np.ones(DIMS[-1])
    opt = _Adam(p0)
    shards = [pkg.shard_range(len(X), world, r) for r in range(world)]
    ref_losses = []
    for ep in range(epochs):
        lr = cosine_lr(1e-2, ep, epochs)
        tot = 0.0
        for st in range(shards[0][1] // batch):
            rows = np.concatenate([f + dp_rows(c, batch, ep, st, 11, r) for r, (f, c) in enumerate(shards)])
            loss, g, _ = mo.forward_backward(opt.p, DIMS, X[rows], Y[rows], *z)
            opt.step(g, lr)
            tot += loss
        ref_losses.append(tot / (shards[0][1] // batch))
    for rank, p, losses, _, _ in res:
        assert np.max(np.abs(p - opt.p)) <= 1e-12 * np.max(np.abs(opt.p)), rank
        assert np.allclose(losses, ref_losses, rtol=1e-12, atol=0), rank
    assert np.max(np.abs(opt.p - p0)) > 1e-3  # the steps moved the parameters
