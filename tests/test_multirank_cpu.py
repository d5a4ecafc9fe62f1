"""The N > 1 path of bench.py on CPU: two gloo ranks, each timing its own profiles;
the reported step time is the max over ranks and the value the whole-job rate."""
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = 100.0 + 50.0 * rank  # rank 1 is the slow one
    m = bench.reduce_max(dist, ms, "cpu")
    out.put((rank, m, bench.weak_scaling_value(world, bench.N_PROF, m)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [150.0, 150.0]
    sys.path.insert(0, str(ROOT))
    import bench
    assert res[0][2] == pytest.approx(2 * bench.N_PROF / 0.150)


def test_single_process_path():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.reduce_max(None, 12.5, "cpu") == 12.5
    assert bench.weak_scaling_value(1, 6, 500.0) == pytest.approx(12.0)
