"""Multi-GPU form of the benchmark, on CPU: every rank is an independent
replica and the whole-job rate is every rank's units over the slowest rank's
time (two gloo ranks stand in for two GPUs; no GPU is touched)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    ctx = bench.Ctx(backend="gloo", device="cpu")
    ctx.barrier()
    # rank r "took" (r + 1) * 10 ms for 1000 units
    seconds = (rank + 1) * 0.010
    slowest = ctx.max_over_ranks(seconds)
    rate = ctx.throughput(1000, seconds)
    out[rank] = (slowest, rate)
    ctx.finish()


@pytest.mark.timeout(120)
def test_replica_rate_uses_the_slowest_rank():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    for slowest, rate in res.values():
        assert slowest == pytest.approx(0.020)
        assert rate == pytest.approx(world * 1000 / 0.020)


def test_single_rank_needs_no_process_group(monkeypatch):
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, ROOT)
    import bench
    ctx = bench.Ctx(backend="gloo", device="cpu")
    assert ctx.world == 1
    assert ctx.throughput(500, 0.5) == pytest.approx(1000.0)
