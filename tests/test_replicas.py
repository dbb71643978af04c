"""bench.py --gpus N runs N independent replicas of the workload (the
path does not shard here); the whole-job figures are the slowest rank's
device time and the cells of all ranks.  Checked with two gloo ranks on
the CPU: every rank gets the same max time and summed cells."""

import importlib.util
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_main", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms, cells = _bench().aggregate(10.0 * (rank + 1), 1000 + rank, world, dist, device="cpu")
        out[rank] = (ms, cells)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


PORT = _free_port()


@pytest.mark.parametrize("world", [2])
def test_replica_aggregation_over_gloo(world):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, PORT, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res == {r: (10.0 * world, float(sum(1000 + q for q in range(world)))) for r in range(world)}


def test_single_rank_aggregation_is_identity():
    assert _bench().aggregate(12.5, 34, 1, None, device="cpu") == (12.5, 34.0)

