"""The N>1 path of bench.py without GPUs: two gloo ranks on CPU exercise the
max-over-ranks timing, the replica aggregation and the barrier, and the CPU
reference arm runs on rank 0 only (the other ranks return without work)."""
import datetime
import multiprocessing
import os
import socket

import pytest

from conftest import ROOT

torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ms = 100.0 + 50.0 * rank  # each rank's device time for its replica
    ms_max = bench.reduce_max(dist, ms, None)
    value = bench.replica_value(world, 10, ms_max)
    bench.barrier(dist)
    ref = bench.run_reference(type("A", (), {"steps": 1, "warmup": 0})(), rank, world) if rank != 0 else None
    out.put((rank, ms_max, value, ref))
    dist.destroy_process_group()


def test_two_rank_replicas_take_the_slowest_rank():
    ctx = multiprocessing.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms_max, value, ref in res:
        assert ms_max == 150.0                       # max over ranks
        assert abs(value - 2 * 10 / 0.150) < 1e-9    # all ranks' cycles / slowest time
        assert ref is None                           # rank 1 runs no reference work
