"""Replicas-only multi-GPU host logic on CPU ranks (gloo, world size 2).

The step does not shard; bench.py runs one jet per rank and reports the
whole-job rate from the slowest rank's time.  These ranks exercise that
reduction and the aggregate with the gloo backend (no GPU)."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        ms = bench.max_over_ranks(times[rank])
        total = bench.sum_over_ranks(times[rank])
        out[rank] = (ms, bench.replica_value(512.0 ** 3, ms, world), total)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_take_slowest_rank():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    times = [10.0, 12.5]
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, times, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for r in range(2):
        ms, value, total = out[r]
        assert ms == 12.5
        assert total == 22.5   # the serving leg's whole-job throughput is the sum of the ranks' own
        assert value == pytest.approx(2 * 512.0 ** 3 / 12.5e-3 / 1e6)


def test_single_process_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.25) == 3.25
    assert bench.sum_over_ranks(3.25) == 3.25
    assert bench.replica_value(100.0, 1.0, 1) == pytest.approx(0.1)
