"""CPU tests of the bench's multi-rank path (one process per GPU under torchrun): the job's
step time is the maximum over ranks and the job's throughput counts every rank's bytes.
Run here as two gloo ranks on CPU; there is no data-path collective to test (each rank
compacts its own column)."""
from __future__ import annotations

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


def _rank_main(rank: int, world: int, port: int, times: list, q) -> None:
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        w, r, local = bench.dist_init(world)
        assert (w, r, local) == (world, rank, rank)
        ms = bench.max_over_ranks(times[rank], dist, "cpu")
        dist.barrier()
        q.put((rank, ms, bench.job_throughput(world, 10**9, ms * 1e-3)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_throughput_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    times = [2.0, 3.5]
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, gbs in got:
        assert ms == pytest.approx(3.5)            # the slowest rank's time, on every rank
        assert gbs == pytest.approx(2 * 1e9 / 3.5e-3 / 1e9)


def test_single_process_path():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(1.25, None, "cpu") == 1.25
    assert bench.job_throughput(1, 10**9, 1.0) == pytest.approx(1.0)
