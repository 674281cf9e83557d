"""bench.py's multi-GPU arithmetic (replicas, no exchange step) on two CPU
ranks over gloo: the job's time is the slowest rank's, the rate counts every
rank's cells, and the reference arm runs on rank 0 only."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        slowest = bench.max_over_ranks(1.0 + rank, world)
        rate = bench.whole_job_rate(1_000_000, 4, world, slowest)
        assert bench.dist_env() == (rank, world, rank)
        # the reference arm: rank 0 alone runs; the others return at once
        ran = None
        if rank != 0:
            args = type("A", (), {"steps": 1, "warmup": 0, "gpus": world, "case": "c4"})()
            ran = bench.run_reference(args)
        out.put((rank, slowest, rate, ran))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_replica_timing():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(out.get(timeout=5) for _ in range(2))
    for rank, slowest, rate, ran in res:
        assert slowest == 2.0                      # max over ranks
        assert rate == pytest.approx(1e6 * 4 * 2 / 2.0 / 1e6)  # both replicas' cells
    assert res[1][3] is None
