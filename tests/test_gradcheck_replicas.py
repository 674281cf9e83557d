"""The finite-difference check's replica mode (3dalm_b200/gradcheck.py) on
two CPU ranks over gloo: the forward runs split between the ranks, every
run is done exactly once, and the assembled central differences equal the
single-process ones and the analytic derivative of a quadratic objective
(for which central differences are exact up to rounding).  The objective
here is a host function; on the GPU each rank's runs are forward solves on
its own device."""
import importlib
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

from conftest import ROOT

BASE = [np.array([0.0, 10.0, 0.0]), np.array([0.0, 0.0, 0.0]), np.array([12.0, 12.0, 12.0])]
COEF = np.array([[0.5, -2.0, 0.25], [1.5, 0.75, -0.5], [-1.0, 3.0, 2.0]])  # [turbine, kind]


def objective(p):
    """sum over turbines and kinds of c p^2 + p: derivative 2 c p + 1"""
    P = np.stack([np.asarray(v, dtype=float) for v in p], axis=1)  # [turbine, kind]
    return float(np.sum(COEF * P * P + P))


def gradcheck_module():
    sys.path.insert(0, ROOT)
    return importlib.import_module("3dalm_b200.gradcheck")


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    gc = gradcheck_module()
    r, w, dev, gather = gc.replicas()
    assert (r, w, dev) == (rank, world, rank)
    jobs = gc.fd_jobs(3, [0, 1, 2], [1e-3, 1e-2])
    local = gc.run_jobs(jobs, objective, BASE, r, w)
    values = gather(local)
    fd = gc.assemble(jobs, values, 3)
    out.put((rank, sorted(local), len(values), {h: v.tolist() for h, v in fd.items()}))
    import torch.distributed as dist
    dist.barrier()
    dist.destroy_process_group()


def test_single_process_assembly():
    gc = gradcheck_module()
    jobs = gc.fd_jobs(3, [0, 1, 2], [1e-3])
    assert len(jobs) == 18
    fd = gc.assemble(jobs, gc.run_jobs(jobs, objective, BASE), 3)[1e-3]
    exact = 2 * COEF * np.stack(BASE, axis=1) + 1
    np.testing.assert_allclose(fd, exact, rtol=1e-9, atol=1e-9)
    # one kind only: the others stay NaN
    jobs = gc.fd_jobs(3, [1], [1e-3])
    fd = gc.assemble(jobs, gc.run_jobs(jobs, objective, BASE), 3)[1e-3]
    assert np.isnan(fd[:, 0]).all() and np.isnan(fd[:, 2]).all() and not np.isnan(fd[:, 1]).any()


def test_two_rank_replicas():
    gc = gradcheck_module()
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
    jobs = gc.fd_jobs(3, [0, 1, 2], [1e-3, 1e-2])
    # each run exactly once, split between the ranks
    assert sorted(res[0][1] + res[1][1]) == list(range(len(jobs)))
    assert not set(res[0][1]) & set(res[1][1])
    single = gc.assemble(jobs, gc.run_jobs(jobs, objective, BASE), 3)
    for rank, _, nvalues, fd in res:
        assert nvalues == len(jobs)
        for h in single:
            np.testing.assert_array_equal(np.array(fd[h]), single[h])
