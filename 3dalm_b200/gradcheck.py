"""Gradient check of dalm_adjoint_power_grad against central finite
differences of the FP64 forward.

    python -m 3dalm_b200.gradcheck [c5] [--steps 200 --t0 101 --ckpt 20 --h 1e-5]

writes the case (default: 256x128x64, three turbines at x = 4, 9, 14 with
yaw 0/10/0 deg, log-law inflow + 8 %, van Albada limiter), computes the
gradient of J = mean total power over steps t0..steps with respect to every
turbine's yaw (deg), collective pitch (deg) and rotor speed (rad/s) by the
discrete adjoint, then each partial derivative by (J(p + h) - J(p - h)) / 2h
from fresh forward runs, and prints one JSON object with both, their
relative differences and the run times.  The pressure solves run to --tol
(RMS residual) so that the forward's solver tolerance enters the finite
differences as little as possible.

Under torchrun (WORLD_SIZE > 1) the check runs as replicas, one per GPU:
the forward runs of the finite differences are independent, so rank r
takes every WORLD_SIZE-th of them on device LOCAL_RANK, rank 0 also runs
the adjoint, and the objective values meet on rank 0 through one host-side
gather (gloo); nothing crosses between GPUs.

    python -m torch.distributed.run --nproc-per-node 8 --master-addr 127.0.0.1 \
        -m 3dalm_b200.gradcheck c5 --tol 1e-13 --h 1e-4
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import shutil
import tempfile
import time

import numpy as np

from . import VAN_ALBADA, Solver
from . import casegen

KINDS = {"yaw": 0, "pitch": 1, "omega": 2}


def fd_jobs(nturb, kinds, hs):
    """The forward runs of the central differences: (h, turbine, kind, sign)
    for every step size, turbine and parameter kind, + before -."""
    return [(h, w, q, sgn) for h in hs for w in range(nturb) for q in kinds for sgn in (1, -1)]


def run_jobs(jobs, objective, base, rank=0, world=1):
    """Objective values of this rank's share of the jobs (every world-th,
    from rank): {job index: J}.  base: (yaw, pitch, omega) arrays."""
    out = {}
    for i in range(rank, len(jobs), world):
        h, w, q, sgn = jobs[i]
        p = [np.array(v, dtype=float) for v in base]
        p[q][w] += sgn * h
        out[i] = objective(p)
    return out


def assemble(jobs, values, nturb):
    """{h: (nturb x 3) central differences} from all jobs' values (NaN where
    a kind was not differenced)."""
    fd = {}
    for i, (h, w, q, sgn) in enumerate(jobs):
        a = fd.setdefault(h, np.full((nturb, 3), np.nan))
        if sgn == 1:
            a[w, q] = (values[i] - values[i + 1]) / (2 * h)
    return fd


def replicas():
    """(rank, world, local_rank, gather) under torchrun, else (0, 1, 0,
    identity).  gather(dict) merges every rank's dict (host-side, gloo)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return 0, 1, 0, lambda d: d
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group("gloo", timeout=datetime.timedelta(hours=4))

    def gather(d):
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, d)
        merged = {}
        for part in parts:
            merged.update(part)
        return merged

    return dist.get_rank(), dist.get_world_size(), int(os.environ.get("LOCAL_RANK", "0")), gather


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("config", nargs="?", default="c5")
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--t0", type=int, default=101)
    ap.add_argument("--ckpt", type=int, default=20)
    ap.add_argument("--h", type=float, default=1e-5)
    ap.add_argument("--h-list", type=float, nargs="*", default=None,
                    help="further step sizes, reported under fd_h")
    ap.add_argument("--only", choices=sorted(KINDS), default=None,
                    help="finite differences of one parameter kind only")
    ap.add_argument("--tol", type=float, default=1e-12)
    ap.add_argument("--max-it", type=int, default=20000)
    ap.add_argument("--case-dir", default=None)
    ap.add_argument("--no-fd", action="store_true", help="adjoint and one forward run only")
    a = ap.parse_args(argv)
    rank, world, device, gather = replicas()

    spec = casegen.config(a.config, steps=a.steps)
    d = (os.path.join(a.case_dir, f"rank{rank}") if a.case_dir and world > 1 else a.case_dir) \
        or tempfile.mkdtemp(prefix="dalm_gradcheck_")
    mesh = casegen.write_case(spec, d)
    U0 = casegen.initial_velocity(spec, mesh)
    prof = casegen.inflow_profile(spec, mesh)

    def make(params=None):
        s = Solver(d, limiter=VAN_ALBADA, time_average=False, device=device)
        if prof is not None:
            s.set_inflow_profile(prof)
        s.set_poisson(a.max_it, a.tol)
        if params is not None:
            s.set_turbine_params(*params)
        s.set_state(U0)
        return s

    def objective(params):
        s = make(params)
        s.step(1)  # step 0: no integration
        J = 0.0
        for n in range(1, a.steps + 1):
            s.step(1)
            if n >= a.t0:
                J += float(np.sum(s.turbines()[2]))
        s.close()
        return J / (a.steps - a.t0 + 1)

    s = make()
    base = s.turbine_params()
    nturb = len(base[0])
    J, g, t_adj, stats = np.nan, np.full((nturb, 3), np.nan), 0.0, {}
    if rank == 0:
        t = time.perf_counter()
        J, g = s.power_gradient(a.t0, a.steps, a.ckpt)
        t_adj = time.perf_counter() - t
        stats = s.adjoint_stats()
    s.close()
    t = time.perf_counter()
    fwd = gather({"J": objective(base), "s": time.perf_counter() - t} if rank == world - 1 else {})
    J_fwd, t_fwd = fwd["J"], fwd["s"]
    out = {
        "config": a.config, "cells": list(spec.n), "turbines": len(base[0]),
        "steps": a.steps, "window": [a.t0, a.steps], "ckpt_every": a.ckpt,
        "limiter": "van Albada", "poisson_tol": a.tol, "polar_step_deg": spec.polar_step_deg,
        "params": {"yaw_deg": base[0].tolist(), "pitch_deg": base[1].tolist(),
                   "omega": base[2].tolist()},
        "J": J, "J_forward": J_fwd, "grad": g.tolist(),
        "adjoint_s": t_adj, "forward_s": t_fwd, "adjoint_over_forward": t_adj / t_fwd,
        "adjoint_stats": stats, "replicas": world,
    }
    kinds = [KINDS[a.only]] if a.only else [0, 1, 2]

    def report(fd):
        m = ~np.isnan(fd)
        rel = np.where(m, np.abs(g - fd) / np.abs(np.where(m, fd, 1.0)), np.nan)
        return {"fd": np.where(m, fd, np.nan).tolist(), "rel_err": rel.tolist(),
                "abs_err": np.where(m, np.abs(g - fd), np.nan).tolist(),
                "max_rel_err": float(np.nanmax(rel)),
                "norm_rel_err": float(np.linalg.norm((g - fd)[m]) / np.linalg.norm(fd[m]))}

    if not a.no_fd:
        hs = [a.h] + list(a.h_list or [])
        jobs = fd_jobs(nturb, kinds, hs)
        t = time.perf_counter()
        values = gather(run_jobs(jobs, objective, base, rank, world))
        fd = assemble(jobs, values, nturb)
        out["fd_s"] = time.perf_counter() - t
        if rank == 0:  # the adjoint gradient lives on rank 0
            out.update(report(fd[a.h]))
            for h in hs[1:]:
                out.setdefault("fd_h", {})[repr(h)] = report(fd[h])
    if rank == 0:
        print(json.dumps(out))
    if not a.case_dir:
        shutil.rmtree(d, ignore_errors=True)


if __name__ == "__main__":
    main()
