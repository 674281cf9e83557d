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
"""
from __future__ import annotations

import argparse
import json
import shutil
import tempfile
import time

import numpy as np

from . import VAN_ALBADA, Solver
from . import casegen

KINDS = {"yaw": 0, "pitch": 1, "omega": 2}


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

    spec = casegen.config(a.config, steps=a.steps)
    d = a.case_dir or tempfile.mkdtemp(prefix="dalm_gradcheck_")
    mesh = casegen.write_case(spec, d)
    U0 = casegen.initial_velocity(spec, mesh)
    prof = casegen.inflow_profile(spec, mesh)

    def make(params=None):
        s = Solver(d, limiter=VAN_ALBADA, time_average=False)
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
    t = time.perf_counter()
    J, g = s.power_gradient(a.t0, a.steps, a.ckpt)
    t_adj = time.perf_counter() - t
    stats = s.adjoint_stats()
    s.close()
    t = time.perf_counter()
    J_fwd = objective(base)
    t_fwd = time.perf_counter() - t
    out = {
        "config": a.config, "cells": list(spec.n), "turbines": len(base[0]),
        "steps": a.steps, "window": [a.t0, a.steps], "ckpt_every": a.ckpt,
        "limiter": "van Albada", "poisson_tol": a.tol, "polar_step_deg": spec.polar_step_deg,
        "params": {"yaw_deg": base[0].tolist(), "pitch_deg": base[1].tolist(),
                   "omega": base[2].tolist()},
        "J": J, "J_forward": J_fwd, "grad": g.tolist(),
        "adjoint_s": t_adj, "forward_s": t_fwd, "adjoint_over_forward": t_adj / t_fwd,
        "adjoint_stats": stats,
    }
    kinds = [KINDS[a.only]] if a.only else [0, 1, 2]

    def central(h):
        fd = np.full_like(g, np.nan)
        for w in range(g.shape[0]):
            for q in kinds:
                pp = [v.copy() for v in base]
                pm = [v.copy() for v in base]
                pp[q][w] += h
                pm[q][w] -= h
                fd[w, q] = (objective(pp) - objective(pm)) / (2 * h)
        return fd

    def report(fd):
        m = ~np.isnan(fd)
        rel = np.where(m, np.abs(g - fd) / np.abs(np.where(m, fd, 1.0)), np.nan)
        return {"fd": np.where(m, fd, np.nan).tolist(), "rel_err": rel.tolist(),
                "abs_err": np.where(m, np.abs(g - fd), np.nan).tolist(),
                "max_rel_err": float(np.nanmax(rel)),
                "norm_rel_err": float(np.linalg.norm((g - fd)[m]) / np.linalg.norm(fd[m]))}

    if not a.no_fd:
        t = time.perf_counter()
        out.update(report(central(a.h)))
        out["fd_s"] = time.perf_counter() - t
        for h in a.h_list or []:
            out.setdefault("fd_h", {})[repr(h)] = report(central(h))
    print(json.dumps(out))
    if not a.case_dir:
        shutil.rmtree(d, ignore_errors=True)


if __name__ == "__main__":
    main()
