"""Mixed-precision form against the FP64 form over a run.

    python -m 3dalm_b200.mixedcheck [c4] [--steps 200 --avg-from 1]

writes the case, runs the FP64 form (the reference's arithmetic and
Jacobi(3)-BiCGStab) and DALM_MIXED from the same initial state for the same
steps, and prints one JSON object: each turbine's power averaged over steps
avg-from..steps in both forms and their relative difference, the relative
L2 difference of u, v, w and p at the end, the largest final pressure
residual of each form, and the wall time of each run.  The flow is chaotic:
step-wise fields drift apart from the solver-tolerance level, averages are
what the two forms must agree on.
"""
from __future__ import annotations

import argparse
import json
import shutil
import tempfile
import time

import numpy as np

from . import FP64, MIXED, Solver
from . import casegen


def run(d, prof, U0, precision, steps, avg_from):
    s = Solver(d, precision=precision, time_average=False)
    if prof is not None:
        s.set_inflow_profile(prof)
    s.set_state(U0)
    s.synchronize()
    power, worst, its = None, 0.0, []
    t = time.perf_counter()
    s.step(1)  # step 0: no integration
    for n in range(1, steps + 1):
        s.step(1)
        st = s.stats()
        worst = max(worst, st["err"])
        its.append(st["it"])
        if n >= avg_from:
            p = s.turbines()[2]
            power = p.copy() if power is None else power + p
    s.synchronize()
    wall = time.perf_counter() - t
    out = {"power": power / (steps - avg_from + 1), "U": s.field("U"), "p": s.field("p"),
           "max_residual": worst, "seconds": wall, "iterations": its}
    s.close()
    return out


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("config", nargs="?", default="c4")
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--avg-from", type=int, default=1)
    ap.add_argument("--dt", type=float, default=None, help="override the case's time step")
    a = ap.parse_args(argv)
    over = {"dt": a.dt} if a.dt else {}
    spec = casegen.config(a.config, steps=a.steps, **over)
    d = tempfile.mkdtemp(prefix="dalm_mixedcheck_")
    mesh = casegen.write_case(spec, d)
    U0, prof = casegen.initial_velocity(spec, mesh), casegen.inflow_profile(spec, mesh)
    f = run(d, prof, U0, FP64, a.steps, a.avg_from)
    m = run(d, prof, U0, MIXED, a.steps, a.avg_from)
    out = {
        "config": a.config, "cells": list(spec.n), "steps": a.steps, "dt": spec.dt,
        "average_over": [a.avg_from, a.steps], "tolerance": spec.tol,
        "mean_power_fp64": f["power"].tolist(), "mean_power_mixed": m["power"].tolist(),
        "mean_power_rel_diff": (np.abs(m["power"] - f["power"]) / np.abs(f["power"])).tolist(),
        "final_rel_l2": {"u": rel(m["U"][..., 0], f["U"][..., 0]),
                         "v": rel(m["U"][..., 1], f["U"][..., 1]),
                         "w": rel(m["U"][..., 2], f["U"][..., 2]), "p": rel(m["p"], f["p"])},
        "max_residual_fp64": f["max_residual"], "max_residual_mixed": m["max_residual"],
        "seconds_fp64": f["seconds"], "seconds_mixed": m["seconds"],
        "speedup": f["seconds"] / m["seconds"],
        "iterations_fp64_mean": float(np.mean(f["iterations"])),
        "iterations_mixed_mean": float(np.mean(m["iterations"])),
    }
    print(json.dumps(out))
    shutil.rmtree(d, ignore_errors=True)


if __name__ == "__main__":
    main()
