"""Kernel timeline of the solver's time step, from the GPU's own records.

    python -m 3dalm_b200.timeline [c4] [--steps 2 --warmup 3 --dt 5e-4 --fp64]

writes the case, runs the warm-up steps, then records every kernel of the
next steps through torch.profiler (CUPTI activity records: start and end of
each kernel as the GPU ran it, CUDA-graph replays included, nothing
serialised) and prints one JSON object: the span from the first kernel's
start to the last one's end, the busy time, the idle gaps, and per kernel
and grid size the launches, the time per step and the mean duration of the
launches that did work (longer than `--noop-us`; the multigrid kernels
enqueued past convergence return at once).
"""
from __future__ import annotations

import argparse
import collections
import json
import os
import re
import shutil
import tempfile

from . import FP64, MIXED, Solver
from . import casegen


def kernel_name(full: str) -> str:
    m = re.search(r"(k_\w+(<\d+>)?)", full)
    return m.group(1) if m else full[:40]


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("config", nargs="?", default="c4")
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--dt", type=float, default=5e-4)
    ap.add_argument("--fp64", action="store_true", help="the FP64 form (default: DALM_MIXED)")
    ap.add_argument("--noop-us", type=float, default=3.0)
    ap.add_argument("--top", type=int, default=40)
    a = ap.parse_args(argv)

    import torch
    from torch.profiler import ProfilerActivity, profile

    spec = casegen.config(a.config, steps=100000, dt=a.dt)
    d = tempfile.mkdtemp(prefix="dalm_timeline_")
    try:
        mesh = casegen.write_case(spec, d)
        s = Solver(d, precision=FP64 if a.fp64 else MIXED)
        s.set_inflow_profile(casegen.inflow_profile(spec, mesh))
        s.set_state(casegen.initial_velocity(spec, mesh))
        s.step(a.warmup)
        s.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as p:
            for _ in range(a.steps):
                s.step(1)
                s.stats()
            s.synchronize()
        s.close()
        trace = os.path.join(d, "trace.json")
        p.export_chrome_trace(trace)
        with open(trace) as f:
            ev = json.load(f)["traceEvents"]
    finally:
        shutil.rmtree(d, ignore_errors=True)
    k = sorted((e for e in ev if e.get("cat") == "kernel"), key=lambda e: e["ts"])
    if not k:
        raise SystemExit("no kernel records (no GPU, or the profiler saw none)")
    span = k[-1]["ts"] + k[-1]["dur"] - k[0]["ts"]
    gaps = [k[n + 1]["ts"] - (k[n]["ts"] + k[n]["dur"]) for n in range(len(k) - 1)]
    by = collections.defaultdict(list)
    for e in k:
        by[(kernel_name(e["name"]), tuple(e.get("args", {}).get("grid", [])))].append(e["dur"])
    rows = []
    for (name, grid), durs in sorted(by.items(), key=lambda kv: -sum(kv[1]))[: a.top]:
        work = [t for t in durs if t > a.noop_us]
        rows.append({"kernel": name, "grid": list(grid), "launches": len(durs),
                     "us_per_step": sum(durs) / a.steps, "working_launches": len(work),
                     "us_per_working_launch": sum(work) / len(work) if work else 0.0})
    print(json.dumps({"config": a.config, "precision": "FP64" if a.fp64 else "MIXED",
                      "steps": a.steps, "kernels": len(k), "span_us_per_step": span / a.steps,
                      "busy_us_per_step": sum(e["dur"] for e in k) / a.steps,
                      "gaps_us_per_step": sum(g for g in gaps if g > 0) / a.steps,
                      "by_kernel": rows}))


if __name__ == "__main__":
    main()
