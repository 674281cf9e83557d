#!/usr/bin/env python
"""Benchmark of the 3dalm time step on one B200 per rank.

Workload (default --case c4): the 3-turbine case, 512x256x128 interior
cells (16.78 M) over a 20x5x5 domain stretched toward the ground, turbines
at x = 4, 9, 14 (yaw 0, 10, 0 deg, 3 blades x 32 points, R = 0.5, TSR 6),
log-law inflow (u* = 0.05, z0 = 1e-3) + seeded 8% Gaussian perturbation,
Re = 1e4, Cs = 0.1, minmod MUSCL, Jacobi(3)-preconditioned BiCGStab to 1e-8,
dt = 5e-4 (BENCH_DT).  Synthetic inputs (no dataset exists for this
solver); every field is larger than the 126 MB L2, so no L2 flush is
needed between steps.

A step is Solver::main_loop_once: predictor, face flux + Poisson RHS, the
Poisson solve to tolerance, projection + BCs, actuator line.  Metric:
Mcell-steps/s = interior cells x steps / time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --compare-forms STEPS     (FP64 vs mixed over a long run)

The headline `value` is the reference's precision (FP64).  The line also
carries `mixed`: the same timed steps with DALM_MIXED (FP32 stencil fields;
FP64 iterative refinement with FP32 multigrid-preconditioned CG inner
solves), its ratio to the FP64 form, its roofline, both forms' largest
final FP64 residual and its per-field / per-turbine errors against the FP64
form; and `e2e`, `roofline`, `cpu_baseline`, `clocks`, `adjoint`.

--impl reference runs the reference's own CPU step (oracle/_ref/ref_mpirun:
its sources compiled with OpenACC off, as MPI ranks on every host core) on
the same case and steps, whole steps within a wall budget.

With N > 1 (torchrun) every rank runs an independent replica of the case on
its own GPU (the path has no exchange step on one domain): weak scaling, no
collective on the data path; the time is the max over ranks.
"""
import argparse
import contextlib
import importlib
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s"
CASE = "c4"
# Time step of the benchmark runs.  At the configured dt = 1e-3 the
# 512x256x128 case diverges in the reference's explicit scheme (both forms
# here, the FP64 one step for step like the reference): the per-cell 8 %
# initial noise gives one 9.5e-4-thick wall cell a Smagorinsky viscosity
# that puts its explicit diffusion number above 1/2, and its velocity grows
# 5-20x per step with alternating sign (max CFL 0.42, 0.72, 2.8, 49, 1.8e4
# over steps 1-5).  At dt = 5e-4 every setting else as configured runs
# stably (max CFL 0.08 falling to 0.02 over 60 steps).
BENCH_DT = 5e-4

def workload_description(case):
    """One line naming the case's grid, rotor count, solver and inflow."""
    cg = importlib.import_module("3dalm_b200.casegen")
    spec = cg.config(case)
    n = "x".join(str(v) for v in spec.n)
    solver = {"SOR": f"red-black SOR w={spec.relax} to {spec.tol:g}",
              "BiCG": f"{spec.pc}({spec.pc_max_it})-BiCGStab to {spec.tol:g}",
              "Jacobi": f"Jacobi to {spec.tol:g}"}[spec.solver]
    inflow = (f"log-law inflow + {spec.intensity:.0%} noise" if spec.loglaw
              else f"uniform inflow + {spec.intensity:.0%} noise")
    rotors = len(spec.turbines)
    pts = rotors * spec.blades * spec.points_per_blade
    what = f"{rotors}-turbine" if rotors else "no-turbine"
    tail = f", {pts} blade points" if rotors else ""
    return f"{what} {n} LES step ({solver}, {inflow}{tail})"


def workload_config(case, cells, iterations, world, dt=BENCH_DT):
    """The `config` object both arms report."""
    return {"workload": workload_description(case),
            "case": case, "dt": dt,
            "dt_note": "configured 1e-3 diverges in the reference's explicit scheme on the "
                       "128-cell stretched z columns (wall-cell diffusion instability); see "
                       "BENCH_DT in bench.py",
            "precision": "FP64", "cells": cells,
            "poisson_iterations": iterations, "parallelism": f"replicas x{world}",
            "l2": "every field > 126 MB L2 (134 MB per scalar field at 512x256x128); no flush"}


@contextlib.contextmanager
def quiet_stdout():
    """Sends what native code prints to stdout (the reference's setup
    report) to stderr, so stdout carries only the JSON line."""
    import ctypes
    sys.stdout.flush()
    libc = ctypes.CDLL(None)
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        yield
    finally:
        libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--case", default=CASE)
    ap.add_argument("--e2e-steps", type=int, default=-1,
                    help="steps of the end-to-end (host buffer) measurement: -1 the same "
                         "steps as the timed region, 0 skips it")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision timing")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint cost run")
    ap.add_argument("--compare-forms", type=int, default=0, metavar="STEPS",
                    help="instead of the benchmark: run the FP64 and the mixed-precision form "
                         "from the same initial state for STEPS steps and print their "
                         "time-averaged turbine power, final field differences and wall times")
    ap.add_argument("--avg-from", type=int, default=1,
                    help="first step of the --compare-forms power average")
    return ap.parse_args()


def grad_interior(p, mesh, gc):
    """Central differences of a cell field over the interior cells along x,
    y, z with the cell-centre coordinates (the pressure gradient the
    projection applies, src/cfd.h:601-783)."""
    import numpy as np
    out = []
    for a in range(3):
        c = mesh[a]
        n = p.shape[a]
        sl = [slice(gc, p.shape[b] - gc) for b in range(3)]
        hi, lo = list(sl), list(sl)
        hi[a], lo[a] = slice(gc + 1, n - gc + 1), slice(gc - 1, n - gc - 1)
        shape = [1, 1, 1]
        shape[a] = n - 2 * gc
        h = (c[gc + 1:n - gc + 1] - c[gc - 1:n - gc - 1]).reshape(shape)
        out.append((p[tuple(hi)] - p[tuple(lo)]) / h)
    return np.stack(out, axis=-1)


def mixed_errors(a, b, mesh=None, gc=2):
    """Relative L2 error of the mixed form's final state against the FP64
    form's after the same steps: per velocity component; the pressure as
    stored, with its mean removed, and its gradient (what the solver
    tolerance pins: two solves that both meet the RMS residual tolerance may
    differ in p's smooth modes); per turbine thrust / power."""
    import numpy as np

    def rel(x, y):
        ny = np.linalg.norm(y)
        return float(np.linalg.norm(x - y) / (ny if ny > 0 else 1.0))
    out = {f"U[{m}]": rel(a["U"][..., m], b["U"][..., m]) for m in range(3)}
    out["p"] = rel(a["p"], b["p"])
    inner = (slice(gc, -gc),) * 3
    pa, pb = a["p"][inner], b["p"][inner]
    out["p_mean_removed"] = rel(pa - pa.mean(), pb - pb.mean())
    if mesh is not None:
        out["grad_p"] = rel(grad_interior(a["p"], mesh, gc), grad_interior(b["p"], mesh, gc))
    (tha, _, pwa), (thb, _, pwb) = a["turbines"], b["turbines"]
    out["thrust"] = [float(abs(x - y) / abs(y)) if y else 0.0 for x, y in zip(tha, thb)]
    out["power"] = [float(abs(x - y) / abs(y)) if y else 0.0 for x, y in zip(pwa, pwb)]
    return out


def max_over_ranks(v, world):
    """The largest of every rank's v (the job's time is its slowest replica's)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(cells, steps, world, seconds):
    """Mcell-steps/s of the whole job: every rank advances its own replica of
    `cells` cells by `steps` steps (weak scaling) in `seconds` (max over ranks)."""
    return cells * steps * world / seconds / 1e6


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms.  start()
    returns once the first sample has arrived (at most 3 s), and stop() waits
    (at most 0.6 s) for one sample after the timed region, so that a region
    shorter than the sampling interval is still covered: the summary takes the
    last sample before the region and every one from it to the first after."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
            return
        t = time.perf_counter()
        while not self.lines and time.perf_counter() - t < 3.0 and self.proc.poll() is None:
            time.sleep(0.01)
        self.first = max(0, len(self.lines) - 1)  # the last sample before the region

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        n, t = len(self.lines), time.perf_counter()
        while len(self.lines) == n and time.perf_counter() - t < 0.6 and self.proc.poll() is None:
            time.sleep(0.01)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[getattr(self, "first", 0):]:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(kernel):
    """DRAM bytes per launch of `kernel` at this workload from the committed
    ncu summary (profiles/traffic.json), or None."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return float(json.load(f)[CASE][kernel]["dram_bytes_per_launch"])
    except (OSError, KeyError, ValueError, TypeError):
        return None


def make_case(name, tmp, dt=BENCH_DT):
    cg = importlib.import_module("3dalm_b200.casegen")
    spec = cg.config(name, steps=100000, dt=dt)
    mesh = cg.write_case(spec, tmp)
    return spec, mesh, cg.initial_velocity(spec, mesh), cg.inflow_profile(spec, mesh)


# ------------------------------------------------------------------ CPU side

REF_MPIRUN = os.path.join(ROOT, "oracle", "_ref", "ref_mpirun")


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# Wall budget of the reference arm: no timed reference step begins after
# this many seconds since the start (every step that runs is whole and
# uncapped; the line says how many ran).  On the 16-core GPU hosts a whole
# step of the 512x256x128 case takes ~0.15-0.25 s per BiCGStab iteration, and
# the warm-up steps from the seeded state take ~3000 iterations.
REF_BUDGET_S = float(os.environ.get("DALM_REF_BUDGET_S", "720"))


def run_reference_ranks(case, warmup, steps, ranks, max_it=None, budget=0.0, timeout=1700):
    """The reference's own time step (oracle/_ref/ref_mpirun: the reference
    compiled from its sources, OpenACC off, with a shared-memory MPI subset)
    as `ranks` MPI ranks on the host cores: the 3-turbine case from its seeded
    initial state, `warmup` untimed steps, then `steps` timed whole steps.
    Returns ref_mpirun's result (per-step seconds, Poisson iterations and
    residuals) plus the case's description."""
    cg = importlib.import_module("3dalm_b200.casegen")
    over = {"steps": 100000, "dt": BENCH_DT}
    if max_it:
        over["max_it"] = max_it
    spec = cg.config(case, **over)
    with tempfile.TemporaryDirectory(prefix="dalm_ref_") as d, quiet_stdout():
        mesh = cg.write_case(spec, d)
        cg.write_state_files(spec, mesh, d)
        out = os.path.join(d, "result.json")
        cmd = [REF_MPIRUN, d, "--ranks", str(ranks), "--warmup", str(warmup), "--steps", str(steps),
               "--out", out, "--state", os.path.join(d, cg.STATE_FILE), "--budget", str(budget)]
        prof = os.path.join(d, cg.PROFILE_FILE)
        if os.path.exists(prof):
            cmd += ["--profile", prof]
        w0 = time.perf_counter()
        r = subprocess.run(cmd, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True,
                           timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"ref_mpirun failed ({r.returncode}): {r.stderr[-2000:]}")
        with open(out) as f:
            res = json.load(f)
        res["wall_seconds"] = time.perf_counter() - w0
    return res


def reference_sample(ranks, iterations, case=CASE):
    """cpu_baseline: a bounded sample of the benchmark workload on the host
    cores: one whole step (step 1 from the seeded initial state) of the full
    512x256x128 case through the reference's own code as `ranks` MPI ranks,
    with its pressure solve capped at the GPU arm's mean iteration count of
    the timed steps (so the sample does the same work per step as they do)."""
    it = max(1, int(round(iterations)))
    res = run_reference_ranks(case, 1, 1, ranks, max_it=it)
    secs = res["seconds"]
    desc = (f"reference (oracle/_ref/ref_mpirun: the reference's own step, OpenACC off) as "
            f"{ranks} MPI ranks on {ranks} host cores; one whole step of the same "
            f"case (step 1 from the seeded initial state) with the pressure "
            f"solve capped at {it} iterations, the GPU arm's mean over its timed steps "
            f"(ran {res['iterations'][0]})")
    return res["cells"] / secs / 1e6, "reference", desc, secs


def run_reference(args):
    """--impl reference: the reference's own CPU implementation of the step
    (MPI ranks on every host core, the reference's x-slab decomposition, OpenACC
    off) on the same case, steps and metric as this benchmark's arm: W untimed
    warm-up steps from the seeded initial state, then K timed whole steps."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    if not os.path.exists(REF_MPIRUN):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/ref_mpirun was not built (the reference sources were "
                          "absent when __graft_entry__.build() ran)"}), flush=True)
        return
    ranks = host_cores()
    res = run_reference_ranks(args.case, args.warmup, args.steps, ranks, budget=REF_BUDGET_S)
    secs = res["seconds"]
    cells = res["cells"]
    timed = res["steps_timed"]
    value = cells * timed / secs / 1e6
    desc = (f"reference (oracle/_ref/ref_mpirun: the reference's own step compiled from its "
            f"sources, OpenACC off, -O3 AVX2/FMA) as {ranks} MPI ranks (x-slabs, shared-memory "
            f"MPI) on {ranks} host cores; steps {args.warmup}..{args.warmup + timed - 1} "
            f"of the case after {args.warmup} untimed warm-up steps from the seeded initial "
            f"state, every step whole (Poisson to its tolerance); {timed} of the {args.steps} "
            f"requested steps fitted the {REF_BUDGET_S:.0f} s wall budget")
    cfg = workload_config(args.case, cells, res["iterations"], args.gpus)
    cfg["reference_residuals"] = res["residuals"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": secs / timed * 1e3, "steps_timed": timed, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": cfg,
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": ranks, "kind": "reference",
                         "sample": desc},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "step_seconds": res["step_seconds"],
        "setup_seconds": res["init_seconds"], "warmup_seconds": res["warmup_seconds"],
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU side

def adjoint_cost(pkg, device, steps=60, t0=31, ckpt=20):
    """Cost of dalm_adjoint_power_grad on the 256x128x64 three-turbine case
    (van Albada, the case's own pressure tolerance): wall time of the
    gradient call (forward run + recomputation + reverse sweep) against the
    same forward steps alone."""
    cg = importlib.import_module("3dalm_b200.casegen")
    tmp = tempfile.mkdtemp(prefix="dalm_bench_adj_")
    spec = cg.config("c5", steps=steps)
    mesh = cg.write_case(spec, tmp)
    U0, prof = cg.initial_velocity(spec, mesh), cg.inflow_profile(spec, mesh)

    def fresh():
        s = pkg.Solver(tmp, device=device, limiter=pkg.VAN_ALBADA, time_average=False)
        s.set_inflow_profile(prof)
        s.set_state(U0)
        s.synchronize()
        return s

    s = fresh()
    w0 = time.perf_counter()
    s.step(steps + 1)
    s.synchronize()
    fwd = time.perf_counter() - w0
    s.finalize()
    s = fresh()
    w0 = time.perf_counter()
    J, g = s.power_gradient(t0, steps, ckpt)
    s.synchronize()
    grad_s = time.perf_counter() - w0
    st = s.adjoint_stats()
    s.finalize()
    shutil.rmtree(tmp, ignore_errors=True)
    return {"workload": f"c5: {spec.n[0]}x{spec.n[1]}x{spec.n[2]} cells, 3 turbines, "
                        f"steps 0..{steps}, J = mean power over steps {t0}..{steps}, "
                        f"restart points every {ckpt} steps, van Albada",
            "forward_s": fwd, "gradient_s": grad_s, "gradient_over_forward": grad_s / fwd,
            "J": J, "grad_yaw_pitch_omega": g.tolist(), "adjoint_solves": st["solves"],
            "adjoint_iterations": st["iterations"], "max_rel_residual": st["max_rel_residual"],
            "recomputed_steps": st["recomputed_steps"], "how": "wall clock of the API calls"}


def run_ours(args):
    import numpy as np
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    pkg = importlib.import_module("3dalm_b200")
    tmp = tempfile.mkdtemp(prefix=f"dalm_bench_r{rank}_")
    spec, mesh, U0, prof = make_case(args.case, tmp)
    n_int = spec.n[0] * spec.n[1] * spec.n[2]

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def fresh_solver(profile, precision=pkg.FP64, inner=pkg.INNER_MULTIGRID):
        """A solver at the start of the timed steps: state set, warm-up run.
        A profiled solver polls the pressure solve after every iteration
        (no iteration is enqueued past convergence), so its per-kernel
        launch counts and bytes are exact."""
        sv = pkg.Solver(tmp, device=local, profile=profile, precision=precision,
                        mixed_inner=inner, poisson_batch=1 if profile else 0)
        sv.set_inflow_profile(prof)
        sv.set_state(U0)
        sv.step(max(args.warmup, 1))
        return sv

    def timed_region(precision, inner=pkg.INNER_MULTIGRID):
        """The K timed steps on the device (CUDA events on the solver's
        stream, no per-kernel instrumentation), max over ranks."""
        s = fresh_solver(False, precision, inner)
        stream = torch.cuda.ExternalStream(s.stream_handle(), device=local)
        s.timings(reset=True)
        clocks = ClockSampler(local)
        barrier()
        torch.cuda.synchronize()
        s.synchronize()
        clocks.start()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        its, errs = [], []
        for _ in range(args.steps):
            s.step(1)
            st = s.stats()
            its.append(st["it"])
            errs.append(st["err"])
        e1.record(stream)
        e1.synchronize()
        s.synchronize()
        clk = clocks.stop()
        ms = e0.elapsed_time(e1)
        _, launches = s.timings()
        ms = max_over_ranks(ms, world)
        final = {"U": s.field("U"), "p": s.field("p"), "turbines": s.turbines(),
                 "mesh": s.mesh(), "gc": s.gc}
        s.finalize()
        return ms, its, errs, clk, launches, final

    # ---- the reference's precision: the headline
    ms, its, errs, clk, launches, final64 = timed_region(pkg.FP64)
    value = whole_job_rate(n_int, args.steps, world, ms / 1e3)
    # ---- the mixed-precision form on the same steps
    mixed = None
    if not args.no_mixed:
        mms, mits, merrs, mclk, _, finalm = timed_region(pkg.MIXED)
        mvalue = whole_job_rate(n_int, args.steps, world, mms / 1e3)
        mixed = {"value": mvalue, "unit": METRIC, "ms_per_step": mms / args.steps,
                 "vs_fp64": mvalue / value, "poisson_iterations": mits,
                 "max_residual": max(merrs), "fp64_max_residual": max(errs),
                 "tolerance": spec.tol, "clocks": mclk,
                 "error_vs_fp64": mixed_errors(finalm, final64, final64["mesh"], final64["gc"]),
                 "how": "DALM_MIXED: FP64 iterative refinement (FP64 residual, norm, pressure "
                        "update and stop test) with capped FP32 inner passes of conjugate "
                        "gradients preconditioned by a geometric multigrid V-cycle; FP64 "
                        "fallback when a pass stalls. poisson_iterations counts inner CG "
                        "iterations (one V-cycle each), not comparable with BiCGStab's"}
        # the same form with the reference's Jacobi(3)-BiCGStab as the FP32
        # inner solver: what precision alone gains
        bms, bits, berrs, bclk, _, finalb = timed_region(pkg.MIXED, pkg.INNER_BICGSTAB)
        bvalue = whole_job_rate(n_int, args.steps, world, bms / 1e3)
        mixed["bicgstab_inner"] = {"value": bvalue, "vs_fp64": bvalue / value,
                                   "ms_per_step": bms / args.steps, "poisson_iterations": bits,
                                   "max_residual": max(berrs),
                                   "error_vs_fp64": mixed_errors(finalb, final64,
                                                                 final64["mesh"], final64["gc"])}

    # ---- end to end through the public API with host (pinned) buffers: a
    # second solver replays the same warm-up and the same timed steps, each
    # step fed from and returned to pinned host memory
    e2e_steps = args.steps if args.e2e_steps < 0 else min(args.e2e_steps, args.steps)
    e2e_value, h2d = None, 0
    if e2e_steps > 0:
        s = fresh_solver(False)
        U_h =torch.empty(s._shape(3), dtype=torch.float64).pin_memory().numpy()
        p_h = torch.empty(s._shape(1), dtype=torch.float64).pin_memory().numpy()
        s.field("U", out=U_h)
        s.field("p", out=p_h)
        barrier()
        torch.cuda.synchronize()
        s.synchronize()
        w0 = time.perf_counter()
        e2e_its = []
        for _ in range(e2e_steps):
            s.set_field("U", U_h)
            s.set_field("p", p_h)
            s.step(1)
            s.field("U", out=U_h)
            s.field("p", out=p_h)
            e2e_its.append(s.stats()["it"])
        s.synchronize()
        e2e_s = time.perf_counter() - w0
        if e2e_its != its[:e2e_steps]:
            raise RuntimeError(f"end-to-end replay took other iteration counts {e2e_its} "
                               f"than the timed region {its[:e2e_steps]}")
        e2e_s = max_over_ranks(e2e_s, world)
        e2e_value = whole_job_rate(n_int, e2e_steps, world, e2e_s)
        h2d = U_h.nbytes + p_h.nbytes
        s.finalize()

    # ---- per-kernel device times: a replay of the same steps with CUDA
    # events around every launch on the solver's stream
    def profiled_replay(precision, expect_its):
        sv = fresh_solver(True, precision)
        sv.timings(reset=True)
        p_its = []
        for _ in range(args.steps):
            sv.step(1)
            p_its.append(sv.stats()["it"])
        kt_ = sv.kernel_timings()
        st_ms, _ = sv.timings()
        if p_its != expect_its:
            raise RuntimeError(f"profiled replay took other iteration counts {p_its} than "
                               f"{expect_its}")
        return sv, kt_, st_ms

    peak, peak_kind = measured_peaks()

    def roofline(kt_, step_ms, traffic_of=None):
        """The kernel with the largest device time (algorithmic bytes per
        launch / mean launch time) and the whole step (all kernels' bytes
        per step / the unprofiled step time), against the measured peak."""
        dom_ = max((k for k in kt_ if kt_[k]["launches"] > 0 and kt_[k]["bytes_per_launch"] > 0),
                   key=lambda k: kt_[k]["ms"])
        d_ = kt_[dom_]
        pl = d_["ms"] / d_["launches"] / 1e3
        ach = d_["bytes_per_launch"] / pl / 1e9
        step_bytes = sum(v["launches"] * v["bytes_per_launch"] for v in kt_.values()) / args.steps
        step_ach = step_bytes / (step_ms / 1e3) / 1e9
        return {"bound": "hbm", "kernel": dom_, "achieved": ach, "peak": peak,
                "peak_source": f"{peak_kind} hbm_gbs", "unit": "GB/s", "frac": ach / peak,
                "traffic": traffic_of(dom_) if traffic_of else None,
                "algorithmic_bytes_per_launch": d_["bytes_per_launch"], "launch_us": pl * 1e6,
                "launches": d_["launches"],
                "share_of_kernel_time": d_["ms"] / max(1e-9, sum(v["ms"] for v in kt_.values())),
                "step": {"algorithmic_bytes": step_bytes, "ms": step_ms,
                         "achieved": step_ach, "frac": step_ach / peak},
                "kernels": {k: {"launches": v["launches"], "ms_per_step": v["ms"] / args.steps,
                                "achieved_gbs": (v["launches"] * v["bytes_per_launch"] /
                                                 (v["ms"] / 1e3) / 1e9) if v["ms"] > 0 else None}
                            for k, v in kt_.items() if v["launches"] > 0}}

    if mixed is not None:
        sm, mkt, _ = profiled_replay(pkg.MIXED, mixed["poisson_iterations"])
        sm.finalize()
        mixed["roofline"] = roofline(mkt, mixed["ms_per_step"])

    s, kt, stage_ms = profiled_replay(pkg.FP64, its)
    rl = roofline(kt, ms / args.steps, profiled_traffic)
    dom = rl["kernel"]
    n_launch = int(launches)  # launches in the unprofiled timed region

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded log-law + 8% Gaussian initial field, generated case files)",
        "config": workload_config(args.case, n_int, its, world),
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": h2d, "steps": e2e_steps,
                "how": "per step: dalm_set_field(U,p) from pinned host, dalm_step(1), "
                       "dalm_get_field(U,p) to pinned host, dalm_get_step_stats; wall clock"},
        "roofline": rl,
        "stage_ms_per_step": {k: v / args.steps for k, v in stage_ms.items()},
        "gpu_launches": n_launch,
        "mixed": mixed,
        "clocks": clk,
    }
    if world == 1 and not args.no_adjoint:
        line["adjoint"] = adjoint_cost(pkg, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline and os.path.exists(REF_MPIRUN):
        ranks = host_cores()
        v, kind, desc, secs = reference_sample(ranks, statistics.mean(its), args.case)
        line["cpu_baseline"] = {"value": v, "unit": METRIC, "cores": ranks, "kind": kind,
                                "sample": desc, "sample_seconds": secs}
    s.finalize()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def compare_forms(args):
    """The FP64 form (the reference's arithmetic and Jacobi(3)-BiCGStab) and
    DALM_MIXED (FP32 stencil fields, FP64 iterative refinement with
    multigrid-CG FP32 inner solves) from the same seeded initial state for the
    same steps: each turbine's power averaged over steps avg-from..STEPS in
    both forms and their relative difference (the running average of
    src/solver.h:1195-1204 applied to the loads of src/alm.h:384-398), the
    final relative L2 differences of u, v, w and p, each form's largest
    pressure residual and wall time.  The flow is chaotic: step-wise fields
    drift apart from the solver-tolerance level; averages are what the two
    forms must agree on."""
    import numpy as np
    import torch
    torch.cuda.set_device(0)
    pkg = importlib.import_module("3dalm_b200")
    tmp = tempfile.mkdtemp(prefix="dalm_compare_")
    spec, mesh, U0, prof = make_case(args.case, tmp)
    steps, avg_from = args.compare_forms, args.avg_from

    def run(precision):
        s = pkg.Solver(tmp, precision=precision, time_average=False)
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
                pw = s.turbines()[2]
                power = pw.copy() if power is None else power + pw
        s.synchronize()
        wall = time.perf_counter() - t
        out = {"power": power / (steps - avg_from + 1), "U": s.field("U"), "p": s.field("p"),
               "turbines": s.turbines(), "max_residual": worst, "seconds": wall,
               "iterations": its, "mesh": s.mesh(), "gc": s.gc}
        s.finalize()
        return out

    with quiet_stdout():
        f = run(pkg.FP64)
        m = run(pkg.MIXED)
    err = mixed_errors(m, f, f["mesh"], f["gc"])
    out = {"workload": workload_description(args.case), "case": args.case, "cells": list(spec.n), "steps": steps,
           "dt": spec.dt, "average_over": [avg_from, steps], "tolerance": spec.tol,
           "mean_power_fp64": f["power"].tolist(), "mean_power_mixed": m["power"].tolist(),
           "mean_power_rel_diff": (np.abs(m["power"] - f["power"]) / np.abs(f["power"])).tolist(),
           "final_rel_l2": err,
           "max_residual_fp64": f["max_residual"], "max_residual_mixed": m["max_residual"],
           "seconds_fp64": f["seconds"], "seconds_mixed": m["seconds"],
           "speedup": f["seconds"] / m["seconds"],
           "iterations_fp64_mean": float(np.mean(f["iterations"])),
           "iterations_mixed_mean": float(np.mean(m["iterations"])),
           "how": "wall time of each run including one host statistics call per step"}
    print(json.dumps(out), flush=True)
    shutil.rmtree(tmp, ignore_errors=True)


def main():
    args = parse()
    if args.compare_forms > 0:
        compare_forms(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
