"""Case generator: writes 3dalm case directories (setup.json, mesh.json,
windturbine.json) for the benchmark configurations, plus the seeded initial
velocity perturbation and the log-law inflow profile.

The files use the reference solver's own input formats:
  * mesh.json       {"guide cell", "x", "y", "z"} cell centres incl. guide
                    cells (read by build_mesh_from_json, src/io.h:98-164);
  * setup.json      keys read by Solver::initialize (src/solver.h:564-708);
  * windturbine.json  {"R", "hub R", "number of blades", "tower", "overhang",
                    "blade": {"airfoil": [...], "attack angle": [...]}}
                    (src/alm.h:35-64, 144-166).

Guide cells follow script/convertmesh.py:22-32: centres are node midpoints and
the guide cells are extrapolated with x[i] = 3x[i+1] - 3x[i+2] + x[i+3].

Two reference quirks shape the turbine file:
  * "r/R" and "chord/R" are used as dimensional r and chord (src/alm.h:52-54,
    72, 86), so dimensional values are written into those keys;
  * a turbine whose three angle slots are all numeric zero gets an
    indeterminate angle type (src/alm.h:150,168-204), so yaw 0 is written as
    {"amp":0,"T":1,"phase":0,"offset":0} in the yaw slot.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass, field

import numpy as np

KAPPA = 0.41  # von Karman constant of the log-law inflow

# ---------------------------------------------------------------- meshes


def _guide_cells(nodes: np.ndarray, gc: int = 2) -> np.ndarray:
    """Cell centres plus gc extrapolated guide cells per side
    (script/convertmesh.py:15-34)."""
    n = len(nodes) - 1
    c = np.zeros(n + 2 * gc)
    c[gc:gc + n] = 0.5 * (nodes[:-1] + nodes[1:])
    for i in range(gc - 1, -1, -1):
        c[i] = 3 * c[i + 1] - 3 * c[i + 2] + c[i + 3]
    for i in range(gc + n, n + 2 * gc):
        c[i] = 3 * c[i - 1] - 3 * c[i - 2] + c[i - 3]
    return c


def tanh_wall_nodes(n: int, length: float, max_ratio: float = 1.05):
    """n+1 nodes on [0, length] clustered toward 0 by
    z(eta) = L * (1 - tanh(beta (1 - eta)) / tanh(beta)); beta is found by
    bisection so that the largest adjacent-cell ratio equals max_ratio."""
    eta = np.linspace(0.0, 1.0, n + 1)

    def nodes(beta):
        return length * (1.0 - np.tanh(beta * (1.0 - eta)) / np.tanh(beta))

    def ratio(beta):
        d = np.diff(nodes(beta))
        return float(np.max(d[1:] / d[:-1]))

    lo, hi = 1e-6, 20.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if ratio(mid) > max_ratio:
            hi = mid
        else:
            lo = mid
    beta = lo
    z = nodes(beta)
    z[0], z[-1] = 0.0, length
    return z, beta


@dataclass
class Mesh:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    gc: int = 2
    beta: float = 0.0

    @property
    def size(self):
        return (len(self.x), len(self.y), len(self.z))


def make_mesh(nx, ny, nz, lx=20.0, ly=5.0, lz=5.0, max_ratio=1.05, gc=2) -> Mesh:
    """Uniform in x and y, tanh-stretched toward the z=0 wall in z."""
    xn = np.linspace(0.0, lx, nx + 1)
    yn = np.linspace(0.0, ly, ny + 1)
    zn, beta = tanh_wall_nodes(nz, lz, max_ratio)
    return Mesh(_guide_cells(xn, gc), _guide_cells(yn, gc), _guide_cells(zn, gc), gc, beta)


def spacing(c: np.ndarray) -> np.ndarray:
    """dx[i] = (x[i+1]-x[i-1])/2 with one-sided ends (src/io.h:112-125)."""
    d = np.empty_like(c)
    d[1:-1] = 0.5 * (c[2:] - c[:-2])
    d[0] = -1.5 * c[0] + 2.0 * c[1] - 0.5 * c[2]
    d[-1] = 1.5 * c[-1] - 2.0 * c[-2] + 0.5 * c[-3]
    return d


# ---------------------------------------------------------------- PRNG


_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(seed: int, n: int) -> np.ndarray:
    """n outputs of splitmix64 (Steele, Lea, Flood 2014) started at `seed`."""
    with np.errstate(over="ignore"):
        k = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed) + k * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def gaussian(seed: int, n: int) -> np.ndarray:
    """n standard normal FP64 deviates: splitmix64 -> 53-bit uniforms ->
    Box-Muller (both outputs of each pair used)."""
    m = (n + 1) // 2
    bits = splitmix64(seed, 2 * m)
    u = (bits >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    u1 = 1.0 - u[0::2]  # (0, 1]
    u2 = u[1::2]
    rad = np.sqrt(-2.0 * np.log(u1))
    z = np.empty(2 * m)
    z[0::2] = rad * np.cos(2.0 * math.pi * u2)
    z[1::2] = rad * np.sin(2.0 * math.pi * u2)
    return z[:n]


# ---------------------------------------------------------------- turbines


@dataclass
class Turbine:
    base: tuple
    yaw_deg: float = 0.0
    omega: float = 12.0


@dataclass
class CaseSpec:
    name: str
    n: tuple                       # interior cells (nx, ny, nz)
    lengths: tuple = (20.0, 5.0, 5.0)
    dt: float = 1e-3
    steps: int = 10
    re: float = 1e4
    cs: float = 0.1
    uin: tuple = (1.0, 0.0, 0.0)
    solver: str = "SOR"            # "SOR" | "BiCG" | "Jacobi"
    pc: str = "Jacobi"             # BiCG preconditioner: "Jacobi" | "SOR"
    tol: float = 1e-6
    max_it: int = 1000
    relax: float = 1.2
    pc_max_it: int = 3
    pc_relax: float = 1.2
    turbines: list = field(default_factory=list)
    points_per_blade: int = 32
    rotor_r: float = 0.5
    hub_r: float = 0.0
    tower: float = 1.5
    overhang: float = 0.0
    blades: int = 3
    intensity: float = 0.05
    seed: int = 0
    loglaw: tuple | None = None     # (u_star, z0)
    tavg_start_time: float = 1e30
    output_start_time: float = 1e30
    output_interval_time: float = 1e30
    polar_step_deg: float = 0.5
    # turbulence-generating grid {"bar", "mesh", "thick", "placement"}, the
    # retracted floor's start x, probe points (the reference's own cases)
    grid: dict | None = None
    floor_start: float | None = None
    probes: list = field(default_factory=list)


def polar_tables(step_deg=0.5):
    """Synthetic polar: Cl = 2 pi clip(alpha, +-15 deg), Cd = 0.01 + 0.02 alpha^2
    (alpha in rad), tabulated every step_deg over [-180, 180] deg."""
    n = int(round(360.0 / step_deg)) + 1
    atk = np.linspace(-180.0, 180.0, n)
    a = np.deg2rad(atk)
    cl = 2.0 * math.pi * np.clip(a, -math.radians(15.0), math.radians(15.0))
    cd = 0.01 + 0.02 * a * a
    return atk, cd, cl


def windturbine_json(spec: CaseSpec, stations: int = 6) -> dict:
    atk, cd, cl = polar_tables(spec.polar_step_deg)
    foils = []
    for s in range(stations):
        frac = s / (stations - 1)
        r = spec.hub_r + frac * (spec.rotor_r - spec.hub_r)
        foils.append({
            "r/R": r,                                   # dimensional (quirk)
            "chord/R": 0.08 + frac * (0.03 - 0.08),     # dimensional (quirk)
            "twist[deg]": 20.0 + frac * (2.0 - 20.0),
            "Cl": cl.tolist(),
            "Cd": cd.tolist(),
        })
    return {
        "R": spec.rotor_r,
        "hub R": spec.hub_r,
        "number of blades": spec.blades,
        "tower": spec.tower,
        "overhang": spec.overhang,
        "blade": {"airfoil": foils, "attack angle": atk.tolist()},
    }


def projection_width(mesh: Mesh, spec: CaseSpec) -> float:
    """epsilon = 2 * min(dx, dy, dz) at the cell holding the first hub."""
    if not spec.turbines:
        return 0.0
    hub = (spec.turbines[0].base[0] - spec.overhang, spec.turbines[0].base[1],
           spec.turbines[0].base[2] + spec.tower)
    widths = []
    for c, h in zip((mesh.x, mesh.y, mesh.z), hub):
        d = spacing(c)
        i = int(np.clip(np.searchsorted(c, h) - 1, mesh.gc, len(c) - mesh.gc - 1))
        widths.append(d[i])
    return 2.0 * float(min(widths))


def setup_json(spec: CaseSpec, mesh: Mesh) -> dict:
    eq = {"tolerance": spec.tol, "max iteration": spec.max_it, "method": spec.solver}
    if spec.solver == "SOR":
        eq["relaxation rate"] = spec.relax
    if spec.solver == "BiCG":
        pc = {"method": spec.pc, "max iteration": spec.pc_max_it}
        if spec.pc == "SOR":
            pc["relaxation rate"] = spec.pc_relax
        eq["preconditioner"] = pc
    js = {
        "runtime": {"dt": spec.dt, "time": spec.steps * spec.dt},
        "output": {"output start time": spec.output_start_time,
                   "output interval time": spec.output_interval_time,
                   "time avg start time": spec.tavg_start_time},
        "inflow": {"value": list(spec.uin)},
        "cfd": {"Re": spec.re, "Cs": spec.cs},
        "eq": eq,
    }
    if spec.grid is not None:
        js["turbulence grid"] = dict(spec.grid)
    if spec.floor_start is not None:
        js["floor start"] = spec.floor_start
    if spec.probes:
        js["probe"] = [list(p) for p in spec.probes]
    if spec.turbines:
        arr = []
        for t in spec.turbines:
            yaw = t.yaw_deg if t.yaw_deg != 0 else {"amp": 0, "T": 1, "phase": 0, "offset": 0}
            arr.append({"base": list(t.base), "angle": [0, 0, yaw], "rotation speed": t.omega})
        js["windturbine array"] = arr
        js["alm"] = {"blade points": spec.points_per_blade,
                     "projection width": projection_width(mesh, spec)}
    return js


def write_case(spec: CaseSpec, case_dir: str) -> Mesh:
    """Write the three JSON files; returns the mesh."""
    os.makedirs(case_dir, exist_ok=True)
    mesh = make_mesh(*spec.n, *spec.lengths)
    with open(os.path.join(case_dir, "mesh.json"), "w") as f:
        json.dump({"guide cell": mesh.gc, "x": mesh.x.tolist(), "y": mesh.y.tolist(),
                   "z": mesh.z.tolist()}, f)
    with open(os.path.join(case_dir, "setup.json"), "w") as f:
        json.dump(setup_json(spec, mesh), f, indent=1)
    if spec.turbines:
        with open(os.path.join(case_dir, "windturbine.json"), "w") as f:
            json.dump(windturbine_json(spec), f)
    return mesh


def inflow_profile(spec: CaseSpec, mesh: Mesh):
    """[NY][NZ][3] inflow ghost values: log-law u = (u*/kappa) ln(z/z0) when
    spec.loglaw is set, else None (uniform Uin)."""
    if spec.loglaw is None:
        return None
    ustar, z0 = spec.loglaw
    ny, nz = len(mesh.y), len(mesh.z)
    prof = np.zeros((ny, nz, 3))
    zc = np.maximum(mesh.z, z0 * 1.0000001)
    u = (ustar / KAPPA) * np.log(zc / z0)
    prof[:, :, 0] = u[None, :]
    return prof


def initial_velocity(spec: CaseSpec, mesh: Mesh) -> np.ndarray:
    """U[NX][NY][NZ][3] (reference AoS layout, guide cells included): the mean
    inflow (uniform Uin or the log-law profile) everywhere, plus N(0, (I*U)^2)
    per component on interior cells with U = |Uin|, from gaussian(seed)."""
    nx, ny, nz = mesh.size
    gc = mesh.gc
    U = np.empty((nx, ny, nz, 3))
    prof = inflow_profile(spec, mesh)
    if prof is None:
        U[...] = np.asarray(spec.uin)
    else:
        U[...] = prof[None, :, :, :]
    if spec.intensity > 0:
        ni = (nx - 2 * gc) * (ny - 2 * gc) * (nz - 2 * gc) * 3
        scale = spec.intensity * float(np.linalg.norm(spec.uin))
        noise = gaussian(spec.seed, ni).reshape(nx - 2 * gc, ny - 2 * gc, nz - 2 * gc, 3)
        U[gc:nx - gc, gc:ny - gc, gc:nz - gc, :] += scale * noise
    return U


# ---------------------------------------------------------------- configs


def _row(x, yaws=(0.0,)):
    return [Turbine(base=(xx, 2.5, 0.0), yaw_deg=yy, omega=12.0) for xx, yy in zip(x, yaws)]


def config(name: str, **over) -> CaseSpec:
    """The benchmark configurations (plus reduced 'tiny' variants for tests).

    c1  128x64x64,  no turbine, RB-SOR w=1.2 tol 1e-6, 5% perturbation
    c2  256x128x128, 1 turbine at x=4, Jacobi(3)-BiCGStab tol 1e-8
    c3  384x192x160, c2 turbine (mixed-precision case)
    c4  512x256x128, 3 turbines at x=4,9,14 yaw 0/10/0, log-law + 8%
    c5  256x128x64,  c4 turbines (adjoint case; polar tabulated every 0.05 deg)
    """
    base = dict(
        c1=CaseSpec("c1", (128, 64, 64), solver="SOR", tol=1e-6, max_it=1000, relax=1.2,
                    steps=100, intensity=0.05),
        c2=CaseSpec("c2", (256, 128, 128), solver="BiCG", pc="Jacobi", pc_max_it=3, tol=1e-8,
                    max_it=10000, steps=500, turbines=_row([4.0]), intensity=0.05),
        c3=CaseSpec("c3", (384, 192, 160), solver="BiCG", pc="Jacobi", pc_max_it=3, tol=1e-8,
                    max_it=10000, steps=500, turbines=_row([4.0]), intensity=0.05),
        c4=CaseSpec("c4", (512, 256, 128), solver="BiCG", pc="Jacobi", pc_max_it=3, tol=1e-8,
                    max_it=20000, steps=2000, turbines=_row([4.0, 9.0, 14.0], (0.0, 10.0, 0.0)),
                    intensity=0.08, loglaw=(0.05, 1e-3)),
        c5=CaseSpec("c5", (256, 128, 64), solver="BiCG", pc="Jacobi", pc_max_it=3, tol=1e-8,
                    max_it=10000, steps=200, turbines=_row([4.0, 9.0, 14.0], (0.0, 10.0, 0.0)),
                    intensity=0.08, loglaw=(0.05, 1e-3), polar_step_deg=0.05),
    )
    if name.startswith("tiny"):
        # tiny-sor / tiny-bicg / tiny-turbine / tiny-loglaw: small grids for tests
        spec = CaseSpec(name, (24, 12, 12), steps=10, solver="SOR", tol=1e-6, max_it=200,
                        relax=1.2, intensity=0.05)
        if "bicg" in name or "turbine" in name or "loglaw" in name:
            spec.solver, spec.pc, spec.pc_max_it, spec.tol, spec.max_it = "BiCG", "Jacobi", 3, 1e-8, 2000
        if "turbine" in name or "loglaw" in name:
            spec.n = (40, 20, 20)
            spec.turbines = _row([4.0])
            spec.points_per_blade = 8
        if "loglaw" in name:
            spec.turbines = _row([4.0, 9.0], (0.0, 10.0))
            spec.loglaw = (0.05, 1e-3)
            spec.intensity = 0.08
        if "sorpc" in name:
            spec.solver, spec.pc, spec.pc_relax = "BiCG", "SOR", 1.2
        if "jacobi" in name:
            spec.solver = "Jacobi"
        if "tgg" in name:
            # a turbulence-generating grid one cell thick at x = 4, a slip
            # floor upstream of x = 3, and probes (the last one outside)
            spec.n = (40, 20, 20)
            spec.grid = {"bar": 0.3, "mesh": 1.0, "thick": 0.5, "placement": [4.0, 2.5, 1.5]}
            spec.floor_start = 3.0
            spec.probes = [[5.0, 2.5, 1.0], [7.3, 1.1, 0.4], [12.0, 3.9, 4.6], [30.0, 2.5, 1.0]]
    else:
        spec = base[name]
    for k, v in over.items():
        setattr(spec, k, v)
    return spec


STATE_FILE = "initial_U.f64"       # U[NX][NY][NZ][3] float64, guide cells included
PROFILE_FILE = "inflow_profile.f64"  # [NY][NZ][3] float64 inflow ghost values


def write_state_files(spec: CaseSpec, mesh: Mesh, case_dir: str) -> None:
    """Raw little-endian float64 files the `dalm` command-line driver loads
    when present: the seeded initial velocity and, for log-law cases, the
    inflow profile."""
    initial_velocity(spec, mesh).astype("<f8").tofile(os.path.join(case_dir, STATE_FILE))
    prof = inflow_profile(spec, mesh)
    if prof is not None:
        prof.astype("<f8").tofile(os.path.join(case_dir, PROFILE_FILE))


def main(argv=None):
    import argparse

    ap = argparse.ArgumentParser(description="write a 3dalm case directory")
    ap.add_argument("config", help="c1..c5 or tiny-*")
    ap.add_argument("case_dir")
    ap.add_argument("--n", type=int, nargs=3, help="interior cells nx ny nz")
    ap.add_argument("--steps", type=int, help="runtime.time = steps * dt")
    ap.add_argument("--max-it", type=int, help="eq.\"max iteration\"")
    ap.add_argument("--tol", type=float, help="eq.\"tolerance\"")
    ap.add_argument("--seed", type=int)
    ap.add_argument("--dt", type=float, help="time step (default: the configuration's)")
    ap.add_argument("--no-state", action="store_true", help="skip the initial-state files")
    a = ap.parse_args(argv)
    over = {}
    if a.n:
        over["n"] = tuple(a.n)
    for key, val in (("steps", a.steps), ("max_it", a.max_it), ("tol", a.tol), ("seed", a.seed),
                     ("dt", a.dt)):
        if val is not None:
            over[key] = val
    spec = config(a.config, **over)
    mesh = write_case(spec, a.case_dir)
    if not a.no_state:
        write_state_files(spec, mesh, a.case_dir)
    print(a.case_dir)


if __name__ == "__main__":
    main()
