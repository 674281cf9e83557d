"""ctypes front end to the two CPU oracles (TEST INFRASTRUCTURE ONLY).

  CRestatement  -> oracle/liboracle.so          (oracle/dalm_oracle.c, own code)
  Reference     -> oracle/_ref/libref3dalm.so   (the reference solver's own
                                                 headers, built by oracle/Makefile)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker / the timed CPU baseline.

Both expose the same interface, in the reference layout (AoS U[NX][NY][NZ][3],
k contiguous, guide cells included):
    set_state(U, JU=None, p=None, flags=...) ; step(n) ; stage(i)
    field(name) ; stats() ; turbines() ; points() ; ...

`load_case` parses the three case JSON files with the semantics of the
reference: build_mesh_from_json (src/io.h:98-164), Solver::initialize
(src/solver.h:564-708), build_wt_props (src/alm.h:144-206) and the
windturbine.json fields read by build_ap_props (src/alm.h:35-64).
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_C = os.path.join(HERE, "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libref3dalm.so")

FIELDS = {"U": (0, 3), "Uold": (1, 3), "JU": (2, 3), "p": (3, 1), "nut": (4, 1),
          "div": (5, 1), "f": (6, 3), "b": (7, 1), "Utavg": (8, 3)}
SET_APPLY_UBC = 1
SET_RECOMPUTE_JU = 2

EULER = {"roll": 0, "pitch": 1, "yaw": 2, "none": 3}
SOLVERS = {"SOR": 0, "BiCG": 1, "Jacobi": 2}
PCS = {"Jacobi": 0, "SOR": 1}

_PD = C.POINTER(C.c_double)
_PI64 = C.POINTER(C.c_int64)


def build(ref: bool = False) -> None:
    """Compile liboracle.so (and _ref when ref=True and the reference sources
    exist) with oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def reference_src() -> str:
    """The reference's source tree (its src/ directory): $DALM_REFERENCE_SRC,
    else oracle/Makefile's REFERENCE_SRC."""
    env = os.environ.get("DALM_REFERENCE_SRC")
    if env:
        return env
    r = subprocess.run(["make", "-s", "--no-print-directory", "-C", HERE, "print-reference-src"],
                       capture_output=True, text=True)
    return r.stdout.strip()


def reference_available() -> bool:
    return os.path.exists(LIB_REF)


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(_PD)


def _angle_slot(slots):
    """First non-zero or object angle slot -> (type, formula[4])
    (src/alm.h:167-204).  All-zero slots leave the type indeterminate in the
    reference; they are reported as 'none' here and rejected by the product."""
    for jj, a in enumerate(slots):
        if isinstance(a, dict) or (isinstance(a, (int, float)) and float(a) != 0.0):
            typ = ("roll", "pitch", "yaw")[jj]
            if isinstance(a, dict):
                f = [float(a["amp"]) * math.pi / 180, 2 * math.pi / float(a["T"]),
                     float(a["phase"]) * math.pi / 180, float(a["offset"]) * math.pi / 180]
            else:
                f = [0.0, 0.0, 0.0, float(a) * math.pi / 180]
            return typ, f
    return "none", [0.0, 0.0, 0.0, 0.0]


class Case:
    """Parsed case directory."""

    def __init__(self, case_dir: str):
        self.case_dir = case_dir
        with open(os.path.join(case_dir, "setup.json")) as f:
            s = json.load(f)
        with open(os.path.join(case_dir, "mesh.json")) as f:
            m = json.load(f)
        self.setup = s
        self.gc = int(m["guide cell"])
        self.x = np.asarray(m["x"], dtype=np.float64)
        self.y = np.asarray(m["y"], dtype=np.float64)
        self.z = np.asarray(m["z"], dtype=np.float64)
        self.size = (len(self.x), len(self.y), len(self.z))
        rt = s["runtime"]
        self.dt = float(rt["dt"])
        self.max_step = int(float(rt["time"]) / self.dt)   # (Int)(time/dt), src/solver.h:194
        self.tavg_start = float(s["output"]["time avg start time"])
        self.uin = [float(v) for v in s["inflow"]["value"]]
        self.re = float(s["cfd"]["Re"])
        self.cs = float(s["cfd"]["Cs"])
        eq = s["eq"]
        self.solver = eq["method"]
        self.tol = float(eq["tolerance"])
        self.max_it = int(float(eq["max iteration"]))
        self.relax = float(eq.get("relaxation rate", 1.0))
        pc = eq.get("preconditioner", {})
        self.pc = pc.get("method", "Jacobi")
        self.pc_max_it = int(pc.get("max iteration", 0))
        self.pc_relax = float(pc.get("relaxation rate", 1.0))
        # turbulence-generating grid and retracted floor (src/solver.h:599-625)
        self.grid = s.get("turbulence grid")
        self.floor_start = s.get("floor start")
        self.turbines = []
        self.wt = None
        if "windturbine array" in s:
            with open(os.path.join(case_dir, "windturbine.json")) as f:
                self.wt = json.load(f)
            alm = s["alm"]
            self.points_per_blade = int(alm["blade points"])
            self.projection_width = float(alm["projection width"])
            for t in s["windturbine array"]:
                typ, form = _angle_slot(t["angle"])
                self.turbines.append({"base": [float(v) for v in t["base"]], "type": typ,
                                      "formula": form, "omega": float(t["rotation speed"])})

    def params(self):
        """Build the oracle_params struct (kept alive by the returned holder)."""
        keep = []

        def arr(v, dt=np.float64):
            a = np.ascontiguousarray(np.asarray(v, dtype=dt))
            keep.append(a)
            return a

        P = OracleParams()
        P.size = (C.c_int64 * 3)(*self.size)
        P.gc = self.gc
        P.x, P.y, P.z = _ptr(arr(self.x)), _ptr(arr(self.y)), _ptr(arr(self.z))
        P.uin = (C.c_double * 3)(*self.uin)
        P.re, P.cs, P.dt = self.re, self.cs, self.dt
        P.max_step = self.max_step
        P.tavg_start_time = self.tavg_start
        P.solver = SOLVERS[self.solver]
        P.pc = PCS[self.pc]
        P.max_it, P.pc_max_it = self.max_it, self.pc_max_it
        P.tol, P.relax, P.pc_relax = self.tol, self.relax, self.pc_relax
        if self.grid is not None:
            P.has_grid = 1
            P.grid_bar = float(self.grid["bar"])
            P.grid_mesh = float(self.grid["mesh"])
            P.grid_thick = float(self.grid["thick"])
            P.grid_at = (C.c_double * 3)(*[float(v) for v in self.grid["placement"]])
        if self.floor_start is not None:
            P.retracted_floor = 1
            P.floor_start = float(self.floor_start)
        if self.turbines:
            wt = self.wt
            P.turbine_count = len(self.turbines)
            P.blades = int(wt["number of blades"])
            P.points_per_blade = self.points_per_blade
            P.projection_width = self.projection_width
            P.rotor_r, P.hub_r = float(wt["R"]), float(wt["hub R"])
            P.tower, P.overhang = float(wt["tower"]), float(wt["overhang"])
            P.base = _ptr(arr([t["base"] for t in self.turbines]))
            at = arr([EULER[t["type"]] for t in self.turbines], np.int32)
            P.angle_type = at.ctypes.data_as(C.POINTER(C.c_int))
            P.formula = _ptr(arr([t["formula"] for t in self.turbines]))
            P.rot_speed = _ptr(arr([t["omega"] for t in self.turbines]))
            foils = wt["blade"]["airfoil"]
            atk = wt["blade"]["attack angle"]
            P.station_count = len(foils)
            P.atk_count = len(atk)
            P.station_r = _ptr(arr([f["r/R"] for f in foils]))
            P.station_chord = _ptr(arr([f["chord/R"] for f in foils]))
            P.station_twist = _ptr(arr([f["twist[deg]"] for f in foils]))
            P.station_cd = _ptr(arr([f["Cd"] for f in foils]))
            P.station_cl = _ptr(arr([f["Cl"] for f in foils]))
            P.atk = _ptr(arr(atk))
        return P, keep


class OracleParams(C.Structure):
    _fields_ = [
        ("size", C.c_int64 * 3), ("gc", C.c_int64),
        ("x", _PD), ("y", _PD), ("z", _PD),
        ("uin", C.c_double * 3), ("re", C.c_double), ("cs", C.c_double), ("dt", C.c_double),
        ("max_step", C.c_int64), ("tavg_start_time", C.c_double),
        ("solver", C.c_int), ("pc", C.c_int),
        ("max_it", C.c_int64), ("pc_max_it", C.c_int64),
        ("tol", C.c_double), ("relax", C.c_double), ("pc_relax", C.c_double),
        ("turbine_count", C.c_int64), ("blades", C.c_int64), ("points_per_blade", C.c_int64),
        ("projection_width", C.c_double), ("rotor_r", C.c_double), ("hub_r", C.c_double),
        ("tower", C.c_double), ("overhang", C.c_double),
        ("base", _PD), ("angle_type", C.POINTER(C.c_int)), ("formula", _PD), ("rot_speed", _PD),
        ("station_count", C.c_int64), ("atk_count", C.c_int64),
        ("station_r", _PD), ("station_chord", _PD), ("station_twist", _PD),
        ("station_cd", _PD), ("station_cl", _PD), ("atk", _PD),
        ("has_grid", C.c_int), ("grid_bar", C.c_double), ("grid_mesh", C.c_double),
        ("grid_thick", C.c_double), ("grid_at", C.c_double * 3),
        ("retracted_floor", C.c_int), ("floor_start", C.c_double),
    ]


class _Base:
    """Common interface over the two oracle libraries."""

    prefix = ""

    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def _setup_common(self):
        self.size = self._size()
        self.nx, self.ny, self.nz, self.gc = self.size
        self.len = self.nx * self.ny * self.nz

    def _size(self):
        out = (C.c_int64 * 4)()
        self._fn("size")(self.h, out)
        return tuple(int(v) for v in out)

    def mesh(self):
        a = [np.zeros(n) for n in (self.nx, self.ny, self.nz, self.nx, self.ny, self.nz)]
        self._fn("mesh")(self.h, *[_ptr(v) for v in a])
        return a

    def max_diag(self):
        f = self._fn("max_diag")
        f.restype = C.c_double
        return f(self.h)

    def matrix(self):
        A = np.zeros((self.nx, self.ny, self.nz, 7))
        self._fn("matrix")(self.h, _ptr(A))
        return A

    def field(self, name):
        which, nc = FIELDS[name]
        shape = (self.nx, self.ny, self.nz) + ((3,) if nc == 3 else ())
        out = np.zeros(shape)
        self._fn("get_field")(self.h, which, _ptr(out))
        return out

    def set_field(self, name, val):
        which, nc = FIELDS[name]
        v = np.ascontiguousarray(val, dtype=np.float64)
        assert v.size == self.len * nc
        self._fn("set_field")(self.h, which, _ptr(v))

    def set_state(self, U, JU=None, p=None, flags=SET_APPLY_UBC | SET_RECOMPUTE_JU):
        U = np.ascontiguousarray(U, dtype=np.float64)
        JU = None if JU is None else np.ascontiguousarray(JU, dtype=np.float64)
        p = None if p is None else np.ascontiguousarray(p, dtype=np.float64)
        self._fn("set_state")(self.h, _ptr(U), _ptr(JU), _ptr(p), flags)

    def set_inflow_profile(self, prof):
        prof = None if prof is None else np.ascontiguousarray(prof, dtype=np.float64)
        self._fn("set_inflow_profile")(self.h, _ptr(prof))

    def set_turbine_params(self, yaw=None, pitch=None, omega=None):
        cv = [None if v is None else np.ascontiguousarray(v, dtype=np.float64)
              for v in (yaw, pitch, omega)]
        self._fn("set_turbine_params")(self.h, *[_ptr(v) for v in cv])

    def step(self, n=1):
        self._fn("step")(self.h, n)

    def stage(self, s):
        self._fn("stage")(self.h, s)

    def advance_clock(self):
        self._fn("advance_clock")(self.h)

    def set_poisson(self, max_it, tol):
        self._fn("set_poisson")(self.h, C.c_int64(max_it), C.c_double(tol))

    def stats(self):
        ints = (C.c_int64 * 4)()
        reals = (C.c_double * 4)()
        self._fn("stats")(self.h, ints, reals)
        return {"step": ints[0], "it": ints[1], "max_step": ints[2], "tavg_count": ints[3],
                "err": reals[0], "avg_div": reals[1], "max_cfl": reals[2], "dt": reals[3]}

    def turbine_count(self):
        return self._turbine_count

    def turbines(self):
        n = self._turbine_count
        tq, th = np.zeros(n), np.zeros(n)
        if n:
            self._fn("turbines")(self.h, _ptr(tq), _ptr(th))
        return tq, th

    def points(self):
        n = self._point_count
        xyz, f, tq, th = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n), np.zeros(n)
        if n:
            self._fn("points")(self.h, _ptr(xyz), _ptr(f), _ptr(tq), _ptr(th))
        return xyz, f, tq, th

    def point_tables(self):
        n, na = self._point_count, self._atk_count
        r, dr, ch, tw = (np.zeros(n) for _ in range(4))
        cd, cl, atk = np.zeros((n, na)), np.zeros((n, na)), np.zeros(na)
        if n:
            self._fn("point_tables")(self.h, *[_ptr(v) for v in (r, dr, ch, tw, cd, cl, atk)])
        return r, dr, ch, tw, cd, cl, atk


class CRestatement(_Base):
    """oracle/dalm_oracle.c through ctypes."""

    prefix = "oracle_"
    _lib = None

    def __init__(self, case_dir: str):
        if CRestatement._lib is None:
            if not os.path.exists(LIB_C):
                build()
            lib = C.CDLL(LIB_C)
            lib.oracle_create.restype = C.c_void_p
            lib.oracle_create.argtypes = [C.POINTER(OracleParams)]
            for n in ("destroy", "size", "mesh", "matrix", "set_inflow_profile",
                      "set_turbine_params", "set_state", "stage", "step", "advance_clock",
                      "get_field", "set_field", "stats", "set_poisson", "turbines", "points",
                      "point_tables", "max_diag", "set_sum_order"):
                getattr(lib, "oracle_" + n).argtypes = None
            CRestatement._lib = lib
        self.lib = CRestatement._lib
        self.case = Case(case_dir)
        P, keep = self.case.params()
        self.h = C.c_void_p(self.lib.oracle_create(C.byref(P)))
        self._setup_common()
        self._turbine_count = len(self.case.turbines)
        wt = self.case.wt
        self._point_count = (self._turbine_count * int(wt["number of blades"]) *
                             self.case.points_per_blade) if wt else 0
        self._atk_count = len(wt["blade"]["attack angle"]) if wt else 0

    def set_sum_order(self, mode: int):
        """Test-only: 1 sums dot products pairwise instead of serially."""
        self.lib.oracle_set_sum_order(self.h, int(mode))

    def set_limiter(self, limiter: int):
        """0: the reference's b=4 limiter; 1: the smooth van Albada limiter."""
        self.lib.oracle_set_limiter(self.h, int(limiter))

    def close(self):
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Reference(_Base):
    """The reference solver (compiled from its own sources) through ctypes."""

    prefix = "ref_"
    _lib = None

    def __init__(self, case_dir: str):
        if Reference._lib is None:
            Reference._lib = C.CDLL(LIB_REF)
            Reference._lib.ref_create.restype = C.c_void_p
            Reference._lib.ref_max_diag.restype = C.c_double
        self.lib = Reference._lib
        self.h = C.c_void_p(self.lib.ref_create(case_dir.encode()))
        self._setup_common()
        counts = (C.c_int64 * 5)()
        self.lib.ref_alm_counts(self.h, counts)
        self._point_count, self._turbine_count, self._atk_count = counts[0], counts[1], counts[2]

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
