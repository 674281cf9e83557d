"""B200-native 3dalm time-step hot path — Python host interface.

`Solver` mirrors the reference's driver object (struct Solver,
src/solver.h:519-1311): `initialize(case_dir)` ~ Solver::initialize,
`main_loop_once()` ~ Solver::main_loop_once, `can_continue()`,
`finalize()`, plus field access in the reference layout (AoS [NX][NY][NZ][3]
velocity, k contiguous, guide cells included).  Every call goes through the
C ABI in include/dalm.h implemented by the in-tree libdalm.so (CUDA, sm_100a).
There is no CPU fallback: if the library cannot be loaded, or no GPU is
present, the constructor raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdalm.so")

DALM_OK = 0
ERRORS = {1: "DALM_ERR_ARG", 2: "DALM_ERR_CASE", 3: "DALM_ERR_CUDA", 4: "DALM_ERR_NONFINITE",
          5: "DALM_ERR_DEVICE_WAIT", 6: "DALM_ERR_UNSUPPORTED"}
FP64, MIXED = 0, 1
MINMOD, VAN_ALBADA = 0, 1
INNER_MULTIGRID, INNER_BICGSTAB = 0, 1
FIELDS = {"U": (0, 3), "Uold": (1, 3), "JU": (2, 3), "p": (3, 1), "nut": (4, 1),
          "div": (5, 1), "f": (6, 3), "b": (7, 1), "Utavg": (8, 3)}
STAGES = {"predict": 0, "flux_rhs": 1, "poisson": 2, "project": 3, "alm": 4, "diag": 5,
          "tavg": 6}
SET_APPLY_UBC = 1
SET_RECOMPUTE_JU = 2

# Every entry point of include/dalm.h (checked by tests/test_abi.py).
EXPORTS = (
    "dalm_default_options", "dalm_create", "dalm_destroy", "dalm_last_error", "dalm_get_size",
    "dalm_get_mesh", "dalm_get_runtime", "dalm_get_max_diag", "dalm_set_state",
    "dalm_get_field", "dalm_set_field", "dalm_set_inflow_profile", "dalm_set_turbine_params",
    "dalm_step", "dalm_run_stage", "dalm_advance_clock", "dalm_get_step_stats",
    "dalm_set_poisson", "dalm_get_counts", "dalm_get_turbines", "dalm_get_points",
    "dalm_synchronize", "dalm_get_stream", "dalm_get_timings", "dalm_kernel_kinds",
    "dalm_get_kernel_timing", "dalm_diagnostics_noalloc", "dalm_get_turbine_params",
    "dalm_adjoint_power_grad", "dalm_get_adjoint_stats",
)


class DalmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("limiter", C.c_int), ("device", C.c_int),
                ("time_average", C.c_int), ("check_finite", C.c_int),
                ("poisson_batch", C.c_int), ("use_graphs", C.c_int), ("profile", C.c_int),
                ("reference_sums", C.c_int), ("fused_krylov", C.c_int),
                ("refine_inner_it", C.c_int), ("write_output", C.c_int),
                ("mixed_inner", C.c_int), ("fused_jacobi", C.c_int), ("reserved", C.c_int * 2)]


_PD = C.POINTER(C.c_double)
_lib = None


def load_library(path: str = LIB_PATH):
    """Load libdalm.so (raises OSError when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise OSError(f"{path} not found: build it with `make -C 3dalm_b200/csrc` "
                          "(or __graft_entry__.build())")
        lib = C.CDLL(path)
        lib.dalm_last_error.restype = C.c_char_p
        lib.dalm_last_error.argtypes = [C.c_void_p]
        lib.dalm_create.argtypes = [C.c_char_p, C.POINTER(Options), C.POINTER(C.c_void_p)]
        lib.dalm_destroy.argtypes = [C.c_void_p]
        lib.dalm_kernel_kinds.restype = C.c_int
        lib.dalm_get_kernel_timing.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_char_p),
                                               C.POINTER(C.c_int64), _PD, _PD]
        _lib = lib
    return _lib


def build():
    """Compile libdalm.so in-tree with the Makefile in csrc/."""
    import subprocess
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "csrc")], check=True)


def _p(a):
    return None if a is None else a.ctypes.data_as(_PD)


class Solver:
    """One case on one GPU (a dalm_handle)."""

    def __init__(self, case_dir: str | None = None, precision: int = FP64, device: int = 0,
                 time_average: bool = True, profile: bool = False, poisson_batch: int = 0,
                 limiter: int = MINMOD, reference_sums: bool = False, fused_krylov: bool = False,
                 refine_inner_it: int = 0, write_output: bool = False,
                 mixed_inner: int = INNER_MULTIGRID, fused_jacobi: bool = False):
        self.lib = load_library()
        self.h = C.c_void_p()
        self.opt = Options()
        self.lib.dalm_default_options(C.byref(self.opt))
        self.opt.precision = precision
        self.opt.limiter = limiter
        self.opt.device = device
        self.opt.time_average = int(time_average)
        self.opt.profile = int(profile)
        self.opt.poisson_batch = poisson_batch
        self.opt.reference_sums = int(reference_sums)
        self.opt.fused_krylov = int(fused_krylov)
        self.opt.refine_inner_it = int(refine_inner_it)
        self.opt.write_output = int(write_output)
        self.opt.mixed_inner = int(mixed_inner)
        self.opt.fused_jacobi = int(fused_jacobi)
        if case_dir is not None:
            self.initialize(case_dir)

    # ---- lifecycle (Solver::initialize / finalize) ----
    def initialize(self, case_dir: str):
        rc = self.lib.dalm_create(case_dir.encode(), C.byref(self.opt), C.byref(self.h))
        if rc != DALM_OK:
            raise DalmError(rc, self.lib.dalm_last_error(None).decode())
        sz = (C.c_int64 * 3)()
        gc = C.c_int64()
        self._check(self.lib.dalm_get_size(self.h, sz, C.byref(gc)))
        self.size = tuple(int(v) for v in sz)
        self.gc = int(gc.value)
        dt = C.c_double()
        ms = C.c_int64()
        self._check(self.lib.dalm_get_runtime(self.h, C.byref(dt), C.byref(ms)))
        self.dt, self.max_step = float(dt.value), int(ms.value)
        cnt = (C.c_int64 * 5)()
        self._check(self.lib.dalm_get_counts(self.h, cnt))
        self.turbine_count, self.point_count = int(cnt[0]), int(cnt[1])
        return self

    def finalize(self):
        if self.h:
            self.lib.dalm_destroy(self.h)
            self.h = C.c_void_p()

    close = finalize

    def __del__(self):
        try:
            self.finalize()
        except Exception:
            pass

    def _check(self, rc):
        if rc != DALM_OK:
            raise DalmError(rc, self.lib.dalm_last_error(self.h).decode())

    # ---- time stepping ----
    def main_loop_once(self):
        self._check(self.lib.dalm_step(self.h, 1))

    def step(self, n: int = 1):
        self._check(self.lib.dalm_step(self.h, int(n)))

    def stage(self, s):
        self._check(self.lib.dalm_run_stage(self.h, STAGES[s] if isinstance(s, str) else int(s)))

    def advance_clock(self):
        self._check(self.lib.dalm_advance_clock(self.h))

    def can_continue(self) -> bool:
        return self.stats()["step"] <= self.max_step

    def synchronize(self):
        self._check(self.lib.dalm_synchronize(self.h))

    def stream_handle(self) -> int:
        """The solver's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        v = C.c_void_p()
        self._check(self.lib.dalm_get_stream(self.h, C.byref(v)))
        return int(v.value or 0)

    # ---- state ----
    def _shape(self, nc):
        nx, ny, nz = self.size
        return (nx, ny, nz, 3) if nc == 3 else (nx, ny, nz)

    def field(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        """Copy a reference-layout array to the host (into `out` when given,
        e.g. a pinned buffer; it must be C-contiguous float64)."""
        which, nc = FIELDS[name]
        if out is None:
            out = np.empty(self._shape(nc))
        elif out.dtype != np.float64 or not out.flags.c_contiguous or out.size != np.prod(
                self._shape(nc)):
            raise ValueError("out must be a C-contiguous float64 array of the field's size")
        self._check(self.lib.dalm_get_field(self.h, which, _p(out)))
        return out

    def set_field(self, name: str, value):
        which, nc = FIELDS[name]
        v = np.ascontiguousarray(value, dtype=np.float64).reshape(self._shape(nc))
        self._check(self.lib.dalm_set_field(self.h, which, _p(v)))

    def set_state(self, U, JU=None, p=None, flags=SET_APPLY_UBC | SET_RECOMPUTE_JU):
        U = np.ascontiguousarray(U, dtype=np.float64)
        JU = None if JU is None else np.ascontiguousarray(JU, dtype=np.float64)
        p = None if p is None else np.ascontiguousarray(p, dtype=np.float64)
        self._check(self.lib.dalm_set_state(self.h, _p(U), _p(JU), _p(p), int(flags)))

    def set_inflow_profile(self, prof):
        prof = None if prof is None else np.ascontiguousarray(prof, dtype=np.float64)
        self._check(self.lib.dalm_set_inflow_profile(self.h, _p(prof)))

    def set_turbine_params(self, yaw=None, pitch=None, omega=None):
        cv = [None if v is None else np.ascontiguousarray(v, dtype=np.float64)
              for v in (yaw, pitch, omega)]
        self._check(self.lib.dalm_set_turbine_params(self.h, *[_p(v) for v in cv]))

    def turbine_params(self):
        """(yaw_deg, pitch_deg, omega) per turbine."""
        n = self.turbine_count
        yaw, pitch, om = np.zeros(n), np.zeros(n), np.zeros(n)
        if n:
            self._check(self.lib.dalm_get_turbine_params(self.h, _p(yaw), _p(pitch), _p(om)))
        return yaw, pitch, om

    def power_gradient(self, t0: int, t1: int, ckpt_every: int = 20):
        """Discrete adjoint (dalm_adjoint_power_grad): runs the steps through
        t1 and returns (J, grad) with J the mean total power over steps
        t0..t1 and grad[w] = dJ/d(yaw_deg, pitch_deg, omega) of turbine w."""
        n = self.turbine_count
        grad = np.zeros(3 * max(n, 1))
        J = C.c_double()
        self._check(self.lib.dalm_adjoint_power_grad(self.h, int(t0), int(t1), int(ckpt_every),
                                                      _p(grad), C.byref(J)))
        return float(J.value), grad[:3 * n].reshape(n, 3)

    def adjoint_stats(self) -> dict:
        solves, its, rec = C.c_int64(), C.c_int64(), C.c_int64()
        res = C.c_double()
        self._check(self.lib.dalm_get_adjoint_stats(self.h, C.byref(solves), C.byref(its),
                                                     C.byref(res), C.byref(rec)))
        return {"solves": solves.value, "iterations": its.value,
                "max_rel_residual": res.value, "recomputed_steps": rec.value}

    def set_poisson(self, max_it: int, tol: float):
        self._check(self.lib.dalm_set_poisson(self.h, C.c_int64(max_it), C.c_double(tol)))

    # ---- outputs ----
    def mesh(self):
        a = [np.empty(n) for n in (self.size[0], self.size[1], self.size[2]) * 2]
        self._check(self.lib.dalm_get_mesh(self.h, *[_p(v) for v in a]))
        return a

    def max_diag(self) -> float:
        v = C.c_double()
        self._check(self.lib.dalm_get_max_diag(self.h, C.byref(v)))
        return float(v.value)

    def stats(self) -> dict:
        step, it = C.c_int64(), C.c_int64()
        err, div, cfl = C.c_double(), C.c_double(), C.c_double()
        self._check(self.lib.dalm_get_step_stats(self.h, C.byref(step), C.byref(it),
                                                 C.byref(err), C.byref(div), C.byref(cfl)))
        return {"step": step.value, "it": it.value, "err": err.value, "avg_div": div.value,
                "max_cfl": cfl.value}

    def turbines(self):
        n = self.turbine_count
        th, tq, pw = np.zeros(n), np.zeros(n), np.zeros(n)
        if n:
            self._check(self.lib.dalm_get_turbines(self.h, _p(th), _p(tq), _p(pw)))
        return th, tq, pw

    def points(self):
        n = self.point_count
        xyz, f, tq, th = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n), np.zeros(n)
        if n:
            self._check(self.lib.dalm_get_points(self.h, _p(xyz), _p(f), _p(tq), _p(th)))
        return xyz, f, tq, th

    def timings(self, reset=False):
        ms = (C.c_double * 7)()
        launches = C.c_int64()
        self._check(self.lib.dalm_get_timings(self.h, ms, C.byref(launches), int(reset)))
        return {k: ms[v] for k, v in STAGES.items()}, int(launches.value)

    def kernel_timings(self):
        out = {}
        for i in range(self.lib.dalm_kernel_kinds()):
            name = C.c_char_p()
            n = C.c_int64()
            ms = C.c_double()
            by = C.c_double()
            self._check(self.lib.dalm_get_kernel_timing(self.h, i, C.byref(name), C.byref(n),
                                                        C.byref(ms), C.byref(by)))
            out[name.value.decode()] = {"launches": int(n.value), "ms": float(ms.value),
                                        "bytes_per_launch": float(by.value)}
        return out
