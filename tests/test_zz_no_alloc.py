"""dalm_diagnostics_noalloc: the allocation-free entry point for callers
that cannot let a library allocate device memory (an OpenACC program that
owns U and JU in its own data region, a caller whose pool owns the device,
code that must not allocate mid-step).  Called through the C ABI on device
arrays in the reference layout, twice in a row, it must give the same
divergence norm and CFL number as the handle-based path (dalm_set_state +
dalm_get_step_stats), within the tolerance used for reductions elsewhere:
1e-12 relative for the summed norm (different summation tree), exact for
the maximum.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from conftest import package

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_diagnostics_match_handle_path(make_case):
    import torch

    pkg = package()
    lib = pkg.load_library()
    lib.dalm_diagnostics_noalloc.argtypes = [C.c_void_p] * 5 + [
        C.POINTER(C.c_int64), C.c_int64, C.c_double, C.c_void_p, C.c_void_p]
    spec, mesh, d, U0, prof = make_case("tiny-turbine")
    s = pkg.Solver(d)
    s.set_state(U0)
    dev = torch.device("cuda", 0)
    x, y, z, dx, dy, dz = s.mesh()
    tdx, tdy, tdz = (torch.from_numpy(a).to(dev) for a in (dx, dy, dz))
    size = (C.c_int64 * 3)(*s.size)
    out = torch.zeros(2, dtype=torch.float64, device=dev)
    for call in range(2):
        want = s.stats()
        tU = torch.from_numpy(s.field("U")).to(dev)
        tJU = torch.from_numpy(s.field("JU")).to(dev)
        out.fill_(-1.0)
        torch.cuda.synchronize()
        rc = lib.dalm_diagnostics_noalloc(_ptr(tU), _ptr(tJU), _ptr(tdx), _ptr(tdy), _ptr(tdz),
                                          size, s.gc, s.dt, _ptr(out), None)
        assert rc == 0, lib.dalm_last_error(None)
        torch.cuda.synchronize()
        avg_div, max_cfl = out.cpu().tolist()
        assert max_cfl == want["max_cfl"], (call, max_cfl, want)
        assert abs(avg_div - want["avg_div"]) <= 1e-12 * want["avg_div"], (call, avg_div, want)
        s.step(2)  # a different state for the second call
    s.finalize()


def test_noalloc_rejects_grids_beyond_its_scratch():
    pkg = package()
    lib = pkg.load_library()
    lib.dalm_diagnostics_noalloc.argtypes = [C.c_void_p] * 5 + [
        C.POINTER(C.c_int64), C.c_int64, C.c_double, C.c_void_p, C.c_void_p]
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    size = (C.c_int64 * 3)(2052, 1028, 516)  # 2048 x 1024 x 512 interior cells
    rc = lib.dalm_diagnostics_noalloc(dummy, dummy, dummy, dummy, dummy, size, 2, 1e-3, dummy,
                                      None)
    assert rc == 6
    assert b"16384" in lib.dalm_last_error(None)
