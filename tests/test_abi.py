"""C-ABI checks that need no GPU: the in-tree libdalm.so loads, exports every
entry point include/dalm.h declares, and reports case errors and the absence
of a GPU through status codes and dalm_last_error (no compute is run)."""
import ctypes as C
import json
import os
import re

import pytest

from conftest import ROOT, package

HEADER = os.path.join(ROOT, "include", "dalm.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char \*)\s*(dalm_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib():
    pkg = package()
    if not os.path.exists(pkg.LIB_PATH):
        pkg.build()
    return pkg.load_library()


def test_header_and_python_mirror_agree():
    assert declared() == sorted(package().EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    for name in declared():
        assert hasattr(lib, name), name


def test_default_options(lib):
    pkg = package()
    o = pkg.Options()
    lib.dalm_default_options(C.byref(o))
    assert (o.precision, o.limiter, o.device, o.time_average) == (pkg.FP64, pkg.MINMOD, 0, 1)
    assert (o.fused_krylov, o.fused_jacobi) == (0, 0)


def test_null_arguments_are_rejected(lib):
    h = C.c_void_p()
    assert lib.dalm_create(None, None, C.byref(h)) == 1
    assert lib.dalm_step(None, 1) == 1
    assert b"null" in lib.dalm_last_error(None)


def test_bad_case_reports_case_error(lib, tmp_path):
    h = C.c_void_p()
    rc = lib.dalm_create(str(tmp_path).encode(), None, C.byref(h))
    assert rc == 2 and not h.value
    assert b"setup.json" in lib.dalm_last_error(None)
    (tmp_path / "setup.json").write_text("{ not json")
    (tmp_path / "mesh.json").write_text("{}")
    assert lib.dalm_create(str(tmp_path).encode(), None, C.byref(h)) == 2
    assert b"JSON" in lib.dalm_last_error(None)


def test_incomplete_turbulence_grid_rejected(lib, make_case):
    spec, mesh, d, U0, prof = make_case("tiny-sor")
    with open(os.path.join(d, "setup.json")) as f:
        s = json.load(f)
    s["turbulence grid"] = {"bar": 0.1, "thick": 0.06, "placement": [1, 1, 1]}  # no "mesh"
    with open(os.path.join(d, "setup.json"), "w") as f:
        json.dump(s, f)
    h = C.c_void_p()
    assert lib.dalm_create(d.encode(), None, C.byref(h)) == 2
    assert b"mesh" in lib.dalm_last_error(None)


def test_valid_case_without_gpu_reports_cuda_error(lib, make_case):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    spec, mesh, d, U0, prof = make_case("tiny-turbine")
    h = C.c_void_p()
    rc = lib.dalm_create(d.encode(), None, C.byref(h))
    assert rc == 3 and not h.value
    assert lib.dalm_last_error(None)


def test_solver_without_gpu_fails_loudly(make_case):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    pkg = package()
    spec, mesh, d, U0, prof = make_case("tiny-sor")
    with pytest.raises(pkg.DalmError):
        pkg.Solver(d)


def test_unknown_options_are_rejected(lib, make_case):
    pkg = package()
    spec, mesh, d, U0, prof = make_case("tiny-bicg")
    for field in ("limiter", "precision"):
        o = pkg.Options()
        lib.dalm_default_options(C.byref(o))
        setattr(o, field, 7)
        h = C.c_void_p()
        assert lib.dalm_create(d.encode(), C.byref(o), C.byref(h)) == 1 and not h.value
        assert b"unknown" in lib.dalm_last_error(None)
