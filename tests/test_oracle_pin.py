"""Pin the C restatement directly against the reference solver compiled from
its own sources (oracle/_ref/libref3dalm.so), field by field and stage by
stage, including the reference's own ALM fixture files (test/turbine.json,
test/turbine_list.json) when the reference tree is present.

Skipped when neither the built _ref library nor the reference sources exist
(the golden-fixture test covers that situation)."""
import json
import os
import shutil

import numpy as np
import pytest

from conftest import casegen
import oracle as O

REF_SRC = os.path.dirname(O.reference_src().rstrip("/"))  # the reference tree


def _have_ref():
    if O.reference_available():
        return True
    if os.path.exists(os.path.join(REF_SRC, "src", "solver.h")):
        O.build(ref=True)
        return O.reference_available()
    return False


pytestmark = pytest.mark.skipif(not _have_ref(), reason="reference oracle not built here")

FIELDS = ("U", "Uold", "JU", "p", "nut", "div", "f", "b", "Utavg")


def pair(make_case, name, params=None, **over):
    spec, mesh, d, U0, prof = make_case(name, **over)
    a, b = O.CRestatement(d), O.Reference(d)
    for o in (a, b):
        if prof is not None:
            o.set_inflow_profile(prof)
        if params:
            o.set_turbine_params(*params)
        o.set_state(U0)
    return a, b


def assert_same(a, b, where):
    for f in FIELDS:
        np.testing.assert_array_equal(a.field(f), b.field(f), err_msg=f"{where}: {f}")
    sa, sb = a.stats(), b.stats()
    assert sa == sb, where
    ta, tb = a.turbines(), b.turbines()
    np.testing.assert_array_equal(ta[0], tb[0])
    np.testing.assert_array_equal(ta[1], tb[1])


@pytest.mark.parametrize("name", ["tiny-sor", "tiny-bicg", "tiny-sorpc", "tiny-turbine",
                                  "tiny-loglaw", "tiny-tgg"])
def test_stage_by_stage_bit_identical(make_case, name):
    a, b = pair(make_case, name, tavg_start_time=0.0)
    assert a.max_diag() == b.max_diag()
    np.testing.assert_array_equal(a.matrix(), b.matrix())
    for x, y in zip(a.mesh(), b.mesh()):
        np.testing.assert_array_equal(x, y)
    assert_same(a, b, "after set_state")
    for o in (a, b):
        o.advance_clock()
    for step in range(3):
        for st in range(7):
            a.stage(st)
            b.stage(st)
            assert_same(a, b, f"step {step} stage {st}")
        a.advance_clock()
        b.advance_clock()


def test_turbine_params_bit_identical(make_case):
    a, b = pair(make_case, "tiny-turbine", params=([12.0], [3.0], [9.0]))
    for _ in range(4):
        a.step(1)
        b.step(1)
    assert_same(a, b, "turbine params")
    xa, fa, tqa, tha = a.points()
    xb, fb, tqb, thb = b.points()
    np.testing.assert_array_equal(xa, xb)
    np.testing.assert_array_equal(fa, fb)


def test_reference_fixture_turbines(tmp_path):
    """The reference's own ALM fixtures: test/turbine.json (12 airfoil
    stations, 40 attack angles) and test/turbine_list.json (an oscillating
    pitch turbine and a static 3-degree pitch turbine), used unchanged as the
    case's windturbine.json and windturbine array."""
    tdir = os.path.join(REF_SRC, "test")
    if not os.path.exists(os.path.join(tdir, "turbine.json")):
        pytest.skip("reference test fixtures not present")
    cg = casegen()
    spec = cg.config("tiny-turbine", n=(48, 24, 24), lengths=(24.0, 6.0, 6.0))
    mesh = cg.write_case(spec, str(tmp_path))
    shutil.copy(os.path.join(tdir, "turbine.json"), tmp_path / "windturbine.json")
    with open(os.path.join(tdir, "turbine_list.json")) as f:
        arr = json.load(f)
    for t in arr:  # place the two rotors inside the small domain
        t["base"] = [t["base"][0] * 0.5 + 6.0, 3.0, 0.5]
    with open(tmp_path / "setup.json") as f:
        setup = json.load(f)
    setup["windturbine array"] = arr
    setup["alm"] = {"blade points": 20, "projection width": 0.6}
    with open(tmp_path / "setup.json", "w") as f:
        json.dump(setup, f)
    a, b = O.CRestatement(str(tmp_path)), O.Reference(str(tmp_path))
    U0 = cg.initial_velocity(spec, mesh)
    for o in (a, b):
        o.set_state(U0)
    ta, tb = a.point_tables(), b.point_tables()
    for x, y in zip(ta, tb):
        np.testing.assert_array_equal(x, y)
    for _ in range(4):
        a.step(1)
        b.step(1)
    assert_same(a, b, "reference fixtures")
    assert np.all(np.isfinite(a.turbines()[0]))
