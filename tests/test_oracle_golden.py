"""Pin the C restatement (oracle/dalm_oracle.c) against golden fixtures that
the reference solver itself produced (tests/golden/make_golden.py).

Everything is FP64 with the reference's operation order, so the comparison
is exact: equal Poisson iteration counts and bit-identical residuals,
diagnostics, turbine loads and field checksums."""
import os

import numpy as np
import pytest

from conftest import casegen
import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_tiny.npz")

CASES = [("tiny-sor", None), ("tiny-bicg", None), ("tiny-sorpc", None), ("tiny-turbine", None),
         ("tiny-loglaw", None), ("tiny-turbine", ([7.5], [2.0], [10.0]))]
FIELDS = ("U", "JU", "p", "nut", "div", "f", "b")


def checksums(a):
    v = a.reshape(-1)
    w = np.sin(np.arange(v.size, dtype=np.float64) * 0.7071)
    return np.array([v.sum(), (v * v).sum(), (v * w).sum()])


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.mark.parametrize("name,params", CASES, ids=[c[0] + ("-params" if c[1] else "") for c in CASES])
def test_restatement_matches_reference_golden(tmp_path, gold, name, params):
    cg = casegen()
    key = name + ("-params" if params else "")
    spec = cg.config(name)
    mesh = cg.write_case(spec, str(tmp_path / key))
    o = O.CRestatement(str(tmp_path / key))
    prof = cg.inflow_profile(spec, mesh)
    if prof is not None:
        o.set_inflow_profile(prof)
    if params:
        o.set_turbine_params(*params)
    o.set_state(cg.initial_velocity(spec, mesh))
    want = gold[key + "/stats"]
    want_t = gold[key + "/turbines"]
    for n in range(len(want)):
        o.step(1)
        s = o.stats()
        got = [s["step"], s["it"], s["err"], s["avg_div"], s["max_cfl"]]
        assert got[1] == want[n][1], f"step {n}: Poisson iterations {got[1]} != {want[n][1]}"
        np.testing.assert_array_equal(np.array(got, dtype=np.float64), want[n])
        if want_t.size:
            tq, th = o.turbines()
            np.testing.assert_array_equal(np.concatenate([tq, th]), want_t[n])
    for f in FIELDS:
        a = o.field(f)
        np.testing.assert_array_equal(checksums(a), gold[key + "/" + f + "/checksums"], err_msg=f)
        np.testing.assert_array_equal(a.reshape(-1)[::97], gold[key + "/" + f + "/sample"], err_msg=f)
    if o.turbine_count():
        r, dr, ch, tw, cd, cl, atk = o.point_tables()
        got = np.concatenate([r, dr, ch, tw, cd.reshape(-1)[::7], cl.reshape(-1)[::7]])
        np.testing.assert_array_equal(got, gold[key + "/point_tables"])
    o.close()


def test_golden_file_is_small():
    assert os.path.getsize(GOLD) < 512 * 1024
