"""Parity of the CUDA path (through the C ABI, libdalm.so) with the oracle
(oracle/dalm_oracle.c, itself pinned bit for bit to the reference).

Tolerances, FP64 form:
  * per-stage fields after one stage: relative L2 <= 1e-13 (differences come
    only from libm cbrt/sin/cos/atan/exp ulps and the order of the global
    dot products);
  * per-step u, v, w, p over the first 10 steps: relative L2 <= 1e-10 and
    equal Poisson iteration counts (the acceptance bar);
  * turbine thrust / torque: relative <= 1e-9.
"""
import numpy as np
import pytest

from conftest import package
import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def setup_pair(make_case, name, params=None, **over):
    pkg = package()
    spec, mesh, d, U0, prof = make_case(name, **over)
    s = pkg.Solver(d)
    o = O.CRestatement(d)
    for x in (s, o):
        if prof is not None:
            x.set_inflow_profile(prof)
        if params:
            x.set_turbine_params(*params)
        x.set_state(U0)
    return s, o


def compare_fields(s, o, names, tol, where):
    for f in names:
        a, b = s.field(f), o.field(f)
        assert np.all(np.isfinite(a)), f"{where}: {f} not finite"
        r = rel(a, b)
        assert r <= tol, f"{where}: {f} rel L2 {r:.3e} > {tol:.0e}"


CASES = ["tiny-sor", "tiny-bicg", "tiny-sorpc", "tiny-jacobi", "tiny-turbine", "tiny-loglaw"]


@pytest.mark.parametrize("name", CASES)
def test_initial_state(make_case, name):
    s, o = setup_pair(make_case, name)
    # BCs and face fluxes involve no libm call: bit-identical
    for f in ("U", "JU"):
        np.testing.assert_array_equal(s.field(f), o.field(f), err_msg=f)
    compare_fields(s, o, ("nut", "div", "f"), 1e-13, "set_state")
    ss, so = s.stats(), o.stats()
    assert abs(ss["avg_div"] - so["avg_div"]) <= 1e-13 * max(abs(so["avg_div"]), 1e-300)
    assert abs(ss["max_cfl"] - so["max_cfl"]) <= 1e-14 * so["max_cfl"]


@pytest.mark.parametrize("name", ["tiny-bicg", "tiny-turbine", "tiny-loglaw"])
def test_stage_by_stage(make_case, name):
    s, o = setup_pair(make_case, name, tavg_start_time=0.0)
    s.advance_clock()
    o.advance_clock()
    checks = {
        0: ("U",),
        1: ("JU", "b"),
        2: ("p",),
        3: ("U", "JU", "p", "nut", "div"),
        4: ("f",),
        6: ("Utavg",),
    }
    for step in range(2):
        for st in range(7):
            s.stage(st)
            o.stage(st)
            if st in checks:
                compare_fields(s, o, checks[st], 1e-12, f"step {step} stage {st}")
            if st == 2:
                assert s.stats()["it"] == o.stats()["it"]
        s.advance_clock()
        o.advance_clock()


@pytest.mark.parametrize("name", CASES)
def test_ten_steps(make_case, name):
    s, o = setup_pair(make_case, name, steps=10)
    for n in range(11):
        s.step(1)
        o.step(1)
        ss, so = s.stats(), o.stats()
        assert ss["step"] == so["step"]
        assert ss["it"] == so["it"], f"step {n}: iterations {ss['it']} != {so['it']}"
        U, Uo = s.field("U"), o.field("U")
        for m in range(3):
            r = rel(U[..., m], Uo[..., m])
            assert r <= 1e-10, f"step {n} U[{m}] rel L2 {r:.3e}"
        r = rel(s.field("p"), o.field("p"))
        assert r <= 1e-10, f"step {n} p rel L2 {r:.3e}"
        if so["step"] > 1:
            assert abs(ss["err"] - so["err"]) <= 1e-8 * abs(so["err"]) + 1e-300
            assert abs(ss["avg_div"] - so["avg_div"]) <= 1e-8 * abs(so["avg_div"])
            assert abs(ss["max_cfl"] - so["max_cfl"]) <= 1e-10 * so["max_cfl"]
        if o.turbine_count():
            th, tq, pw = s.turbines()
            tqo, tho = o.turbines()
            np.testing.assert_allclose(th, tho, rtol=1e-9)
            np.testing.assert_allclose(tq, tqo, rtol=1e-9)


def test_turbine_params_and_points(make_case):
    params = ([12.0], [3.0], [9.0])
    s, o = setup_pair(make_case, "tiny-turbine", params=params)
    for _ in range(4):
        s.step(1)
        o.step(1)
    xs, fs, tqs, ths = s.points()
    xo, fo, tqo, tho = o.points()
    np.testing.assert_allclose(xs, xo, rtol=0, atol=1e-13)
    np.testing.assert_allclose(fs, fo, rtol=1e-9, atol=1e-15)
    th, tq, pw = s.turbines()
    np.testing.assert_allclose(pw, tq * 9.0, rtol=1e-15)
    compare_fields(s, o, ("U", "p", "f"), 1e-11, "params")


def test_time_average(make_case):
    s, o = setup_pair(make_case, "tiny-bicg", tavg_start_time=0.0)
    for _ in range(5):
        s.step(1)
        o.step(1)
    compare_fields(s, o, ("Utavg",), 1e-11, "tavg")


def test_field_round_trip(make_case):
    pkg = package()
    spec, mesh, d, U0, prof = make_case("tiny-sor")
    s = pkg.Solver(d)
    rng = np.random.default_rng(0)
    for name in ("U", "p", "JU", "f", "b"):
        v = rng.standard_normal(s.field(name).shape)
        s.set_field(name, v)
        np.testing.assert_array_equal(s.field(name), v)


def test_poisson_iteration_cap(make_case):
    s, o = setup_pair(make_case, "tiny-bicg")
    for x in (s, o):
        x.set_poisson(3, 0.0)
    for _ in range(3):
        s.step(1)
        o.step(1)
    assert s.stats()["it"] == 3 == o.stats()["it"]
    compare_fields(s, o, ("U", "p"), 1e-11, "capped")


def test_nonfinite_state_is_reported(make_case):
    pkg = package()
    spec, mesh, d, U0, prof = make_case("tiny-sor")
    s = pkg.Solver(d)
    bad = U0.copy()
    bad[5, 6, 7, 0] = np.nan
    s.set_state(bad)
    with pytest.raises(pkg.DalmError) as e:
        s.step(3)
    assert e.value.code == 4


def test_kernel_timings(make_case):
    pkg = package()
    spec, mesh, d, U0, prof = make_case("tiny-turbine")
    s = pkg.Solver(d, profile=True)
    s.set_state(U0)
    s.step(3)
    kt = s.kernel_timings()
    assert kt["predict"]["launches"] == 2
    assert kt["bicg_xr"]["launches"] >= s.stats()["it"]
    assert kt["jacobi_sweep"]["bytes_per_launch"] > 0
    stages, launches = s.timings()
    assert stages["poisson"] > 0 and launches > 0
