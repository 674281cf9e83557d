"""Parity of the CUDA path (through the C ABI, libdalm.so) with the oracle
(oracle/dalm_oracle.c, itself pinned bit for bit to the reference).

Two modes of the same kernels:

  reference_sums=True   every global sum (Krylov dots, residual and
                        divergence norms) is accumulated in the reference's
                        serial cell order, and the actuator line (blade-point
                        model and Gaussian projection) runs on the host with
                        the host's libm.  Every other operation already keeps
                        the reference's order and rounding (FP64, no FMA
                        contraction, host-libm Smagorinsky filter), so the GPU
                        step must be BIT-IDENTICAL to the reference: fields,
                        Poisson iteration counts, residuals, blade-point
                        positions, forces and turbine loads.
  default (fast)        the sums use a deterministic parallel tree.  The
                        reference algorithm itself moves by the envelope
                        ENVELOPE under a change of summation order alone
                        (tests/test_oracle_sensitivity.py), so the fast mode
                        is held to that envelope over 10 steps:
                        |d it| <= max(3, 10%), u,v,w rel L2 <= 1e-7,
                        p rel L2 <= 1e-3, thrust/torque rel <= 1e-6.
"""
import numpy as np
import pytest

from conftest import package
import oracle as O
from test_oracle_sensitivity import ENVELOPE

pytestmark = pytest.mark.gpu

NO_TURBINE = ["tiny-sor", "tiny-bicg", "tiny-sorpc", "tiny-jacobi", "tiny-tgg"]
TURBINE = ["tiny-turbine", "tiny-loglaw"]


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def setup_pair(make_case, name, params=None, reference_sums=False, **over):
    pkg = package()
    spec, mesh, d, U0, prof = make_case(name, **over)
    s = pkg.Solver(d, reference_sums=reference_sums)
    o = O.CRestatement(d)
    for x in (s, o):
        if prof is not None:
            x.set_inflow_profile(prof)
        if params:
            x.set_turbine_params(*params)
        x.set_state(U0)
    return s, o


def assert_identical(s, o, names, where):
    for f in names:
        np.testing.assert_array_equal(s.field(f), o.field(f), err_msg=f"{where}: {f}")


def assert_close(s, o, names, tol, where):
    for f in names:
        a, b = s.field(f), o.field(f)
        assert np.all(np.isfinite(a)), f"{where}: {f} not finite"
        r = rel(a, b)
        assert r <= tol, f"{where}: {f} rel L2 {r:.3e} > {tol:.0e}"


@pytest.mark.parametrize("name", NO_TURBINE + TURBINE)
def test_initial_state(make_case, name):
    s, o = setup_pair(make_case, name)
    # boundary conditions, face fluxes, eddy viscosity, divergence: no
    # device libm call, bit-identical
    assert_identical(s, o, ("U", "JU", "nut", "div"), "set_state")
    assert_close(s, o, ("f",), 1e-13, "set_state")
    ss, so = s.stats(), o.stats()
    assert ss["max_cfl"] == so["max_cfl"]
    assert abs(ss["avg_div"] - so["avg_div"]) <= 1e-14 * abs(so["avg_div"])


@pytest.mark.parametrize("name", NO_TURBINE)
def test_reference_sums_bit_identical_10_steps(make_case, name):
    s, o = setup_pair(make_case, name, reference_sums=True, tavg_start_time=0.0)
    for n in range(11):
        s.step(1)
        o.step(1)
        ss, so = s.stats(), o.stats()
        assert ss["it"] == so["it"], f"step {n}: iterations {ss['it']} != {so['it']}"
        assert ss["err"] == so["err"] and ss["avg_div"] == so["avg_div"], f"step {n}"
        assert ss["max_cfl"] == so["max_cfl"], f"step {n}"
        assert_identical(s, o, ("U", "p"), f"step {n}")
    assert_identical(s, o, ("JU", "nut", "div", "b", "Uold", "Utavg"), "after 10 steps")


@pytest.mark.parametrize("name", NO_TURBINE[1:3])
def test_reference_sums_stage_by_stage(make_case, name):
    s, o = setup_pair(make_case, name, reference_sums=True, tavg_start_time=0.0)
    s.advance_clock()
    o.advance_clock()
    checks = {0: ("U",), 1: ("JU", "b"), 2: ("p",), 3: ("U", "JU", "p", "nut", "div"),
              4: ("f",), 6: ("Utavg",)}
    for step in range(2):
        for st in range(7):
            s.stage(st)
            o.stage(st)
            if st in checks:
                assert_identical(s, o, checks[st], f"step {step} stage {st}")
            if st == 2:
                assert s.stats()["it"] == o.stats()["it"]
        s.advance_clock()
        o.advance_clock()


def within_envelope(s, o, n, label):
    ss, so = s.stats(), o.stats()
    assert ss["step"] == so["step"]
    assert abs(ss["it"] - so["it"]) <= max(ENVELOPE["it_abs"], ENVELOPE["it_rel"] * so["it"]), \
        f"{label} step {n}: iterations {ss['it']} vs {so['it']}"
    U, Uo = s.field("U"), o.field("U")
    for m in range(3):
        r = rel(U[..., m], Uo[..., m])
        assert r <= ENVELOPE["U"], f"{label} step {n} U[{m}] rel L2 {r:.3e}"
    r = rel(s.field("p"), o.field("p"))
    assert r <= ENVELOPE["p"], f"{label} step {n} p rel L2 {r:.3e}"
    if o.turbine_count():
        th, tq, pw = s.turbines()
        tqo, tho = o.turbines()
        np.testing.assert_allclose(th, tho, rtol=1e-6)
        np.testing.assert_allclose(tq, tqo, rtol=1e-6)


@pytest.mark.parametrize("name", NO_TURBINE + TURBINE)
def test_fast_mode_10_steps_within_envelope(make_case, name):
    s, o = setup_pair(make_case, name)
    for n in range(11):
        s.step(1)
        o.step(1)
        within_envelope(s, o, n, "fast")


@pytest.mark.parametrize("name", TURBINE)
def test_reference_sums_turbines_bit_identical_10_steps(make_case, name):
    """With reference-order sums the blade-point model and the Gaussian
    projection run on the host with the host's libm (the reference's), so
    turbine cases are bit-identical too: fields, iteration counts, residuals,
    blade-point positions, forces and turbine loads at every step."""
    s, o = setup_pair(make_case, name, reference_sums=True)
    assert_points_identical(s, o, "set_state")
    assert_identical(s, o, ("U", "JU", "f", "nut", "div"), "set_state")
    for n in range(11):
        s.step(1)
        o.step(1)
        ss, so = s.stats(), o.stats()
        assert ss["it"] == so["it"], f"step {n}: iterations {ss['it']} != {so['it']}"
        assert ss["err"] == so["err"] and ss["avg_div"] == so["avg_div"], f"step {n}"
        assert ss["max_cfl"] == so["max_cfl"], f"step {n}"
        assert_identical(s, o, ("U", "p", "f"), f"step {n}")
        assert_points_identical(s, o, f"step {n}")
    assert_identical(s, o, ("JU", "nut", "div", "b", "Uold"), "after 10 steps")


def assert_points_identical(s, o, where):
    xs, fs, tqs, ths = s.points()
    xo, fo, tqo, tho = o.points()
    np.testing.assert_array_equal(xs, xo, err_msg=f"{where}: blade-point positions")
    np.testing.assert_array_equal(fs, fo, err_msg=f"{where}: blade-point forces")
    np.testing.assert_array_equal(tqs, tqo, err_msg=f"{where}: blade-point torque")
    np.testing.assert_array_equal(ths, tho, err_msg=f"{where}: blade-point thrust")
    th, tq, _ = s.turbines()
    tqo_w, tho_w = o.turbines()
    np.testing.assert_array_equal(th, tho_w, err_msg=f"{where}: turbine thrust")
    np.testing.assert_array_equal(tq, tqo_w, err_msg=f"{where}: turbine torque")


@pytest.mark.parametrize("name", TURBINE)
def test_fast_mode_blade_points(make_case, name):
    """The fast mode evaluates the blade points on the device (device sin,
    cos, atan) and projects with the device exp, truncated at r^2 <= 40 eps^2:
    positions within 1e-13 absolute, forces and the force field within
    1e-12 relative of the oracle's on the same velocity."""
    s, o = setup_pair(make_case, name)
    xs, fs, _, _ = s.points()
    xo, fo, _, _ = o.points()
    np.testing.assert_allclose(xs, xo, rtol=0, atol=1e-13)
    np.testing.assert_allclose(fs, fo, rtol=1e-12, atol=1e-16)
    assert_close(s, o, ("f",), 1e-12, "set_state")


def test_turbine_params_and_points(make_case):
    params = ([12.0], [3.0], [9.0])
    s, o = setup_pair(make_case, "tiny-turbine", params=params, reference_sums=True)
    assert_points_identical(s, o, "set_state")
    s.step(1)
    o.step(1)
    assert_points_identical(s, o, "step 1")
    th, tq, pw = s.turbines()
    np.testing.assert_allclose(pw, tq * 9.0, rtol=1e-15)
    assert_identical(s, o, ("f", "U", "p"), "params")


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
    s, o = setup_pair(make_case, "tiny-bicg", reference_sums=True)
    for x in (s, o):
        x.set_poisson(3, 0.0)
    for _ in range(3):
        s.step(1)
        o.step(1)
    assert s.stats()["it"] == 3 == o.stats()["it"]
    assert_identical(s, o, ("U", "p"), "capped")


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


@pytest.mark.parametrize("name", ["tiny-sor", "tiny-bicg"])
def test_van_albada_reference_sums_bit_identical(make_case, name):
    """The smooth limiter (extension) against its restatement in the oracle."""
    pkg = package()
    spec, mesh, d, U0, prof = make_case(name)
    s = pkg.Solver(d, reference_sums=True, limiter=pkg.VAN_ALBADA)
    o = O.CRestatement(d)
    o.set_limiter(1)
    for x in (s, o):
        x.set_state(U0)
    for n in range(6):
        s.step(1)
        o.step(1)
        assert s.stats()["it"] == o.stats()["it"], n
        assert_identical(s, o, ("U", "p"), f"van Albada step {n}")


def test_van_albada_fast_mode_with_turbines(make_case):
    pkg = package()
    spec, mesh, d, U0, prof = make_case("tiny-turbine")
    s = pkg.Solver(d, limiter=pkg.VAN_ALBADA)
    o = O.CRestatement(d)
    o.set_limiter(1)
    for x in (s, o):
        x.set_state(U0)
    for n in range(6):
        s.step(1)
        o.step(1)
        within_envelope(s, o, n, "van Albada")
