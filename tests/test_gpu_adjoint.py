"""The discrete adjoint on the GPU (dalm_adjoint_power_grad).

Checked three ways on the 40x20x20 two-turbine log-law case with the van
Albada limiter and tight pressure solves: against central finite
differences of the GPU's own FP64 forward (the oracle the north star names
for the gradient), against the host-side adjoint of the same arithmetic
over the oracle's trajectory, and for independence of the checkpoint
interval.  The gradient run must also leave the handle exactly where
dalm_step would."""
import numpy as np
import pytest

from conftest import package
from test_adjoint_math import Setup, adjoint_gradient

pytestmark = pytest.mark.gpu

TOL = 1e-13  # pressure solves: finite differences need a converged forward


def solver(d, prof, U0, params=None):
    pkg = package()
    s = pkg.Solver(d, limiter=pkg.VAN_ALBADA)
    if prof is not None:
        s.set_inflow_profile(prof)
    s.set_poisson(20000, TOL)
    if params is not None:
        s.set_turbine_params(*params)
    s.set_state(U0)
    return s


def objective(d, prof, U0, params, t0, t1):
    s = solver(d, prof, U0, params)
    s.step(1)
    J = 0.0
    for n in range(1, t1 + 1):
        s.step(1)
        if n >= t0:
            J += np.sum(s.turbines()[2])
    return J / (t1 - t0 + 1)


def test_gradient_matches_finite_differences(make_case):
    spec, mesh, d, U0, prof = make_case("tiny-loglaw", steps=24)
    t0, t1 = 13, 24
    s = solver(d, prof, U0)
    base = s.turbine_params()
    J, g = s.power_gradient(t0, t1, ckpt_every=5)
    st = s.adjoint_stats()
    print("J", J, "stats", st)
    assert st["max_rel_residual"] <= 1e-9
    assert abs(J - objective(d, prof, U0, base, t0, t1)) <= 1e-12 * abs(J)
    h = 1e-5
    fd = np.zeros_like(g)
    for w in range(g.shape[0]):
        for q in range(3):
            pp = [v.copy() for v in base]
            pm = [v.copy() for v in base]
            pp[q][w] += h
            pm[q][w] -= h
            fd[w, q] = (objective(d, prof, U0, pp, t0, t1) -
                        objective(d, prof, U0, pm, t0, t1)) / (2 * h)
    rel = np.abs(g - fd) / np.abs(fd)
    print("adjoint\n", g, "\nfinite differences\n", fd, "\nrelative", rel)
    # the bar of the gradient check: 1e-4 relative per parameter
    assert np.all(np.abs(g - fd) <= 1e-4 * np.abs(fd) + 1e-7 * np.abs(fd).max())


def test_gradient_matches_host_adjoint(make_case):
    """Same arithmetic on the host over the oracle's trajectory (6 steps)."""
    host = Setup(make_case, steps=6)
    try:
        g_host = adjoint_gradient(host, 6, 3)
    finally:
        host.close()
    spec, mesh, d, U0, prof = make_case("tiny-loglaw", steps=6)
    s = solver(d, prof, U0)
    J, g = s.power_gradient(3, 6, ckpt_every=2)
    err = np.abs(g - g_host) / np.abs(g_host).max()
    print("GPU\n", g, "\nhost\n", g_host, "\nerr", err)
    assert np.all(err <= 1e-7)


def test_checkpoint_interval_does_not_change_the_gradient(make_case):
    spec, mesh, d, U0, prof = make_case("tiny-loglaw", steps=12)
    out = []
    for k in (1, 4, 5, 100):
        s = solver(d, prof, U0)
        J, g = s.power_gradient(7, 12, ckpt_every=k)
        st = s.adjoint_stats()
        print(k, J, st)
        out.append((J, g, st))
    for J, g, st in out[1:]:
        assert J == out[0][0]
        np.testing.assert_array_equal(g, out[0][1])
    # restart points every step: nothing is recomputed except from them
    assert out[3][2]["recomputed_steps"] == 0  # one segment, recorded by the forward run
    assert out[0][2]["recomputed_steps"] == 11


def test_handle_ends_where_dalm_step_would(make_case):
    spec, mesh, d, U0, prof = make_case("tiny-loglaw", steps=9)
    a = solver(d, prof, U0)
    a.power_gradient(4, 9, ckpt_every=3)
    b = solver(d, prof, U0)
    b.step(10)  # steps 0..9
    assert a.stats()["step"] == b.stats()["step"] == 10
    for f in ("U", "Uold", "JU", "p", "f"):
        np.testing.assert_array_equal(a.field(f), b.field(f), err_msg=f)
    for x, y in zip(a.turbines(), b.turbines()):
        np.testing.assert_array_equal(x, y)
    sa, sb = a.stats(), b.stats()
    assert (sa["it"], sa["err"], sa["avg_div"]) == (sb["it"], sb["err"], sb["avg_div"])
    # and it continues identically
    a.step(2)
    b.step(2)
    np.testing.assert_array_equal(a.field("U"), b.field("U"))


def test_rejects_bad_windows(make_case):
    pkg = package()
    spec, mesh, d, U0, prof = make_case("tiny-loglaw", steps=4)
    s = solver(d, prof, U0)
    for t0, t1, k in ((0, 3, 2), (3, 2, 2), (1, 3, 0)):
        with pytest.raises(pkg.DalmError):
            s.power_gradient(t0, t1, k)
    spec, mesh, d, U0, prof = make_case("tiny-bicg", steps=4)
    s2 = pkg.Solver(d)
    with pytest.raises(pkg.DalmError, match="UNSUPPORTED"):
        s2.power_gradient(1, 2, 1)


def test_torch_autograd_function(make_case):
    """The gradient through a torch.autograd.Function (test harness only):
    backward returns dalm_adjoint_power_grad's gradient, checked against a
    central difference of the Function along a random direction."""
    torch = pytest.importorskip("torch")
    spec, mesh, d, U0, prof = make_case("tiny-loglaw", steps=10)
    t0, t1 = 6, 10

    class MeanPower(torch.autograd.Function):
        @staticmethod
        def forward(ctx, params):  # (turbines, 3): yaw deg, pitch deg, rotor speed rad/s
            p = params.detach().cpu().numpy()
            s = solver(d, prof, U0, (p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy()))
            J, g = s.power_gradient(t0, t1, ckpt_every=4)
            s.close()
            ctx.save_for_backward(torch.from_numpy(g))
            return params.new_tensor(J)

        @staticmethod
        def backward(ctx, gJ):
            (g,) = ctx.saved_tensors
            return gJ * g.to(gJ.dtype)

    s0 = solver(d, prof, U0)
    yaw, pitch, om = s0.turbine_params()
    params = torch.tensor(np.stack([yaw, pitch, om], axis=1), dtype=torch.float64,
                          requires_grad=True)
    J = MeanPower.apply(params)
    J.backward()
    v = torch.from_numpy(np.random.default_rng(0).standard_normal(tuple(params.shape)))
    h = 1e-5
    with torch.no_grad():
        dd = (MeanPower.apply(params + h * v) - MeanPower.apply(params - h * v)) / (2 * h)
    dg = float((params.grad * v).sum())
    print("directional derivative: autograd", dg, "central difference", float(dd))
    assert abs(dg - float(dd)) <= 1e-5 * abs(float(dd))


def test_gradient_with_grid_and_floor(make_case):
    """The transposed solid scaling and retracted-floor wall: a
    turbulence-generating grid upstream of the rotors and a slip floor up to
    x = 2, against central differences."""
    grid = {"bar": 0.4, "mesh": 1.25, "thick": 0.5, "placement": [2.5, 2.5, 1.5]}
    spec, mesh, d, U0, prof = make_case("tiny-loglaw", steps=12, grid=grid, floor_start=2.0)
    t0, t1 = 7, 12
    s = solver(d, prof, U0)
    base = s.turbine_params()
    J, g = s.power_gradient(t0, t1, ckpt_every=4)
    h = 1e-5
    fd = np.zeros_like(g)
    for w in range(g.shape[0]):
        for q in range(3):
            pp = [v.copy() for v in base]
            pm = [v.copy() for v in base]
            pp[q][w] += h
            pm[q][w] -= h
            fd[w, q] = (objective(d, prof, U0, pp, t0, t1) -
                        objective(d, prof, U0, pm, t0, t1)) / (2 * h)
    print("adjoint\n", g, "\nfinite differences\n", fd, "\nrelative", np.abs(g - fd) / np.abs(fd))
    assert np.all(np.abs(g - fd) <= 1e-4 * np.abs(fd) + 1e-7 * np.abs(fd).max())


def test_three_turbine_gradient_each_component(make_case):
    """Every one of the 9 components (yaw, pitch, rotor speed of three
    turbines, the middle one yawed 10 deg) within 1e-4 relative of central
    finite differences, with no absolute floor: the C5 configuration (log-law
    inflow + 8 %, van Albada, polar every 0.05 deg) reduced to 64x32x32 cells
    and 30 steps, J over steps 16-30.  The unyawed rotors' yaw derivatives
    are one to two orders smaller than the others; with pressure solves to
    1e-14 and h = 1e-4 the finite differences resolve them (measured on a
    B200: every component within 1e-7)."""
    pkg = package()
    spec, mesh, d, U0, prof = make_case("c5", n=(64, 32, 32), steps=30)
    t0, t1, tol = 16, 30, 1e-14

    def make(params=None):
        s = pkg.Solver(d, limiter=pkg.VAN_ALBADA, time_average=False)
        s.set_inflow_profile(prof)
        s.set_poisson(20000, tol)
        if params is not None:
            s.set_turbine_params(*params)
        s.set_state(U0)
        return s

    def J(params):
        s = make(params)
        s.step(1)
        acc = 0.0
        for n in range(1, t1 + 1):
            s.step(1)
            if n >= t0:
                acc += float(np.sum(s.turbines()[2]))
        s.finalize()
        return acc / (t1 - t0 + 1)

    s = make()
    base = s.turbine_params()
    assert len(base[0]) == 3 and base[0][1] == pytest.approx(10.0)
    Ja, g = s.power_gradient(t0, t1, ckpt_every=10)
    s.finalize()
    assert abs(Ja - J(base)) <= 1e-13 * abs(Ja)
    h = 1e-4
    fd = np.zeros_like(g)
    for w in range(3):
        for q in range(3):
            pp = [v.copy() for v in base]
            pm = [v.copy() for v in base]
            pp[q][w] += h
            pm[q][w] -= h
            fd[w, q] = (J(pp) - J(pm)) / (2 * h)
    rel = np.abs(g - fd) / np.abs(fd)
    print("adjoint\n", g, "\nfinite differences\n", fd, "\nrelative\n", rel)
    assert np.all(rel <= 1e-4), rel
