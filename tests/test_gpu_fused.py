"""The fused BiCGStab kernels (poisson_fused.cu) against the unfused ones and
the oracle.

The fused half-iterations compute every cell value with the same operations
in the same order as the unfused fast kernels; only the order of the global
sums (alpha, omega, rho) differs.  So after ONE iteration the two paths
agree to a few ulps of alpha and omega, and over many steps the fused path
is held to the summation-order envelope (ENVELOPE) like the unfused one.
The grids below span several 32 x 8 tiles in k and j, partial tiles and
several i-chunks, so the halo recomputation at tile, chunk and domain
boundaries is exercised."""
import numpy as np
import pytest

from conftest import package
import oracle as O
from test_gpu_parity import rel
from test_oracle_sensitivity import ENVELOPE, ENVELOPE_MULTI, MULTI_GRID

pytestmark = pytest.mark.gpu

# interior sizes: several k tiles (72 = 32 + 32 + 8), several j tiles
# (20 = 8 + 8 + 4), several i chunks; and a grid narrower than one tile
GRIDS = [MULTI_GRID, (40, 12, 12)]
# each grid's summation-order envelope, measured on the oracle
# (tests/test_oracle_sensitivity.py)
ENVELOPES = {MULTI_GRID: ENVELOPE_MULTI, (40, 12, 12): ENVELOPE}


def solver_pair(make_case, n, **over):
    pkg = package()
    spec, mesh, d, U0, prof = make_case("tiny-loglaw", n=n, **over)
    out = []
    for fused in (True, False):
        s = pkg.Solver(d, fused_krylov=fused)
        s.set_inflow_profile(prof)
        s.set_state(U0)
        out.append(s)
    return spec, d, U0, prof, out


@pytest.mark.parametrize("n", GRIDS)
def test_one_iteration_matches_unfused(make_case, n):
    spec, d, U0, prof, (f, u) = solver_pair(make_case, n)
    for s in (f, u):
        s.set_poisson(1, 0.0)
        s.step(2)
    assert f.stats()["it"] == u.stats()["it"] == 1
    # p = 0 + alpha pp + omega ss after one iteration from p = 0 at step 1
    assert rel(f.field("p"), u.field("p")) <= 1e-13
    for name in ("U", "JU"):
        assert rel(f.field(name), u.field(name)) <= 1e-14


@pytest.mark.parametrize("n", GRIDS)
def test_five_iterations_match_unfused(make_case, n):
    # exercises the ping-pong of p and q across iterations; the paths differ
    # only through the sums' order, which five iterations barely amplify
    spec, d, U0, prof, (f, u) = solver_pair(make_case, n)
    for s in (f, u):
        s.set_poisson(5, 0.0)
        s.step(2)
    assert f.stats()["it"] == u.stats()["it"] == 5
    assert rel(f.field("p"), u.field("p")) <= 1e-10


@pytest.mark.parametrize("n", GRIDS)
def test_fused_within_envelope_of_oracle(make_case, n):
    pkg = package()
    spec, mesh, d, U0, prof = make_case("tiny-loglaw", n=n)
    s = pkg.Solver(d, fused_krylov=True)
    o = O.CRestatement(d)
    for x in (s, o):
        x.set_inflow_profile(prof)
        x.set_state(U0)
    env = ENVELOPES[n]
    for step in range(5):
        s.step(1)
        o.step(1)
        ss, so = s.stats(), o.stats()
        assert abs(ss["it"] - so["it"]) <= max(env["it_abs"], env["it_rel"] * so["it"]), (step, ss, so)
        U, Uo = s.field("U"), o.field("U")
        for m in range(3):
            assert rel(U[..., m], Uo[..., m]) <= env["U"], (step, m)
        assert rel(s.field("p"), o.field("p")) <= env["p"], step
        if step >= 1:
            assert ss["err"] <= spec.tol or ss["it"] == spec.max_it


def test_fused_iteration_cap_and_kernels(make_case):
    pkg = package()
    spec, mesh, d, U0, prof = make_case("tiny-loglaw", n=GRIDS[0])
    s = pkg.Solver(d, profile=True, fused_krylov=True)
    s.set_inflow_profile(prof)
    s.set_state(U0)
    s.set_poisson(7, 0.0)
    s.step(3)
    assert s.stats()["it"] == 7
    kt = s.kernel_timings()
    assert kt["bicg_p_fused"]["launches"] >= 14 and kt["bicg_s_fused"]["launches"] >= 14
    assert kt["jacobi_sweep"]["launches"] == 0 and kt["bicg_p"]["launches"] == 0
    cells = int(np.prod(GRIDS[0]))
    assert kt["bicg_p_fused"]["bytes_per_launch"] == 7 * 8.0 * cells
    assert kt["bicg_s_fused"]["bytes_per_launch"] == 5 * 8.0 * cells
