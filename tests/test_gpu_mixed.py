"""Mixed-precision pressure solve (DALM_MIXED) against the oracle.

DALM_MIXED solves A p = b by FP64 iterative refinement: the residual
r = b - A p, its norm and the pressure are FP64; each correction A e = r is
an FP32 inner solve (capped): conjugate gradients preconditioned by a
multigrid V-cycle (default) or the case's Jacobi(k)-BiCGStab; a pass that
makes the FP64 residual worse is taken back, and one that stalls or breaks
down hands the rest of the solve to the reference's FP64 BiCGStab.  Every solve that is not capped therefore
ends with its residual below the case's tolerance, like the reference's, but
at a different iterate: the pressure differs from the reference's by what two
solutions that both meet the tolerance may differ by, and the iteration
counts are not comparable.  The fields are held to MIXED_ENVELOPE over ten
steps; SOR and Jacobi solves are FP64 under either precision."""
import numpy as np
import pytest

from conftest import package
import oracle as O
from test_gpu_parity import rel

pytestmark = pytest.mark.gpu

BICG = ["tiny-bicg", "tiny-sorpc", "tiny-turbine", "tiny-loglaw"]

# rel L2 against the FP64 oracle over ten steps (u, v, w per component)
MIXED_ENVELOPE = {"U": 1e-6, "p": 1e-2}


def setup(make_case, name, precision, with_oracle=True, **kw):
    pkg = package()
    spec, mesh, d, U0, prof = make_case(name)
    s = pkg.Solver(d, precision=precision, **kw)
    xs = [s]
    o = None
    if with_oracle:
        o = O.CRestatement(d)
        xs.append(o)
    for x in xs:
        if prof is not None:
            x.set_inflow_profile(prof)
        x.set_state(U0)
    return spec, s, o


INNER = {"multigrid": 0, "bicgstab": 1}


@pytest.mark.parametrize("inner", sorted(INNER))
@pytest.mark.parametrize("name", BICG)
def test_mixed_10_steps_within_envelope(make_case, name, inner):
    pkg = package()
    spec, s, o = setup(make_case, name, pkg.MIXED, mixed_inner=INNER[inner])
    worst = {"U": 0.0, "p": 0.0}
    for n in range(11):
        s.step(1)
        o.step(1)
        ss, so = s.stats(), o.stats()
        assert ss["step"] == so["step"]
        if n >= 1 and ss["it"] < spec.max_it:
            assert ss["err"] <= spec.tol, f"step {n}: residual {ss['err']:.3e} > tol"
        U, Uo = s.field("U"), o.field("U")
        for m in range(3):
            worst["U"] = max(worst["U"], rel(U[..., m], Uo[..., m]))
        worst["p"] = max(worst["p"], rel(s.field("p"), o.field("p")))
    print(f"{name}: mixed vs oracle worst rel L2 over 10 steps: U {worst['U']:.2e} p {worst['p']:.2e}")
    assert worst["U"] <= MIXED_ENVELOPE["U"] and worst["p"] <= MIXED_ENVELOPE["p"], worst


@pytest.mark.parametrize("name", ["tiny-sor", "tiny-jacobi"])
def test_mixed_is_fp64_without_bicgstab(make_case, name):
    pkg = package()
    _, a, _ = setup(make_case, name, pkg.MIXED, with_oracle=False)
    _, b, _ = setup(make_case, name, pkg.FP64, with_oracle=False)
    a.step(5)
    b.step(5)
    assert a.stats()["it"] == b.stats()["it"]
    for f in ("U", "p"):
        np.testing.assert_array_equal(a.field(f), b.field(f))


@pytest.mark.parametrize("inner", sorted(INNER))
def test_mixed_iteration_cap(make_case, inner):
    pkg = package()
    spec, s, _ = setup(make_case, "tiny-bicg", pkg.MIXED, with_oracle=False, refine_inner_it=3,
                       mixed_inner=INNER[inner])
    s.set_poisson(5, 0.0)
    s.step(2)
    # the cap counts FP32 and FP64 iterations together
    assert s.stats()["it"] == 5


def test_mixed_kernels(make_case):
    pkg = package()
    spec, s, _ = setup(make_case, "tiny-loglaw", pkg.MIXED, with_oracle=False, profile=True,
                       mixed_inner=pkg.INNER_BICGSTAB)
    s.step(3)
    kt = s.kernel_timings()
    assert kt["refine_residual"]["launches"] >= 2 * 2
    assert kt["refine_update"]["launches"] >= 2
    assert kt["bicg_xr32"]["launches"] >= 1 and kt["jacobi_sweep32"]["launches"] >= 2
    cells = int(np.prod([n - 2 * s.gc for n in s.size]))
    assert kt["bicg_q32"]["bytes_per_launch"] == 4.0 * 3 * cells
    assert kt["refine_residual"]["bytes_per_launch"] == 28.0 * cells


def test_multigrid_inner_solves(make_case):
    """The multigrid-CG inner solves run (their kernels launch, no BiCGStab
    FP32 kernel does) and need a small fraction of the FP64 form's
    iterations for the same stop test."""
    pkg = package()
    spec, s, _ = setup(make_case, "tiny-loglaw", pkg.MIXED, with_oracle=False, profile=True)
    _, f, _ = setup(make_case, "tiny-loglaw", pkg.FP64, with_oracle=False)
    its_m, its_f = [], []
    for n in range(6):
        s.step(1)
        f.step(1)
        if n >= 1:
            its_m.append(s.stats()["it"])
            its_f.append(f.stats()["it"])
            assert s.stats()["err"] <= spec.tol
    kt = s.kernel_timings()
    print("iterations per solve: multigrid-CG", its_m, "FP64 BiCGStab", its_f)
    assert kt["mg_smooth"]["launches"] > 0 and kt["mg_coarse"]["launches"] > 0
    assert kt["mg_pcg"]["launches"] > 0
    assert kt["bicg_xr32"]["launches"] == 0 and kt["jacobi_sweep32"]["launches"] == 0
    assert sum(its_m) * 5 <= sum(its_f)
    # the FP64 residual writes only the FP32 residual for multigrid-CG
    cells = int(np.prod([n - 2 * s.gc for n in s.size]))
    assert kt["refine_residual"]["bytes_per_launch"] == 20.0 * cells


def is_fp32(v):
    return np.array_equal(v, v.astype(np.float32).astype(np.float64))


def test_mixed_stencil_fields_are_fp32(make_case):
    """DALM_MIXED stores the stencil fields U (both time levels), JU and f in
    FP32 and keeps p in FP64: every U, Uold, JU and f value the ABI returns
    is an FP32 number, p is not; the flow kernels' algorithmic bytes are
    those of 4-byte stencil fields."""
    pkg = package()
    spec, s, _ = setup(make_case, "tiny-loglaw", pkg.MIXED, with_oracle=False, profile=True)
    s.step(4)
    for f in ("U", "Uold", "JU", "f"):
        v = s.field(f)
        assert np.all(np.isfinite(v)) and np.any(v != 0), f
        assert is_fp32(v), f"{f} is not stored in FP32"
    assert not is_fp32(s.field("p"))
    kt = s.kernel_timings()
    cells = int(np.prod([n - 2 * s.gc for n in s.size]))
    assert kt["project"]["bytes_per_launch"] == (12 * 4 + 8) * cells
    assert kt["flux_rhs"]["bytes_per_launch"] == (6 * 4 + 8) * cells
    assert kt["mg_smooth"]["bytes_per_launch"] > 0 and kt["mg_pcg"]["bytes_per_launch"] > 0


def test_mixed_fp32_fields_set_and_step(make_case):
    """Setting a field through the ABI rounds it into the FP32 field the
    stages use; stepping from a state set that way equals stepping a solver
    whose state was set identically (deterministic FP32 stages)."""
    pkg = package()
    spec, a, _ = setup(make_case, "tiny-turbine", pkg.MIXED, with_oracle=False)
    _, b, _ = setup(make_case, "tiny-turbine", pkg.MIXED, with_oracle=False)
    U = a.field("U")
    rng = np.random.default_rng(3)
    U2 = U + 1e-3 * rng.standard_normal(U.shape)
    for x in (a, b):
        x.set_state(U2)
    got = a.field("U")
    assert is_fp32(got)
    gc = a.gc
    inner = (slice(gc, -gc), slice(gc, -gc), slice(gc, -gc))
    np.testing.assert_array_equal(got[inner], U2[inner].astype(np.float32).astype(np.float64))
    a.step(3)
    b.step(3)
    for f in ("U", "p", "JU"):
        np.testing.assert_array_equal(a.field(f), b.field(f))
    np.testing.assert_array_equal(a.turbines()[0], b.turbines()[0])


def test_mixed_adjoint_is_refused(make_case):
    pkg = package()
    spec, s, _ = setup(make_case, "tiny-turbine", pkg.MIXED, with_oracle=False)
    with pytest.raises(pkg.DalmError):
        s.power_gradient(1, 2, 1)


TGG_BICG = dict(solver="BiCG", pc="Jacobi", pc_max_it=3, tol=1e-8, max_it=2000)


def test_mixed_with_grid_floor_and_probes(make_case):
    """The FP32 stencil fields carry the turbulence-generating grid (solid
    scaling in the projection), the retracted floor (slip rows of the
    velocity BCs) and the probes: a BiCGStab version of the grid case stays
    within the mixed envelope of the FP64 oracle over ten steps."""
    pkg = package()
    spec, mesh, d, U0, prof = make_case("tiny-tgg", **TGG_BICG)
    s = pkg.Solver(d, precision=pkg.MIXED)
    o = O.CRestatement(d)
    for x in (s, o):
        x.set_state(U0)
    worst = 0.0
    for n in range(11):
        s.step(1)
        o.step(1)
        if n >= 1:
            assert s.stats()["err"] <= spec.tol
        U, Uo = s.field("U"), o.field("U")
        for m in range(3):
            worst = max(worst, rel(U[..., m], Uo[..., m]))
    assert is_fp32(s.field("U"))
    assert worst <= MIXED_ENVELOPE["U"], worst


def test_mixed_output_files(make_case):
    """With write_output the mixed form writes the reference's files from
    its FP32 fields: the inst_ velocity is FP32-valued and close to the FP64
    form's at the same step."""
    import os
    from test_gpu_output import read_binary
    pkg = package()
    out = dict(output_start_time=0.0, output_interval_time=0.002, tavg_start_time=0.003)
    spec, mesh, d, U0, prof = make_case("tiny-turbine", steps=4, **out)
    files = {}
    for prec in (pkg.MIXED, pkg.FP64):
        s = pkg.Solver(d, precision=prec, write_output=True)
        s.set_state(U0)
        s.step(spec.steps + 1)
        s.finalize()
        odir = os.path.join(d, "output")
        names = sorted(n for n in os.listdir(odir) if n.startswith("inst_"))
        assert names, "no inst_ files written"
        files[prec] = read_binary(os.path.join(odir, names[-1]))[4]
        for n in os.listdir(odir):
            os.remove(os.path.join(odir, n))
    um, uf = files[pkg.MIXED]["U"], files[pkg.FP64]["U"]
    assert is_fp32(um)
    assert np.linalg.norm(um - uf) / np.linalg.norm(uf) <= 1e-6


def test_mixed_multi_tile_grid(make_case):
    """The FP32 flow kernels' tile seams (plane tile halos, the y-face
    exchange between rows, the carried x faces at chunk starts): on the
    72x20x100 grid (several k tiles, partial j and k tiles, several i
    chunks; dt = 5e-4, at which the stretched 100-cell columns are stable)
    the mixed form stays within the multi-tile envelope of the FP64 oracle
    over six steps.  Its coarsest multigrid level (9x5x25 cells) is above
    the dense-inverse limit, so this also covers the FP32 BiCGStab inner
    solves.  (On multi-tile grids the reference algorithm
    itself moves by 1.5e-6 in U and 5e-3 in p under a change of summation
    order alone; the bound here is that envelope with room for the FP32
    fields.)"""
    pkg = package()
    spec, mesh, d, U0, prof = make_case("tiny-bicg", n=(72, 20, 100), dt=5e-4)
    s = pkg.Solver(d, precision=pkg.MIXED)
    o = O.CRestatement(d)
    for x in (s, o):
        x.set_state(U0)
    worst = {"U": 0.0, "p": 0.0}
    for n in range(7):
        s.step(1)
        o.step(1)
        if n >= 1:
            assert s.stats()["err"] <= spec.tol
        U, Uo = s.field("U"), o.field("U")
        for m in range(3):
            worst["U"] = max(worst["U"], rel(U[..., m], Uo[..., m]))
        worst["p"] = max(worst["p"], rel(s.field("p"), o.field("p")))
    print("multi-tile mixed vs oracle:", worst)
    assert worst["U"] <= 5e-6 and worst["p"] <= 2e-2, worst


# (case, cells, overrides): z columns of exactly 32 R cells, R = 2 and 4.
# The second grid is 20 tall so that its wall cells (3.5e-3) keep the
# explicit scheme stable at dt = 2.5e-4 (at height 5 the 8.8e-4 wall cells
# under the uniform inflow's wall shear put the Smagorinsky diffusion number
# near 2, and the reference's scheme diverges).
VEC_ROWS = [("tiny-loglaw", (48, 24, 64), {"dt": 5e-4}),
            ("tiny-bicg", (32, 16, 128), {"dt": 2.5e-4, "lengths": (2.0, 1.0, 20.0)})]


@pytest.mark.parametrize("name,n,over", VEC_ROWS, ids=["R2", "R4"])
def test_multigrid_vector_rows(make_case, monkeypatch, capfd, name, n, over):
    """The multigrid-CG inner solve's level-0 kernels on z columns of exactly
    32 R cells, where the SpMV and the smoother take the vector-row layout
    (one warp per row, lane l owning rows R l .. R l + R - 1): every solve
    meets the case's tolerance by FP32 passes alone, in few multigrid-CG
    iterations (an operator that is not K would stall conjugate gradients
    and hand the solve to the FP64 fallback), and U stays within the
    envelope of the FP64 form."""
    pkg = package()
    spec, mesh, d, U0, prof = make_case(name, n=n, **over)
    monkeypatch.setenv("DALM_TRACE_POISSON", "1")
    s = pkg.Solver(d, precision=pkg.MIXED)
    monkeypatch.delenv("DALM_TRACE_POISSON")
    f = pkg.Solver(d, precision=pkg.FP64)
    for x in (s, f):
        if prof is not None:
            x.set_inflow_profile(prof)
        x.set_state(U0)
    worst = 0.0
    for k in range(6):
        s.step(1)
        f.step(1)
        if k >= 1:
            assert s.stats()["err"] <= spec.tol, (k, s.stats())
        U, Uf = s.field("U"), f.field("U")
        worst = max(worst, max(rel(U[..., m], Uf[..., m]) for m in range(3)))
    solves = []
    for line in capfd.readouterr().err.splitlines():
        if "poisson it" in line and "FP32" in line:
            t = line.split("(FP32 ")[1]
            fp32, rest = t.split(" in ")
            passes, fp64 = rest.split(" passes, FP64 ")
            solves.append((int(fp32), int(passes), int(fp64.rstrip(")"))))
    print(n, "FP32 its, passes, FP64 its per solve:", solves, "U vs FP64:", worst)
    assert len(solves) >= 5
    for fp32, passes, fp64 in solves:
        assert fp64 == 0 and passes <= 3 and fp32 <= 8 * max(passes, 1), solves
    assert worst <= MIXED_ENVELOPE["U"], worst
