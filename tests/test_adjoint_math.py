"""The discrete adjoint's arithmetic on the CPU, against the oracle.

tests/adjoint_host.cu runs the product's adjoint building blocks
(3dalm_b200/csrc/adjoint_cell.cuh, the same __host__ __device__ functions
the CUDA kernels call) in plain host loops.  Each transposed stage is
checked with the dot-product identity  <lambda, dG delta> = <dG^T lambda,
delta>, where dG delta is a central finite difference of the oracle's own
forward stage; the last test chains the stages over several time steps
(the orchestration the device code follows) and compares the gradient of
the mean turbine power with central finite differences of the oracle's
time stepping.  Van Albada limiter throughout (smooth convection)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from conftest import ROOT, casegen
import oracle as O

BUILD = os.path.join(ROOT, "tests", "_build")
SRC = os.path.join(ROOT, "tests", "adjoint_host.cu")
LIB = os.path.join(BUILD, "libadjoint_host.so")
CSRC = os.path.join(ROOT, "3dalm_b200", "csrc")
DEPS = [SRC] + [os.path.join(CSRC, f) for f in
                ("adjoint_cell.cuh", "dual.cuh", "alm.cuh", "flow.cuh", "common.cuh")]

PD = C.POINTER(C.c_double)
PPD = C.POINTER(PD)


def harness():
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(f) for f in DEPS):
        os.makedirs(BUILD, exist_ok=True)
        subprocess.run(["nvcc", "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-shared",
                        SRC, "-o", LIB], check=True)
    lib = C.CDLL(LIB)
    lib.hx_create.restype = C.c_void_p
    lib.hx_create.argtypes = [C.c_int] * 4 + [PD] * 6 + [C.c_double] * 3 + [C.c_int, PD]
    lib.hx_total.restype = C.c_longlong
    lib.hx_total.argtypes = [C.c_void_p]
    lib.hx_set_alm.argtypes = ([C.c_void_p] + [C.c_int] * 5 + [C.c_double] * 3 + [PD] * 4 +
                               [C.POINTER(C.c_int)] + [PD] * 7)
    lib.hx_alm_points.argtypes = [C.c_void_p, PPD, C.c_double, PD, PD, PD, PD]
    lib.hx_adj_alm.argtypes = [C.c_void_p, PPD, PPD, C.c_double, C.c_double, PPD, PD]
    lib.hx_adj_velocity_bc.argtypes = [C.c_void_p, PPD, PPD, PPD]
    lib.hx_adj_project.restype = C.c_double
    lib.hx_adj_project.argtypes = [C.c_void_p, PPD, PPD, PD]
    lib.hx_adj_faces.argtypes = [C.c_void_p, PPD, PD, PPD]
    lib.hx_adj_predict.argtypes = [C.c_void_p] + [PPD] * 6
    lib.hx_destroy.argtypes = [C.c_void_p]
    return lib


def _p(a):
    return a.ctypes.data_as(PD)


def _pp(fields):
    arr = (PD * len(fields))(*[_p(f) for f in fields])
    arr.keep = fields  # the arrays must outlive the call
    return arr


class Layout:
    """The product's padded SoA layout (Grid::make in common.cuh)."""

    def __init__(self, nx, ny, nz, gc):
        self.n = (nx, ny, nz)
        self.gc = gc
        self.off = (8 - gc % 8) % 8
        self.sy = ((self.off + nz + 7) // 8) * 8
        self.total = self.sy * ny * nx

    def to_soa(self, a):
        nx, ny, nz = self.n
        comps = [a[..., m] for m in range(3)] if a.ndim == 4 else [a]
        out = []
        for f in comps:
            v = np.zeros(self.total)
            v.reshape(nx, ny, self.sy)[:, :, self.off:self.off + nz] = f
            out.append(v)
        return out

    def from_soa(self, fields):
        nx, ny, nz = self.n
        comps = [f.reshape(nx, ny, self.sy)[:, :, self.off:self.off + nz].copy() for f in fields]
        return np.stack(comps, axis=-1) if len(comps) == 3 else comps[0]

    def zeros(self, nc=3):
        return [np.zeros(self.total) for _ in range(nc)]


class Setup:
    """Oracle + harness on one case, van Albada limiter, tight Poisson."""

    def __init__(self, make_case, name="tiny-loglaw", **over):
        cg = casegen()
        self.spec, self.mesh, self.dir, self.U0, self.prof = make_case(name, **over)
        self.o = O.CRestatement(self.dir)
        self.o.set_limiter(1)
        if self.prof is not None:
            self.o.set_inflow_profile(self.prof)
        self.o.set_poisson(20000, 1e-13)
        self.o.set_state(self.U0)
        nx, ny, nz, gc = self.o.size
        self.lay = Layout(nx, ny, nz, gc)
        self.x, self.y, self.z, self.dx, self.dy, self.dz = self.o.mesh()
        self.dt = self.o.stats()["dt"]
        self.md = self.o.max_diag()
        case = O.Case(self.dir)
        self.case = case
        vol = self.dx[:, None, None] * self.dy[None, :, None] * self.dz[None, None, :]
        filt = np.zeros((nx, ny, nz))
        filt[gc:-gc, gc:-gc, gc:-gc] = (case.cs * np.cbrt(vol[gc:-gc, gc:-gc, gc:-gc])) ** 2
        self.filter2 = self.lay.to_soa(filt)[0]
        self.vol = vol
        self.lib = harness()
        self.keep = [self.x, self.y, self.z, self.dx, self.dy, self.dz, self.filter2]
        self.ctx = self.lib.hx_create(nx, ny, nz, gc, *[_p(v) for v in self.keep[:6]], case.re,
                                      self.dt, self.md, 1, _p(self.filter2))
        assert self.lib.hx_total(self.ctx) == self.lay.total
        if case.turbines:
            self._set_alm()

    def _set_alm(self, yaw=None, pitch=None, omega=None):
        case = self.case
        T = len(case.turbines)
        wt = case.wt
        r, dr, ch, tw, cd, cl, atk = self.o.point_tables()
        base = np.array([t["base"] for t in case.turbines], dtype=np.float64)
        rc = np.tile(np.array([-float(wt["overhang"]), 0.0, float(wt["tower"])]), (T, 1))
        form = np.array([t["formula"] for t in case.turbines], dtype=np.float64)
        om = np.array([t["omega"] for t in case.turbines], dtype=np.float64)
        typ = np.array([O.EULER[t["type"]] for t in case.turbines], dtype=np.int32)
        pw = case.projection_width
        self.alm_keep = [base, rc, form, om, typ, r, dr, ch, tw, cd, cl, atk]
        self.T = T
        self.omega = om
        self.ap = len(r)
        self.lib.hx_set_alm(self.ctx, T, int(wt["number of blades"]) * case.points_per_blade,
                            case.points_per_blade, int(wt["number of blades"]), len(atk),
                            pw * pw, 1.0 / (pw * np.sqrt(np.pi)) ** 3, 40.0 * pw * pw,
                            _p(base), _p(rc), _p(form), _p(om),
                            typ.ctypes.data_as(C.POINTER(C.c_int)),
                            *[_p(np.ascontiguousarray(v)) for v in (r, dr, ch, tw, cd, cl, atk)])

    def base_params(self):
        yaw = np.array([t["formula"][3] * 180 / np.pi for t in self.case.turbines])
        return yaw, np.zeros(self.T), self.omega.copy()

    def close(self):
        self.lib.hx_destroy(self.ctx)


def interior_mask(lay):
    nx, ny, nz = lay.n
    gc = lay.gc
    m = np.zeros((nx, ny, nz), bool)
    m[gc:-gc, gc:-gc, gc:-gc] = True
    return m


def slab_mask(lay):
    """guide cells of the six face slabs (not edges or corners)"""
    nx, ny, nz = lay.n
    gc = lay.gc
    ii = np.zeros((nx, ny, nz), bool)
    I, J, K = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    inx = (I >= gc) & (I < nx - gc)
    iny = (J >= gc) & (J < ny - gc)
    inz = (K >= gc) & (K < nz - gc)
    ii |= (~inx) & iny & inz
    ii |= inx & (~iny) & inz
    ii |= inx & iny & (~inz)
    return ii


def active_faces(lay):
    """[3] masks of the JU faces the projection changes (non-override faces
    with interior tangential indices, normal index in [gc-1, N-gc-1])"""
    nx, ny, nz = lay.n
    gc = lay.gc
    I, J, K = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    inx = (I >= gc) & (I < nx - gc)
    iny = (J >= gc) & (J < ny - gc)
    inz = (K >= gc) & (K < nz - gc)
    fx = (I >= gc) & (I <= nx - gc - 1) & iny & inz
    fy = (J >= gc) & (J <= ny - gc - 2) & inx & inz
    fz = (K >= gc) & (K <= nz - gc - 2) & inx & iny
    return [fx, fy, fz]


def rel_gap(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


@pytest.fixture
def setup(make_case):
    s = Setup(make_case)
    yield s
    s.close()


def test_predictor_transpose(setup):
    """U* = U^n + dt(-conv + diff + f) on the interior (stage 0)."""
    s, o, lay = setup, setup.o, setup.lay
    rng = np.random.default_rng(1)
    o.step(3)
    V, JU, f = o.field("U"), o.field("JU"), o.field("f")
    inside = interior_mask(lay)
    dV = rng.standard_normal(V.shape) * 1e-2
    dV[~(inside | slab_mask(lay))] = 0
    dJ = rng.standard_normal(JU.shape) * 1e-4
    df = rng.standard_normal(f.shape) * 1e-2
    df[~inside] = 0
    lam = rng.standard_normal(V.shape)
    lam[~inside] = 0

    def G(eps):
        o.set_state(V + eps * dV, JU + eps * dJ, None, flags=0)
        o.set_field("f", f + eps * df)
        o.stage(0)
        return o.field("U")

    h = 1e-6
    fd = np.sum(lam * (G(h) - G(-h))) / (2 * h)
    aV, aJU, af = lay.zeros(), lay.zeros(), lay.zeros()
    s.lib.hx_adj_predict(s.ctx, _pp(lay.to_soa(V)), _pp(lay.to_soa(JU)), _pp(lay.to_soa(lam)),
                         _pp(aV), _pp(aJU), _pp(af))
    # aV holds the identity term a_us too (U* = U^n + ...): part of the map
    adj = (np.sum(lay.from_soa(aV) * dV) + np.sum(lay.from_soa(aJU) * dJ) +
           np.sum(lay.from_soa(af) * df))
    print("predictor: fd", fd, "adjoint", adj)
    assert rel_gap(fd, adj) < 1e-7


def test_velocity_bc_transpose(setup):
    """apply_Ubc after the projection: guide cells from the projected
    interior and U^n (stage 3 with p = 0 leaves the interior unchanged)."""
    s, o, lay = setup, setup.o, setup.lay
    rng = np.random.default_rng(2)
    o.step(3)
    Un = o.field("U")
    o.step(1)
    U1 = o.field("U")
    inside, slabs = interior_mask(lay), slab_mask(lay)
    dV = rng.standard_normal(Un.shape) * 1e-2
    dV[~(inside | slabs)] = 0
    dU = rng.standard_normal(Un.shape) * 1e-2
    dU[~inside] = 0
    lam = rng.standard_normal(Un.shape)
    lam[~slabs] = 0
    p0 = np.zeros(o.field("p").shape)

    def H(eps):
        V = Un + eps * dV
        U = U1 + eps * dU
        U[~inside] = V[~inside]  # before the BC the guide cells hold U^n's
        o.set_field("U", U)
        o.set_field("Uold", V)
        o.set_field("p", p0)
        o.stage(3)
        return o.field("U")

    h = 1e-6
    fd = np.sum(lam * (H(h) - H(-h))) / (2 * h)
    aU = lay.to_soa(lam)
    aV = lay.zeros()
    s.lib.hx_adj_velocity_bc(s.ctx, _pp(lay.to_soa(Un)), _pp(aU), _pp(aV))
    aUa = lay.from_soa(aU)
    assert np.all(aUa[slabs] == 0)
    adj = np.sum(aUa * dU) + np.sum(lay.from_soa(aV) * dV)
    print("velocity bc: fd", fd, "adjoint", adj)
    assert rel_gap(fd, adj) < 1e-7


def test_projection_transpose(setup):
    """U^{n+1}, JU^{n+1} from U*, JU*, p (apply_pbc + project_p): the
    adjoint pressure right-hand side times the cell volume is the adjoint
    of p on the interior."""
    s, o, lay = setup, setup.o, setup.lay
    rng = np.random.default_rng(3)
    o.step(3)
    U, JU, p = o.field("U"), o.field("JU"), o.field("p")
    inside = interior_mask(lay)
    act = active_faces(lay)
    dp = rng.standard_normal(p.shape) * 1e-3
    dp[~inside] = 0
    lu = rng.standard_normal(U.shape)
    lu[~inside] = 0
    lj = rng.standard_normal(JU.shape)
    for a in range(3):
        lj[..., a][~act[a]] = 0

    def K(eps):
        o.set_field("U", U)
        o.set_field("Uold", U)
        o.set_field("JU", JU)
        o.set_field("p", p + eps * dp)
        o.stage(3)
        return o.field("U"), o.field("JU")

    h = 1.0  # the map is affine in p
    (u1, j1), (u0, j0) = K(h), K(-h)
    fd = (np.sum(lu * (u1 - u0)) + np.sum(lj * (j1 - j0))) / (2 * h)
    rhs = np.zeros(lay.total)
    s.lib.hx_adj_project(s.ctx, _pp(lay.to_soa(lu)), _pp(lay.to_soa(lj)), _p(rhs))
    lp = lay.from_soa([rhs]) * s.vol
    adj = np.sum(lp * dp)
    print("projection: fd", fd, "adjoint", adj)
    assert rel_gap(fd, adj) < 1e-7


def test_poisson_operator_symmetrises(setup):
    """A = M^-1 L / max_diag with L symmetric and M = diag(cell volume)."""
    s, o, lay = setup, setup.o, setup.lay
    A, idx = poisson_matrix(o)
    nx, ny, nz = lay.n
    gc = lay.gc
    vol = s.vol[gc:-gc, gc:-gc, gc:-gc].ravel()
    MA = sp.diags(vol) @ A
    asym = abs(MA - MA.T).max()
    print("max |MA - (MA)^T|", asym, "max |MA|", abs(MA).max())
    assert asym <= 1e-12 * abs(MA).max()


def test_faces_transpose(setup):
    """b and JU* from U* (interpolate_JU + apply_JUbc + calc_poisson_rhs);
    the adjoint of b enters as y = lambda_b / vol."""
    s, o, lay = setup, setup.o, setup.lay
    rng = np.random.default_rng(4)
    o.step(3)
    U = o.field("U")
    inside, slabs = interior_mask(lay), slab_mask(lay)
    act = active_faces(lay)
    dU = rng.standard_normal(U.shape) * 1e-2
    dU[~(inside | slabs)] = 0
    lb = rng.standard_normal(o.field("p").shape)
    lb[~inside] = 0
    lj = rng.standard_normal(U.shape)
    for a in range(3):
        lj[..., a][~act[a]] = 0

    def F(eps):
        o.set_field("U", U + eps * dU)
        o.stage(1)
        return o.field("b"), o.field("JU")

    h = 1.0  # the map is affine in U*
    (b1, j1), (b0, j0) = F(h), F(-h)
    fd = (np.sum(lb * (b1 - b0)) + np.sum(lj * (j1 - j0))) / (2 * h)
    y = lay.to_soa(np.where(inside, lb / s.vol, 0.0))[0]
    aus = lay.zeros()
    s.lib.hx_adj_faces(s.ctx, _pp(lay.to_soa(lj)), _p(y), _pp(aus))
    adj = np.sum(lay.from_soa(aus) * dU)
    print("faces: fd", fd, "adjoint", adj)
    assert rel_gap(fd, adj) < 1e-7


def test_actuator_line_transpose(setup):
    """Force field and weighted power from U and the turbine parameters."""
    s, o, lay = setup, setup.o, setup.lay
    rng = np.random.default_rng(5)
    o.step(4)
    U = o.field("U")
    inside = interior_mask(lay)
    dU = rng.standard_normal(U.shape) * 1e-2
    dU[~inside] = 0
    lf = rng.standard_normal(U.shape)
    lf[~inside] = 0
    yaw0, pitch0, om0 = s.base_params()
    dth = rng.standard_normal((3, s.T))
    weight = 0.37
    t = o.stats()["step"] * s.dt

    def A(eps):
        o.set_turbine_params(yaw0 + eps * dth[0], pitch0 + eps * dth[1], om0 + eps * dth[2])
        o.set_field("U", U + eps * dU)
        o.stage(4)
        tq, _ = o.turbines()
        return o.field("f"), np.sum(tq * np.abs(om0 + eps * dth[2]))

    h = 1e-6
    (f1, p1), (f0, p0) = A(h), A(-h)
    fd = (np.sum(lf * (f1 - f0)) + weight * (p1 - p0)) / (2 * h)
    aU = lay.zeros()
    grad = np.zeros(3 * s.T)
    s.lib.hx_adj_alm(s.ctx, _pp(lay.to_soa(U)), _pp(lay.to_soa(lf)), t, weight, _pp(aU), _p(grad))
    adj = np.sum(lay.from_soa(aU) * dU) + np.sum(grad.reshape(s.T, 3).T * dth)
    print("actuator line: fd", fd, "adjoint", adj)
    assert rel_gap(fd, adj) < 1e-6


# ------------------------------------------------------------- full chain


def poisson_matrix(o):
    A7 = o.matrix()
    nx, ny, nz, gc = o.size
    ni, nj, nk = nx - 2 * gc, ny - 2 * gc, nz - 2 * gc
    idx = np.arange(ni * nj * nk).reshape(ni, nj, nk)
    a = A7[gc:-gc, gc:-gc, gc:-gc]
    rows, cols, vals = [idx.ravel()], [idx.ravel()], [a[..., 0].ravel()]
    offs = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    for m, (di, dj, dk) in enumerate(offs, start=1):
        sl = (slice(max(0, -di), ni - max(0, di)), slice(max(0, -dj), nj - max(0, dj)),
              slice(max(0, -dk), nk - max(0, dk)))
        sl2 = (slice(max(0, di), ni - max(0, -di)), slice(max(0, dj), nj - max(0, -dj)),
               slice(max(0, dk), nk - max(0, -dk)))
        rows.append(idx[sl].ravel())
        cols.append(idx[sl2].ravel())
        vals.append(a[sl][..., m].ravel())
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(idx.size,) * 2)
    return A, idx


def run_objective(s, params, n_steps, t0):
    """J = mean over steps t0..n_steps of the total power, by the oracle."""
    o = O.CRestatement(s.dir)
    o.set_limiter(1)
    if s.prof is not None:
        o.set_inflow_profile(s.prof)
    o.set_poisson(20000, 1e-13)
    o.set_turbine_params(*params)
    o.set_state(s.U0)
    o.step(1)  # step 0: no integration
    J = 0.0
    for n in range(1, n_steps + 1):
        o.step(1)
        if n >= t0:
            tq, _ = o.turbines()
            J += np.sum(tq * np.abs(params[2]))
    o.close()
    return J / (n_steps - t0 + 1)


def adjoint_gradient(s, n_steps, t0):
    """Reverse sweep over the oracle's trajectory with the harness stages."""
    o, lay, lib = s.o, s.lay, s.lib
    o.set_state(s.U0)
    o.step(1)
    traj_U, traj_JU = {}, {}
    for n in range(1, n_steps + 1):
        traj_U[n], traj_JU[n] = o.field("U"), o.field("JU")
        o.step(1)
    traj_U[n_steps + 1] = o.field("U")
    A, idx = poisson_matrix(o)
    solve = spla.factorized(A.tocsc())
    gc = lay.gc
    c = 1.0 / (n_steps - t0 + 1)
    aU, aJU, af = lay.zeros(), lay.zeros(), lay.zeros()
    grad = np.zeros(3 * s.T)
    for n in range(n_steps, 0, -1):
        U1 = _pp(lay.to_soa(traj_U[n + 1]))
        lib.hx_adj_alm(s.ctx, U1, _pp(af), n * s.dt, c if n >= t0 else 0.0, _pp(aU), _p(grad))
        V = lay.to_soa(traj_U[n])
        aV = lay.zeros()
        lib.hx_adj_velocity_bc(s.ctx, _pp(V), _pp(aU), _pp(aV))
        rhs = np.zeros(lay.total)
        lib.hx_adj_project(s.ctx, _pp(aU), _pp(aJU), _p(rhs))
        r = lay.from_soa([rhs])[gc:-gc, gc:-gc, gc:-gc].ravel()
        y = np.zeros(lay.n)
        y[gc:-gc, gc:-gc, gc:-gc] = solve(r).reshape(idx.shape)
        ys = lay.to_soa(y)[0]
        lib.hx_adj_faces(s.ctx, _pp(aJU), _p(ys), _pp(aU))
        nJU, nf = lay.zeros(), lay.zeros()
        lib.hx_adj_predict(s.ctx, _pp(V), _pp(lay.to_soa(traj_JU[n])), _pp(aU), _pp(aV),
                           _pp(nJU), _pp(nf))
        aU, aJU, af = aV, nJU, nf
    # the forces of step 1 came from the actuator line at t = 0 on U^1
    lib.hx_adj_alm(s.ctx, _pp(lay.to_soa(traj_U[1])), _pp(af), 0.0, 0.0, _pp(aU), _p(grad))
    return grad.reshape(s.T, 3)


def test_gradient_matches_finite_differences(setup):
    """d(mean power)/d(yaw, pitch, rotor speed) over 6 steps (window 3-6)."""
    s = setup
    n_steps, t0 = 6, 3
    g = adjoint_gradient(s, n_steps, t0)
    base = s.base_params()
    h = 1e-5
    fd = np.zeros((s.T, 3))
    for w in range(s.T):
        for q in range(3):
            pp = [v.copy() for v in base]
            pm = [v.copy() for v in base]
            pp[q][w] += h
            pm[q][w] -= h
            fd[w, q] = (run_objective(s, pp, n_steps, t0) - run_objective(s, pm, n_steps, t0)) / (2 * h)
    err = np.abs(g - fd)
    print("adjoint\n", g, "\nfinite differences\n", fd, "\nrelative", err / np.abs(fd))
    assert np.all(err <= 1e-4 * np.abs(fd) + 1e-6 * np.abs(fd).max())
