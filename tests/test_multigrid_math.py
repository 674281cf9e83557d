"""The multigrid preconditioner of the mixed-precision inner solves, on the
CPU: tests/mg_host.cu runs the product's level set-up and V-cycle schedule
with the same __host__ __device__ per-cell functions the CUDA kernels call.

Checks: the finest-level operator K equals -max_diag vol A with A the
reference's pressure matrix (from the oracle, build_A of src/eq.h:701-798);
the V-cycle is a symmetric positive definite operator (conjugate gradients
need one); and conjugate gradients preconditioned by it converge in a few
tens of iterations where plain conjugate gradients need hundreds, on the
stretched meshes of the benchmark configurations."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, casegen
import oracle as O

BUILD = os.path.join(ROOT, "tests", "_build")
SRC = os.path.join(ROOT, "tests", "mg_host.cu")
LIB = os.path.join(BUILD, "libmg_host.so")
CSRC = os.path.join(ROOT, "3dalm_b200", "csrc")
DEPS = [SRC] + [os.path.join(CSRC, f) for f in ("multigrid.cuh", "multigrid_setup.hpp", "common.cuh")]

PD = C.POINTER(C.c_double)
PF = C.POINTER(C.c_float)


def harness():
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(f) for f in DEPS):
        os.makedirs(BUILD, exist_ok=True)
        subprocess.run(["nvcc", "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-Xcompiler", "-fPIC", "-shared", SRC, "-o", LIB], check=True)
    lib = C.CDLL(LIB)
    lib.mgx_create.restype = C.c_void_p
    lib.mgx_create.argtypes = [C.c_int] * 3 + [PD] * 6
    lib.mgx_destroy.argtypes = [C.c_void_p]
    lib.mgx_levels.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    lib.mgx_total.restype = C.c_longlong
    lib.mgx_total.argtypes = [C.c_void_p]
    lib.mgx_apply.argtypes = [C.c_void_p, PF, PF]
    lib.mgx_vcycle.argtypes = [C.c_void_p, PF, PF]
    PI = C.POINTER(C.c_int)
    lib.mgx_vcycle_folded.argtypes = [C.c_void_p, PF, PF]
    lib.mgx_layout.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_longlong)]
    lib.mgx_level_arrays.argtypes = [C.c_void_p, C.c_int, C.c_int, PF, PF]
    lib.mgx_line_table.argtypes = [C.c_void_p, C.c_int, PI, PI, PI, PF]
    return lib


class HostMg:
    def __init__(self, x, y, z, gc=2):
        """x, y, z: cell centres with guide cells (mesh.json); widths by the
        reference's rule (src/io.h:112-125)."""
        cg = casegen()
        self.lib = harness()
        cen = [np.ascontiguousarray(c[gc:-gc]) for c in (x, y, z)]
        wid = [np.ascontiguousarray(cg.spacing(c)[gc:-gc]) for c in (x, y, z)]
        self.keep = cen + wid
        self.n = tuple(len(c) for c in cen)
        self.h = self.lib.mgx_create(*self.n, *[v.ctypes.data_as(PD) for v in self.keep])
        out = (C.c_int * 48)()
        nl = self.lib.mgx_levels(self.h, out)
        self.levels = [tuple(out[3 * l:3 * l + 3]) for l in range(nl)]
        self.total = self.lib.mgx_total(self.h)
        self.off = (8 - gc % 8) % 8
        nk = self.n[2] + 2 * gc
        self.sy = ((self.off + nk + 7) // 8) * 8
        self.shape = (self.n[0] + 2 * gc, self.n[1] + 2 * gc, self.sy)
        self.gc = gc

    def pad(self, v):
        """interior array (n0, n1, n2) -> padded float32 vector"""
        out = np.zeros(self.total, np.float32)
        g = self.gc
        out.reshape(self.shape)[g:-g, g:-g, self.off + g:self.off + g + self.n[2]] = v
        return out

    def unpad(self, p):
        g = self.gc
        return p.reshape(self.shape)[g:-g, g:-g, self.off + g:self.off + g + self.n[2]].astype(np.float64)

    def apply(self, v):
        x = self.pad(v)
        y = np.zeros_like(x)
        self.lib.mgx_apply(self.h, x.ctypes.data_as(PF), y.ctypes.data_as(PF))
        return self.unpad(y)

    def vcycle(self, v):
        f = self.pad(v)
        x = np.zeros_like(f)
        assert self.lib.mgx_vcycle(self.h, f.ctypes.data_as(PF), x.ctypes.data_as(PF)) == 0
        return self.unpad(x)

    def vcycle_folded(self, v):
        f = self.pad(v)
        x = np.zeros_like(f)
        assert self.lib.mgx_vcycle_folded(self.h, f.ctypes.data_as(PF), x.ctypes.data_as(PF)) == 0
        return self.unpad(x)

    def level_arrays(self, l):
        """(cf, w) per axis of level l, FP32 as the device holds them"""
        out = []
        for a in range(3):
            n = self.levels[l][a]
            cf, w = np.zeros(n + 1, np.float32), np.zeros(n, np.float32)
            self.lib.mgx_level_arrays(self.h, l, a, cf.ctypes.data_as(PF), w.ctypes.data_as(PF))
            out.append((cf.astype(np.float64), w.astype(np.float64)))
        return out

    def line_table(self, l):
        """the smoother's z-line factor table of level l, or None"""
        info = np.zeros(4, np.int32)
        PI = C.POINTER(C.c_int)
        self.lib.mgx_line_table(self.h, l, info.ctypes.data_as(PI), None, None, None)
        if not info[0]:
            return None
        n = self.levels[l]
        cx, cy = np.zeros(n[0], np.int32), np.zeros(n[1], np.int32)
        tab = np.zeros(info[2] * info[3] * 32, np.float32)
        self.lib.mgx_line_table(self.h, l, info.ctypes.data_as(PI), cx.ctypes.data_as(PI),
                                cy.ctypes.data_as(PI), tab.ctypes.data_as(PF))
        return {"ky": int(info[1]), "nclass": int(info[2]), "nf": int(info[3]), "cls_x": cx,
                "cls_y": cy, "tab": tab.reshape(info[2], info[3], 32).astype(np.float64)}

    def close(self):
        self.lib.mgx_destroy(self.h)


def pcg(apply, precond, f, rtol, maxit=2000):
    x = np.zeros_like(f)
    r = f.copy()
    z = precond(r)
    p = z.copy()
    rz = np.sum(r * z)
    n0 = np.linalg.norm(r)
    for it in range(1, maxit + 1):
        q = apply(p)
        a = rz / np.sum(p * q)
        x += a * p
        r -= a * q
        if np.linalg.norm(r) <= rtol * n0:
            return x, it
        z = precond(r)
        rz2 = np.sum(r * z)
        p = z + (rz2 / rz) * p
        rz = rz2
    return x, maxit


def test_finest_operator_is_the_reference_matrix(make_case):
    spec, mesh, d, U0, prof = make_case("tiny-loglaw")
    o = O.CRestatement(d)
    A7 = o.matrix()
    md = o.max_diag()
    x, y, z, dx, dy, dz = o.mesh()
    gc = o.size[3]
    mg = HostMg(x, y, z, gc)
    try:
        rng = np.random.default_rng(0)
        v = rng.standard_normal(mg.n)
        vp = np.zeros(A7.shape[:3])
        vp[gc:-gc, gc:-gc, gc:-gc] = v
        a = A7[gc:-gc, gc:-gc, gc:-gc]
        Av = a[..., 0] * v
        for m, (di, dj, dk) in enumerate([(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0),
                                          (0, 0, 1), (0, 0, -1)], start=1):
            Av += a[..., m] * vp[gc + di:vp.shape[0] - gc + di, gc + dj:vp.shape[1] - gc + dj,
                                 gc + dk:vp.shape[2] - gc + dk]
        vol = (dx[:, None, None] * dy[None, :, None] * dz[None, None, :])[gc:-gc, gc:-gc, gc:-gc]
        ref = -md * vol * Av
        got = mg.apply(v)
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        print("levels", mg.levels, "K vs -max_diag vol A:", err)
        assert err < 1e-5
    finally:
        mg.close()


@pytest.mark.parametrize("n", [(40, 20, 20), (48, 20, 72), (64, 32, 16)])
def test_vcycle_is_symmetric_positive_definite(n):
    cg = casegen()
    mesh = cg.make_mesh(*n)
    mg = HostMg(mesh.x, mesh.y, mesh.z, mesh.gc)
    try:
        rng = np.random.default_rng(1)
        u, v = rng.standard_normal(mg.n), rng.standard_normal(mg.n)
        Mu, Mv = mg.vcycle(u), mg.vcycle(v)
        a, b = np.sum(u * Mv), np.sum(Mu * v)
        print(n, "levels", mg.levels, "<u,Mv>", a, "<Mu,v>", b)
        assert abs(a - b) <= 1e-4 * np.sqrt(np.sum(u * Mu) * np.sum(v * Mv))
        assert np.sum(u * Mu) > 0 and np.sum(v * Mv) > 0
    finally:
        mg.close()


@pytest.mark.parametrize("n", [(40, 20, 20), (64, 32, 16), (128, 64, 32)])
def test_preconditioned_cg_converges_in_few_iterations(n):
    cg = casegen()
    mesh = cg.make_mesh(*n)
    mg = HostMg(mesh.x, mesh.y, mesh.z, mesh.gc)
    try:
        rng = np.random.default_rng(2)
        f = rng.standard_normal(mg.n)
        x, it = pcg(mg.apply, mg.vcycle, f, 1e-5)
        res = np.linalg.norm(f - mg.apply(x)) / np.linalg.norm(f)
        print(n, "levels", mg.levels, "multigrid-CG iterations to 1e-5:", it, "residual", res)
        assert it <= 30 and res <= 2e-5
        if n == (64, 32, 16):
            _, it_plain = pcg(mg.apply, lambda r: r, f, 1e-5, 5000)
            print("unpreconditioned CG:", it_plain)
            assert it_plain > 5 * it
    finally:
        mg.close()


# field layout of the factor table (multigrid.cuh, mglf_*)
def _f_q(s): return 5 * s
def _f_a(s): return 5 * s + 1
def _f_g(s): return 5 * s + 2
def _f_xa(s): return 5 * s + 3
def _f_xc(s): return 5 * s + 4
def _f_al(R): return 5 * (R - 1)
def _f_cl(R): return 5 * (R - 1) + 1
def _f_alpha(R, t): return 5 * (R - 1) + (2 if R > 1 else 0) + 2 * t
def _f_gamma(R, t): return _f_alpha(R, t) + 1
def _f_invrb(R): return _f_alpha(R, 5)


def line_solve_table(T, R, d):
    """k_mg_smooth's table path (line_solve_table) lane by lane: T[field][lane],
    d[lane, s] the right-hand sides of rows R lane + s"""
    lanes = np.arange(32)
    e = np.zeros((32, R))
    if R > 1:
        for s in range(R - 1):
            e[:, s] = (d[:, 0] if s == 0 else d[:, s] - T[_f_a(s)] * e[:, s - 1]) * T[_f_q(s)]
        for s in range(R - 3, -1, -1):
            e[:, s] -= T[_f_g(s)] * e[:, s + 1]
        dn = np.roll(e[:, 0], -1)
        dn[31] = 0
        rd = d[:, R - 1] - T[_f_al(R)] * e[:, R - 2] - T[_f_cl(R)] * dn
    else:
        rd = d[:, 0].copy()
    for t in range(5):
        dl = 1 << t
        dm, dp = np.roll(rd, dl), np.roll(rd, -dl)
        dm[lanes < dl] = 0
        dp[lanes + dl >= 32] = 0
        rd = rd + T[_f_alpha(R, t)] * dm + T[_f_gamma(R, t)] * dp
    y = rd * T[_f_invrb(R)]
    ym = np.roll(y, 1)
    ym[0] = 0
    x = np.zeros((32, R))
    x[:, R - 1] = y
    for s in range(R - 1):
        x[:, s] = e[:, s] - T[_f_xa(s)] * ym - T[_f_xc(s)] * y
    return x


@pytest.mark.parametrize("n", [(40, 20, 20), (48, 20, 72), (64, 32, 128), (16, 8, 200)])
def test_line_factor_table_solves_every_column(n):
    """On every level, the smoother's factored z-line solve (the table from
    the product's set-up, applied as the kernel's table path does) matches a
    dense solve of each column's line matrix, for columns of every class."""
    cg = casegen()
    mesh = cg.make_mesh(*n)
    mg = HostMg(mesh.x, mesh.y, mesh.z, mesh.gc)
    rng = np.random.default_rng(3)
    try:
        for l, (n0, n1, nk) in enumerate(mg.levels):
            tb = mg.line_table(l)
            assert tb is not None, "uniform x and y spacing: few classes"
            assert tb["nclass"] <= 16, tb["nclass"]
            R = (nk + 31) // 32
            (cf0, w0), (cf1, w1), (cf2, w2) = mg.level_arrays(l)
            for i in sorted({0, n0 - 1, n0 // 2}):
                for j in sorted({0, n1 - 1, n1 // 2}):
                    az = w0[i] * w1[j]
                    sxy = w1[j] * (cf0[i + 1] + cf0[i]) + w0[i] * (cf1[j + 1] + cf1[j])
                    lo, hi = az * cf2[:nk], az * cf2[1:nk + 1]
                    M = np.diag(w2 * sxy + lo + hi) - np.diag(lo[1:], -1) - np.diag(hi[:-1], 1)
                    rhs = rng.standard_normal(nk)
                    ref = np.linalg.solve(M, rhs)
                    d = np.zeros(32 * R)
                    d[:nk] = rhs
                    T = tb["tab"][tb["cls_x"][i] * tb["ky"] + tb["cls_y"][j]]
                    got = line_solve_table(T, R, d.reshape(32, R)).reshape(-1)[:nk]
                    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
                    assert err < 2e-5, (l, i, j, err)
    finally:
        mg.close()


def test_line_factor_table_falls_back_on_irregular_meshes():
    """x spacing with more distinct cells than the table takes: no table,
    the smoother forms each column's matrix itself."""
    cg = casegen()
    mesh = cg.make_mesh(160, 8, 16)
    x = mesh.x.copy()
    x[2:-2] += 0.01 * np.sin(np.arange(len(x) - 4) ** 1.5)  # every x cell different
    mg = HostMg(x, mesh.y, mesh.z, mesh.gc)
    try:
        assert mg.line_table(0) is None
    finally:
        mg.close()


@pytest.mark.parametrize("n", [(40, 20, 20), (48, 20, 72), (64, 32, 16)])
def test_folded_vcycle_equals_the_plain_one(n):
    """The CUDA executor's two shortcuts keep the V-cycle's operator: the
    restriction without the children of the colour smoothed last (their
    lines were just solved exactly, so their residual is zero) and the
    prolongation applied by the next half-sweep's neighbour reads (the two
    half-sweeps after it overwrite both colours) give the plain V-cycle's
    result up to FP32 rounding (the dropped residuals are rounding-level, and
    a V-cycle over z-merged levels amplifies rounding to ~1e-5), and a
    symmetric positive operator as conjugate gradients need."""
    cg = casegen()
    mesh = cg.make_mesh(*n)
    mg = HostMg(mesh.x, mesh.y, mesh.z, mesh.gc)
    try:
        rng = np.random.default_rng(4)
        for _ in range(2):
            f = rng.standard_normal(mg.n)
            a, b = mg.vcycle(f), mg.vcycle_folded(f)
            err = np.linalg.norm(a - b) / np.linalg.norm(a)
            print(n, "levels", mg.levels, "folded vs plain V-cycle:", err)
            assert err < 1e-4
        u, v = rng.standard_normal(mg.n), rng.standard_normal(mg.n)
        Mu, Mv = mg.vcycle_folded(u), mg.vcycle_folded(v)
        assert abs(np.sum(u * Mv) - np.sum(Mu * v)) <= 1e-4 * np.sqrt(np.sum(u * Mu) * np.sum(v * Mv))
        assert np.sum(u * Mu) > 0 and np.sum(v * Mv) > 0
    finally:
        mg.close()


@pytest.mark.parametrize("n", [(40, 20, 20), (64, 32, 128), (48, 20, 72)])
def test_rows_start_on_32_byte_boundaries(n):
    """The smoother's vector path loads each lane's rows with float2/float4
    accesses: it relies on every level's row start (k = 0 of an interior
    row) and both strides being multiples of 8 elements, which the storage
    layout (Grid::make: guide cells shifted so that k = 0 is aligned, rows
    padded to 8) gives on every level."""
    cg = casegen()
    mesh = cg.make_mesh(*n)
    mg = HostMg(mesh.x, mesh.y, mesh.z, mesh.gc)
    try:
        out = (C.c_longlong * 3)()
        for l in range(len(mg.levels)):
            mg.lib.mgx_layout(mg.h, l, out)
            assert out[0] % 8 == 0 and out[1] % 8 == 0 and out[2] % 8 == 0, (l, list(out))
    finally:
        mg.close()
