// Geometric multigrid for the pressure equation in FP32: the preconditioner
// of the conjugate-gradient inner solves of DALM_MIXED.
//
// The pressure operator of build_A (src/eq.h:701-798) is A = M^-1 L /
// max_diag with M = diag(cell volume) and L the symmetric finite-volume
// Laplacian: each face between cells c and c' couples them with area / dist
// (dist = distance of the two centres), the x+ outlet face couples the last
// cell to p = 0 at area / (dx / 2), the inflow and wall faces are closed.
// The inner solve A e = r is therefore K e = f with K = -L (symmetric
// positive definite) and f = -max_diag vol r.  Each level stores K
// matrix-free as one conductance per face and axis (cf[a][f + 1] couples
// cells f and f + 1 along axis a; cf[a][0] and cf[a][n] are the boundary
// faces) and the cell widths (the face areas).  The wall-stretched z
// spacing makes the coupling strongly anisotropic, and in opposite senses
// at the bottom (z dominates by ~400x) and the top (x, y dominate), which
// point smoothers cannot handle; the robust combination used here is
// z-line relaxation with semi-coarsening in x and y: coarser levels merge
// pairs of cells along x and y while their counts are even and at least 4,
// and along z only once neither can, down to the first level of at most
// MG_COARSE_TARGET cells.  Each level's operator is the same
// finite-volume Laplacian on the merged cells (centre = mean of the
// children's centres, width = sum).  Transfers are piecewise constant: the
// restriction sums the children's residuals (K is in integrated form), the
// prolongation copies the coarse correction.  The smoother solves every
// z-column exactly (zebra Gauss-Seidel over columns coloured (i + j) % 2),
// colour 0 then 1 before the coarse correction and 1 then 0 after, mg_nu
// (level) times each, and the
// coarsest level is solved exactly with its precomputed inverse: the
// V-cycle is a symmetric positive definite linear operator, as conjugate
// gradients require of a preconditioner.
//
// Everything here is __host__ __device__ so that host-side checks run the
// kernels' arithmetic.
#pragma once

#include "common.cuh"

#ifndef DALM_HD
#define DALM_HD __host__ __device__ __forceinline__
#endif

namespace dalm {

constexpr int MG_MAX_LEVELS = 24;
constexpr int MG_MAX_COARSE = 1024;   // cells of the coarsest level at most (dense inverse)
constexpr int MG_COARSE_TARGET = 512;  // coarsening stops at the first level this small

struct MgLevel {
    Grid g;              // storage: level 0 is the solver's grid, coarser levels gc = 1
    int n[3];            // interior cells per axis
    int fac[3];          // children per coarse cell along each axis (1 or 2); finest: 1
    const float *cf[3];  // face conductances, [n + 1]
    const float *w[3];   // cell widths, [n]
    // z-line factor table (or null): the line matrix of column (i, j) depends
    // on (i, j) only through (w0[i], cf0[i + 1], cf0[i]) and (w1[j], cf1[j + 1],
    // cf1[j]); lcls[0][i] and lcls[1][j] number those triples, and column
    // (i, j) uses class lcls[0][i] * lky + lcls[1][j] of ltab (layout: mglf_*)
    const int *lcls[2] = {nullptr, nullptr};
    int lky = 0;
    const float *ltab = nullptr;
    DALM_HD long long at(int i, int j, int k) const {
        return g.at(i + g.gc, j + g.gc, k + g.gc);
    }
    DALM_HD long long cells() const { return (long long)n[0] * n[1] * n[2]; }
};

// Field layout of the z-line factor table, per class [field][lane] (32
// lanes): the partition-method line solve of k_mg_smooth with every
// quantity that depends only on the line matrix precomputed, for R rows
// per lane (rows R l + s):
//   Q(s), A(s)   forward sweep  e_s = (d_s - A(s) e_{s-1}) Q(s)   (s < R-1)
//   G(s)         back sweep     e_s -= G(s) e_{s+1}
//   XA(s), XC(s) expansion      x_s = e_s - XA(s) y_{l-1} - XC(s) y_l
//   AL, CL       the last row's couplings (R > 1)
//   ALPHA(t), GAMMA(t)  cyclic-reduction step t (stride 2^t) multipliers
//   INVRB        1 / the reduced diagonal after the reduction
DALM_HD constexpr int mglf_q(int s) { return 5 * s; }
DALM_HD constexpr int mglf_a(int s) { return 5 * s + 1; }
DALM_HD constexpr int mglf_g(int s) { return 5 * s + 2; }
DALM_HD constexpr int mglf_xa(int s) { return 5 * s + 3; }
DALM_HD constexpr int mglf_xc(int s) { return 5 * s + 4; }
DALM_HD constexpr int mglf_al(int R) { return 5 * (R - 1); }
DALM_HD constexpr int mglf_cl(int R) { return 5 * (R - 1) + 1; }
DALM_HD constexpr int mglf_alpha(int R, int t) { return 5 * (R - 1) + (R > 1 ? 2 : 0) + 2 * t; }
DALM_HD constexpr int mglf_gamma(int R, int t) { return mglf_alpha(R, t) + 1; }
DALM_HD constexpr int mglf_invrb(int R) { return mglf_alpha(R, 5); }
DALM_HD constexpr int mglf_count(int R) { return mglf_invrb(R) + 1; }

// Sum over the faces of cell (i,j,k) of area * conductance * x_neighbour
// (x = 0 beyond the boundary, where the guide cells hold zeros), and the
// diagonal sum of area * conductance: (K x)_c = diag x_c - nb.
DALM_HD float mg_neighbours(const MgLevel &L, const float *x, int i, int j, int k,
                            float &diag) {
    const long long c = L.at(i, j, k);
    const long long sx = L.g.sx, sy = L.g.sy;
    const float ax = L.w[1][j] * L.w[2][k], ay = L.w[0][i] * L.w[2][k],
                az = L.w[0][i] * L.w[1][j];
    const float xe = L.cf[0][i + 1], xw = L.cf[0][i];
    const float yn = L.cf[1][j + 1], ys = L.cf[1][j];
    const float zt = L.cf[2][k + 1], zb = L.cf[2][k];
    diag = ax * (xe + xw) + ay * (yn + ys) + az * (zt + zb);
    return ax * (xe * x[c + sx] + xw * x[c - sx]) + ay * (yn * x[c + sy] + ys * x[c - sy]) +
           az * (zt * x[c + 1] + zb * x[c - 1]);
}

DALM_HD float mg_apply(const MgLevel &L, const float *x, int i, int j, int k) {
    float d;
    float nb = mg_neighbours(L, x, i, j, k, d);
    return d * x[L.at(i, j, k)] - nb;
}

// z-line Gauss-Seidel: column (i,j) solved exactly along k with its x and
// y neighbours' current values on the right; columns coloured (i + j) % 2.
// Row k of the column:  -lo x_{k-1} + b x_k - hi x_{k+1} = d_k.
DALM_HD void mg_zline_coef(const MgLevel &L, int i, int j, int k, float &lo, float &hi,
                           float &b) {
    const float wi = L.w[0][i], wj = L.w[1][j];
    const float az = wi * wj, ax = wj * L.w[2][k], ay = wi * L.w[2][k];
    lo = az * L.cf[2][k];
    hi = az * L.cf[2][k + 1];
    b = ax * (L.cf[0][i + 1] + L.cf[0][i]) + ay * (L.cf[1][j + 1] + L.cf[1][j]) + lo + hi;
}

// d_k: the right-hand side plus the x and y neighbours (zero_start: they
// are still zero)
DALM_HD float mg_zline_rhs(const MgLevel &L, const float *x, const float *f, int i, int j, int k,
                           bool zero_start) {
    const long long c = L.at(i, j, k);
    if (zero_start) return f[c];
    const float wi = L.w[0][i], wj = L.w[1][j];
    const float ax = wj * L.w[2][k], ay = wi * L.w[2][k];
    return f[c] + ax * (L.cf[0][i + 1] * x[c + L.g.sx] + L.cf[0][i] * x[c - L.g.sx]) +
           ay * (L.cf[1][j + 1] * x[c + L.g.sy] + L.cf[1][j] * x[c - L.g.sy]);
}

// Thomas algorithm on column (i,j): d[k * s] holds d_k on entry and x_k on
// exit, cp[k * s] is scratch.  The rows are diagonally dominant, so the
// elimination needs no pivoting.
DALM_HD void mg_thomas(const MgLevel &L, int i, int j, float *d, float *cp, int s) {
    float prev_c = 0.f, prev_d = 0.f;
    for (int k = 0; k < L.n[2]; k++) {
        float lo, hi, b;
        mg_zline_coef(L, i, j, k, lo, hi, b);
        const float m = b - lo * prev_c;
        prev_c = hi / m;
        prev_d = (d[k * s] + lo * prev_d) / m;
        cp[k * s] = prev_c;
        d[k * s] = prev_d;
    }
    float next = 0.f;
    for (int k = L.n[2] - 1; k >= 0; k--) {
        next = d[k * s] + cp[k * s] * next;
        d[k * s] = next;
    }
}

// the whole line update in place in x (cp: scratch of the level's layout);
// the kernels stage the column in shared memory instead
DALM_HD void mg_zline_column(const MgLevel &L, float *x, const float *f, float *cp, int i, int j,
                             bool zero_start) {
    const long long c0 = L.at(i, j, 0);
    for (int k = 0; k < L.n[2]; k++) x[c0 + k] = mg_zline_rhs(L, x, f, i, j, k, zero_start);
    mg_thomas(L, i, j, x + c0, cp + c0, 1);
}

// column number n of colour `color` ((i + j) % 2): false when past the end
DALM_HD bool mg_color_column(const MgLevel &L, long long n, int color, int &i, int &j) {
    const int njh = (L.n[1] + 1) / 2;
    if (n >= (long long)njh * L.n[0]) return false;
    i = (int)(n / njh);
    j = 2 * (int)(n % njh) + ((i + color) & 1);
    return j < L.n[1];
}

// coarse cell (I,J,K): the sum of its children's residuals f - K x, leaving
// out the children of colour `skip` ((i + j) % 2; -1: none), whose residual
// the caller knows to be zero
DALM_HD float mg_restrict_sum(const MgLevel &F, const MgLevel &C, const float *x, const float *f,
                              int I, int J, int K, int skip = -1) {
    float s = 0;
    for (int a = 0; a < C.fac[0]; a++)
        for (int b = 0; b < C.fac[1]; b++) {
            const int i = I * C.fac[0] + a, j = J * C.fac[1] + b;
            if (((i + j) & 1) == skip) continue;
            for (int c = 0; c < C.fac[2]; c++) {
                const int k = K * C.fac[2] + c;
                s += f[F.at(i, j, k)] - mg_apply(F, x, i, j, k);
            }
        }
    return s;
}

DALM_HD void mg_restrict_cell(const MgLevel &F, const MgLevel &C, const float *x, const float *f,
                              float *fc, int I, int J, int K) {
    fc[C.at(I, J, K)] = mg_restrict_sum(F, C, x, f, I, J, K);
}

// fine cell (i,j,k) += its parent's correction
DALM_HD void mg_prolong_cell(const MgLevel &F, const MgLevel &C, float *x, const float *xc, int i,
                             int j, int k) {
    x[F.at(i, j, k)] += xc[C.at(i / C.fac[0], j / C.fac[1], k / C.fac[2])];
}

// coarsest level: row r of x = K^-1 f with the inverse dense, row-major,
// unknowns ordered (i n1 + j) n2 + k
DALM_HD long long mg_cell_index(const MgLevel &L, int r) {
    const int k = r % L.n[2], j = (r / L.n[2]) % L.n[1], i = r / (L.n[2] * L.n[1]);
    return L.at(i, j, k);
}

// The V-cycle's order of operations, shared by the CUDA launcher and the
// host-side checks.  E provides smooth(level, colour, zero_start) (a
// half-sweep over the z-columns of one colour),
// restrict(level) (f of level + 1 from level's residual), coarse() (x of
// the last level from its f) and prolong(level) (x of level += P x of
// level + 1).  x of level 0 = V-cycle(f of level 0).
template <class E, class Nu>
void mg_vcycle_nu(E &e, int levels, Nu nu) {
    for (int l = 0; l + 1 < levels; l++) {
        e.smooth(l, 0, true);
        e.smooth(l, 1, false);
        for (int s = 1; s < nu(l); s++) {
            e.smooth(l, 0, false);
            e.smooth(l, 1, false);
        }
        e.restrict(l);
    }
    e.coarse();
    for (int l = levels - 2; l >= 0; l--) {
        e.prolong(l);
        for (int s = 0; s < nu(l); s++) {
            e.smooth(l, 1, false);
            e.smooth(l, 0, false);
        }
    }
}
template <class E>
void mg_vcycle(E &e, int levels, int nu) {
    mg_vcycle_nu(e, levels, [nu](int) { return nu; });
}

// smoothing sweeps per level before and after the coarse correction: MG_NU
// on the coarser levels, more on the two finest, where each sweep saves
// more outer iterations than it costs (C4, dt 5e-4: 4, 3, 2 ... gives 3
// conjugate-gradient iterations per step where 2 everywhere gives 5-7, at
// 0.86x the step time)
constexpr int MG_NU = 2;
DALM_HD int mg_nu(int level) { return level == 0 ? 4 : level == 1 ? 3 : MG_NU; }

// Device state of the preconditioner (multigrid.cu).
struct MgDev {
    int levels = 0;
    MgLevel L[MG_MAX_LEVELS];
    float *x[MG_MAX_LEVELS] = {}, *f[MG_MAX_LEVELS] = {};  // level 0: the caller's z and r
    const float *kinv = nullptr;  // coarsest inverse, [n][n]
    int ncoarse = 0;
};

struct KrylovState;

// False when the levels' z-columns are longer than the line smoother takes
// (256 cells); the mixed form then keeps its BiCGStab inner solves.
bool mg_prepare(const MgDev &M);

// x[0] = V-cycle(f[0]); every kernel returns at once when st->done is set.
void launch_mg_vcycle(const LaunchCtx &L, const MgDev &M, const KrylovState *st);

// Conjugate gradients on K e = f, preconditioned by the V-cycle, for the
// inner solves of iterative refinement.  r holds the FP32 residual of A on
// entry to begin (made into f = -max_diag vol r in place), e the correction
// (zeroed by begin); z, p, q are work vectors of the finest grid with zero
// guide cells.  The stop test is the RMS of the A-form residual
// r / (-max_diag vol) against st->tol, as for the Krylov inner solves.
struct MgPcgBufs {
    float *r, *e, *z, *p, *q;
};
void launch_mg_begin(const LaunchCtx &L, const MgDev &M, const MgPcgBufs &B, double max_diag,
                     Partials<1> part, KrylovState *st);
void launch_mg_iteration(const LaunchCtx &L, const MgDev &M, const MgPcgBufs &B,
                         double max_diag, Partials<1> part, KrylovState *st);

}  // namespace dalm
