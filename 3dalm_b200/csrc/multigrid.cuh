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
// faces) and the cell widths (the face areas).  Coarser levels merge pairs
// of cells along every axis whose count is even and at least 4 (semi-
// coarsening where an axis can no longer halve); their operator is the same
// finite-volume Laplacian on the merged cells (centre = mean of the
// children's centres, width = sum).  Transfers are piecewise constant: the
// restriction sums the children's residuals (K is in integrated form), the
// prolongation copies the coarse correction.  The smoother is red-black
// Gauss-Seidel, pre-smoothing red then black from zero and post-smoothing
// black then red, and the coarsest level is solved exactly with its
// precomputed inverse: the V-cycle is a symmetric positive definite linear
// operator, as conjugate gradients require of a preconditioner.
//
// Everything here is __host__ __device__ so that host-side checks run the
// kernels' arithmetic.
#pragma once

#include "common.cuh"

#ifndef DALM_HD
#define DALM_HD __host__ __device__ __forceinline__
#endif

namespace dalm {

constexpr int MG_MAX_LEVELS = 16;
constexpr int MG_MAX_COARSE = 1024;  // cells of the coarsest level (dense inverse)

struct MgLevel {
    Grid g;              // storage: level 0 is the solver's grid, coarser levels gc = 1
    int n[3];            // interior cells per axis
    int fac[3];          // children per coarse cell along each axis (1 or 2); finest: 1
    const float *cf[3];  // face conductances, [n + 1]
    const float *w[3];   // cell widths, [n]
    DALM_HD long long at(int i, int j, int k) const {
        return g.at(i + g.gc, j + g.gc, k + g.gc);
    }
    DALM_HD long long cells() const { return (long long)n[0] * n[1] * n[2]; }
};

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

DALM_HD float mg_diag(const MgLevel &L, int i, int j, int k) {
    const float ax = L.w[1][j] * L.w[2][k], ay = L.w[0][i] * L.w[2][k],
                az = L.w[0][i] * L.w[1][j];
    return ax * (L.cf[0][i + 1] + L.cf[0][i]) + ay * (L.cf[1][j + 1] + L.cf[1][j]) +
           az * (L.cf[2][k + 1] + L.cf[2][k]);
}

// One Gauss-Seidel update of cell (i,j,k); zero_start: the other colour is
// still zero (the first half-sweep from x = 0 reads no neighbour).
DALM_HD void mg_smooth_cell(const MgLevel &L, float *x, const float *f, int i, int j, int k,
                            bool zero_start) {
    const long long c = L.at(i, j, k);
    if (zero_start) {
        x[c] = f[c] / mg_diag(L, i, j, k);
        return;
    }
    float d;
    float nb = mg_neighbours(L, x, i, j, k, d);
    x[c] = (f[c] + nb) / d;
}

// cell of colour `color` ((i + j + k) % 2) number n of a level: false when
// past the end
DALM_HD bool mg_color_cell(const MgLevel &L, long long n, int color, int &i, int &j, int &k) {
    const int nkh = (L.n[2] + 1) / 2;
    const long long per_i = (long long)L.n[1] * nkh;
    if (n >= per_i * L.n[0]) return false;
    i = (int)(n / per_i);
    const long long r = n % per_i;
    j = (int)(r / nkh);
    k = 2 * (int)(r % nkh) + ((i + j + color) & 1);
    return k < L.n[2];
}

// coarse cell (I,J,K): the sum of its children's residuals f - K x
DALM_HD void mg_restrict_cell(const MgLevel &F, const MgLevel &C, const float *x, const float *f,
                              float *fc, int I, int J, int K) {
    float s = 0;
    for (int a = 0; a < C.fac[0]; a++)
        for (int b = 0; b < C.fac[1]; b++)
            for (int c = 0; c < C.fac[2]; c++) {
                const int i = I * C.fac[0] + a, j = J * C.fac[1] + b, k = K * C.fac[2] + c;
                s += f[F.at(i, j, k)] - mg_apply(F, x, i, j, k);
            }
    fc[C.at(I, J, K)] = s;
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
// host-side checks.  E provides smooth(level, colour, zero_start),
// restrict(level) (f of level + 1 from level's residual), coarse() (x of
// the last level from its f) and prolong(level) (x of level += P x of
// level + 1).  x of level 0 = V-cycle(f of level 0).
template <class E>
void mg_vcycle(E &e, int levels, int nu) {
    for (int l = 0; l + 1 < levels; l++) {
        e.smooth(l, 0, true);
        e.smooth(l, 1, false);
        for (int s = 1; s < nu; s++) {
            e.smooth(l, 0, false);
            e.smooth(l, 1, false);
        }
        e.restrict(l);
    }
    e.coarse();
    for (int l = levels - 2; l >= 0; l--) {
        e.prolong(l);
        for (int s = 0; s < nu; s++) {
            e.smooth(l, 1, false);
            e.smooth(l, 0, false);
        }
    }
}

// smoothing sweeps per level before and after the coarse correction
constexpr int MG_NU = 2;

// Device state of the preconditioner (multigrid.cu).
struct MgDev {
    int levels = 0;
    MgLevel L[MG_MAX_LEVELS];
    float *x[MG_MAX_LEVELS] = {}, *f[MG_MAX_LEVELS] = {};  // level 0: the caller's z and r
    const float *kinv = nullptr;  // coarsest inverse, [n][n]
    int ncoarse = 0;
};

struct KrylovState;

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
