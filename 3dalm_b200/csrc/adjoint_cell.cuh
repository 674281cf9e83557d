// Discrete adjoint of one time step: the per-cell and per-blade-point
// building blocks.  Everything here is __host__ __device__ so that the CUDA
// kernels (adjoint.cu) and host-side checks run the same arithmetic.
//
// The forward step being differentiated (Solver::main_loop_once,
// src/solver.h:1034-1193), for the state (U^n, JU^n, f^n) with guide cells:
//   U*  = U^n + dt (-conv(U^n, JU^n) + diff(U^n; nut(U^n)) + f^n)   interior
//   U*  = U^n                                                      guide cells
//   JU* = face interpolation of U* with the inflow / wall overrides
//   b   = div(JU*) / (dt max_diag);   p = A^-1 b;   p guide cells by apply_pbc
//   U^{n+1} = U* - dt grad_c p (interior), JU^{n+1} = JU* - dt area grad_f p
//   U^{n+1} guide cells by apply_Ubc (convective outflow reads U^n)
//   f^{n+1}, torque: actuator line on U^{n+1} at t_n
// Each function below is the transpose (reverse mode) of one of these maps,
// written as a gather so that every output element is owned by one thread.
// Kinks (the b=4 limiter, |JU| in the upwind flux, fabs in the torque, the
// table lookup, trilinear cell switches) take the derivative of the branch
// the forward takes; with the van Albada limiter the convection is smooth.
#pragma once

#include <cmath>

#include "alm.cuh"

#define DALM_HD __host__ __device__ __forceinline__

#include "dual.cuh"

namespace dalm {
namespace adj {

DALM_HD double sgn(double v) { return (double)((v > 0.) - (v < 0.)); }

DALM_HD bool interior(const Grid &g, int i, int j, int k) {
    return i >= g.gc && i < g.nx - g.gc && j >= g.gc && j < g.ny - g.gc && k >= g.gc &&
           k < g.nz - g.gc;
}

// Axis helpers: stored extent, coordinate and width arrays, element stride.
struct Axes {
    int n[3];
    const double *x[3], *d[3];
    long long s[3];
    DALM_HD Axes(const StepParams &P) {
        n[0] = P.g.nx; n[1] = P.g.ny; n[2] = P.g.nz;
        x[0] = P.m.x; x[1] = P.m.y; x[2] = P.m.z;
        d[0] = P.m.dx; d[1] = P.m.dy; d[2] = P.m.dz;
        s[0] = P.g.sx; s[1] = P.g.sy; s[2] = 1;
    }
    DALM_HD bool in(int a, int v, int gc) const { return v >= gc && v < n[a] - gc; }
};

// ------------------------------------------------------------ convection

// A reconstructed face state v0 + limited slope term, as a function of the
// cell value v0 and the two differences a (upwind side) and b (face side),
// with its partial derivatives.  This is the form of all four face values
// of src/cfd.h:37-60:  the left state at face f+1/2 is recon(v_f, v_f -
// v_{f-1}, v_{f+1} - v_f), the right state recon(v_{f+1}, v_{f+1} - v_{f+2},
// v_f - v_{f+1}) (both limiters are odd in (a, b)).
struct Recon {
    double v, da, db;
};

// b=4 limiter term s_a max(0, min(|a|, s_a bb b)) and its partials.
DALM_HD void minmod_b(double a, double b, double bb, double &v, double &d1, double &d2) {
    double s = sgn(a);
    double m1 = fabs(a), m2 = s * bb * b;
    double mn = fmin(m1, m2);
    v = s * fmax(0., mn);
    d1 = d2 = 0;
    if (s == 0 || !(mn > 0)) return;
    if (m1 <= m2) d1 = 1;
    else d2 = bb;
}

DALM_HD Recon recon(double v0, double a, double b, int limiter) {
    const double kap = 1. / 3.;
    Recon r;
    if (limiter == 1) {
        // van Albada switch s = (2ab + eps)/(a^2 + b^2 + eps)
        const double eps = 1e-12;
        double N = 2. * a * b + eps, D = a * a + b * b + eps;
        double s = N / D;
        double dsa = (2. * b * D - N * 2. * a) / (D * D);
        double dsb = (2. * a * D - N * 2. * b) / (D * D);
        double T = (s / 4.) * ((1. - kap * s) * a + (1. + kap * s) * b);
        double dTds = (a + b) / 4. + (kap * s / 2.) * (b - a);
        r.v = v0 + T;
        r.da = s / 4. - kap * s * s / 4. + dTds * dsa;
        r.db = s / 4. + kap * s * s / 4. + dTds * dsb;
        return r;
    }
    const double bb = (3. - kap) / (1. - kap);
    double lab, lab_1, lab_2, lba, lba_1, lba_2;
    minmod_b(a, b, bb, lab, lab_1, lab_2);
    minmod_b(b, a, bb, lba, lba_1, lba_2);
    r.v = v0 + 0.25 * ((1. - kap) * lab + (1. + kap) * lba);
    r.da = 0.25 * ((1. - kap) * lab_1 + (1. + kap) * lba_2);
    r.db = 0.25 * ((1. - kap) * lab_2 + (1. + kap) * lba_1);
    return r;
}

// Partials of the upwind face flux F = (J (fR + fL) - |J| (fR - fL)) / 2 at
// face f+1/2 with respect to v_{f-1}, v_f, v_{f+1}, v_{f+2} and J.
struct FaceAdj {
    double dv[4];
    double dJ;
};

DALM_HD FaceAdj face_flux_adj(double a0, double a1, double a2, double a3, double J, int limiter) {
    Recon L = recon(a1, a1 - a0, a2 - a1, limiter);
    Recon R = recon(a2, a2 - a3, a1 - a2, limiter);
    double cl = 0.5 * (J + fabs(J)), cr = 0.5 * (J - fabs(J));
    FaceAdj f;
    f.dv[0] = cl * (-L.da);
    f.dv[1] = cl * (1. + L.da - L.db) + cr * R.db;
    f.dv[2] = cl * L.db + cr * (1. + R.da - R.db);
    f.dv[3] = cr * (-R.da);
    f.dJ = 0.5 * ((R.v + L.v) - sgn(J) * (R.v - L.v));
    return f;
}

// ------------------------------------------------- predictor (K1) adjoint

// Index of dS/d(d_a u_m) in the six per-cell strain products (symmetric).
DALM_HD int strain_slot(int m, int a) { return m == a ? m : 2 + m + a; }

// Pass 1 over interior cells c: with L = adjoint of U* (a_us), forms
//   nu(c) = 1/Re + nut(c)                  (the forward's viscosity)
//   s6(c) = lS(c) dS/d(grad)               (six strain products)
// where lnu = dt sum_m L_m Lap_m(c) and lS = lnu filter2 / (2 sqrt S).
struct AdjNutArgs {
    StepParams P;
    Vec3<const double> V;    // U^n
    Vec3<const double> aus;  // adjoint of U*
    double *nu;
    double *s6[6];
};

DALM_HD void adj_nut_cell(const AdjNutArgs &A, int i, int j, int k) {
    const StepParams &P = A.P;
    const Grid &g = P.g;
    long long c = g.at(i, j, k);
    long long e = g.at(i + 1, j, k), w = g.at(i - 1, j, k), n = g.at(i, j + 1, k),
              s = g.at(i, j - 1, k), t = c + 1, b = c - 1;
    const double *x = P.m.x, *y = P.m.y, *z = P.m.z;
    double dxew = x[i + 1] - x[i - 1], dyns = y[j + 1] - y[j - 1], dztb = z[k + 1] - z[k - 1];
    double G[3][3];  // G[m][a] = d_a u_m
    for (int m = 0; m < 3; m++) {
        const double *v = A.V.c[m];
        G[m][0] = (v[e] - v[w]) / dxew;
        G[m][1] = (v[n] - v[s]) / dyns;
        G[m][2] = (v[t] - v[b]) / dztb;
    }
    double S = 2 * G[0][0] * G[0][0] + 2 * G[1][1] * G[1][1] + 2 * G[2][2] * G[2][2] +
               (G[0][1] + G[1][0]) * (G[0][1] + G[1][0]) +
               (G[0][2] + G[2][0]) * (G[0][2] + G[2][0]) +
               (G[1][2] + G[2][1]) * (G[1][2] + G[2][1]);
    double shear = sqrt(S);
    double f2 = P.filter2[c];
    A.nu[c] = 1 / P.re + f2 * shear;
    double lnu = 0;
    double dxc = P.m.dx[i], dyc = P.m.dy[j], dzc = P.m.dz[k];
    for (int m = 0; m < 3; m++) {
        const double *v = A.V.c[m];
        double fc = v[c];
        double lap = ((v[e] - fc) / (x[i + 1] - x[i]) - (fc - v[w]) / (x[i] - x[i - 1])) / dxc +
                     ((v[n] - fc) / (y[j + 1] - y[j]) - (fc - v[s]) / (y[j] - y[j - 1])) / dyc +
                     ((v[t] - fc) / (z[k + 1] - z[k]) - (fc - v[b]) / (z[k] - z[k - 1])) / dzc;
        lnu += A.aus.c[m][c] * lap;
    }
    lnu *= P.dt;
    double lS = shear > 0 ? lnu * f2 / (2 * shear) : 0.0;
    A.s6[0][c] = lS * 4 * G[0][0];
    A.s6[1][c] = lS * 4 * G[1][1];
    A.s6[2][c] = lS * 4 * G[2][2];
    A.s6[3][c] = lS * 2 * (G[0][1] + G[1][0]);
    A.s6[4][c] = lS * 2 * (G[0][2] + G[2][0]);
    A.s6[5][c] = lS * 2 * (G[1][2] + G[2][1]);
}

// Pass 2 over every stored cell q: the transposed predictor stencil.
//   aV(q)  += a_us(q)                       (U* = U^n + ..., and on guide cells)
//            + sum over faces f whose MUSCL stencil holds q of lF(f) dF/dv_q
//            + transposed diffusion and eddy-viscosity terms
//   aJU(q)  = sum_m lF_m dF_m/dJ at the three faces q owns
//   af(q)   = dt a_us(q) on interior cells
// with lF(f) = -dt L(f)/vol(f) + dt L(f+1)/vol(f+1), L = a_us on interior cells.
struct AdjPredictArgs {
    StepParams P;
    Vec3<const double> V, JU, aus;
    const double *nu;
    const double *s6[6];
    Vec3<double> aV, aJU, af;
};

DALM_HD double cell_volume(const StepParams &P, int i, int j, int k) {
    return P.m.dx[i] * P.m.dy[j] * P.m.dz[k];
}

DALM_HD void adj_predict_cell(const AdjPredictArgs &A, int i, int j, int k) {
    const StepParams &P = A.P;
    const Grid &g = P.g;
    const Axes X(P);
    const int gc = g.gc;
    const long long q = g.at(i, j, k);
    const int idx[3] = {i, j, k};
    const double dt = P.dt;
    double add[3], lJ[3] = {0, 0, 0};
    for (int m = 0; m < 3; m++) add[m] = A.aus.c[m][q];

    for (int a = 0; a < 3; a++) {
        const int b1 = (a + 1) % 3, b2 = (a + 2) % 3;
        if (!X.in(b1, idx[b1], gc) || !X.in(b2, idx[b2], gc)) continue;  // no face flux here
        const int ia = idx[a];
        const long long sa = X.s[a];
        for (int f = ia - 2; f <= ia + 1; f++) {
            if (f < gc - 1 || f > X.n[a] - gc - 1) continue;
            const long long cf = q + (long long)(f - ia) * sa;  // cell f (lower cell of the face)
            int cidx[3] = {i, j, k};
            cidx[a] = f;
            const double vol_f = X.in(a, f, gc) ? cell_volume(P, cidx[0], cidx[1], cidx[2]) : 0.0;
            cidx[a] = f + 1;
            const double vol_f1 = X.in(a, f + 1, gc) ? cell_volume(P, cidx[0], cidx[1], cidx[2]) : 0.0;
            const double J = A.JU.c[a][cf];
            const int pos = ia - (f - 1);
            double ljf = 0;
            for (int m = 0; m < 3; m++) {
                const double *v = A.V.c[m];
                double lF = 0;
                if (vol_f != 0.0) lF -= dt * A.aus.c[m][cf] / vol_f;
                if (vol_f1 != 0.0) lF += dt * A.aus.c[m][cf + sa] / vol_f1;
                if (lF == 0.0) continue;
                FaceAdj fa = face_flux_adj(v[cf - sa], v[cf], v[cf + sa], v[cf + 2 * sa], J,
                                           P.limiter);
                add[m] += lF * fa.dv[pos];
                ljf += lF * fa.dJ;
            }
            if (f == ia) lJ[a] = ljf;
        }
    }

    // diffusion nu(c) Lap(c) and eddy viscosity nut(c) = filter2 sqrt(S)
    const bool qin = interior(g, i, j, k);
    if (qin) {
        double cq = 0;
        for (int a = 0; a < 3; a++) {
            const int ia = idx[a];
            cq -= (1. / (X.x[a][ia + 1] - X.x[a][ia]) + 1. / (X.x[a][ia] - X.x[a][ia - 1])) /
                  X.d[a][ia];
        }
        for (int m = 0; m < 3; m++) add[m] += dt * A.nu[q] * A.aus.c[m][q] * cq;
    }
    for (int a = 0; a < 3; a++) {
        const int ia = idx[a];
        const long long sa = X.s[a];
        int lo[3] = {i, j, k}, hi[3] = {i, j, k};
        lo[a] = ia - 1;
        hi[a] = ia + 1;
        if (interior(g, lo[0], lo[1], lo[2])) {  // q is the + neighbour of c = q - e_a
            const long long c = q - sa;
            const double kc = 1. / ((X.x[a][ia] - X.x[a][ia - 1]) * X.d[a][ia - 1]);
            const double D = X.x[a][ia] - X.x[a][ia - 2];
            for (int m = 0; m < 3; m++)
                add[m] += dt * A.nu[c] * A.aus.c[m][c] * kc + A.s6[strain_slot(m, a)][c] / D;
        }
        if (interior(g, hi[0], hi[1], hi[2])) {  // q is the - neighbour of c = q + e_a
            const long long c = q + sa;
            const double kc = 1. / ((X.x[a][ia + 1] - X.x[a][ia]) * X.d[a][ia + 1]);
            const double D = X.x[a][ia + 2] - X.x[a][ia];
            for (int m = 0; m < 3; m++)
                add[m] += dt * A.nu[c] * A.aus.c[m][c] * kc - A.s6[strain_slot(m, a)][c] / D;
        }
    }
    for (int m = 0; m < 3; m++) {
        A.aV.c[m][q] += add[m];
        A.aJU.c[m][q] = lJ[m];
        A.af.c[m][q] = qin ? dt * A.aus.c[m][q] : 0.0;
    }
}

// set_solid_U (src/cfd.h:1143-1160) transposed: the projected interior
// velocity was scaled by 1 - solid
DALM_HD void adj_solid_cell(const StepParams &P, Vec3<double> aU, int i, int j, int k) {
    const long long c = P.g.at(i, j, k);
    const double sf = P.solid[c];
    for (int m = 0; m < 3; m++) aU.c[m][c] = (1. - sf) * aU.c[m][c];
}

// ---------------------------------------------- projection and Poisson

// JU faces the projection changes and the next predictor reads: normal
// index f along axis a in [gc-1, N-gc-1] with interior tangential indices,
// minus the faces apply_JUbc overrides with constants (src/bc.h:235-302):
// the inflow face x = gc-1 and the wall faces y, z = gc-1 and N-gc-1.
DALM_HD bool face_active(const Axes &X, int a, int f, int gc) {
    if (a == 0) return f >= gc && f <= X.n[0] - gc - 1;
    return f >= gc && f <= X.n[a] - gc - 2;
}

DALM_HD double face_area(const StepParams &P, int a, int i, int j, int k) {
    if (a == 0) return P.m.dy[j] * P.m.dz[k];
    if (a == 1) return P.m.dx[i] * P.m.dz[k];
    return P.m.dx[i] * P.m.dy[j];
}

// Interior cell q: the adjoint of the pressure, lp(q), from the projection
// of U and JU (src/cfd.h:601-783), with the guide-cell values of apply_pbc
// (src/bc.h:304-411) folded onto the interior cells they copy; returns the
// right-hand side of the adjoint pressure solve, lp(q) / vol(q).
// (A = M^-1 L / max_diag with M = diag(vol) and L symmetric, so A^T = M A
// M^-1 and A^T y = lp  <=>  A (y / vol) = lp / vol.)
struct AdjProjectArgs {
    StepParams P;
    Vec3<const double> aU, aJU;
    double *rhs;
};

DALM_HD double adj_project_cell(const AdjProjectArgs &A, int i, int j, int k) {
    const StepParams &P = A.P;
    const Grid &g = P.g;
    const Axes X(P);
    const int gc = g.gc;
    const long long q = g.at(i, j, k);
    const int idx[3] = {i, j, k};
    const double dt = P.dt;
    double lp = 0;
    for (int a = 0; a < 3; a++) {
        const int ia = idx[a];
        const long long sa = X.s[a];
        const double *x = X.x[a];
        const double area = face_area(P, a, i, j, k);
        // central gradient of the cell velocities
        if (X.in(a, ia + 1, gc)) lp += dt * A.aU.c[a][q + sa] / (x[ia + 2] - x[ia]);
        if (X.in(a, ia - 1, gc)) lp -= dt * A.aU.c[a][q - sa] / (x[ia] - x[ia - 2]);
        // compact gradient of the face fluxes
        if (face_active(X, a, ia, gc)) lp += dt * area * A.aJU.c[a][q] / (x[ia + 1] - x[ia]);
        if (face_active(X, a, ia - 1, gc)) lp -= dt * area * A.aJU.c[a][q - sa] / (x[ia] - x[ia - 1]);
        // guide cells written by apply_pbc from this cell
        if (ia == gc) {  // copy (x-: Neumann inflow side; y-, z- walls)
            lp += dt * A.aU.c[a][q] / (x[ia + 1] - x[ia - 1]);
        }
        if (ia == X.n[a] - gc - 1) {
            double lg = -dt * A.aU.c[a][q] / (x[ia + 1] - x[ia - 1]);
            if (a == 0) {
                // outlet: p_o = -p_i (ho / hi), and the outlet face reads p_o
                if (face_active(X, 0, ia, gc)) lg -= dt * area * A.aJU.c[0][q] / (x[ia + 1] - x[ia]);
                double hi = 0.5 * P.m.dx[ia], ho = 0.5 * P.m.dx[ia + 1];
                lp += -(ho / hi) * lg;
            } else {
                lp += lg;  // copy (y+, z+ walls)
            }
        }
    }
    double r = lp / cell_volume(P, i, j, k);
    A.rhs[q] = r;
    return r * r;
}

// Cells q with i in [gc, nx-gc] (the interior plus the first outflow guide
// plane) and interior j, k: the adjoint of the face fluxes JU* (the
// projection passes them through; the Poisson right-hand side takes their
// divergence, src/cfd.h:569-598) mapped back onto U* by the transposed face
// interpolation (src/cfd.h:395-493).  y = the adjoint pressure solution
// scaled by 1/vol (the solve's unknown); adds into aus in place.
struct AdjFacesArgs {
    StepParams P;
    Vec3<const double> aJU;
    const double *y;
    Vec3<double> aus;
};

DALM_HD void adj_faces_cell(const AdjFacesArgs &A, int i, int j, int k) {
    const StepParams &P = A.P;
    const Grid &g = P.g;
    const Axes X(P);
    const int gc = g.gc;
    const long long q = g.at(i, j, k);
    const int idx[3] = {i, j, k};
    const double scale = 1. / (P.dt * P.max_diag);
    for (int a = 0; a < 3; a++) {
        const int b1 = (a + 1) % 3, b2 = (a + 2) % 3;
        if (!X.in(b1, idx[b1], gc) || !X.in(b2, idx[b2], gc)) continue;
        const int ia = idx[a];
        const long long sa = X.s[a];
        const double half_area = 0.5 * face_area(P, a, i, j, k);
        double acc = 0;
        for (int f = ia - 1; f <= ia; f++) {
            if (!face_active(X, a, f, gc)) continue;
            const long long cf = q + (long long)(f - ia) * sa;
            double lj = A.aJU.c[a][cf];
            if (X.in(a, f, gc)) lj += A.y[cf] * scale;
            if (X.in(a, f + 1, gc)) lj -= A.y[cf + sa] * scale;
            acc += half_area * lj;
        }
        A.aus.c[a][q] += acc;
    }
}

// ------------------------------------------------- velocity BC adjoint

// Three-point Lagrange weights (src/util.h:201-212) at x3.
DALM_HD void lagrange3(double x0, double x1, double x2, double x3, double &l0, double &l1,
                       double &l2) {
    l0 = ((x3 - x1) * (x3 - x2)) / ((x0 - x1) * (x0 - x2));
    l1 = ((x3 - x0) * (x3 - x2)) / ((x1 - x0) * (x1 - x2));
    l2 = ((x3 - x0) * (x3 - x1)) / ((x2 - x0) * (x2 - x1));
}

// apply_Ubc after the projection (src/bc.h:5-233), transposed for one
// boundary column n of the forward's enumeration (2 nyz x-columns, then
// 2 nxz y-columns, then 2 nxy z-columns).  The guide values' adjoint moves
// to the interior cells they extrapolate (aU) or, for the convective
// outflow, which reads U^n only, to the adjoint of U^n (aV); the guide
// cells' adjoint is then zero.  Columns of the y faces and of the z faces
// both add into the same near-wall cells, so they run as separate passes.
struct AdjBcArgs {
    StepParams P;
    Vec3<const double> V;  // U^n
    Vec3<double> aU, aV;
};

DALM_HD void adj_velocity_bc_column(const AdjBcArgs &A, long long n) {
    const StepParams &P = A.P;
    const Grid &g = P.g;
    const int GC = g.gc;
    const long long nyz = (long long)g.nj() * g.nk(), nxz = (long long)g.ni() * g.nk();
    long long r = n;
    if (r < 2 * nyz) {
        int side = (int)(r / nyz);
        long long qq = r % nyz;
        int j = GC + (int)(qq / g.nk()), k = GC + (int)(qq % g.nk());
        if (side == 0) {
            for (int i = 0; i < GC; i++)
                for (int m = 0; m < 3; m++) A.aU.c[m][g.at(i, j, k)] = 0;
            return;
        }
        for (int i = g.nx - GC; i < g.nx; i++) {
            long long i0 = g.at(i, j, k), i1 = g.at(i - 1, j, k), i2 = g.at(i - 2, j, k);
            double uout = A.V.c[0][i0];
            double c1 = uout * P.dt / P.m.dx[i];
            double lux = 0;
            for (int m = 0; m < 3; m++) {
                double a = A.aU.c[m][i0];
                if (a == 0.0) continue;
                double f0 = A.V.c[m][i0], f1 = A.V.c[m][i1], f2 = A.V.c[m][i2];
                double grad = (3 * f0 - 4 * f1 + f2) / 2;
                A.aV.c[m][i0] += a * (1. - 1.5 * c1);
                A.aV.c[m][i1] += a * (2. * c1);
                A.aV.c[m][i2] += a * (-0.5 * c1);
                lux -= a * P.dt * grad / P.m.dx[i];
                A.aU.c[m][i0] = 0;
            }
            A.aV.c[0][i0] += lux;
        }
        return;
    }
    r -= 2 * nyz;
    int side, i, j, k, a0i, a1i, a3i, a4i, axis;
    if (r < 2 * nxz) {
        axis = 1;
        side = (int)(r / nxz);
        long long qq = r % nxz;
        i = GC + (int)(qq / g.nk());
        k = GC + (int)(qq % g.nk());
        j = 0;
        a0i = side ? g.ny - GC - 2 : GC + 1;
        a1i = side ? g.ny - GC - 1 : GC;
        a3i = side ? g.ny - GC : GC - 1;
        a4i = side ? g.ny - GC + 1 : GC - 2;
    } else {
        r -= 2 * nxz;
        axis = 2;
        long long nxy = (long long)g.ni() * g.nj();
        side = (int)(r / nxy);
        long long qq = r % nxy;
        i = GC + (int)(qq / g.nj());
        j = GC + (int)(qq % g.nj());
        k = 0;
        a0i = side ? g.nz - GC - 2 : GC + 1;
        a1i = side ? g.nz - GC - 1 : GC;
        a3i = side ? g.nz - GC : GC - 1;
        a4i = side ? g.nz - GC + 1 : GC - 2;
    }
    const double *c = axis == 1 ? P.m.y : P.m.z;
    const double *d = axis == 1 ? P.m.dy : P.m.dz;
    auto at = [&](int v) { return axis == 1 ? g.at(i, v, k) : g.at(i, j, v); };
    long long a0 = at(a0i), a1 = at(a1i), a3 = at(a3i), a4 = at(a4i);
    double x0 = c[a0i], x1 = c[a1i];
    double x2 = side ? c[a1i] + 0.5 * d[a1i] : c[a1i] - 0.5 * d[a1i];
    double l30, l31, l32, l40, l41, l42;
    lagrange3(x0, x1, x2, c[a3i], l30, l31, l32);
    lagrange3(x0, x1, x2, c[a4i], l40, l41, l42);
    for (int m = 0; m < 3; m++) {
        // the wall value equals the adjacent cell's (slip components) or 0:
        // y-/y+ slip (v = 0), z+ slip (w = 0), z- no slip (all 0) or slip
        // upstream of a retracted floor's start
        bool slip = axis == 1 ? (m != 1)
                              : ((side == 1 || (P.retracted && P.m.x[i] < P.floor_start)) && m != 2);
        double g3 = A.aU.c[m][a3], g4 = A.aU.c[m][a4];
        A.aU.c[m][a0] += l30 * g3 + l40 * g4;
        A.aU.c[m][a1] += (l31 + (slip ? l32 : 0.0)) * g3 + (l41 + (slip ? l42 : 0.0)) * g4;
        A.aU.c[m][a3] = 0;
        A.aU.c[m][a4] = 0;
    }
}


// ------------------------------------------------------ actuator line

constexpr double ADJ_PI = 3.14159265358979323846;  // M_PI (src/type.h:12)

// find_floor_index (src/util.h:119-146)
DALM_HD int floor_index(const double *a, double v, int n) {
    if (v < a[0]) return -1;
    if (v >= a[n - 1]) return n - 1;
    int lo = 0, hi = n - 1, found = -1;
    while (lo <= hi) {
        int mid = lo + (hi - lo) / 2;
        if (a[mid] <= v) {
            found = mid;
            lo = mid + 1;
        } else {
            hi = mid - 1;
        }
    }
    return found;
}

// frame_transform (src/euler_angle.h:34-62) on a generic scalar
template <class S>
DALM_HD void frame_transform(const S (&in)[3], S (&out)[3], const S &angle, int type) {
    S c = cos(angle), s = sin(angle);
    switch (type) {
    case EULER_ROLL: out[0] = in[0]; out[1] = c * in[1] + s * in[2]; out[2] = -s * in[1] + c * in[2]; break;
    case EULER_PITCH: out[0] = c * in[0] - s * in[2]; out[1] = in[1]; out[2] = -s * in[0] + c * in[2]; break;
    case EULER_YAW: out[0] = c * in[0] + s * in[1]; out[1] = -s * in[0] + c * in[1]; out[2] = in[2]; break;
    default: out[0] = in[0]; out[1] = in[1]; out[2] = in[2]; break;
    }
}

// frame_transform_U (src/euler_angle.h:64-127) with its two typos
template <class S>
DALM_HD void frame_transform_U(const S (&p)[3], const S (&U)[3], S (&out)[3], const S &angle,
                               double ow, int type) {
    S c = cos(angle), s = sin(angle);
    const S &x = p[0], &y = p[1], &z = p[2], &u = U[0], &v = U[1], &w = U[2];
    switch (type) {
    case EULER_ROLL:
        out[0] = 0. + u;
        out[1] = ow * (-s * y + c * z) + (c * v + s * w);
        out[2] = ow * (-c * y - s * z) + (-s * v + v * w);
        break;
    case EULER_PITCH:
        out[0] = ow * (-s * x - c * z) + (c * u - s * w);
        out[1] = 0. + v;
        out[2] = ow * (c * x - s * z) + (s * u + c * w);
        break;
    case EULER_YAW:
        out[0] = ow * (-s * x + c * y) + (c * u + s * v);
        out[1] = ow * (-c * s - s * y) + (-s * u + c * v);
        out[2] = 0. + w;
        break;
    default: out[0] = u; out[1] = v; out[2] = w; break;
    }
}

template <class S>
DALM_HD S lin_interp(double v0, double v1, double x0, double x1, const S &xp) {
    S fx = (xp - x0) / (x1 - x0);  // src/util.h:166-174
    return v0 * (1 - fx) + v1 * fx;
}

template <class S>
struct PointEval {
    S xyz[3], f[3], torque, thrust;
    long long id[8];  // trilinear stencil (-1: point outside the interior)
    double w[8];      // its weights
};

// One blade point (update_ap_position + calc_ap_force, src/alm.h:233-370)
// on a generic scalar: the turbine's angle offset (rad), the collective
// pitch (deg, added to the twist), the rotor speed (rad/s) and a shift of
// the sampled velocity are inputs, so dual numbers seeded in them give the
// point's position, force and torque derivatives.  With plain doubles the
// operation order is that of k_alm_points.
template <class S>
DALM_HD void alm_point_eval(const StepParams &P, const AlmDev &A, const TurbineDev &wt, int a,
                            double t, Vec3<const double> U, const S &angle_offset,
                            const S &pitch, const S &omega, const S (&ushift)[3],
                            PointEval<S> &o) {
    const Grid &g = P.g;
    S angle = wt.formula[0] * ::sin(wt.formula[1] * t + wt.formula[2]) + angle_offset;
    double ow = wt.formula[0] * wt.formula[1] * ::cos(wt.formula[1] * t + wt.formula[2]);
    int bid = (a % A.ap_per_wt) / A.ap_per_blade;
    double r = A.r[a];
    S theta = bid * (2 * ADJ_PI / A.blades) + t * omega;
    S loc[3] = {S(wt.rot_center[0]), wt.rot_center[1] + r * cos(theta),
                wt.rot_center[2] + r * sin(theta)};
    S xyz[3];
    frame_transform(loc, xyz, -angle, wt.type);
    for (int m = 0; m < 3; m++) xyz[m] = xyz[m] + wt.base[m];
    for (int m = 0; m < 3; m++) {
        o.xyz[m] = xyz[m];
        o.f[m] = S(0.0);
    }
    o.torque = S(0.0);
    o.thrust = S(0.0);
    for (int q = 0; q < 8; q++) {
        o.id[q] = -1;
        o.w[q] = 0;
    }
    int i = floor_index(P.m.x, value(xyz[0]), g.nx);
    int j = floor_index(P.m.y, value(xyz[1]), g.ny);
    int k = floor_index(P.m.z, value(xyz[2]), g.nz);
    if (!(i >= g.gc && i < g.nx - g.gc && j >= g.gc && j < g.ny - g.gc && k >= g.gc &&
          k < g.nz - g.gc))
        return;
    long long id[8] = {g.at(i, j, k),         g.at(i + 1, j, k),
                       g.at(i, j + 1, k),     g.at(i + 1, j + 1, k),
                       g.at(i, j, k + 1),     g.at(i + 1, j, k + 1),
                       g.at(i, j + 1, k + 1), g.at(i + 1, j + 1, k + 1)};
    double x0 = P.m.x[i], x1 = P.m.x[i + 1], y0 = P.m.y[j], y1 = P.m.y[j + 1];
    double z0 = P.m.z[k], z1 = P.m.z[k + 1];
    S fx = (xyz[0] - x0) / (x1 - x0), fy = (xyz[1] - y0) / (y1 - y0),
      fz = (xyz[2] - z0) / (z1 - z0);
    S Uap[3];
    for (int m = 0; m < 3; m++) {
        const double *v = U.c[m];
        S v01 = v[id[0]] * (1 - fx) + v[id[1]] * fx;
        S v23 = v[id[2]] * (1 - fx) + v[id[3]] * fx;
        S v45 = v[id[4]] * (1 - fx) + v[id[5]] * fx;
        S v67 = v[id[6]] * (1 - fx) + v[id[7]] * fx;
        S v0123 = v01 * (1 - fy) + v23 * fy;
        S v4567 = v45 * (1 - fy) + v67 * fy;
        Uap[m] = v0123 * (1 - fz) + v4567 * fz + ushift[m];
    }
    S rel[3] = {xyz[0] - wt.base[0], xyz[1] - wt.base[1], xyz[2] - wt.base[2]};
    S Ur[3];
    frame_transform_U(rel, Uap, Ur, angle, ow, wt.type);
    S ux_ = Ur[0];
    S ut_ = r * omega + Ur[1] * sin(theta) - Ur[2] * cos(theta);
    S urel2 = ux_ * ux_ + ut_ * ut_;
    S phi = atan(ux_ / ut_);
    S atk = phi * 180 / ADJ_PI - (A.twist[a] + pitch);
    const double *cdt = A.cd + (long long)a * A.atk_count;
    const double *clt = A.cl + (long long)a * A.atk_count;
    int ti = floor_index(A.atk, value(atk), A.atk_count);
    S cd, cl;
    if (ti < 0) {
        cd = S(cdt[0]);
        cl = S(clt[0]);
    } else if (ti >= A.atk_count - 1) {
        cd = S(cdt[A.atk_count - 1]);
        cl = S(clt[A.atk_count - 1]);
    } else {
        cd = lin_interp(cdt[ti], cdt[ti + 1], A.atk[ti], A.atk[ti + 1], atk);
        cl = lin_interp(clt[ti], clt[ti + 1], A.atk[ti], A.atk[ti + 1], atk);
    }
    S fd = 0.5 * cd * urel2 * A.chord[a] * A.dr[a];
    S fl = 0.5 * cl * urel2 * A.chord[a] * A.dr[a];
    S fx_ = fl * cos(phi) + fd * sin(phi);
    S ft_ = fl * sin(phi) - fd * cos(phi);
    ft_ = ft_ * sgn(value(omega));
    S f_[3] = {-fx_, ft_ * sin(theta), -ft_ * cos(theta)};
    frame_transform(f_, o.f, -angle, wt.type);
    o.torque = fabs(ft_) * r;
    o.thrust = fx_;
    double wx = value(fx), wy = value(fy), wz = value(fz);
    double w[8] = {(1 - wx) * (1 - wy) * (1 - wz), wx * (1 - wy) * (1 - wz),
                   (1 - wx) * wy * (1 - wz),       wx * wy * (1 - wz),
                   (1 - wx) * (1 - wy) * wz,       wx * (1 - wy) * wz,
                   (1 - wx) * wy * wz,             wx * wy * wz};
    for (int q = 0; q < 8; q++) {
        o.id[q] = id[q];
        o.w[q] = w[q];
    }
}

// Adjoint of distribute_ap_force (src/alm.h:416-448), one cell's term for
// point a: with w = e_coef exp(-r^2/eps^2) the cell adds
//   acc[m]   += w af_m                                (adjoint of f_ap)
//   acc[3+d] += w 2 (x_d - p_d)/eps^2 (af . f_ap)     (adjoint of the position)
// where af is the adjoint of the projected force field.
DALM_HD void adj_alm_gather_term(const StepParams &P, const AlmDev &A, Vec3<const double> af,
                                 int a, int i, int j, int k, double (&acc)[6]) {
    double px = A.pt_xyz[a * 3], py = A.pt_xyz[a * 3 + 1], pz = A.pt_xyz[a * 3 + 2];
    double dx = P.m.x[i] - px, dy = P.m.y[j] - py, dz = P.m.z[k] - pz;
    double r2 = dx * dx + dy * dy + dz * dz;
    if (!(r2 <= A.cutoff2)) return;
    double w = A.e_coef * ::exp(-r2 / A.pw2);
    long long c = P.g.at(i, j, k);
    double l0 = af.c[0][c], l1 = af.c[1][c], l2 = af.c[2][c];
    acc[0] += w * l0;
    acc[1] += w * l1;
    acc[2] += w * l2;
    double dot = l0 * A.pt_f[a * 3] + l1 * A.pt_f[a * 3 + 1] + l2 * A.pt_f[a * 3 + 2];
    double s = w * 2 * dot / A.pw2;
    acc[3] += s * dx;
    acc[4] += s * dy;
    acc[5] += s * dz;
}

// The interior cells whose centre can lie within the support radius of
// point a (the exact test is in adj_alm_gather_term): [lo, hi) per axis.
DALM_HD void alm_support_box(const StepParams &P, const AlmDev &A, int a, int (&lo)[3],
                             int (&hi)[3]) {
    const Grid &g = P.g;
    const double *c[3] = {P.m.x, P.m.y, P.m.z};
    const int n[3] = {g.nx, g.ny, g.nz};
    double R = ::sqrt(A.cutoff2);
    for (int m = 0; m < 3; m++) {
        double p = A.pt_xyz[a * 3 + m];
        int l = floor_index(c[m], p - R, n[m]);
        int h = floor_index(c[m], p + R, n[m]) + 2;
        lo[m] = l < g.gc ? g.gc : l;
        hi[m] = h > n[m] - g.gc ? n[m] - g.gc : h;
    }
}

// Reverse mode through one blade point: forward-mode derivatives of the
// point model in 6 directions (angle offset per degree, pitch, rotor speed,
// the 3 sampled velocity components), contracted with the adjoints of the
// point's force (gather[0..2]), position (gather[3..5]) and torque (weight
// |Omega|: the objective is weight * torque * |Omega| per turbine).
// Writes the point's parameter gradient gth[3], the adjoint of its sampled
// velocity lU[3], its trilinear stencil and its torque.
struct AdjAlmPointArgs {
    StepParams P;
    AlmDev A;
    Vec3<const double> U;  // the velocity the actuator line sampled
    double t, weight;
    const double *gather;  // [ap][6]
    long long *ids;        // [ap][8]
    double *w;             // [ap][8]
    double *lU, *gth;      // [ap][3]
    double *torque;        // [ap]
};

DALM_HD void adj_alm_point(const AdjAlmPointArgs &X, int a) {
    typedef Dual<6> D;
    const TurbineDev &wt = X.A.wt[a / X.A.ap_per_wt];
    D off = D::seed(wt.formula[3], 0, ADJ_PI / 180);
    D pitch = D::seed(0.0, 1);
    D om = D::seed(wt.rot_speed, 2);
    D us[3] = {D::seed(0.0, 3), D::seed(0.0, 4), D::seed(0.0, 5)};
    PointEval<D> e;
    alm_point_eval(X.P, X.A, wt, a, X.t, X.U, off, pitch, om, us, e);
    const double *gq = X.gather + 6 * (long long)a;
    double lt = X.weight * ::fabs(wt.rot_speed);
    double acc[6];
    for (int p = 0; p < 6; p++) {
        double v = lt * e.torque.d[p];
        for (int m = 0; m < 3; m++) v += gq[m] * e.f[m].d[p] + gq[3 + m] * e.xyz[m].d[p];
        acc[p] = v;
    }
    for (int p = 0; p < 3; p++) {
        X.gth[3 * (long long)a + p] = acc[p];
        X.lU[3 * (long long)a + p] = acc[3 + p];
    }
    for (int q = 0; q < 8; q++) {
        X.ids[8 * (long long)a + q] = e.id[q];
        X.w[8 * (long long)a + q] = e.w[q];
    }
    X.torque[a] = e.torque.v;
}

// Turbine t's gradient (yaw deg, pitch deg, rotor speed): its points' terms
// in blade-point order, then the explicit |Omega| factor of the power.
DALM_HD void adj_alm_turbine_grad(const AlmDev &A, const double *gth, const double *torque,
                                  double weight, int t, double *grad) {
    double g[3] = {grad[3 * t], grad[3 * t + 1], grad[3 * t + 2]};
    double tau = 0;
    for (int a = t * A.ap_per_wt; a < (t + 1) * A.ap_per_wt; a++) {
        tau += torque[a];
        for (int p = 0; p < 3; p++) g[p] += gth[3 * (long long)a + p];
    }
    g[2] += weight * tau * sgn(A.wt[t].rot_speed);
    for (int p = 0; p < 3; p++) grad[3 * t + p] = g[p];
}

// Serial, in blade-point order: the sampled-velocity adjoints onto the grid
// (entry e = 8 a + q adds w[e] lU[a] to cell ids[e]) and the per-turbine
// gradient.  The device form (k_adj_alm_scatter) sums each cell's entries
// in the same order and so gives the same bits.
DALM_HD void adj_alm_scatter(const AlmDev &A, const long long *ids, const double *w,
                             const double *lU, const double *gth, const double *torque,
                             double weight, Vec3<double> aU, double *grad) {
    for (int t = 0; t < A.wt_count; t++) adj_alm_turbine_grad(A, gth, torque, weight, t, grad);
    for (long long e = 0; e < 8 * (long long)A.ap_count; e++) {
        long long c = ids[e];
        if (c < 0) continue;
        for (int m = 0; m < 3; m++) aU.c[m][c] += w[e] * lU[3 * (e / 8) + m];
    }
}

}  // namespace adj
}  // namespace dalm
