// FP64 stencil kernels of one time step.
//
// Compiled with --fmad=false: every expression keeps the reference's
// operation order and rounding (no contraction), so these stages agree with
// the reference bit for bit; the only libm call is cbrt in the eddy
// viscosity.
#include "flow.cuh"

namespace dalm {

namespace {

__device__ __forceinline__ double sgn(double v) { return (double)((v > 0.) - (v < 0.)); }

// The smooth van Albada limiter (DALM_LIMITER_VAN_ALBADA, an extension: the
// reference has only the limiter above): the face value of a cell with
// backward / forward differences a, b is  f +- (s/4)[(1 - k s) a + (1 + k s) b]
// with the switch s = (2ab + eps)/(a^2 + b^2 + eps) (van Albada, van Leer &
// Roberts 1982, in the kappa-MUSCL form), eps = 1e-12; differentiable
// everywhere, unlike the b=4 limiter.
__device__ __forceinline__ double va_switch(double a, double b) {
    const double eps = 1e-12;
    return (2. * a * b + eps) / (a * a + b * b + eps);
}

// κ=1/3 MUSCL reconstruction with the b=(3-κ)/(1-κ) limiter and the upwind
// face flux along one axis (src/cfd.h:37-60): returns flux(+) - flux(-).
__device__ __forceinline__ void muscl_axis(double fmm, double fm, double fc, double fp,
                                           double fpp, double Jp, double Jm, double &flux_p,
                                           double &flux_m, int limiter) {
    const double kap = 1. / 3.;
    const double bb = (3. - kap) / (1. - kap);
    const double e = 1.;
    double d4 = fpp - fp, d3 = fp - fc, d2 = fc - fm, d1 = fm - fmm;
    if (limiter == 1) {
        const double sp = va_switch(d4, d3), sc = va_switch(d3, d2), sm = va_switch(d2, d1);
        const double fpr = fp - (sp / 4.) * ((1. - kap * sp) * d4 + (1. + kap * sp) * d3);
        const double fpl = fc + (sc / 4.) * ((1. - kap * sc) * d2 + (1. + kap * sc) * d3);
        const double fmr = fc - (sc / 4.) * ((1. - kap * sc) * d3 + (1. + kap * sc) * d2);
        const double fml = fm + (sm / 4.) * ((1. - kap * sm) * d1 + (1. + kap * sm) * d2);
        flux_p = 0.5 * (Jp * (fpr + fpl) - fabs(Jp) * (fpr - fpl));
        flux_m = 0.5 * (Jm * (fmr + fml) - fabs(Jm) * (fmr - fml));
        return;
    }
    double s4 = sgn(d4), s3 = sgn(d3), s2 = sgn(d2), s1 = sgn(d1);
    double g6 = s4 * fmax(0., fmin(fabs(d4), s4 * bb * d3));
    double g5 = s3 * fmax(0., fmin(fabs(d3), s3 * bb * d4));
    double g4 = s3 * fmax(0., fmin(fabs(d3), s3 * bb * d2));
    double g3 = s2 * fmax(0., fmin(fabs(d2), s2 * bb * d3));
    double g2 = s2 * fmax(0., fmin(fabs(d2), s2 * bb * d1));
    double g1 = s1 * fmax(0., fmin(fabs(d1), s1 * bb * d2));
    double fpr = fp - (e / 4.) * ((1. - kap) * g6 + (1. + kap) * g5);
    double fpl = fc + (e / 4.) * ((1. - kap) * g3 + (1. + kap) * g4);
    double fmr = fc - (e / 4.) * ((1. - kap) * g4 + (1. + kap) * g3);
    double fml = fm + (e / 4.) * ((1. - kap) * g1 + (1. + kap) * g2);
    flux_p = 0.5 * (Jp * (fpr + fpl) - fabs(Jp) * (fpr - fpl));
    flux_m = 0.5 * (Jm * (fmr + fml) - fabs(Jm) * (fmr - fml));
}

__device__ __forceinline__ double sq(double v) { return v * v; }

// Loop over the cells of a Segments box: each block takes (32 k) x (8 j)
// column segments and marches along i, so the per-cell index arithmetic is
// done once per segment instead of per cell.  The body sees i, j, k;
// `continue` skips to the next cell.
#define TILE_LOOP(S)                                                      \
    for (int u_ = blockIdx.x; u_ < (S).count; u_ += gridDim.x) {          \
        int i0_, i1_, j, k;                                               \
        if (!(S).column(u_, i0_, i1_, j, k)) continue;                    \
        for (int i = i0_; i < i1_; i++) {
#define TILE_END \
        }        \
    }

// Smagorinsky viscosity at (i,j,k) from the velocity (src/cfd.h:786-825).
// The filter factor (Cs cbrt(dx dy dz))^2 comes precomputed per cell.
__device__ __forceinline__ double smagorinsky(const StepParams &P, Vec3<const double> U, int i,
                                              int j, int k) {
    const Grid &g = P.g;
    long long c = g.at(i, j, k);
    long long e = g.at(i + 1, j, k), w = g.at(i - 1, j, k), n = g.at(i, j + 1, k),
              s = g.at(i, j - 1, k), t = c + 1, b = c - 1;
    double dxew = P.m.x[i + 1] - P.m.x[i - 1];
    double dyns = P.m.y[j + 1] - P.m.y[j - 1];
    double dztb = P.m.z[k + 1] - P.m.z[k - 1];
    double dudx = (U.c[0][e] - U.c[0][w]) / dxew;
    double dudy = (U.c[0][n] - U.c[0][s]) / dyns;
    double dudz = (U.c[0][t] - U.c[0][b]) / dztb;
    double dvdx = (U.c[1][e] - U.c[1][w]) / dxew;
    double dvdy = (U.c[1][n] - U.c[1][s]) / dyns;
    double dvdz = (U.c[1][t] - U.c[1][b]) / dztb;
    double dwdx = (U.c[2][e] - U.c[2][w]) / dxew;
    double dwdy = (U.c[2][n] - U.c[2][s]) / dyns;
    double dwdz = (U.c[2][t] - U.c[2][b]) / dztb;
    double s1 = 2 * sq(dudx), s2 = 2 * sq(dvdy), s3 = 2 * sq(dwdz);
    double s4 = sq(dudy + dvdx), s5 = sq(dudz + dwdx), s6 = sq(dvdz + dwdy);
    double shear = sqrt(s1 + s2 + s3 + s4 + s5 + s6);
    return P.filter2[c] * shear;
}

__device__ __forceinline__ bool interior(const Grid &g, int i, int j, int k) {
    return i >= g.gc && i < g.nx - g.gc && j >= g.gc && j < g.ny - g.gc && k >= g.gc &&
           k < g.nz - g.gc;
}

// ---------------------------------------------------------------- predictor
//
// cpy_array(Uold, U) + calc_intermediate_U (src/solver.h:1042-1053,
// src/cfd.h:176-322).  The copy is a buffer swap on the host; this kernel
// writes the interior of the new buffer and copies its guide cells from the
// old one.  nut is the Smagorinsky viscosity of Uold, which is exactly the
// array the reference computed at the end of the previous step (calc_nut
// after apply_Ubc, src/solver.h:1157-1164), so it is evaluated inline.
__global__ void __launch_bounds__(TILE_THREADS, 2)
k_predict(StepParams P, Segments T, Vec3<const double> V, Vec3<double> Un, Vec3<const double> JU,
          Vec3<const double> F) {
    const Grid &g = P.g;
    TILE_LOOP(T)
        long long c = g.at(i, j, k);
        if (!interior(g, i, j, k)) {
            Un.c[0][c] = V.c[0][c];
            Un.c[1][c] = V.c[1][c];
            Un.c[2][c] = V.c[2][c];
            continue;
        }
        long long e = g.at(i + 1, j, k), ee = g.at(i + 2, j, k);
        long long w = g.at(i - 1, j, k), ww = g.at(i - 2, j, k);
        long long n = g.at(i, j + 1, k), nn = g.at(i, j + 2, k);
        long long s = g.at(i, j - 1, k), ss = g.at(i, j - 2, k);
        long long t = c + 1, tt = c + 2, b = c - 1, bb = c - 2;
        double dxc = P.m.dx[i], dyc = P.m.dy[j], dzc = P.m.dz[k];
        double J = dxc * dyc * dzc;
        double visc = 1 / P.re + smagorinsky(P, V, i, j, k);
        double JUE = JU.c[0][c], JUW = JU.c[0][w];
        double JVN = JU.c[1][c], JVS = JU.c[1][s];
        double JWT = JU.c[2][c], JWB = JU.c[2][b];
        double xi = P.m.x[i], xe = P.m.x[i + 1], xw = P.m.x[i - 1];
        double yj = P.m.y[j], yn = P.m.y[j + 1], ys = P.m.y[j - 1];
        double zk = P.m.z[k], zt = P.m.z[k + 1], zb = P.m.z[k - 1];
        bool has_f = P.fbox.contains(i, j, k);
#pragma unroll
        for (int m = 0; m < 3; m++) {
            const double *v = V.c[m];
            double fc = v[c];
            double fE, fW, fN, fS, fT, fB;
            muscl_axis(v[ww], v[w], fc, v[e], v[ee], JUE, JUW, fE, fW, P.limiter);
            muscl_axis(v[ss], v[s], fc, v[n], v[nn], JVN, JVS, fN, fS, P.limiter);
            muscl_axis(v[bb], v[b], fc, v[t], v[tt], JWT, JWB, fT, fB, P.limiter);
            double conv = (fE - fW + fN - fS + fT - fB) / J;
            double diff = visc * (((v[e] - fc) / (xe - xi) - (fc - v[w]) / (xi - xw)) / dxc +
                                  ((v[n] - fc) / (yn - yj) - (fc - v[s]) / (yj - ys)) / dyc +
                                  ((v[t] - fc) / (zt - zk) - (fc - v[b]) / (zk - zb)) / dzc);
            double fm = has_f ? F.c[m][c] : 0.0;
            Un.c[m][c] = fc + P.dt * (-conv + diff + fm);
        }
    TILE_END
}

// ------------------------------------------- face fluxes, their BCs, RHS

// interpolate_JU face values (src/cfd.h:395-420) with apply_JUbc overrides
// (src/bc.h:235-302, inflow profile extension) for the faces the override
// touches.  Faces are identified by their lower cell (i,j,k).
__device__ __forceinline__ double face_x(const StepParams &P, Vec3<const double> U, int i, int j,
                                         int k) {
    const Grid &g = P.g;
    double yz = P.m.dy[j] * P.m.dz[k];
    if (i == g.gc - 1 && j >= g.gc && j < g.ny - g.gc && k >= g.gc && k < g.nz - g.gc) {
        double u = P.prof ? P.prof[((long long)j * g.nz + k) * 3] : P.uin[0];
        return yz * u;
    }
    return 0.5 * (U.c[0][g.at(i, j, k)] * yz + U.c[0][g.at(i + 1, j, k)] * yz);
}
__device__ __forceinline__ double face_y(const StepParams &P, Vec3<const double> U, int i, int j,
                                         int k) {
    const Grid &g = P.g;
    if ((j == g.gc - 1 || j == g.ny - g.gc - 1) && i >= g.gc && i < g.nx - g.gc && k >= g.gc &&
        k < g.nz - g.gc)
        return 0;
    double xz = P.m.dx[i] * P.m.dz[k];
    return 0.5 * (U.c[1][g.at(i, j, k)] * xz + U.c[1][g.at(i, j + 1, k)] * xz);
}
__device__ __forceinline__ double face_z(const StepParams &P, Vec3<const double> U, int i, int j,
                                         int k) {
    const Grid &g = P.g;
    if ((k == g.gc - 1 || k == g.nz - g.gc - 1) && i >= g.gc && i < g.nx - g.gc && j >= g.gc &&
        j < g.ny - g.gc)
        return 0;
    double xy = P.m.dx[i] * P.m.dy[j];
    return 0.5 * (U.c[2][g.at(i, j, k)] * xy + U.c[2][g.at(i, j, k + 1)] * xy);
}

// interpolate_JU + apply_JUbc + calc_poisson_rhs (src/solver.h:1055-1077).
// Covers faces i,j,k in [gc-1, N-gc); the RHS of an interior cell needs its
// west/south/bottom faces, which it recomputes (same arithmetic, same bits).
template <bool RHS>
__global__ void __launch_bounds__(TILE_THREADS)
k_flux_rhs(StepParams P, Segments T, Vec3<const double> U, Vec3<double> JU, double *b) {
    const Grid &g = P.g;
    TILE_LOOP(T)
        long long c = g.at(i, j, k);
        double fe = face_x(P, U, i, j, k), fn = face_y(P, U, i, j, k), ft = face_z(P, U, i, j, k);
        JU.c[0][c] = fe;
        JU.c[1][c] = fn;
        JU.c[2][c] = ft;
        if (RHS && interior(g, i, j, k)) {
            double fw = face_x(P, U, i - 1, j, k), fs = face_y(P, U, i, j - 1, k),
                   fb = face_z(P, U, i, j, k - 1);
            double J = P.m.dx[i] * P.m.dy[j] * P.m.dz[k];
            double divergence = (fe - fw + fn - fs + ft - fb) / J;
            b[c] = divergence / (P.dt * P.max_diag);
        }
    TILE_END
}

// ------------------------------------------------------------- projection

// apply_pbc (src/bc.h:304-411): one thread per guide cell of the six faces.
__global__ void k_pressure_bc(StepParams P, double *p) {
    const Grid &g = P.g;
    int GC = g.gc;
    long long nyz = (long long)g.nj() * g.nk(), nxz = (long long)g.ni() * g.nk(),
              nxy = (long long)g.ni() * g.nj();
    long long tot = 2 * (nyz + nxz + nxy);
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < tot;
         n += (long long)gridDim.x * blockDim.x) {
        long long r = n;
        if (r < 2 * nyz) {
            int side = (int)(r / nyz);
            long long q = r % nyz;
            int j = GC + (int)(q / g.nk()), k = GC + (int)(q % g.nk());
            if (side == 0) {
                p[g.at(GC - 1, j, k)] = p[g.at(GC, j, k)];
            } else {
                int ii = g.nx - GC - 1, io = g.nx - GC;
                double hi = 0.5 * P.m.dx[ii], ho = 0.5 * P.m.dx[io], pbc = 0;
                p[g.at(io, j, k)] = pbc - (p[g.at(ii, j, k)] - pbc) * (ho / hi);
            }
            continue;
        }
        r -= 2 * nyz;
        if (r < 2 * nxz) {
            int side = (int)(r / nxz);
            long long q = r % nxz;
            int i = GC + (int)(q / g.nk()), k = GC + (int)(q % g.nk());
            if (side == 0) p[g.at(i, GC - 1, k)] = p[g.at(i, GC, k)];
            else p[g.at(i, g.ny - GC, k)] = p[g.at(i, g.ny - GC - 1, k)];
            continue;
        }
        r -= 2 * nxz;
        int side = (int)(r / nxy);
        long long q = r % nxy;
        int i = GC + (int)(q / g.nj()), j = GC + (int)(q % g.nj());
        if (side == 0) p[g.at(i, j, GC - 1)] = p[g.at(i, j, GC)];
        else p[g.at(i, j, g.nz - GC)] = p[g.at(i, j, g.nz - GC - 1)];
    }
}

// Projected face flux with the apply_JUbc override: project_p's compact
// correction (src/cfd.h:716-740) then the BC (src/bc.h:235-302).
__device__ __forceinline__ double proj_face(const StepParams &P, Vec3<double> JU, const double *p,
                                            int axis, int i, int j, int k) {
    const Grid &g = P.g;
    long long c = g.at(i, j, k);
    if (axis == 0) {
        if (i == g.gc - 1 && j >= g.gc && j < g.ny - g.gc && k >= g.gc && k < g.nz - g.gc) {
            double u = P.prof ? P.prof[((long long)j * g.nz + k) * 3] : P.uin[0];
            return (P.m.dy[j] * P.m.dz[k]) * u;
        }
        double yz = P.m.dy[j] * P.m.dz[k];
        double dpdx = (p[g.at(i + 1, j, k)] - p[c]) / (P.m.x[i + 1] - P.m.x[i]);
        return JU.c[0][c] - P.dt * yz * dpdx;
    } else if (axis == 1) {
        if ((j == g.gc - 1 || j == g.ny - g.gc - 1) && i >= g.gc && i < g.nx - g.gc &&
            k >= g.gc && k < g.nz - g.gc)
            return 0;
        double xz = P.m.dx[i] * P.m.dz[k];
        double dpdy = (p[g.at(i, j + 1, k)] - p[c]) / (P.m.y[j + 1] - P.m.y[j]);
        return JU.c[1][c] - P.dt * xz * dpdy;
    } else {
        if ((k == g.gc - 1 || k == g.nz - g.gc - 1) && i >= g.gc && i < g.nx - g.gc &&
            j >= g.gc && j < g.ny - g.gc)
            return 0;
        double xy = P.m.dx[i] * P.m.dy[j];
        double dpdz = (p[g.at(i, j, k + 1)] - p[c]) / (P.m.z[k + 1] - P.m.z[k]);
        return JU.c[2][c] - P.dt * xy * dpdz;
    }
}

// project_p (src/cfd.h:601-783) + set_solid_U + the apply_JUbc that follows it
// + calc_divergence norm + calc_max_cfl (src/solver.h:1122-1186).  The
// velocity BCs (apply_Ubc) run in k_velocity_bc after this kernel; they touch
// guide cells only, so the interior velocity used for the CFL here is final.
// A thread owns the three faces of its lower cell; the divergence of an
// interior cell also needs its west/south/bottom faces, which it recomputes
// from the pre-projection flux.  Because other threads overwrite those faces
// in the same launch, the projected flux goes to a second buffer (JUout) and
// the host swaps the two.
__global__ void __launch_bounds__(TILE_THREADS)
k_project(StepParams P, Segments T, Vec3<double> U, Vec3<double> JUin, Vec3<double> JUout,
          const double *p, Partials<2> part, DiagState *diag) {
    const Grid &g = P.g;
    double div2 = 0, cfl = 0;
    TILE_LOOP(T)
        long long c = g.at(i, j, k);
        double fe = proj_face(P, JUin, p, 0, i, j, k);
        double fn = proj_face(P, JUin, p, 1, i, j, k);
        double ft = proj_face(P, JUin, p, 2, i, j, k);
        JUout.c[0][c] = fe;
        JUout.c[1][c] = fn;
        JUout.c[2][c] = ft;
        if (interior(g, i, j, k)) {
            double u = U.c[0][c] - P.dt * (p[g.at(i + 1, j, k)] - p[g.at(i - 1, j, k)]) /
                                       (P.m.x[i + 1] - P.m.x[i - 1]);
            double v = U.c[1][c] - P.dt * (p[g.at(i, j + 1, k)] - p[g.at(i, j - 1, k)]) /
                                       (P.m.y[j + 1] - P.m.y[j - 1]);
            double w = U.c[2][c] - P.dt * (p[c + 1] - p[c - 1]) / (P.m.z[k + 1] - P.m.z[k - 1]);
            if (P.solid) {  // set_solid_U (src/cfd.h:1143-1160)
                const double sf = P.solid[c];
                u = (1. - sf) * u;
                v = (1. - sf) * v;
                w = (1. - sf) * w;
            }
            U.c[0][c] = u;
            U.c[1][c] = v;
            U.c[2][c] = w;
            double fw = proj_face(P, JUin, p, 0, i - 1, j, k);
            double fs = proj_face(P, JUin, p, 1, i, j - 1, k);
            double fb = proj_face(P, JUin, p, 2, i, j, k - 1);
            double J = P.m.dx[i] * P.m.dy[j] * P.m.dz[k];
            double d = (fe - fw + fn - fs + ft - fb) / J;
            div2 += d * d;
            double local = fabs(u) * P.dt / P.m.dx[i] + fabs(v) * P.dt / P.m.dy[j] +
                           fabs(w) * P.dt / P.m.dz[k];
            cfl = local > cfl ? local : cfl;
        }
    TILE_END
    if (P.reference_sums) return;  // k_seq_diag sums in the reference's order
    double v[2] = {div2, cfl};
    if (grid_reduce<2>(v, 2u, part) && threadIdx.x == 0) {
        diag->div2 = v[0];
        diag->max_cfl = v[1];
        diag->avg_div = sqrt(v[0]) / sqrt(diag->ncell);
    }
}

// divergence of cell c from the face fluxes (src/cfd.h:1093-1105) and the
// cell CFL number (src/cfd.h:1126-1130)
template <typename T>
__device__ __forceinline__ double cell_div(const StepParams &P, Vec3<const T> JU, int i, int j,
                                           int k) {
    const Grid &g = P.g;
    long long c = g.at(i, j, k);
    double J = P.m.dx[i] * P.m.dy[j] * P.m.dz[k];
    return ((double)JU.c[0][c] - (double)JU.c[0][g.at(i - 1, j, k)] + (double)JU.c[1][c] -
            (double)JU.c[1][g.at(i, j - 1, k)] + (double)JU.c[2][c] - (double)JU.c[2][c - 1]) / J;
}
template <typename T>
__device__ __forceinline__ double cell_cfl(const StepParams &P, Vec3<const T> U, int i, int j,
                                           int k) {
    long long c = P.g.at(i, j, k);
    return fabs((double)U.c[0][c]) * P.dt / P.m.dx[i] + fabs((double)U.c[1][c]) * P.dt / P.m.dy[j] +
           fabs((double)U.c[2][c]) * P.dt / P.m.dz[k];
}

// Diagnostics alone (after set_state): sum div^2 and max CFL.
template <typename T>
__global__ void __launch_bounds__(TILE_THREADS)
k_diag(StepParams P, Segments S, Vec3<const T> U, Vec3<const T> JU, Partials<2> part,
       DiagState *diag) {
    double div2 = 0, cfl = 0;
    TILE_LOOP(S)
        double d = cell_div(P, JU, i, j, k);
        div2 += d * d;
        double local = cell_cfl(P, U, i, j, k);
        cfl = local > cfl ? local : cfl;
    TILE_END
    double v[2] = {div2, cfl};
    if (grid_reduce<2>(v, 2u, part) && threadIdx.x == 0) {
        diag->div2 = v[0];
        diag->max_cfl = v[1];
        diag->avg_div = sqrt(v[0]) / sqrt(diag->ncell);
    }
}

// The same diagnostics summed in the reference's serial order by one warp:
// calc_l2_norm(div) (src/mv.h:33-55) and calc_max_cfl (src/cfd.h:1109-1141).
__global__ void k_seq_diag(StepParams P, Vec3<const double> U, Vec3<const double> JU,
                           DiagState *diag) {
    const Grid &g = P.g;
    double tot[2];
    warp_serial_sums<2>(
        g,
        [&](long long c, double (&t)[2]) {
            long long r = c - g.off;
            int i = (int)(r / g.sx), j = (int)((r % g.sx) / g.sy), k = (int)(r % g.sy);
            double d = cell_div(P, JU, i, j, k);
            t[0] = d * d;
            t[1] = 0;
        },
        tot);
    // max is exact in any order
    double cfl = 0;
    int lane = threadIdx.x & 31;
    for (int i = g.gc; i < g.nx - g.gc; i++)
        for (int j = g.gc; j < g.ny - g.gc; j++)
            for (int k = g.gc + lane; k < g.nz - g.gc; k += 32) {
                double local = cell_cfl(P, U, i, j, k);
                cfl = local > cfl ? local : cfl;
            }
    for (int o = 16; o > 0; o >>= 1) {
        double other = __shfl_down_sync(0xffffffffu, cfl, o);
        cfl = other > cfl ? other : cfl;
    }
    if (lane == 0) {
        diag->div2 = tot[0];
        diag->max_cfl = cfl;
        diag->avg_div = sqrt(tot[0]) / sqrt(diag->ncell);
    }
}

// Three-point Lagrange extrapolation (src/util.h:201-212).
__device__ __forceinline__ double quad_poly(double x0, double x1, double x2, double f0, double f1,
                                            double f2, double x3) {
    double l0 = ((x3 - x1) * (x3 - x2)) / ((x0 - x1) * (x0 - x2));
    double l1 = ((x3 - x0) * (x3 - x2)) / ((x1 - x0) * (x1 - x2));
    double l2 = ((x3 - x0) * (x3 - x1)) / ((x2 - x0) * (x2 - x1));
    return f0 * l0 + f1 * l1 + f2 * l2;
}

// apply_Ubc (src/bc.h:5-233): inflow (uniform Uin or profile), convective
// outflow on Uold, slip y-/y+/z+, no-slip z-.  One thread per face column;
// each writes the gc guide cells of its column.  Reads only interior cells
// of U and the old guide values, so the faces are independent.
// T is the storage type of U (double; float for the FP32 stencil fields of
// the mixed form): the arithmetic is FP64 either way.
template <typename T>
__global__ void k_velocity_bc(StepParams P, Vec3<T> U, Vec3<const T> V) {
    const Grid &g = P.g;
    int GC = g.gc;
    long long nyz = (long long)g.nj() * g.nk(), nxz = (long long)g.ni() * g.nk(),
              nxy = (long long)g.ni() * g.nj();
    long long tot = 2 * (nyz + nxz + nxy);
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < tot;
         n += (long long)gridDim.x * blockDim.x) {
        long long r = n;
        if (r < 2 * nyz) {
            int side = (int)(r / nyz);
            long long q = r % nyz;
            int j = GC + (int)(q / g.nk()), k = GC + (int)(q % g.nk());
            if (side == 0) {
                for (int i = 0; i < GC; i++) {
                    long long id = g.at(i, j, k);
                    for (int m = 0; m < 3; m++)
                        U.c[m][id] = (T)(P.prof ? P.prof[((long long)j * g.nz + k) * 3 + m] : P.uin[m]);
                }
            } else {
                for (int i = g.nx - GC; i < g.nx; i++) {
                    long long i0 = g.at(i, j, k), i1 = g.at(i - 1, j, k), i2 = g.at(i - 2, j, k);
                    double uout = (double)U.c[0][i0];
                    double nv[3];
                    for (int m = 0; m < 3; m++) {
                        double f0 = (double)V.c[m][i0], f1 = (double)V.c[m][i1], f2 = (double)V.c[m][i2];
                        double grad = (3 * f0 - 4 * f1 + f2) / 2;
                        nv[m] = f0 - uout * P.dt * grad / P.m.dx[i];
                    }
                    for (int m = 0; m < 3; m++) U.c[m][i0] = (T)nv[m];
                }
            }
            continue;
        }
        r -= 2 * nyz;
        if (r < 2 * nxz) {
            int side = (int)(r / nxz);
            long long q = r % nxz;
            int i = GC + (int)(q / g.nk()), k = GC + (int)(q % g.nk());
            int j0 = side ? g.ny - GC - 2 : GC + 1, j1 = side ? g.ny - GC - 1 : GC;
            int j3 = side ? g.ny - GC : GC - 1, j4 = side ? g.ny - GC + 1 : GC - 2;
            long long a0 = g.at(i, j0, k), a1 = g.at(i, j1, k), a3 = g.at(i, j3, k),
                      a4 = g.at(i, j4, k);
            double y0 = P.m.y[j0], y1 = P.m.y[j1];
            double y2 = side ? P.m.y[j1] + 0.5 * P.m.dy[j1] : P.m.y[j1] - 0.5 * P.m.dy[j1];
            double y3 = P.m.y[j3], y4 = P.m.y[j4];
            double ubc[3] = {(double)U.c[0][a1], 0, (double)U.c[2][a1]};
            for (int m = 0; m < 3; m++) {
                double f0 = (double)U.c[m][a0], f1 = (double)U.c[m][a1], f2 = ubc[m];
                U.c[m][a3] = (T)quad_poly(y0, y1, y2, f0, f1, f2, y3);
                U.c[m][a4] = (T)quad_poly(y0, y1, y2, f0, f1, f2, y4);
            }
            continue;
        }
        r -= 2 * nxz;
        int side = (int)(r / nxy);
        long long q = r % nxy;
        int i = GC + (int)(q / g.nj()), j = GC + (int)(q % g.nj());
        int k0 = side ? g.nz - GC - 2 : GC + 1, k1 = side ? g.nz - GC - 1 : GC;
        int k3 = side ? g.nz - GC : GC - 1, k4 = side ? g.nz - GC + 1 : GC - 2;
        long long a0 = g.at(i, j, k0), a1 = g.at(i, j, k1), a3 = g.at(i, j, k3),
                  a4 = g.at(i, j, k4);
        double z0 = P.m.z[k0], z1 = P.m.z[k1];
        double z2 = side ? P.m.z[k1] + 0.5 * P.m.dz[k1] : P.m.z[k1] - 0.5 * P.m.dz[k1];
        double z3 = P.m.z[k3], z4 = P.m.z[k4];
        double ubc[3] = {0, 0, 0};
        // z+ slip; z- no slip, or slip upstream of a retracted floor's start
        // (src/bc.h:140-160)
        if (side || (P.retracted && P.m.x[i] < P.floor_start)) {
            ubc[0] = (double)U.c[0][a1];
            ubc[1] = (double)U.c[1][a1];
        }
        for (int m = 0; m < 3; m++) {
            double f0 = (double)U.c[m][a0], f1 = (double)U.c[m][a1], f2 = ubc[m];
            U.c[m][a3] = (T)quad_poly(z0, z1, z2, f0, f1, f2, z3);
            U.c[m][a4] = (T)quad_poly(z0, z1, z2, f0, f1, f2, z4);
        }
    }
}

__global__ void __launch_bounds__(TILE_THREADS)
k_nut_field(StepParams P, Segments T, Vec3<const double> U, double *nut) {
    TILE_LOOP(T)
        nut[P.g.at(i, j, k)] = smagorinsky(P, U, i, j, k);
    TILE_END
}

__global__ void __launch_bounds__(TILE_THREADS)
k_div_field(StepParams P, Segments T, Vec3<const double> JU, double *div) {
    const Grid &g = P.g;
    TILE_LOOP(T)
        long long c = g.at(i, j, k);
        double J = P.m.dx[i] * P.m.dy[j] * P.m.dz[k];
        div[c] = (JU.c[0][c] - JU.c[0][g.at(i - 1, j, k)] + JU.c[1][c] -
                  JU.c[1][g.at(i, j - 1, k)] + JU.c[2][c] - JU.c[2][c - 1]) / J;
    TILE_END
}

// Q-criterion on the interior (calc_q_at_cell, src/cfd.h:949-975): central
// differences over x[i+1] - x[i-1] etc., same operation order.
__global__ void __launch_bounds__(TILE_THREADS)
k_q_field(StepParams P, Segments T, Vec3<const double> U, double *q) {
    const Grid &g = P.g;
    TILE_LOOP(T)
        const long long c = g.at(i, j, k);
        const long long ce = g.at(i + 1, j, k), cw = g.at(i - 1, j, k);
        const long long cn = g.at(i, j + 1, k), cs = g.at(i, j - 1, k);
        const long long ct = c + 1, cb = c - 1;
        const double dxew = P.m.x[i + 1] - P.m.x[i - 1];
        const double dyns = P.m.y[j + 1] - P.m.y[j - 1];
        const double dztb = P.m.z[k + 1] - P.m.z[k - 1];
        const double dudx = (U.c[0][ce] - U.c[0][cw]) / dxew;
        const double dudy = (U.c[0][cn] - U.c[0][cs]) / dyns;
        const double dudz = (U.c[0][ct] - U.c[0][cb]) / dztb;
        const double dvdx = (U.c[1][ce] - U.c[1][cw]) / dxew;
        const double dvdy = (U.c[1][cn] - U.c[1][cs]) / dyns;
        const double dvdz = (U.c[1][ct] - U.c[1][cb]) / dztb;
        const double dwdx = (U.c[2][ce] - U.c[2][cw]) / dxew;
        const double dwdy = (U.c[2][cn] - U.c[2][cs]) / dyns;
        const double dwdz = (U.c[2][ct] - U.c[2][cb]) / dztb;
        q[c] = -0.5 * (dudx * dudx + dvdy * dvdy + dwdz * dwdz +
                       2 * (dudy * dvdx + dudz * dwdx + dvdz * dwdy));
    TILE_END
}

// Running time average over every stored cell (calc_ax_plus_by,
// src/mv.h:322-335 as used at src/solver.h:1198-1203).
template <typename T>
__global__ void k_tavg(Grid g, Vec3<double> A, Vec3<const T> U, double w) {
    long long tot = (long long)g.nx * g.ny * g.nz;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < tot;
         n += (long long)gridDim.x * blockDim.x) {
        int k = (int)(n % g.nz);
        long long r = n / g.nz;
        int j = (int)(r % g.ny), i = (int)(r / g.ny);
        long long c = g.at(i, j, k);
        for (int m = 0; m < 3; m++) A.c[m][c] = (1. - w) * A.c[m][c] + w * (double)U.c[m][c];
    }
}

__global__ void k_to_device(Grid g, const double *ref, int nc, double *d0, double *d1, double *d2) {
    long long tot = (long long)g.nx * g.ny * g.nz;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < tot;
         n += (long long)gridDim.x * blockDim.x) {
        int k = (int)(n % g.nz);
        long long r = n / g.nz;
        int j = (int)(r % g.ny), i = (int)(r / g.ny);
        long long c = g.at(i, j, k);
        if (nc == 1) {
            d0[c] = ref[n];
        } else {
            d0[c] = ref[3 * n];
            d1[c] = ref[3 * n + 1];
            d2[c] = ref[3 * n + 2];
        }
    }
}

__global__ void k_to_ref(Grid g, const double *s0, const double *s1, const double *s2, int nc,
                         double *ref) {
    long long tot = (long long)g.nx * g.ny * g.nz;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < tot;
         n += (long long)gridDim.x * blockDim.x) {
        int k = (int)(n % g.nz);
        long long r = n / g.nz;
        int j = (int)(r % g.ny), i = (int)(r / g.ny);
        long long c = g.at(i, j, k);
        if (nc == 1) {
            ref[n] = s0[c];
        } else {
            ref[3 * n] = s0[c];
            ref[3 * n + 1] = s1[c];
            ref[3 * n + 2] = s2[c];
        }
    }
}

__global__ void k_fill(double *p, long long n, double v) {
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < n;
         x += (long long)gridDim.x * blockDim.x)
        p[x] = v;
}

Box interior_box(const Grid &g) {
    return Box{{g.gc, g.gc, g.gc}, {g.nx - g.gc, g.ny - g.gc, g.nz - g.gc}};
}
Box face_box(const Grid &g) {
    return Box{{g.gc - 1, g.gc - 1, g.gc - 1}, {g.nx - g.gc, g.ny - g.gc, g.nz - g.gc}};
}
Box full_box(const Grid &g) { return Box{{0, 0, 0}, {g.nx, g.ny, g.nz}}; }

int plane_blocks(const Grid &g) {
    long long tot = 2 * ((long long)g.nj() * g.nk() + (long long)g.ni() * g.nk() +
                         (long long)g.ni() * g.nj());
    long long b = (tot + 255) / 256;
    return (int)(b < 4096 ? (b > 0 ? b : 1) : 4096);
}

template <typename T>
__global__ void k_gather_points(Vec3<const T> U, const long long *idx, int n, double *out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    for (int m = 0; m < 3; m++) out[3 * t + m] = (double)U.c[m][idx[t]];
}

// element-wise precision conversions over whole allocations (same layout)
__global__ void k_widen(const float *src, double *dst, long long n) {
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < n;
         x += (long long)gridDim.x * blockDim.x)
        dst[x] = (double)src[x];
}
__global__ void k_narrow(const double *src, float *dst, long long n) {
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < n;
         x += (long long)gridDim.x * blockDim.x)
        dst[x] = (float)src[x];
}

}  // namespace

void launch_predict(const LaunchCtx &L, const StepParams &P, Vec3<const double> uold,
                    Vec3<double> unew, Vec3<const double> ju, Vec3<const double> f) {
    Segments T = Segments::make(full_box(P.g), L.blocks);
    L.pre(KK_PREDICT);
    k_predict<<<L.blocks, TILE_THREADS, 0, L.s>>>(P, T, uold, unew, ju, f);
    L.post(KK_PREDICT);
}

void launch_flux_rhs(const LaunchCtx &L, const StepParams &P, Vec3<const double> u,
                     Vec3<double> ju, double *b) {
    Segments T = Segments::make(face_box(P.g), L.blocks);
    L.pre(KK_FLUX_RHS);
    k_flux_rhs<true><<<L.blocks, TILE_THREADS, 0, L.s>>>(P, T, u, ju, b);
    L.post(KK_FLUX_RHS);
}

void launch_flux_only(const LaunchCtx &L, const StepParams &P, Vec3<const double> u,
                      Vec3<double> ju) {
    Segments T = Segments::make(face_box(P.g), L.blocks);
    L.pre(KK_FLUX_RHS);
    k_flux_rhs<false><<<L.blocks, TILE_THREADS, 0, L.s>>>(P, T, u, ju, nullptr);
    L.post(KK_FLUX_RHS);
}

void launch_pressure_bc(const LaunchCtx &L, const StepParams &P, double *p) {
    L.pre(KK_PBC);
    k_pressure_bc<<<plane_blocks(P.g), 256, 0, L.s>>>(P, p);
    L.post(KK_PBC);
}

void launch_project(const LaunchCtx &L, const StepParams &P, Vec3<double> u,
                    Vec3<double> ju_in, Vec3<double> ju_out, const double *p, Partials<2> part,
                    DiagState *diag) {
    Segments T = Segments::make(face_box(P.g), L.blocks);
    L.pre(KK_PROJECT);
    k_project<<<L.blocks, TILE_THREADS, 0, L.s>>>(P, T, u, ju_in, ju_out, p, part, diag);
    L.post(KK_PROJECT);
    if (P.reference_sums) {
        L.pre(KK_DIAG);
        k_seq_diag<<<1, 32, 0, L.s>>>(P, {{u.c[0], u.c[1], u.c[2]}},
                                      {{ju_out.c[0], ju_out.c[1], ju_out.c[2]}}, diag);
        L.post(KK_DIAG);
    }
}

template <typename T>
void launch_velocity_bc(const LaunchCtx &L, const StepParams &P, Vec3<T> u, Vec3<const T> uold) {
    L.pre(KK_UBC);
    k_velocity_bc<T><<<plane_blocks(P.g), 256, 0, L.s>>>(P, u, uold);
    L.post(KK_UBC);
}
template void launch_velocity_bc<double>(const LaunchCtx &, const StepParams &, Vec3<double>,
                                         Vec3<const double>);
template void launch_velocity_bc<float>(const LaunchCtx &, const StepParams &, Vec3<float>,
                                        Vec3<const float>);

void launch_diag(const LaunchCtx &L, const StepParams &P, Vec3<const double> u,
                 Vec3<const double> ju, Partials<2> part, DiagState *diag) {
    Segments T = Segments::make(interior_box(P.g), L.blocks);
    L.pre(KK_DIAG);
    if (P.reference_sums)
        k_seq_diag<<<1, 32, 0, L.s>>>(P, u, ju, diag);
    else
        k_diag<double><<<L.blocks, TILE_THREADS, 0, L.s>>>(P, T, u, ju, part, diag);
    L.post(KK_DIAG);
}

void launch_diag(const LaunchCtx &L, const StepParams &P, Vec3<const float> u,
                 Vec3<const float> ju, Partials<2> part, DiagState *diag) {
    Segments T = Segments::make(interior_box(P.g), L.blocks);
    L.pre(KK_DIAG);
    k_diag<float><<<L.blocks, TILE_THREADS, 0, L.s>>>(P, T, u, ju, part, diag);
    L.post(KK_DIAG);
}

void launch_nut_field(const LaunchCtx &L, const StepParams &P, Vec3<const double> u, double *nut) {
    Segments T = Segments::make(interior_box(P.g), L.blocks);
    L.pre(KK_LAYOUT);
    k_nut_field<<<L.blocks, TILE_THREADS, 0, L.s>>>(P, T, u, nut);
    L.post(KK_LAYOUT);
}

void launch_div_field(const LaunchCtx &L, const StepParams &P, Vec3<const double> ju, double *div) {
    Segments T = Segments::make(interior_box(P.g), L.blocks);
    L.pre(KK_LAYOUT);
    k_div_field<<<L.blocks, TILE_THREADS, 0, L.s>>>(P, T, ju, div);
    L.post(KK_LAYOUT);
}

void launch_q_field(const LaunchCtx &L, const StepParams &P, Vec3<const double> u, double *q) {
    Segments T = Segments::make(interior_box(P.g), L.blocks);
    L.pre(KK_LAYOUT);
    k_q_field<<<L.blocks, TILE_THREADS, 0, L.s>>>(P, T, u, q);
    L.post(KK_LAYOUT);
}

template <typename T>
void launch_tavg(const LaunchCtx &L, const Grid &g, Vec3<double> tavg, Vec3<const T> u, double w) {
    L.pre(KK_TAVG);
    k_tavg<T><<<L.blocks, 256, 0, L.s>>>(g, tavg, u, w);
    L.post(KK_TAVG);
}
template void launch_tavg<double>(const LaunchCtx &, const Grid &, Vec3<double>,
                                  Vec3<const double>, double);
template void launch_tavg<float>(const LaunchCtx &, const Grid &, Vec3<double>, Vec3<const float>,
                                 double);

void launch_to_device_layout(const LaunchCtx &L, const Grid &g, const double *ref, int ncomp,
                             double *const *dst) {
    L.pre(KK_LAYOUT);
    k_to_device<<<L.blocks, 256, 0, L.s>>>(g, ref, ncomp, dst[0], ncomp == 3 ? dst[1] : nullptr,
                                           ncomp == 3 ? dst[2] : nullptr);
    L.post(KK_LAYOUT);
}

void launch_to_ref_layout(const LaunchCtx &L, const Grid &g, double *const *src, int ncomp,
                          double *ref) {
    L.pre(KK_LAYOUT);
    k_to_ref<<<L.blocks, 256, 0, L.s>>>(g, src[0], ncomp == 3 ? src[1] : nullptr,
                                        ncomp == 3 ? src[2] : nullptr, ncomp, ref);
    L.post(KK_LAYOUT);
}

template <typename T>
void launch_gather_points(const LaunchCtx &L, Vec3<const T> u, const long long *idx, int n,
                          double *out) {
    if (n <= 0) return;
    L.pre(KK_LAYOUT);
    k_gather_points<T><<<(n + 127) / 128, 128, 0, L.s>>>(u, idx, n, out);
    L.post(KK_LAYOUT);
}
template void launch_gather_points<double>(const LaunchCtx &, Vec3<const double>,
                                           const long long *, int, double *);
template void launch_gather_points<float>(const LaunchCtx &, Vec3<const float>, const long long *,
                                          int, double *);

void launch_widen(const LaunchCtx &L, const float *src, double *dst, long long n) {
    L.pre(KK_LAYOUT);
    k_widen<<<L.blocks, 256, 0, L.s>>>(src, dst, n);
    L.post(KK_LAYOUT);
}
void launch_narrow(const LaunchCtx &L, const double *src, float *dst, long long n) {
    L.pre(KK_LAYOUT);
    k_narrow<<<L.blocks, 256, 0, L.s>>>(src, dst, n);
    L.post(KK_LAYOUT);
}

void launch_fill(const LaunchCtx &L, double *p, long long n, double v) {
    L.pre(KK_LAYOUT);
    k_fill<<<L.blocks, 256, 0, L.s>>>(p, n, v);
    L.post(KK_LAYOUT);
}

}  // namespace dalm
