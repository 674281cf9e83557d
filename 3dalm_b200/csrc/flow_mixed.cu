// Flow stages of the mixed-precision form (DALM_MIXED) on FP32 stencil
// fields: the velocity U (both time levels), the face fluxes JU and the
// actuator-line force f are stored in FP32; the pressure p, the Poisson
// right-hand side b (the divergence residual) and every sum stay FP64.
//
//   k_predict32   cpy_array(Uold, U) + calc_intermediate_U
//                 (src/cfd.h:176-322, src/solver.h:1042-1053) with the
//                 Smagorinsky viscosity of Uold inline (calc_nut,
//                 src/cfd.h:786-904)
//   k_flux32      interpolate_JU + apply_JUbc + calc_poisson_rhs
//                 (src/cfd.h:395-598, src/bc.h:235-302); b in FP64
//   k_project32   project_p + set_solid_U + apply_JUbc + the divergence
//                 norm and max CFL (src/cfd.h:601-783, 1079-1141); the
//                 pressure-gradient corrections and the divergence in FP64
//
// Compiled with contraction and fast quotients: this form has no parity to
// keep with the reference; its error against the FP64 form is measured.
//
// All three kernels walk column segments (a block owns 32 k x 8 j cells and
// marches through a chunk of i-planes).  The predictor keeps each thread's
// five i-neighbours in a register ring and stages the current plane with a
// two-cell halo in j and k in shared memory (double-buffered, one barrier per
// plane).  A face flux is the same number for the two cells that share the
// face (the kappa-MUSCL face states of src/cfd.h:37-60 depend only on the
// four values around the face), so each x face is computed once and carried
// to the next plane, and each y face once and passed to the next row through
// shared memory; z faces are computed by both cells (a warp's row).
#include <algorithm>

#include "flow.cuh"

namespace dalm {

namespace {

__device__ __forceinline__ float qf(float a, float b) { return __fdividef(a, b); }

__device__ __forceinline__ float va_switch_f(float a, float b) {
    const float eps = 1e-12f;
    return qf(2.f * a * b + eps, a * a + b * b + eps);
}

// the b=4 limiter term s_a max(0, min(|a|, s_a bb b)) for (a, b) and
// (b, a): zero unless a and b have the same sign, else min(|a|, bb |b|)
// with a's sign
__device__ __forceinline__ void minmod_pair(float a, float b, float bb, float &gab, float &gba) {
    const bool same = a * b > 0.f;
    gab = same ? copysignf(fminf(fabsf(a), bb * fabsf(b)), a) : 0.f;
    gba = same ? copysignf(fminf(fabsf(b), bb * fabsf(a)), b) : 0.f;
}

// Upwind flux through the face between cells c and p = c + 1 along one axis
// from the values at c - 1, c, c + 1, c + 2 and the face's volume flux J
// (src/cfd.h:37-60: kappa = 1/3 MUSCL with the b = 4 limiter, or the smooth
// van Albada limiter of DALM_LIMITER_VAN_ALBADA).  The reference blends the
// left and right states, 0.5 (J (fr + fl) - |J| (fr - fl)), which is J fl
// for J > 0 and J fr otherwise; only that upwind state is formed here, so
// each face takes one limiter evaluation instead of two.  The two states are
// one reconstruction mirrored: with centre u, forward difference a and
// backward difference b (fl: u = fc, a = fp - fc, b = fc - fm; fr: u = fp,
// a = fc - fp, b = fp - fpp) the state is
//   u + 1/4 [(1 - kappa) L(b, a) + (1 + kappa) L(a, b)]
// with L(x, y) = minmod(x, bb y) for b = 4 (odd in its arguments) or
// s x, s = (2ab + eps) / (a^2 + b^2 + eps), for van Albada (even).
__device__ __forceinline__ float face_flux(float fm, float fc, float fp, float fpp, float J,
                                           int limiter) {
    const float kap = 1.f / 3.f;
    const float bb = (3.f - kap) / (1.f - kap);
    const bool pos = J > 0.f;
    const float u = pos ? fc : fp;
    const float a = pos ? fp - fc : fc - fp;
    const float b = pos ? fc - fm : fp - fpp;
    float st;
    if (limiter == 1) {
        const float s = va_switch_f(a, b);
        st = u + (s * 0.25f) * ((1.f - kap * s) * b + (1.f + kap * s) * a);
    } else {
        float lab, lba;  // L(a, b), L(b, a)
        minmod_pair(a, b, bb, lab, lba);
        st = u + 0.25f * ((1.f - kap) * lba + (1.f + kap) * lab);
    }
    return J * st;
}

constexpr int HR = TJ + 4;  // tile rows: j - 2 .. j + 9
constexpr int HC = TK + 4;  // tile columns: k - 2 .. k + 33

// The operands a cell of the predictor reads besides the velocity: its six
// face fluxes' JU (east, north, south, top, bottom; west is carried) and the
// actuator-line force.
struct PredictOperands {
    float ju[5], f[3];
};

__device__ __forceinline__ void load_operands(const StepParams &P, Vec3<const float> JU,
                                              Vec3<const float> F, long long c, long long sy, int i,
                                              int j, int k, PredictOperands &o) {
    o.ju[0] = JU.c[0][c];
    o.ju[1] = JU.c[1][c];
    o.ju[2] = JU.c[1][c - sy];
    o.ju[3] = JU.c[2][c];
    o.ju[4] = JU.c[2][c - 1];
    const bool has_f = P.fbox.contains(i, j, k);
#pragma unroll
    for (int m = 0; m < 3; m++) o.f[m] = has_f ? F.c[m][c] : 0.f;
}

// The predictor (see the file comment).  Software-pipelined along i: the
// loads of plane i + 1 (the ring's next column value, this thread's halo
// cell, the face fluxes and the force) are issued before plane i is computed
// and consumed after it, so their latency overlaps the arithmetic.  Threads
// whose (j, k) lies outside the interior but inside the stored grid still
// load their column: their values are the guide-cell neighbours of the
// interior cells in the tile.
__global__ void __launch_bounds__(TILE_THREADS, 2)
k_predict32(StepParams P, Segments T, MixedGeom Gm, float inv_re, float dt, Vec3<const float> V,
            Vec3<float> Un, Vec3<const float> JU, Vec3<const float> F) {
    __shared__ float tile[2][3][HR][HC];
    __shared__ float fny[2][3][TJ][TK];
    const Grid &g = P.g;
    const int lane = threadIdx.x & 31, row = threadIdx.x >> 5;
    const long long sx = g.sx, sy = g.sy;
    for (int u = blockIdx.x; u < T.count; u += gridDim.x) {
        int i0, i1, j, k;
        const bool valid = T.column(u, i0, i1, j, k);
        const bool inmem = j < g.ny && k < g.nz;
        const int j0 = j - row, k0 = k - lane;
        const long long c0 = inmem ? g.at(i0, j, k) : 0;
        // halo loads of a plane: warps 0-3 the rows j0-2, j0-1, j0+8, j0+9
        // (lanes along k), warp 4 the columns k0-2, k0-1, k0+32, k0+33 of
        // the 8 rows; -1 where outside the stored grid
        int hrow = -1, hcol = -1;
        long long hidx = 0;  // stored index of this thread's halo cell in plane i0
        if (row < 4) {
            const int r = row < 2 ? row : row + TJ;  // tile row 0, 1, 10, 11
            const int jj = j0 - 2 + r;
            if (jj >= 0 && jj < g.ny && k < g.nz) {
                hrow = r;
                hcol = lane + 2;
                hidx = g.at(i0, jj, k);
            }
        } else if (row == 4) {
            const int q = lane >> 3, rr = lane & 7;
            const int col = q < 2 ? q : q + TK;  // tile column 0, 1, 34, 35
            const int kk = k0 - 2 + col, jj = j0 + rr;
            if (kk >= 0 && kk < g.nz && jj < g.ny) {
                hrow = rr + 2;
                hcol = col;
                hidx = g.at(i0, jj, kk);
            }
        }
        const float4 gy = Gm.ax[1][min(j, g.ny - 1)], gz = Gm.ax[2][min(k, g.nz - 1)];
        const float wyz = Gm.wd[1][min(j, g.ny - 1)].y * Gm.wd[2][min(k, g.nz - 1)].y;
        // register ring: r[m][d] = V at (i - 2 + d, j, k)
        float r[3][5], nxt[3] = {0.f, 0.f, 0.f}, hv[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
            for (int d = 0; d < 5; d++) r[m][d] = inmem ? V.c[m][c0 + (d - 2) * sx] : 0.f;
        PredictOperands cur{}, next{};
        // the west face of the chunk's first plane
        float fW[3] = {0.f, 0.f, 0.f};
        if (valid) {
            const float JUW = JU.c[0][c0 - sx];
            load_operands(P, JU, F, c0, sy, i0, j, k, cur);
#pragma unroll
            for (int m = 0; m < 3; m++)
                fW[m] = face_flux(r[m][0], r[m][1], r[m][2], r[m][3], JUW, P.limiter);
        }
        // the first plane's tile
#pragma unroll
        for (int m = 0; m < 3; m++) {
            tile[0][m][row + 2][lane + 2] = r[m][2];
            if (hrow >= 0) tile[0][m][hrow][hcol] = V.c[m][hidx];
        }
        __syncthreads();
        for (int i = i0; i < i1; i++) {
            const int b = (i - i0) & 1;
            const long long c = c0 + (long long)(i - i0) * sx;
            const bool more = i + 1 < i1;
            // plane i + 1's loads, issued now, consumed after this plane
            if (more) {
                if (inmem)
#pragma unroll
                    for (int m = 0; m < 3; m++) nxt[m] = V.c[m][c + 3 * sx];
                if (hrow >= 0)
#pragma unroll
                    for (int m = 0; m < 3; m++) hv[m] = V.c[m][hidx + (long long)(i + 1 - i0) * sx];
                if (valid) load_operands(P, JU, F, c + sx, sy, i + 1, j, k, next);
            }
            float fE[3], fN[3], fT[3], fB[3], G[3][3];
            float4 gx = make_float4(0.f, 0.f, 0.f, 0.f);
            if (valid) {
                gx = Gm.ax[0][i];
#pragma unroll
                for (int m = 0; m < 3; m++) {
                    const float(*t)[HC] = tile[b][m];
                    const float fc = r[m][2];
                    const float yn = t[row + 3][lane + 2], ynn = t[row + 4][lane + 2];
                    const float ys = t[row + 1][lane + 2];
                    const float zt = t[row + 2][lane + 3], ztt = t[row + 2][lane + 4];
                    const float zb = t[row + 2][lane + 1], zbb = t[row + 2][lane];
                    fE[m] = face_flux(r[m][1], fc, r[m][3], r[m][4], cur.ju[0], P.limiter);
                    fN[m] = face_flux(ys, fc, yn, ynn, cur.ju[1], P.limiter);
                    fT[m] = face_flux(zb, fc, zt, ztt, cur.ju[3], P.limiter);
                    fB[m] = face_flux(zbb, zb, fc, zt, cur.ju[4], P.limiter);
                    // central differences over x[n+1] - x[n-1] (calc_nut_at_cell)
                    G[m][0] = (r[m][3] - r[m][1]) * gx.w;
                    G[m][1] = (yn - ys) * gy.w;
                    G[m][2] = (zt - zb) * gz.w;
                    fny[b][m][row][lane] = fN[m];
                }
            }
            // the next plane's tile (center from the ring, halo loaded above)
            if (more) {
#pragma unroll
                for (int m = 0; m < 3; m++) {
                    tile[b ^ 1][m][row + 2][lane + 2] = r[m][3];
                    if (hrow >= 0) tile[b ^ 1][m][hrow][hcol] = hv[m];
                }
            }
            __syncthreads();
            if (valid) {
                const float inv_vol = gx.x * gy.x * gz.x;
                const float S = 2.f * (G[0][0] * G[0][0] + G[1][1] * G[1][1] + G[2][2] * G[2][2]) +
                                (G[0][1] + G[1][0]) * (G[0][1] + G[1][0]) +
                                (G[0][2] + G[2][0]) * (G[0][2] + G[2][0]) +
                                (G[1][2] + G[2][1]) * (G[1][2] + G[2][1]);
                const float visc = inv_re + Gm.cs2 * Gm.wd[0][i].y * wyz * sqrtf(S);
#pragma unroll
                for (int m = 0; m < 3; m++) {
                    const float(*t)[HC] = tile[b][m];
                    const float fc = r[m][2];
                    float fS;
                    if (row > 0) {
                        fS = fny[b][m][row - 1][lane];
                    } else {
                        fS = face_flux(t[row][lane + 2], t[row + 1][lane + 2], fc,
                                       t[row + 3][lane + 2], cur.ju[2], P.limiter);
                    }
                    const float conv = (fE[m] - fW[m] + fN[m] - fS + fT[m] - fB[m]) * inv_vol;
                    const float yn = t[row + 3][lane + 2], ys = t[row + 1][lane + 2];
                    const float zt = t[row + 2][lane + 3], zb = t[row + 2][lane + 1];
                    const float diff =
                        visc * (((r[m][3] - fc) * gx.y - (fc - r[m][1]) * gx.z) * gx.x +
                                ((yn - fc) * gy.y - (fc - ys) * gy.z) * gy.x +
                                ((zt - fc) * gz.y - (fc - zb) * gz.z) * gz.x);
                    Un.c[m][c] = fc + dt * (-conv + diff + cur.f[m]);
                    fW[m] = fE[m];
                }
                // the guide cells at the ends of this k row (U* = U^n there)
                if (k == g.gc || k == g.nz - g.gc - 1) {
                    const long long d = k == g.gc ? -1 : 1;
                    for (int tt = 1; tt <= g.gc; tt++)
#pragma unroll
                        for (int m = 0; m < 3; m++) Un.c[m][c + tt * d] = V.c[m][c + tt * d];
                }
            }
            // shift the ring and the operands
#pragma unroll
            for (int m = 0; m < 3; m++) {
                r[m][0] = r[m][1];
                r[m][1] = r[m][2];
                r[m][2] = r[m][3];
                r[m][3] = r[m][4];
                r[m][4] = nxt[m];
            }
            cur = next;
        }
        __syncthreads();  // the tiles are rewritten by the next segment
    }
}

// U* = U^n on the guide cells of the rows (i, j) outside the interior (no
// boundary condition after the predictor; k_predict32 copies the k ends of
// the interior rows): one warp per row, 2 gc planes of ny rows, then 2 gc
// strips of nx - 2 gc rows.
__global__ void __launch_bounds__(256) k_copy_guides32(Grid g, Vec3<const float> V, Vec3<float> Un) {
    const int gc = g.gc, ni = g.nx - 2 * gc;
    const int lane = threadIdx.x & 31;
    const unsigned a = 2u * gc * g.ny;
    const unsigned rows = a + 2u * gc * ni;
    const unsigned nw = gridDim.x * (blockDim.x >> 5);
    for (unsigned r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += nw) {
        int i, j;
        if (r < a) {
            const int p = (int)(r / g.ny);
            i = p < gc ? p : g.nx - 2 * gc + p;
            j = (int)(r - (unsigned)p * g.ny);
        } else {
            const unsigned q = r - a;
            const int p = (int)(q / ni);
            j = p < gc ? p : g.ny - 2 * gc + p;
            i = gc + (int)(q - (unsigned)p * ni);
        }
        const long long c0 = g.at(i, j, 0);
        for (int k = lane; k < g.nz; k += 32)
            for (int m = 0; m < 3; m++) Un.c[m][c0 + k] = V.c[m][c0 + k];
    }
}

// Face flux with the apply_JUbc overrides (src/bc.h:235-302 and the inflow
// profile extension); faces are named by their lower cell.  FP32.
__device__ __forceinline__ float flux_x32(const StepParams &P, float u0, float u1, float yz, int i,
                                          int j, int k) {
    const Grid &g = P.g;
    if (i == g.gc - 1 && j >= g.gc && j < g.ny - g.gc && k >= g.gc && k < g.nz - g.gc)
        return yz * (float)(P.prof ? P.prof[((long long)j * g.nz + k) * 3] : P.uin[0]);
    return 0.5f * (u0 * yz + u1 * yz);
}
__device__ __forceinline__ float flux_y32(const StepParams &P, float v0, float v1, float xz, int i,
                                          int j, int k) {
    const Grid &g = P.g;
    if ((j == g.gc - 1 || j == g.ny - g.gc - 1) && i >= g.gc && i < g.nx - g.gc && k >= g.gc &&
        k < g.nz - g.gc)
        return 0.f;
    return 0.5f * (v0 * xz + v1 * xz);
}
__device__ __forceinline__ float flux_z32(const StepParams &P, float w0, float w1, float xy, int i,
                                          int j, int k) {
    const Grid &g = P.g;
    if ((k == g.gc - 1 || k == g.nz - g.gc - 1) && i >= g.gc && i < g.nx - g.gc && j >= g.gc &&
        j < g.ny - g.gc)
        return 0.f;
    return 0.5f * (w0 * xy + w1 * xy);
}

// Face fluxes on faces [gc-1, N-gc) per axis, and for RHS the Poisson
// right-hand side b = div(JU) / (dt max_diag) of the interior cells in FP64
// from the stored FP32 faces.  The west face of a cell is the previous
// plane's east face (carried); the south and bottom faces are recomputed.
// Software-pipelined along i: plane i + 1's velocities are loaded before
// plane i is computed.
struct FluxOps {
    float ue, v, vn, vs, w, wt, wb;  // U0 at i + 1; U1 at j, j + 1, j - 1; U2 at k, k + 1, k - 1
};

__device__ __forceinline__ void load_flux_ops(Vec3<const float> U, long long c, long long sx,
                                              long long sy, bool rhs, FluxOps &o) {
    o.ue = U.c[0][c + sx];
    o.v = U.c[1][c];
    o.vn = U.c[1][c + sy];
    o.w = U.c[2][c];
    o.wt = U.c[2][c + 1];
    o.vs = rhs ? U.c[1][c - sy] : 0.f;
    o.wb = rhs ? U.c[2][c - 1] : 0.f;
}

template <bool RHS>
__global__ void __launch_bounds__(TILE_THREADS)
k_flux32(StepParams P, Segments T, MixedGeom Gm, Vec3<const float> U, Vec3<float> JU, double *b) {
    const Grid &g = P.g;
    const long long sx = g.sx, sy = g.sy;
    const double inv_dtm = 1.0 / (P.dt * P.max_diag);
    for (int u = blockIdx.x; u < T.count; u += gridDim.x) {
        int i0, i1, j, k;
        if (!T.column(u, i0, i1, j, k)) continue;
        const float dy = Gm.wd[1][j].x, dz = Gm.wd[2][k].x;
        const double dyz64 = P.m.dy[j] * P.m.dz[k];
        const float yz = dy * dz;
        const bool jk_in = j >= g.gc && j < g.ny - g.gc && k >= g.gc && k < g.nz - g.gc;
        long long c = g.at(i0, j, k);
        float u_c = U.c[0][c];
        float fw = 0.f;
        if (RHS && i0 > g.gc - 1) fw = flux_x32(P, U.c[0][c - sx], u_c, yz, i0 - 1, j, k);
        // rhs loads only where b is computed (interior j, k; any interior i)
        FluxOps cur{}, nxt{};
        load_flux_ops(U, c, sx, sy, RHS && jk_in, cur);
        for (int i = i0; i < i1; i++, c += sx) {
            if (i + 1 < i1) load_flux_ops(U, c + sx, sx, sy, RHS && jk_in, nxt);
            const float dx = Gm.wd[0][i].x;
            const float fe = flux_x32(P, u_c, cur.ue, yz, i, j, k);
            const float fn = flux_y32(P, cur.v, cur.vn, dx * dz, i, j, k);
            const float ft = flux_z32(P, cur.w, cur.wt, dx * dy, i, j, k);
            JU.c[0][c] = fe;
            JU.c[1][c] = fn;
            JU.c[2][c] = ft;
            if (RHS && jk_in && i >= g.gc && i < g.nx - g.gc) {
                const float fs = flux_y32(P, cur.vs, cur.v, dx * dz, i, j - 1, k);
                const float fb = flux_z32(P, cur.wb, cur.w, dx * dy, i, j, k - 1);
                const double vol = P.m.dx[i] * dyz64;
                const double div = ((double)fe - (double)fw + (double)fn - (double)fs +
                                    (double)ft - (double)fb) / vol;
                b[c] = div * inv_dtm;
            }
            fw = fe;
            u_c = cur.ue;
            cur = nxt;
        }
    }
}

// project_p with the apply_JUbc overrides, set_solid_U, the divergence norm
// and max CFL.  Corrections dt A (p_{n+1} - p_n) / (x_{n+1} - x_n) of the
// faces and dt (p_{n+1} - p_{n-1}) / (x_{n+1} - x_{n-1}) of the cell velocity
// in FP64 (reciprocal tables Gm.inv64), results stored in FP32; the
// divergence of the projected faces in FP64 before they are rounded.
// Software-pipelined along i: plane i + 1's operands are loaded before plane
// i is computed.  Three blocks per SM (80 registers, a few bytes spilled):
// the kernel is latency-bound, and the extra warps cut it from 452 to
// 395 us per step on 512x256x128 against two blocks at 114 registers.
struct ProjectOps {
    double pee, pn, ps, pt, pb;  // p at i + 2 (the ring's next), j +- 1, k +- 1
    float ju[3], jus, jub, u[3];  // JU at the cell, JU1 at j - 1, JU2 at k - 1, U
};

__device__ __forceinline__ void load_project_ops(Vec3<const float> JU, Vec3<float> U,
                                                 const double *p, long long c, long long sx,
                                                 long long sy, bool cell, ProjectOps &o) {
    o.pee = p[c + sx];
    o.pn = p[c + sy];
    o.pt = p[c + 1];
#pragma unroll
    for (int m = 0; m < 3; m++) o.ju[m] = JU.c[m][c];
    if (cell) {
        o.ps = p[c - sy];
        o.pb = p[c - 1];
        o.jus = JU.c[1][c - sy];
        o.jub = JU.c[2][c - 1];
#pragma unroll
        for (int m = 0; m < 3; m++) o.u[m] = U.c[m][c];
    }
}

__global__ void __launch_bounds__(TILE_THREADS, 3)
k_project32(StepParams P, Segments T, MixedGeom Gm, Vec3<float> U, Vec3<const float> JUin,
            Vec3<float> JUout, const double *p, Partials<2> part, DiagState *diag) {
    const Grid &g = P.g;
    const long long sx = g.sx, sy = g.sy;
    const double dt = P.dt;
    double div2 = 0, cfl = 0;
    for (int u = blockIdx.x; u < T.count; u += gridDim.x) {
        int i0, i1, j, k;
        if (!T.column(u, i0, i1, j, k)) continue;
        const bool jk_in = j >= g.gc && j < g.ny - g.gc && k >= g.gc && k < g.nz - g.gc;
        const double uin = P.prof ? P.prof[((long long)j * g.nz + k) * 3] : P.uin[0];
        const bool ywall_n = (j == g.gc - 1 || j == g.ny - g.gc - 1) && k >= g.gc && k < g.nz - g.gc;
        const bool zwall_t = (k == g.gc - 1 || k == g.nz - g.gc - 1) && j >= g.gc && j < g.ny - g.gc;
        const bool ywall_s = j - 1 == g.gc - 1 || j - 1 == g.ny - g.gc - 1;
        const bool zwall_b = k - 1 == g.gc - 1 || k - 1 == g.nz - g.gc - 1;
        long long c = g.at(i0, j, k);
        double p_w = p[c - sx], p_c = p[c];
        double fw = 0.0;
        if (i0 > g.gc - 1)
            fw = (i0 - 1 == g.gc - 1 && jk_in)
                     ? P.m.dy[j] * P.m.dz[k] * uin
                     : (double)JUin.c[0][c - sx] -
                           dt * (P.m.dy[j] * P.m.dz[k]) * ((p_c - p_w) * Gm.inv64[0][i0 - 1].x);
        ProjectOps cur{}, nxt{};
        load_project_ops(JUin, U, p, c, sx, sy, jk_in && i0 >= g.gc, cur);
        for (int i = i0; i < i1; i++, c += sx) {
            const bool cell = jk_in && i >= g.gc && i < g.nx - g.gc;
            if (i + 1 < i1)
                load_project_ops(JUin, U, p, c + sx, sx, sy, jk_in && i + 1 >= g.gc && i + 1 < g.nx - g.gc,
                                 nxt);
            const double p_e = cur.pee;
            const double dx = P.m.dx[i], dy = P.m.dy[j], dz = P.m.dz[k];
            const bool iin = i >= g.gc && i < g.nx - g.gc;
            const double fe = (i == g.gc - 1 && jk_in)
                                  ? dy * dz * uin
                                  : (double)cur.ju[0] - dt * (dy * dz) * ((p_e - p_c) * Gm.inv64[0][i].x);
            const double fn = (ywall_n && iin)
                                  ? 0.0
                                  : (double)cur.ju[1] - dt * (dx * dz) * ((cur.pn - p_c) * Gm.inv64[1][j].x);
            const double ft = (zwall_t && iin)
                                  ? 0.0
                                  : (double)cur.ju[2] - dt * (dx * dy) * ((cur.pt - p_c) * Gm.inv64[2][k].x);
            JUout.c[0][c] = (float)fe;
            JUout.c[1][c] = (float)fn;
            JUout.c[2][c] = (float)ft;
            if (cell) {
                double uu = (double)cur.u[0] - dt * (p_e - p_w) * Gm.inv64[0][i].y;
                double vv = (double)cur.u[1] - dt * (cur.pn - cur.ps) * Gm.inv64[1][j].y;
                double ww = (double)cur.u[2] - dt * (cur.pt - cur.pb) * Gm.inv64[2][k].y;
                if (P.solid) {  // set_solid_U (src/cfd.h:1143-1160)
                    const double sf = P.solid[c];
                    uu = (1. - sf) * uu;
                    vv = (1. - sf) * vv;
                    ww = (1. - sf) * ww;
                }
                U.c[0][c] = (float)uu;
                U.c[1][c] = (float)vv;
                U.c[2][c] = (float)ww;
                const double fs = ywall_s ? 0.0
                                          : (double)cur.jus -
                                                dt * (dx * dz) * ((p_c - cur.ps) * Gm.inv64[1][j - 1].x);
                const double fb = zwall_b ? 0.0
                                          : (double)cur.jub -
                                                dt * (dx * dy) * ((p_c - cur.pb) * Gm.inv64[2][k - 1].x);
                const double d = (fe - fw + fn - fs + ft - fb) / (dx * dy * dz);
                div2 += d * d;
                const double local = (fabs(uu) / dx + fabs(vv) / dy + fabs(ww) / dz) * dt;
                cfl = local > cfl ? local : cfl;
            }
            fw = fe;
            p_w = p_c;
            p_c = p_e;
            cur = nxt;
        }
    }
    double v[2] = {div2, cfl};
    if (grid_reduce<2>(v, 2u, part) && threadIdx.x == 0) {
        diag->div2 = v[0];
        diag->max_cfl = v[1];
        diag->avg_div = sqrt(v[0]) / sqrt(diag->ncell);
    }
}

Box interior_box32(const Grid &g) {
    return Box{{g.gc, g.gc, g.gc}, {g.nx - g.gc, g.ny - g.gc, g.nz - g.gc}};
}
Box face_box32(const Grid &g) {
    return Box{{g.gc - 1, g.gc - 1, g.gc - 1}, {g.nx - g.gc, g.ny - g.gc, g.nz - g.gc}};
}

}  // namespace

void launch_predict32(const LaunchCtx &L, const StepParams &P, const MixedGeom &geo,
                      Vec3<const float> uold, Vec3<float> unew, Vec3<const float> ju,
                      Vec3<const float> f) {
    const Grid &g = P.g;
    const Segments T = Segments::make(interior_box32(g), L.blocks);
    L.pre(KK_PREDICT);
    k_predict32<<<L.blocks, TILE_THREADS, 0, L.s>>>(P, T, geo, (float)(1.0 / P.re), (float)P.dt,
                                                    uold, unew, ju, f);
    L.post(KK_PREDICT);
    // the guide-cell copy is counted as a layout kernel, so the predictor's
    // launches and bytes are its own
    const long long outer = 2LL * g.gc * g.ny + 2LL * g.gc * (g.nx - 2 * g.gc);
    L.pre(KK_LAYOUT);
    k_copy_guides32<<<(int)std::min<long long>((outer + 7) / 8, 2 * 148), 256, 0, L.s>>>(g, uold,
                                                                                      unew);
    L.post(KK_LAYOUT);
}

void launch_flux32(const LaunchCtx &L, const StepParams &P, const MixedGeom &geo,
                   Vec3<const float> u, Vec3<float> ju, double *b) {
    const Segments T = Segments::make(face_box32(P.g), L.blocks);
    L.pre(KK_FLUX_RHS);
    if (b)
        k_flux32<true><<<L.blocks, TILE_THREADS, 0, L.s>>>(P, T, geo, u, ju, b);
    else
        k_flux32<false><<<L.blocks, TILE_THREADS, 0, L.s>>>(P, T, geo, u, ju, nullptr);
    L.post(KK_FLUX_RHS);
}

void launch_project32(const LaunchCtx &L, const StepParams &P, const MixedGeom &geo, Vec3<float> u,
                      Vec3<const float> ju_in, Vec3<float> ju_out, const double *p,
                      Partials<2> part, DiagState *diag) {
    const Segments T = Segments::make(face_box32(P.g), L.blocks);
    L.pre(KK_PROJECT);
    k_project32<<<L.blocks, TILE_THREADS, 0, L.s>>>(P, T, geo, u, ju_in, ju_out, p, part, diag);
    L.post(KK_PROJECT);
}

}  // namespace dalm
