// Multigrid-preconditioned conjugate gradients in FP32 (the inner solves of
// DALM_MIXED); the arithmetic is in multigrid.cuh.  Vectors are FP32, sums
// FP64 through the deterministic grid reduction, Krylov scalars on the
// device; every kernel returns at once once the solve is done, so batches
// of iterations can be enqueued (and replayed as CUDA graphs) ahead of the
// host's convergence check.
#include <algorithm>
#include <cfloat>
#include <cstdint>

#include "multigrid.cuh"
#include "poisson.cuh"

namespace dalm {

namespace {

constexpr int MG_THREADS = 256;

// Interior cells of a level: one warp per (i, j) row, lane l taking
// k = k0 + l + 32 u (u < U) for k0 = 0, 32 U, ... (coalesced rows; one
// 32-bit division per row).  `prep(i, j)` makes the row's constants once;
// `load(row, k)` runs for all U cells before `store(row, k, value)` runs for
// any, so every lane keeps U cells' loads in flight: the compiler may not
// move a later cell's loads above an earlier cell's stores, which it cannot
// prove do not alias them.
template <int U, typename Prep, typename Ld, typename St>
__device__ __forceinline__ void level_loop(const MgLevel &L, Prep prep, Ld load, St store) {
    using Row = decltype(prep(0, 0));
    using T = decltype(load(prep(0, 0), 0));
    const int lane = threadIdx.x & 31;
    const int nk = L.n[2];
    const unsigned nj = (unsigned)L.n[1];
    const unsigned rows = (unsigned)L.n[0] * nj;
    const unsigned nw = gridDim.x * (blockDim.x >> 5);
    for (unsigned row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); row < rows;
         row += nw) {
        const int i = (int)(row / nj), j = (int)(row - (unsigned)i * nj);
        const Row R = prep(i, j);
        for (int k0 = 0; k0 < nk; k0 += 32 * U) {
            T v[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int k = k0 + lane + 32 * u;
                if (k < nk) v[u] = load(R, k);
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int k = k0 + lane + 32 * u;
                if (k < nk) store(R, k, v[u]);
            }
        }
    }
}

// Row (i, j) of a level with its constants: (K x) at k is mg_apply with the
// row's factors taken out of the per-cell sums.
struct MgRow {
    long long c0;
    int sx, sy;
    float w0, w1, az, xe, xw, yn, ys, sxy;
    MgRow() = default;
    __device__ __forceinline__ MgRow(const MgLevel &L, int i, int j) {
        c0 = L.at(i, j, 0);
        sx = (int)L.g.sx;
        sy = (int)L.g.sy;
        w0 = L.w[0][i];
        w1 = L.w[1][j];
        az = w0 * w1;
        xe = L.cf[0][i + 1];
        xw = L.cf[0][i];
        yn = L.cf[1][j + 1];
        ys = L.cf[1][j];
        sxy = w1 * (xe + xw) + w0 * (yn + ys);
    }
    __device__ __forceinline__ float apply(const MgLevel &L, const float *x, int k) const {
        const float *xr = x + c0 + k;
        const float w2 = L.w[2][k], zt = L.cf[2][k + 1], zb = L.cf[2][k];
        const float diag = w2 * sxy + az * (zt + zb);
        const float nb =
            w2 * (w1 * (xe * xr[sx] + xw * xr[-sx]) + w0 * (yn * xr[sy] + ys * xr[-sy])) +
            az * (zt * xr[1] + zb * xr[-1]);
        return diag * xr[0] - nb;
    }
};

// a row's storage offset and area factor w0 w1 (cell volume = w01 w2[k])
struct MgRowBase {
    long long c0;
    float w01;
};
__device__ __forceinline__ MgRowBase row_base(const MgLevel &L, int i, int j) {
    return MgRowBase{L.at(i, j, 0), L.w[0][i] * L.w[1][j]};
}

// Steps 2 and 3 of the line solve for the lane's rows d[] (right-hand
// sides in, solution out in x[]): the row coefficients from the column's
// constants, the lane's Thomas sweeps and the cyclic reduction over lanes.
template <int R>
__device__ __forceinline__ void line_solve(float az, float sxy, const float *w2, const float *cf2,
                                           int nk, int lane, const float (&d)[R], float (&x)[R]) {
    const unsigned full = 0xffffffffu;
    float a[R], b[R], c[R];
#pragma unroll
    for (int s = 0; s < R; s++) {
        const int k = R * lane + s;
        if (k < nk) {
            const float lo = az * cf2[k], hi = az * cf2[k + 1];
            a[s] = -lo;
            b[s] = w2[k] * sxy + lo + hi;
            c[s] = -hi;
        } else {
            a[s] = 0.f;
            b[s] = 1.f;
            c[s] = 0.f;
        }
    }
    // 2. rows s < R - 1: x_s = D_s - A_s y_{l-1} - C_s y_l (in e, fa, g)
    float e[R], fa[R], g[R];
    float ra = a[R - 1], rb = b[R - 1], rc = c[R - 1], rd = d[R - 1];
    if (R > 1) {
#pragma unroll
        for (int s = 0; s < R - 1; s++) {
            const float den = s == 0 ? b[0] : b[s] - a[s] * g[s > 0 ? s - 1 : 0];
            const float q = __fdividef(1.f, den);
            e[s] = (s == 0 ? d[0] : d[s] - a[s] * e[s > 0 ? s - 1 : 0]) * q;
            fa[s] = (s == 0 ? a[0] : -a[s] * fa[s > 0 ? s - 1 : 0]) * q;
            g[s] = c[s] * q;
        }
#pragma unroll
        for (int s = R - 3; s >= 0; s--) {
            e[s] -= g[s] * e[s + 1];
            fa[s] -= g[s] * fa[s + 1];
            g[s] = -g[s] * g[s + 1];
        }
        // 3. the last row, with x of the next lane's first row
        float An = __shfl_down_sync(full, fa[0], 1), Cn = __shfl_down_sync(full, g[0], 1);
        float Dn = __shfl_down_sync(full, e[0], 1);
        if (lane == 31) An = Cn = Dn = 0.f;
        const float al = a[R - 1], cl = c[R - 1];
        ra = -al * fa[R - 2];
        rb = b[R - 1] - al * g[R - 2] - cl * An;
        rc = -cl * Cn;
        rd = d[R - 1] - al * e[R - 2] - cl * Dn;
    }
#pragma unroll
    for (int delta = 1; delta < 32; delta <<= 1) {
        float am = __shfl_up_sync(full, ra, delta), bm = __shfl_up_sync(full, rb, delta);
        float cm = __shfl_up_sync(full, rc, delta), dm = __shfl_up_sync(full, rd, delta);
        float ap = __shfl_down_sync(full, ra, delta), bp = __shfl_down_sync(full, rb, delta);
        float cp = __shfl_down_sync(full, rc, delta), dp = __shfl_down_sync(full, rd, delta);
        if (lane < delta) am = 0.f, bm = 1.f, cm = 0.f, dm = 0.f;  // identity rows
        if (lane + delta >= 32) ap = 0.f, bp = 1.f, cp = 0.f, dp = 0.f;
        // approximate quotients (2 ulp): the preconditioner needs no
        // correctly rounded division
        const float alpha = -__fdividef(ra, bm), gamma = -__fdividef(rc, bp);
        rb += alpha * cm + gamma * ap;
        rd += alpha * dm + gamma * dp;
        ra = alpha * am;
        rc = gamma * cp;
    }
    const float y = __fdividef(rd, rb);
    float ym = __shfl_up_sync(full, y, 1);
    if (lane == 0) ym = 0.f;
#pragma unroll
    for (int s = 0; s < R; s++)
        x[s] = s == R - 1 ? y : e[s < R - 1 ? s : 0] - fa[s < R - 1 ? s : 0] * ym -
                                    g[s < R - 1 ? s : 0] * y;
}

// The same with every matrix-only quantity read from the level's factor
// table (MgLevel::ltab, mglf_* layout; T points at this lane's entry of
// the column's class): two shuffles and two FMAs per reduction step.
template <int R>
__device__ __forceinline__ void line_solve_table(const float *T, int lane, const float (&d)[R],
                                                 float (&x)[R]) {
    const unsigned full = 0xffffffffu;
    float e[R];
    float rd = d[R - 1];
    if (R > 1) {
#pragma unroll
        for (int s = 0; s < R - 1; s++)
            e[s] = (s == 0 ? d[0] : d[s] - T[32 * mglf_a(s)] * e[s > 0 ? s - 1 : 0]) *
                   T[32 * mglf_q(s)];
#pragma unroll
        for (int s = R - 3; s >= 0; s--) e[s] -= T[32 * mglf_g(s)] * e[s + 1];
        float Dn = __shfl_down_sync(full, e[0], 1);
        if (lane == 31) Dn = 0.f;
        rd = d[R - 1] - T[32 * mglf_al(R)] * e[R - 2] - T[32 * mglf_cl(R)] * Dn;
    }
#pragma unroll
    for (int t = 0; t < 5; t++) {
        const int delta = 1 << t;
        float dm = __shfl_up_sync(full, rd, delta), dp = __shfl_down_sync(full, rd, delta);
        if (lane < delta) dm = 0.f;
        if (lane + delta >= 32) dp = 0.f;
        rd += T[32 * mglf_alpha(R, t)] * dm + T[32 * mglf_gamma(R, t)] * dp;
    }
    const float y = rd * T[32 * mglf_invrb(R)];
    float ym = __shfl_up_sync(full, y, 1);
    if (lane == 0) ym = 0.f;
#pragma unroll
    for (int s = 0; s < R; s++)
        x[s] = s == R - 1 ? y
                          : e[s < R - 1 ? s : 0] - T[32 * mglf_xa(s < R - 1 ? s : 0)] * ym -
                                T[32 * mglf_xc(s < R - 1 ? s : 0)] * y;
}

// R consecutive floats at p (VEC path: p is 4R-byte aligned)
template <int R>
__device__ __forceinline__ void load_seg(const float *p, float (&v)[R]) {
    if constexpr (R == 8) {
        const float4 a = reinterpret_cast<const float4 *>(p)[0], b = reinterpret_cast<const float4 *>(p)[1];
        v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
    } else if constexpr (R == 4) {
        const float4 a = *reinterpret_cast<const float4 *>(p);
        v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w;
    } else if constexpr (R == 2) {
        const float2 a = *reinterpret_cast<const float2 *>(p);
        v[0] = a.x, v[1] = a.y;
    } else {
#pragma unroll
        for (int s = 0; s < R; s++) v[s] = p[s];
    }
}

template <int R>
__device__ __forceinline__ void store_seg(float *p, const float (&v)[R]) {
    if constexpr (R == 8) {
        reinterpret_cast<float4 *>(p)[0] = make_float4(v[0], v[1], v[2], v[3]);
        reinterpret_cast<float4 *>(p)[1] = make_float4(v[4], v[5], v[6], v[7]);
    } else if constexpr (R == 4) {
        *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
    } else if constexpr (R == 2) {
        *reinterpret_cast<float2 *>(p) = make_float2(v[0], v[1]);
    } else {
#pragma unroll
        for (int s = 0; s < R; s++) p[s] = v[s];
    }
}

// Zebra z-line half-sweep, one warp per column, by the partition method.
// Lane l owns the R consecutive rows k = R l + s (s < R):
//  1. the right-hand sides are formed in the coalesced layout k = l + 32 r
//     and pass to the lanes' own rows through a per-warp shared-memory slab
//     (slot k + k / 32: no bank conflicts either way for R = 1, 2, 4, 8);
//  2. each lane eliminates its first R - 1 rows by a Thomas forward and back
//     sweep into x_k = D_k - A_k y_{l-1} - C_k y_l, y_l being the value of
//     its last row;
//  3. the 32 last rows then form a tridiagonal system in the y_l alone,
//     solved by parallel cyclic reduction over the lanes (5 shuffle steps);
//  4. each lane expands its rows and the solution leaves through the slab in
//     the coalesced layout.
// Rows past the column are identity rows.  The line operator is diagonally
// dominant, which keeps both eliminations stable without pivoting; the result
// is mg_thomas's up to rounding (this file is compiled with contraction and
// fast quotients).  Blocks only read columns of the other colour and only
// write their own.  FAC: steps 2-3 read the matrix-only quantities from the
// level's factor table (line_solve_table) instead of forming and
// eliminating the column's matrix (line_solve).  VEC (columns of exactly
// 32 R cells, R = 1, 2, 4, 8, on rows whose k = 0 is 32-byte aligned, which
// Grid's layout gives every interior row): each lane loads and stores its
// own R rows with vector accesses, and no slab is needed.
//
// With xc set, the half-sweep also applies the pending prolongation of the
// coarse correction xc (level C): it reads each interior x or y neighbour
// as x + xc(parent).  This is the first half-sweep after the coarse
// correction; it overwrites its own colour, and the next half-sweep
// overwrites the other colour from these values, so adding xc to the
// neighbours it reads gives the prolongate-then-smooth result without the
// separate pass over the level.
struct ZlineArgs {
    MgLevel L;
    float *x;
    const float *f;
    int color, zero_start;
    const float *xc;  // pending prolongation (or nullptr)
    MgLevel C;
};

// Position (i, h) of items t0, t0 + nw, t0 + 2 nw, ... of a row-major
// enumeration with nh items per i, advanced without a division per step.
struct Stepper {
    unsigned i, h, di, dh, nh;
    __device__ __forceinline__ Stepper(unsigned t0, unsigned nw, unsigned nh_) : nh(nh_) {
        i = t0 / nh;
        h = t0 - i * nh;
        di = nw / nh;
        dh = nw - di * nh;
    }
    __device__ __forceinline__ void next() {
        i += di;
        h += dh;
        if (h >= nh) {
            h -= nh;
            i++;
        }
    }
};

// The operands of one column's right-hand side in the VEC layout: f and the
// four x/y neighbours' x of this lane's R rows.
template <int R>
struct ColumnLoads {
    float f[R], e[R], w[R], n[R], s[R];
};

// Column `col` of the half-sweep's colour: (i, j), false past the grid.
__device__ __forceinline__ bool zline_column(const MgLevel &L, unsigned col, unsigned njh, int color,
                                             int &i, int &j) {
    i = (int)(col / njh);
    j = 2 * (int)(col - (unsigned)i * njh) + ((i + color) & 1);
    return j < L.n[1];
}

template <int R>
__device__ __forceinline__ void zline_load(const MgLevel &L, const float *x, const float *f, int i,
                                           int j, int lane, ColumnLoads<R> &v) {
    const long long c0 = L.at(i, j, 0) + R * lane;
    load_seg<R>(f + c0, v.f);
    load_seg<R>(x + c0 + L.g.sx, v.e);
    load_seg<R>(x + c0 - L.g.sx, v.w);
    load_seg<R>(x + c0 + L.g.sy, v.n);
    load_seg<R>(x + c0 - L.g.sy, v.s);
}

// The VEC half-sweep without a pending prolongation (all but the first
// half-sweep after a coarse correction), software-pipelined over the
// columns a warp takes: the next column's operands are loaded before the
// current column is solved, so their latency overlaps the line solve.  Same
// arithmetic as k_mg_smooth's VEC path.
template <int R, bool FAC>
__global__ void __launch_bounds__(MG_THREADS) k_mg_smooth_pipe(ZlineArgs A, const KrylovState *st) {
    pdl_wait();
    if (st->done) return;
    const MgLevel &L = A.L;
    float *__restrict__ x = A.x;
    const float *__restrict__ f = A.f;
    const int lane = threadIdx.x & 31;
    const unsigned njh = (unsigned)(L.n[1] + 1) / 2;
    const unsigned ncol = (unsigned)L.n[0] * njh;
    const unsigned nw = gridDim.x * (blockDim.x >> 5);
    const int nk = L.n[2];
    const bool zero = A.zero_start != 0;
    const float *w2 = L.w[2], *cf2 = L.cf[2];
    float vw2[R];
    load_seg<R>(w2 + R * lane, vw2);
    unsigned col = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    int i = 0, j = 0;
    bool ok = col < ncol && zline_column(L, col, njh, A.color, i, j);
    ColumnLoads<R> cur, nxt;
    if (ok) zline_load<R>(L, x, f, i, j, lane, cur);
    while (col < ncol) {
        const unsigned ncol2 = col + nw;
        int i2 = 0, j2 = 0;
        const bool ok2 = ncol2 < ncol && zline_column(L, ncol2, njh, A.color, i2, j2);
        if (ok2) zline_load<R>(L, x, f, i2, j2, lane, nxt);
        if (ok) {
            const float wi = L.w[0][i], wj = L.w[1][j];
            const float xe = L.cf[0][i + 1], xw = L.cf[0][i], yn = L.cf[1][j + 1], ys = L.cf[1][j];
            float d[R], xs[R];
#pragma unroll
            for (int q = 0; q < R; q++)
                d[q] = zero ? cur.f[q]
                            : cur.f[q] + vw2[q] * (wj * (xe * cur.e[q] + xw * cur.w[q]) +
                                                   wi * (yn * cur.n[q] + ys * cur.s[q]));
            if (FAC) {
                line_solve_table<R>(L.ltab + (size_t)(L.lcls[0][i] * L.lky + L.lcls[1][j]) *
                                                 mglf_count(R) * 32 + lane,
                                    lane, d, xs);
            } else {
                const float az = wi * wj, sxy = wj * (xe + xw) + wi * (yn + ys);
                line_solve<R>(az, sxy, w2, cf2, nk, lane, d, xs);
            }
            store_seg<R>(x + L.at(i, j, 0) + R * lane, xs);
        }
        col = ncol2;
        i = i2;
        j = j2;
        ok = ok2;
        cur = nxt;
    }
}

// One column (i, j) of a zebra z-line half-sweep (see above); sl is the
// warp's slab of 33 R floats (unused on the VEC path).
template <int R, bool FAC, bool VEC>
__device__ __forceinline__ void zline_solve_column(const ZlineArgs &A, int i, int j, int lane,
                                                   float *sl) {
    const MgLevel &L = A.L;
    float *__restrict__ x = A.x;
    const float *__restrict__ f = A.f;
    const float *__restrict__ xc = A.xc;
    const int nk = L.n[2];
    const bool zero = A.zero_start != 0;
    const int kshift = A.C.fac[2] == 2 ? 1 : 0;
    const long long c0 = L.at(i, j, 0);
    // parents of the interior x and y neighbours (-1: boundary, no correction)
    long long pe = -1, pw = -1, pn = -1, ps = -1;
    if (xc) {
        const MgLevel &C = A.C;
        const int I = i / C.fac[0], J = j / C.fac[1];
        if (i + 1 < L.n[0]) pe = C.at((i + 1) / C.fac[0], J, 0);
        if (i > 0) pw = C.at((i - 1) / C.fac[0], J, 0);
        if (j + 1 < L.n[1]) pn = C.at(I, (j + 1) / C.fac[1], 0);
        if (j > 0) ps = C.at(I, (j - 1) / C.fac[1], 0);
    }
    // the column's constants (mg_zline_coef and mg_zline_rhs per row)
    const float wi = L.w[0][i], wj = L.w[1][j];
    const float xe = L.cf[0][i + 1], xw = L.cf[0][i], yn = L.cf[1][j + 1], ys = L.cf[1][j];
    const float az = wi * wj, sxy = wj * (xe + xw) + wi * (yn + ys);
    const float *w2 = L.w[2], *cf2 = L.cf[2];
    // the column and its x and y neighbours, from k = 0
    const float *fr = f + c0, *xre = x + c0 + L.g.sx, *xrw = x + c0 - L.g.sx,
                *xrn = x + c0 + L.g.sy, *xrs = x + c0 - L.g.sy;
    float d[R], xs[R];
    if (VEC) {
        // this lane's rows k = R lane + s, with vector loads
        const int k0 = R * lane;
        float vf[R], vw2[R], ve[R], vw[R], vn[R], vs[R];
        load_seg<R>(fr + k0, vf);
        if (!zero) {
            load_seg<R>(w2 + k0, vw2);
            load_seg<R>(xre + k0, ve);
            load_seg<R>(xrw + k0, vw);
            load_seg<R>(xrn + k0, vn);
            load_seg<R>(xrs + k0, vs);
            if (xc) {
#pragma unroll
                for (int q = 0; q < R; q++) {
                    const int K = (k0 + q) >> kshift;
                    if (pe >= 0) ve[q] += xc[pe + K];
                    if (pw >= 0) vw[q] += xc[pw + K];
                    if (pn >= 0) vn[q] += xc[pn + K];
                    if (ps >= 0) vs[q] += xc[ps + K];
                }
            }
        }
#pragma unroll
        for (int q = 0; q < R; q++)
            d[q] = zero ? vf[q]
                        : vf[q] + vw2[q] * (wj * (xe * ve[q] + xw * vw[q]) +
                                            wi * (yn * vn[q] + ys * vs[q]));
    } else {
        // all of the column's loads first, then the slab
        float rhs[R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int k = lane + 32 * r;
            rhs[r] = 0.f;
            if (k < nk) {
                rhs[r] = fr[k];
                if (!zero) {
                    float ve = xre[k], vw = xrw[k], vn = xrn[k], vs = xrs[k];
                    if (xc) {
                        const int K = k >> kshift;
                        if (pe >= 0) ve += xc[pe + K];
                        if (pw >= 0) vw += xc[pw + K];
                        if (pn >= 0) vn += xc[pn + K];
                        if (ps >= 0) vs += xc[ps + K];
                    }
                    rhs[r] += w2[k] * (wj * (xe * ve + xw * vw) + wi * (yn * vn + ys * vs));
                }
            }
        }
        __syncwarp();  // the previous column's reads of the slab are done
#pragma unroll
        for (int r = 0; r < R; r++) sl[lane + 33 * r] = rhs[r];
        __syncwarp();
#pragma unroll
        for (int s = 0; s < R; s++) {
            const int k = R * lane + s;
            d[s] = sl[k + (k >> 5)];
        }
    }
    if (FAC)
        line_solve_table<R>(L.ltab + (size_t)(L.lcls[0][i] * L.lky + L.lcls[1][j]) *
                                         mglf_count(R) * 32 + lane,
                            lane, d, xs);
    else
        line_solve<R>(az, sxy, w2, cf2, nk, lane, d, xs);
    // 4. store (through the slab into the coalesced layout unless VEC)
    if (VEC) {
        store_seg<R>(x + c0 + R * lane, xs);
    } else {
#pragma unroll
        for (int s = 0; s < R; s++) {
            const int k = R * lane + s;
            sl[k + (k >> 5)] = xs[s];
        }
        __syncwarp();
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int k = lane + 32 * r;
            if (k < nk) x[c0 + k] = sl[k + r];
        }
    }
}

template <int R, bool FAC, bool VEC>
__global__ void __launch_bounds__(MG_THREADS) k_mg_smooth(ZlineArgs A, const KrylovState *st) {
    pdl_wait();
    __shared__ float slab[MG_THREADS / 32][33 * R];
    if (st->done) return;
    const int lane = threadIdx.x & 31;
    float *sl = slab[threadIdx.x >> 5];
    const unsigned njh = (unsigned)(A.L.n[1] + 1) / 2;
    const unsigned ncol = (unsigned)A.L.n[0] * njh;
    const unsigned nw = gridDim.x * (blockDim.x >> 5);
    for (unsigned col = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); col < ncol;
         col += nw) {
        int i, j;
        if (!zline_column(A.L, col, njh, A.color, i, j)) continue;  // uniform in the warp
        zline_solve_column<R, FAC, VEC>(A, i, j, lane, sl);
    }
}

// longest line the warp solver takes (32 rows per register slot)
constexpr int ZL_MAX_R = 8;

// the VEC path's conditions: full 32 R columns, R a power of two up to 8,
// every row start (k = 0) and stride a multiple of 8 elements, and 16-byte
// aligned arrays
bool zline_vec_ok(const ZlineArgs &a, int R) {
    const MgLevel &v = a.L;
    auto al = [](const void *p) { return ((uintptr_t)p & 15) == 0; };
    bool ok = v.n[2] == 32 * R && (R == 1 || R == 2 || R == 4 || R == 8) &&
              v.at(0, 0, 0) % 8 == 0 && v.g.sx % 8 == 0 && v.g.sy % 8 == 0 && al(a.x) &&
              al(a.f) && al(v.w[2]);
    return ok;
}

template <int R>
void zline_launch(const LaunchCtx &L, const ZlineArgs &a, const KrylovState *st, int blocks) {
    const bool vec = zline_vec_ok(a, R);
    if (vec && !a.xc && a.L.ltab)
        pdl_launch(k_mg_smooth_pipe<R, true>, blocks, MG_THREADS, 0, L.s, a, st);
    else if (vec && !a.xc)
        pdl_launch(k_mg_smooth_pipe<R, false>, blocks, MG_THREADS, 0, L.s, a, st);
    else if (a.L.ltab && vec)
        pdl_launch(k_mg_smooth<R, true, true>, blocks, MG_THREADS, 0, L.s, a, st);
    else if (a.L.ltab)
        pdl_launch(k_mg_smooth<R, true, false>, blocks, MG_THREADS, 0, L.s, a, st);
    else if (vec)
        pdl_launch(k_mg_smooth<R, false, true>, blocks, MG_THREADS, 0, L.s, a, st);
    else
        pdl_launch(k_mg_smooth<R, false, false>, blocks, MG_THREADS, 0, L.s, a, st);
}

void zline_dispatch(const LaunchCtx &L, const ZlineArgs &a, const KrylovState *st) {
    const MgLevel &v = a.L;
    const long long ncol = (long long)v.n[0] * ((v.n[1] + 1) / 2);
    long long nb = (ncol + MG_THREADS / 32 - 1) / (MG_THREADS / 32);
    if (nb > L.blocks) nb = L.blocks;
    const int R = (v.n[2] + 31) / 32;
    switch (R) {
    case 1: zline_launch<1>(L, a, st, (int)nb); break;
    case 2: zline_launch<2>(L, a, st, (int)nb); break;
    case 3: zline_launch<3>(L, a, st, (int)nb); break;
    case 4: zline_launch<4>(L, a, st, (int)nb); break;
    case 5: zline_launch<5>(L, a, st, (int)nb); break;
    case 6: zline_launch<6>(L, a, st, (int)nb); break;
    case 7: zline_launch<7>(L, a, st, (int)nb); break;
    default: zline_launch<8>(L, a, st, (int)nb); break;
    }
}

// coarse cell (I,J,K) = the sum of its children's residuals f - K x,
// leaving out the children of colour `skip` (as mg_restrict_sum).  One warp
// per coarse row (warps w0, w0 + nw, ...), U coarse cells per lane at a
// time: the child rows (at most 2 x 2, levels merge at most two cells per
// axis) are visited one after the other, each with its row constants, and
// the sums are stored at the end.
__device__ __forceinline__ void mg_restrict_rows(const MgLevel &F, const MgLevel &C, const float *x,
                                                 const float *f, float *fc, int skip, unsigned w0,
                                                 unsigned nw) {
    constexpr int U = 4;
    const int lane = threadIdx.x & 31;
    const int nk = C.n[2], f2 = C.fac[2];
    const unsigned nj = (unsigned)C.n[1];
    const unsigned rows = (unsigned)C.n[0] * nj;
    for (unsigned row = w0; row < rows; row += nw) {
        const int I = (int)(row / nj), J = (int)(row - (unsigned)I * nj);
        const long long cc = C.at(I, J, 0);
        for (int k0 = 0; k0 < nk; k0 += 32 * U) {
            float s[U];
#pragma unroll
            for (int u = 0; u < U; u++) s[u] = 0.f;
            for (int a = 0; a < C.fac[0]; a++)
                for (int b = 0; b < C.fac[1]; b++) {
                    const int i = I * C.fac[0] + a, j = J * C.fac[1] + b;
                    if (((i + j) & 1) == skip) continue;
                    const MgRow R(F, i, j);
#pragma unroll
                    for (int u = 0; u < U; u++) {
                        const int K = k0 + lane + 32 * u;
                        if (K < nk)
                            for (int c = 0; c < f2; c++) {
                                const int k = K * f2 + c;
                                s[u] += f[R.c0 + k] - R.apply(F, x, k);
                            }
                    }
                }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int K = k0 + lane + 32 * u;
                if (K < nk) fc[cc + K] = s[u];
            }
        }
    }
}

__global__ void __launch_bounds__(MG_THREADS)
k_mg_restrict(MgLevel F, MgLevel C, const float *x, const float *f, float *fc, int skip,
              const KrylovState *st) {
    pdl_wait();
    if (st->done) return;
    mg_restrict_rows(F, C, x, f, fc, skip, blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5),
                     gridDim.x * (blockDim.x >> 5));
}

// x = K^-1 f on the coarsest level: one warp per row of the dense inverse
__device__ __forceinline__ void mg_coarse_rows(const MgLevel &C, const float *kinv, int n,
                                               const float *f, float *x, int w0, int nw) {
    const int lane = threadIdx.x & 31;
    for (int r = w0; r < n; r += nw) {
        const float *row = kinv + (long long)r * n;
        float s = 0;
        for (int c = lane; c < n; c += 32) s += row[c] * f[mg_cell_index(C, c)];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) x[mg_cell_index(C, r)] = s;
    }
}

__global__ void __launch_bounds__(MG_THREADS)
k_mg_coarse(MgLevel C, const float *kinv, int n, const float *f, float *x,
            const KrylovState *st) {
    pdl_wait();
    if (st->done) return;
    mg_coarse_rows(C, kinv, n, f, x, blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5),
                   gridDim.x * (blockDim.x >> 5));
}

// f = -max_diag vol r (in place), e = 0
__global__ void __launch_bounds__(MG_THREADS)
k_mg_rhs(MgLevel L, float *r, float *e, float md, const KrylovState *st) {
    pdl_wait();
    if (st->done) return;
    level_loop<4>(
        L, [&](int i, int j) { return row_base(L, i, j); },
        [&](const MgRowBase &R, int k) { return r[R.c0 + k]; },
        [&](const MgRowBase &R, int k, float rv) {
            r[R.c0 + k] = -md * (R.w01 * L.w[2][k]) * rv;
            e[R.c0 + k] = 0.f;
        });
}

__device__ __forceinline__ void breakdown(KrylovState *st) {
    st->breakdown = 1;
    st->done = 1;
}

// p = z; rho = <r, z>
__global__ void __launch_bounds__(MG_THREADS)
k_mg_first(MgLevel L, const float *r, const float *z, float *p, Partials<1> part,
           KrylovState *st) {
    pdl_wait();
    if (st->done) return;
    double acc = 0;
    level_loop<4>(
        L, [&](int i, int j) { return L.at(i, j, 0); },
        [&](long long c0, int k) { return make_float2(r[c0 + k], z[c0 + k]); },
        [&](long long c0, int k, float2 v) {
            p[c0 + k] = v.y;
            acc += (double)v.x * (double)v.y;
        });
    double v[1] = {acc};
    if (grid_reduce<1>(v, 0u, part) && threadIdx.x == 0) {
        st->rho = v[0];
        if (v[0] == 0.0) st->done = 1;
        else if (!(v[0] > 0.0) || !isfinite(v[0])) breakdown(st);
    }
}

// q = K p; alpha = rho / <p, q>
__global__ void __launch_bounds__(MG_THREADS)
k_mg_spmv(MgLevel L, const float *p, float *q, Partials<1> part, KrylovState *st) {
    pdl_wait();
    if (st->done) return;
    double acc = 0;
    level_loop<4>(
        L, [&](int i, int j) { return MgRow(L, i, j); },
        [&](const MgRow &R, int k) { return make_float2(R.apply(L, p, k), p[R.c0 + k]); },
        [&](const MgRow &R, int k, float2 v) {
            q[R.c0 + k] = v.x;
            acc += (double)v.y * (double)v.x;
        });
    double v[1] = {acc};
    if (grid_reduce<1>(v, 0u, part) && threadIdx.x == 0) {
        if (!(v[0] > 0.0) || !isfinite(v[0])) breakdown(st);
        else st->alpha = st->rho / v[0];
    }
}

// The operands of one row of the VEC SpMV: p at the lane's R rows and at
// its four x/y neighbours, and the values below the lane's first row and
// above its last row from the guide cells (lanes 0 and 31 only; the other
// lanes take them from their neighbours by shuffles).
template <int R>
struct SpmvLoads {
    float c[R], e[R], w[R], n[R], s[R];
    float below, above;
};

template <int R>
__device__ __forceinline__ void spmv_load(const MgLevel &L, const float *p, int i, int j,
                                          int lane, SpmvLoads<R> &v) {
    const int sx = (int)L.g.sx, sy = (int)L.g.sy;
    const int c0 = (int)L.at(i, j, 0), cl = c0 + R * lane;  // stored grids have < 2^31 cells
    load_seg<R>(p + cl, v.c);
    load_seg<R>(p + (cl + sx), v.e);
    load_seg<R>(p + (cl - sx), v.w);
    load_seg<R>(p + (cl + sy), v.n);
    load_seg<R>(p + (cl - sy), v.s);
    v.below = lane == 0 ? p[c0 - 1] : 0.f;
    v.above = lane == 31 ? p[c0 + 32 * R] : 0.f;
}

// (K p) at the lane's R rows of row (i, j) from the row's operands: the z
// neighbours across lanes by shuffles (every lane of the warp calls this)
template <int R>
__device__ __forceinline__ void row_apply(const MgLevel &L, const SpmvLoads<R> &v, int i, int j,
                                          int lane, const float (&w2)[R], const float (&zb)[R],
                                          const float (&zt)[R], float (&out)[R]) {
    const unsigned full = 0xffffffffu;
    const float w0 = L.w[0][i], w1 = L.w[1][j];
    const float xe = L.cf[0][i + 1], xw = L.cf[0][i], yn = L.cf[1][j + 1], ys = L.cf[1][j];
    const float up = __shfl_down_sync(full, v.c[0], 1);
    const float dn = __shfl_up_sync(full, v.c[R - 1], 1);
    const float az = w0 * w1;
    const float sxy = w1 * (xe + xw) + w0 * (yn + ys);
#pragma unroll
    for (int s = 0; s < R; s++) {
        const float bl = s > 0 ? v.c[s > 0 ? s - 1 : 0] : (lane == 0 ? v.below : dn);
        const float ab = s < R - 1 ? v.c[s < R - 1 ? s + 1 : 0] : (lane == 31 ? v.above : up);
        const float diag = w2[s] * sxy + az * (zt[s] + zb[s]);
        const float nb = w2[s] * (w1 * (xe * v.e[s] + xw * v.w[s]) + w0 * (yn * v.n[s] + ys * v.s[s])) +
                         az * (zt[s] * ab + zb[s] * bl);
        out[s] = diag * v.c[s] - nb;
    }
}

// the lane's z widths and face conductances: w2, zb (below), zt (above)
template <int R>
__device__ __forceinline__ void lane_z(const MgLevel &L, int lane, float (&w2)[R], float (&zb)[R],
                                       float (&zt)[R]) {
    load_seg<R>(L.w[2] + R * lane, w2);
    load_seg<R>(L.cf[2] + R * lane, zb);
#pragma unroll
    for (int s = 0; s < R - 1; s++) zt[s] = zb[s + 1];
    zt[R - 1] = L.cf[2][R * lane + R];
}

// q = K p and alpha = rho / <p, q> on rows of exactly 32 R cells (the
// smoother's VEC layout and conditions): one warp per (i, j) row, lane l
// owning rows k = R l + s, every access a vector access; the z conductances
// and widths of the lane's rows stay in registers for all the rows the warp
// visits, and the next row's operands are loaded before this row is
// computed.  Same operator as MgRow::apply.
template <int R>
__global__ void __launch_bounds__(MG_THREADS, R <= 4 ? 3 : 1)
k_mg_spmv_vec(MgLevel L, const float *p, float *q, Partials<1> part, KrylovState *st) {
    pdl_wait();
    if (st->done) return;
    const int lane = threadIdx.x & 31;
    const unsigned nj = (unsigned)L.n[1], rows = (unsigned)L.n[0] * nj;
    const unsigned nw = gridDim.x * (blockDim.x >> 5);
    float w2[R], zb[R], zt[R];
    lane_z<R>(L, lane, w2, zb, zt);
    double acc = 0;
    unsigned row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    Stepper pos(row, nw, nj);
    SpmvLoads<R> cur, nxt;
    if (row < rows) spmv_load<R>(L, p, (int)pos.i, (int)pos.h, lane, cur);
    while (row < rows) {
        const unsigned row2 = row + nw;
        const int i = (int)pos.i, j = (int)pos.h;
        pos.next();
        if (row2 < rows) spmv_load<R>(L, p, (int)pos.i, (int)pos.h, lane, nxt);
        float out[R];
        row_apply<R>(L, cur, i, j, lane, w2, zb, zt, out);
#pragma unroll
        for (int s = 0; s < R; s++) acc += (double)cur.c[s] * (double)out[s];
        store_seg<R>(q + ((int)L.at(i, j, 0) + R * lane), out);
        row = row2;
        cur = nxt;
    }
    double v[1] = {acc};
    if (grid_reduce<1>(v, 0u, part) && threadIdx.x == 0) {
        if (!(v[0] > 0.0) || !isfinite(v[0])) breakdown(st);
        else st->alpha = st->rho / v[0];
    }
}

// The restriction (as k_mg_restrict) from a level of rows of exactly 32 R
// cells to a coarser one that merges cells along x and/or y only (same z
// cells, the same vector-row layout on both): one warp per coarse row, the
// residuals f - K x of its kept children (one or two rows: the colour
// smoothed last is left out) in the SpMV's row form, their operands loaded
// together.
template <int R>
__global__ void __launch_bounds__(MG_THREADS, R <= 2 ? 3 : R <= 4 ? 2 : 1)
k_mg_restrict_vec(MgLevel F, MgLevel C, const float *x, const float *f, float *fc, int skip,
                  const KrylovState *st) {
    pdl_wait();
    if (st->done) return;
    const int lane = threadIdx.x & 31;
    const unsigned nJ = (unsigned)C.n[1], rows = (unsigned)C.n[0] * nJ;
    const unsigned nw = gridDim.x * (blockDim.x >> 5);
    float w2[R], zb[R], zt[R];
    lane_z<R>(F, lane, w2, zb, zt);
    unsigned row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    Stepper pos(row, nw, nJ);
    for (; row < rows; row += nw, pos.next()) {
        const int I = (int)pos.i, J = (int)pos.h;
        int ci[2] = {0, 0}, cj[2] = {0, 0}, kept = 0;
        for (int a = 0; a < C.fac[0]; a++)
            for (int b = 0; b < C.fac[1]; b++) {
                const int i = I * C.fac[0] + a, j = J * C.fac[1] + b;
                if (((i + j) & 1) != skip && kept < 2) {
                    ci[kept] = i;
                    cj[kept] = j;
                    kept++;
                }
            }
        SpmvLoads<R> v[2];
        float fv[2][R];
#pragma unroll
        for (int c = 0; c < 2; c++)
            if (c < kept) {
                spmv_load<R>(F, x, ci[c], cj[c], lane, v[c]);
                load_seg<R>(f + F.at(ci[c], cj[c], 0) + R * lane, fv[c]);
            }
        float sum[R];
#pragma unroll
        for (int s = 0; s < R; s++) sum[s] = 0.f;
#pragma unroll
        for (int c = 0; c < 2; c++)
            if (c < kept) {
                float kx[R];
                row_apply<R>(F, v[c], ci[c], cj[c], lane, w2, zb, zt, kx);
#pragma unroll
                for (int s = 0; s < R; s++) sum[s] += fv[c][s] - kx[s];
            }
        store_seg<R>(fc + C.at(I, J, 0) + R * lane, sum);
    }
}

// e += alpha p, r -= alpha q; err = RMS of r / (-max_diag vol); stop test
__global__ void __launch_bounds__(MG_THREADS)
k_mg_update(MgLevel L, float *e, float *r, const float *p, const float *q, float md,
            Partials<1> part, KrylovState *st) {
    pdl_wait();
    if (st->done) return;
    const float a = (float)st->alpha;
    double acc = 0;
    level_loop<4>(
        L, [&](int i, int j) { return row_base(L, i, j); },
        [&](const MgRowBase &R, int k) {
            const long long c = R.c0 + k;
            return make_float4(e[c], p[c], r[c], q[c]);
        },
        [&](const MgRowBase &R, int k, float4 v) {
            const long long c = R.c0 + k;
            e[c] = v.x + a * v.y;
            const float rn = v.z - a * v.w;
            r[c] = rn;
            const double ra = (double)rn / ((double)md * (double)(R.w01 * L.w[2][k]));
            acc += ra * ra;
        });
    double v[1] = {acc};
    if (grid_reduce<1>(v, 0u, part) && threadIdx.x == 0) {
        st->err = sqrt(v[0] / st->ncell);
        st->it += 1;
        if (!isfinite(st->err)) breakdown(st);
        else if (!(st->err > st->tol) || st->it >= st->max_it) st->done = 1;
    }
}

// beta = <r, z> / rho, rho = <r, z>
__global__ void __launch_bounds__(MG_THREADS)
k_mg_rz(MgLevel L, const float *r, const float *z, Partials<1> part, KrylovState *st) {
    pdl_wait();
    if (st->done) return;
    double acc = 0;
    level_loop<4>(
        L, [&](int i, int j) { return L.at(i, j, 0); },
        [&](long long c0, int k) { return make_float2(r[c0 + k], z[c0 + k]); },
        [&](long long, int, float2 v) { acc += (double)v.x * (double)v.y; });
    double v[1] = {acc};
    if (grid_reduce<1>(v, 0u, part) && threadIdx.x == 0) {
        if (!isfinite(v[0])) {
            breakdown(st);
        } else {
            st->beta = v[0] / st->rho;
            st->rho = v[0];
        }
    }
}

// p = z + beta p
__global__ void __launch_bounds__(MG_THREADS)
k_mg_pupdate(MgLevel L, const float *z, float *p, const KrylovState *st) {
    pdl_wait();
    if (st->done) return;
    const float b = (float)st->beta;
    level_loop<4>(
        L, [&](int i, int j) { return L.at(i, j, 0); },
        [&](long long c0, int k) { return make_float2(z[c0 + k], p[c0 + k]); },
        [&](long long c0, int k, float2 v) { p[c0 + k] = v.x + b * v.y; });
}

// R of the VEC SpMV for this level and these vectors (rows of exactly 32 R
// cells, R = 1, 2, 4, 8; every row start and stride a multiple of 8
// elements; 16-byte aligned vectors and z arrays), else 0
int spmv_vec_r(const MgLevel &v, const float *p, const float *q) {
    auto al = [](const void *x) { return ((uintptr_t)x & 15) == 0; };
    const int nk = v.n[2], R = nk / 32;
    const bool ok = nk % 32 == 0 && (R == 1 || R == 2 || R == 4 || R == 8) &&
                    v.at(0, 0, 0) % 8 == 0 && v.g.sx % 8 == 0 && v.g.sy % 8 == 0 && al(p) &&
                    al(q) && al(v.w[2]) && al(v.cf[2]);
    return ok ? R : 0;
}

int blocks_for(long long n, int cap) {
    long long b = (n + MG_THREADS - 1) / MG_THREADS;
    if (b < 1) b = 1;
    return (int)(b < cap ? b : cap);
}

// launches the V-cycle's steps (mg_vcycle's executor)
// The V-cycle's steps (mg_vcycle's executor).  Two steps are folded into
// the smoothing: the restriction sums only the children of the colour
// smoothed before the last half-sweep (the last half-sweep leaves its own
// colour's residual at zero: each of its lines is solved exactly with
// neighbours it did not change), and each prolongation is applied by the
// next half-sweep (ZlineArgs::xc) instead of a pass of its own.
struct DeviceCycle {
    const LaunchCtx &L;
    const MgDev &M;
    const KrylovState *st;
    int last_color[MG_MAX_LEVELS];
    bool pending[MG_MAX_LEVELS] = {};
    void smooth(int l, int color, bool zero) {
        ZlineArgs a{M.L[l], M.x[l], M.f[l], color, zero ? 1 : 0, nullptr, M.L[l]};
        if (pending[l]) {
            a.xc = M.x[l + 1];
            a.C = M.L[l + 1];
            pending[l] = false;
        }
        L.pre(KK_MG_SMOOTH);
        zline_dispatch(L, a, st);
        L.post(KK_MG_SMOOTH);
        // R f and the other colour's x, W this colour's x: half the level each
        L.bytes(KK_MG_SMOOTH, 4.0 * 1.5 * (double)M.L[l].cells());
        last_color[l] = color;
    }
    void restrict(int l) {
        const MgLevel &F = M.L[l], &C = M.L[l + 1];
        const int nb = blocks_for(C.cells(), L.blocks);
        const int r = C.fac[2] == 1 && C.n[2] == F.n[2] && spmv_vec_r(C, M.f[l + 1], M.f[l + 1])
                          ? spmv_vec_r(F, M.x[l], M.f[l])
                          : 0;
        L.pre(KK_MG_TRANSFER);
        switch (r) {
        case 1: pdl_launch(k_mg_restrict_vec<1>, nb, MG_THREADS, 0, L.s, F, C, M.x[l], M.f[l], M.f[l + 1], last_color[l], st); break;
        case 2: pdl_launch(k_mg_restrict_vec<2>, nb, MG_THREADS, 0, L.s, F, C, M.x[l], M.f[l], M.f[l + 1], last_color[l], st); break;
        case 4: pdl_launch(k_mg_restrict_vec<4>, nb, MG_THREADS, 0, L.s, F, C, M.x[l], M.f[l], M.f[l + 1], last_color[l], st); break;
        case 8: pdl_launch(k_mg_restrict_vec<8>, nb, MG_THREADS, 0, L.s, F, C, M.x[l], M.f[l], M.f[l + 1], last_color[l], st); break;
        default:
            pdl_launch(k_mg_restrict, nb, MG_THREADS, 0, L.s, F, C, M.x[l], M.f[l], M.f[l + 1], last_color[l], st);
            break;
        }
        L.post(KK_MG_TRANSFER);
        // R x, f of half the children; W the coarse f
        L.bytes(KK_MG_TRANSFER, 4.0 * ((double)M.L[l].cells() + 0.5 * (double)M.L[l].cells() +
                                       (double)M.L[l + 1].cells()));
    }
    void coarse() {
        const int l = M.levels - 1;
        L.pre(KK_MG_COARSE);
        pdl_launch(k_mg_coarse, blocks_for((long long)M.ncoarse * 32, L.blocks), MG_THREADS, 0, L.s,
                   M.L[l], M.kinv, M.ncoarse, M.f[l], M.x[l], st);
        L.post(KK_MG_COARSE);
        L.bytes(KK_MG_COARSE, 4.0 * ((double)M.ncoarse * M.ncoarse + 2.0 * M.ncoarse));
    }
    void prolong(int l) { pending[l] = true; }
};
static_assert(MG_NU >= 1, "the prolongation is applied by the first smoothing after it");

}  // namespace

bool mg_prepare(const MgDev &M) {
    for (int l = 0; l < M.levels; l++)
        if (M.L[l].n[2] > 32 * ZL_MAX_R) return false;
    return true;
}

void launch_mg_vcycle(const LaunchCtx &L, const MgDev &M, const KrylovState *st) {
    DeviceCycle e{L, M, st};
    mg_vcycle_nu(e, M.levels, mg_nu);
}

void launch_mg_begin(const LaunchCtx &L, const MgDev &M, const MgPcgBufs &B, double max_diag,
                     Partials<1> part, KrylovState *st) {
    const MgLevel &v = M.L[0];
    const int nb = blocks_for(v.cells(), L.blocks);
    const double n = (double)v.cells();
    L.pre(KK_MG_PCG);
    pdl_launch(k_mg_rhs, nb, MG_THREADS, 0, L.s, v, B.r, B.e, (float)max_diag, st);
    L.post(KK_MG_PCG);
    L.bytes(KK_MG_PCG, 12.0 * n);  // R r; W r, e
    MgDev m = M;
    m.f[0] = B.r;
    m.x[0] = B.z;
    launch_mg_vcycle(L, m, st);
    L.pre(KK_MG_PCG);
    pdl_launch(k_mg_first, L.blocks, MG_THREADS, 0, L.s, v, B.r, B.z, B.p, part, st);
    L.post(KK_MG_PCG);
    L.bytes(KK_MG_PCG, 12.0 * n);  // R r, z; W p
}

void launch_mg_iteration(const LaunchCtx &L, const MgDev &M, const MgPcgBufs &B,
                         double max_diag, Partials<1> part, KrylovState *st) {
    const MgLevel &v = M.L[0];
    const double n = (double)v.cells();
    L.pre(KK_MG_PCG);
    switch (spmv_vec_r(v, B.p, B.q)) {
    case 1: pdl_launch(k_mg_spmv_vec<1>, L.blocks, MG_THREADS, 0, L.s, v, B.p, B.q, part, st); break;
    case 2: pdl_launch(k_mg_spmv_vec<2>, L.blocks, MG_THREADS, 0, L.s, v, B.p, B.q, part, st); break;
    case 4: pdl_launch(k_mg_spmv_vec<4>, L.blocks, MG_THREADS, 0, L.s, v, B.p, B.q, part, st); break;
    case 8: pdl_launch(k_mg_spmv_vec<8>, L.blocks, MG_THREADS, 0, L.s, v, B.p, B.q, part, st); break;
    default: pdl_launch(k_mg_spmv, L.blocks, MG_THREADS, 0, L.s, v, B.p, B.q, part, st); break;
    }
    L.post(KK_MG_PCG);
    L.bytes(KK_MG_PCG, 8.0 * n);  // R p; W q
    L.pre(KK_MG_PCG);
    pdl_launch(k_mg_update, L.blocks, MG_THREADS, 0, L.s, v, B.e, B.r, B.p, B.q, (float)max_diag, part, st);
    L.post(KK_MG_PCG);
    L.bytes(KK_MG_PCG, 24.0 * n);  // R e, p, r, q; W e, r
    MgDev m = M;
    m.f[0] = B.r;
    m.x[0] = B.z;
    launch_mg_vcycle(L, m, st);
    L.pre(KK_MG_PCG);
    pdl_launch(k_mg_rz, L.blocks, MG_THREADS, 0, L.s, v, B.r, B.z, part, st);
    L.post(KK_MG_PCG);
    L.bytes(KK_MG_PCG, 8.0 * n);  // R r, z
    L.pre(KK_MG_PCG);
    pdl_launch(k_mg_pupdate, blocks_for(v.cells(), L.blocks), MG_THREADS, 0, L.s, v, B.z, B.p, st);
    L.post(KK_MG_PCG);
    L.bytes(KK_MG_PCG, 12.0 * n);  // R z, p; W p
}

}  // namespace dalm
