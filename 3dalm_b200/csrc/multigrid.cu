// Multigrid-preconditioned conjugate gradients in FP32 (the inner solves of
// DALM_MIXED); the arithmetic is in multigrid.cuh.  Vectors are FP32, sums
// FP64 through the deterministic grid reduction, Krylov scalars on the
// device; every kernel returns at once once the solve is done, so batches
// of iterations can be enqueued (and replayed as CUDA graphs) ahead of the
// host's convergence check.
#include <cfloat>

#include "multigrid.cuh"
#include "poisson.cuh"

namespace dalm {

namespace {

constexpr int MG_THREADS = 256;

// interior cells of a level, k fastest
template <typename F>
__device__ __forceinline__ void level_loop(const MgLevel &L, F f) {
    const long long tot = L.cells();
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < tot;
         n += (long long)gridDim.x * blockDim.x) {
        int k = (int)(n % L.n[2]);
        long long r = n / L.n[2];
        int j = (int)(r % L.n[1]);
        int i = (int)(r / L.n[1]);
        f(i, j, k);
    }
}

// Zebra z-line half-sweep, one warp per column: lane l holds rows
// k = l + 32 r (r < R, so the warp's loads and stores are coalesced rows)
// and the tridiagonal system is solved by parallel cyclic reduction:
// step delta combines every row with rows k -+ delta (through shuffles for
// delta < 32, within the lane above) until each row stands alone; rows past
// the column are identity rows.  The line operator is diagonally dominant,
// which keeps the reduction stable without pivoting.  Same result as the
// Thomas elimination of mg_thomas up to rounding (this file is compiled
// with contraction and fast quotients).  Blocks only read columns
// of the other colour and only write their own.
template <int R>
__global__ void __launch_bounds__(MG_THREADS)
k_mg_smooth(MgLevel L, float *x, const float *f, int color, int zero_start,
            const KrylovState *st) {
    if (st->done) return;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long ncol = (long long)L.n[0] * ((L.n[1] + 1) / 2);
    const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
    const int nk = L.n[2];
    const bool zero = zero_start != 0;
    for (long long col = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5);
         col < ncol; col += nw) {
        int i, j;
        if (!mg_color_column(L, col, color, i, j)) continue;  // uniform in the warp
        float a[R], b[R], c[R], d[R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int k = lane + 32 * r;
            if (k < nk) {
                float lo, hi, bb;
                mg_zline_coef(L, i, j, k, lo, hi, bb);
                a[r] = -lo;
                c[r] = -hi;
                b[r] = bb;
                d[r] = mg_zline_rhs(L, x, f, i, j, k, zero);
            } else {
                a[r] = 0.f;
                c[r] = 0.f;
                b[r] = 1.f;
                d[r] = 0.f;
            }
        }
#pragma unroll
        for (int delta = 1; delta < 32 * R; delta <<= 1) {
            float na[R], nb[R], nc[R], nd[R];
#pragma unroll
            for (int r = 0; r < R; r++) {
                // row k - delta and row k + delta (identity outside the column)
                float am = 0.f, bm = 1.f, cm = 0.f, dm = 0.f, ap = 0.f, bp = 1.f, cp = 0.f, dp = 0.f;
                if (delta < 32) {
                    const int src_m = (lane - delta) & 31, src_p = (lane + delta) & 31;
                    const bool wrap_m = lane < delta, wrap_p = lane + delta >= 32;
                    // same register r, or r - 1 / r + 1 across the lane wrap
                    const float a0 = __shfl_sync(full, a[r], src_m), b0 = __shfl_sync(full, b[r], src_m);
                    const float c0 = __shfl_sync(full, c[r], src_m), d0 = __shfl_sync(full, d[r], src_m);
                    const float a1 = __shfl_sync(full, r > 0 ? a[r > 0 ? r - 1 : 0] : 0.f, src_m);
                    const float b1 = __shfl_sync(full, r > 0 ? b[r > 0 ? r - 1 : 0] : 1.f, src_m);
                    const float c1 = __shfl_sync(full, r > 0 ? c[r > 0 ? r - 1 : 0] : 0.f, src_m);
                    const float d1 = __shfl_sync(full, r > 0 ? d[r > 0 ? r - 1 : 0] : 0.f, src_m);
                    am = wrap_m ? a1 : a0; bm = wrap_m ? b1 : b0; cm = wrap_m ? c1 : c0; dm = wrap_m ? d1 : d0;
                    const float a2 = __shfl_sync(full, a[r], src_p), b2 = __shfl_sync(full, b[r], src_p);
                    const float c2 = __shfl_sync(full, c[r], src_p), d2 = __shfl_sync(full, d[r], src_p);
                    const float a3 = __shfl_sync(full, r + 1 < R ? a[r + 1 < R ? r + 1 : r] : 0.f, src_p);
                    const float b3 = __shfl_sync(full, r + 1 < R ? b[r + 1 < R ? r + 1 : r] : 1.f, src_p);
                    const float c3 = __shfl_sync(full, r + 1 < R ? c[r + 1 < R ? r + 1 : r] : 0.f, src_p);
                    const float d3 = __shfl_sync(full, r + 1 < R ? d[r + 1 < R ? r + 1 : r] : 0.f, src_p);
                    ap = wrap_p ? a3 : a2; bp = wrap_p ? b3 : b2; cp = wrap_p ? c3 : c2; dp = wrap_p ? d3 : d2;
                } else {
                    const int m = delta / 32;
                    if (r - m >= 0) {
                        am = a[r - m >= 0 ? r - m : 0]; bm = b[r - m >= 0 ? r - m : 0];
                        cm = c[r - m >= 0 ? r - m : 0]; dm = d[r - m >= 0 ? r - m : 0];
                    }
                    if (r + m < R) {
                        ap = a[r + m < R ? r + m : 0]; bp = b[r + m < R ? r + m : 0];
                        cp = c[r + m < R ? r + m : 0]; dp = d[r + m < R ? r + m : 0];
                    }
                }
                // approximate quotients (2 ulp): the preconditioner needs no
                // correctly rounded division
                const float al = -__fdividef(a[r], bm), ga = -__fdividef(c[r], bp);
                na[r] = al * am;
                nc[r] = ga * cp;
                nb[r] = b[r] + al * cm + ga * ap;
                nd[r] = d[r] + al * dm + ga * dp;
            }
#pragma unroll
            for (int r = 0; r < R; r++) {
                a[r] = na[r];
                b[r] = nb[r];
                c[r] = nc[r];
                d[r] = nd[r];
            }
        }
        const long long c0 = L.at(i, j, 0);
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int k = lane + 32 * r;
            if (k < nk) x[c0 + k] = __fdividef(d[r], b[r]);
        }
    }
}

// longest line the warp solver takes (32 rows per register slot)
constexpr int ZL_MAX_R = 8;

template <int R>
void zline_launch(const LaunchCtx &L, const MgLevel &v, float *x, const float *f, int color,
                  int zero, const KrylovState *st, int blocks) {
    k_mg_smooth<R><<<blocks, MG_THREADS, 0, L.s>>>(v, x, f, color, zero, st);
}

void zline_dispatch(const LaunchCtx &L, const MgLevel &v, float *x, const float *f, int color,
                    int zero, const KrylovState *st) {
    const long long ncol = (long long)v.n[0] * ((v.n[1] + 1) / 2);
    long long nb = (ncol + MG_THREADS / 32 - 1) / (MG_THREADS / 32);
    if (nb > L.blocks) nb = L.blocks;
    const int R = (v.n[2] + 31) / 32;
    switch (R) {
    case 1: zline_launch<1>(L, v, x, f, color, zero, st, (int)nb); break;
    case 2: zline_launch<2>(L, v, x, f, color, zero, st, (int)nb); break;
    case 3: zline_launch<3>(L, v, x, f, color, zero, st, (int)nb); break;
    case 4: zline_launch<4>(L, v, x, f, color, zero, st, (int)nb); break;
    case 5: zline_launch<5>(L, v, x, f, color, zero, st, (int)nb); break;
    case 6: zline_launch<6>(L, v, x, f, color, zero, st, (int)nb); break;
    case 7: zline_launch<7>(L, v, x, f, color, zero, st, (int)nb); break;
    default: zline_launch<8>(L, v, x, f, color, zero, st, (int)nb); break;
    }
}

__global__ void __launch_bounds__(MG_THREADS)
k_mg_restrict(MgLevel F, MgLevel C, const float *x, const float *f, float *fc,
              const KrylovState *st) {
    if (st->done) return;
    level_loop(C, [&](int I, int J, int K) { mg_restrict_cell(F, C, x, f, fc, I, J, K); });
}

__global__ void __launch_bounds__(MG_THREADS)
k_mg_prolong(MgLevel F, MgLevel C, float *x, const float *xc, const KrylovState *st) {
    if (st->done) return;
    level_loop(F, [&](int i, int j, int k) { mg_prolong_cell(F, C, x, xc, i, j, k); });
}

// x = K^-1 f on the coarsest level: one warp per row of the dense inverse
__global__ void __launch_bounds__(MG_THREADS)
k_mg_coarse(MgLevel C, const float *kinv, int n, const float *f, float *x,
            const KrylovState *st) {
    if (st->done) return;
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n; r += warps) {
        const float *row = kinv + (long long)r * n;
        float s = 0;
        for (int c = lane; c < n; c += 32) s += row[c] * f[mg_cell_index(C, c)];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) x[mg_cell_index(C, r)] = s;
    }
}

__device__ __forceinline__ float cell_volume(const MgLevel &L, int i, int j, int k) {
    return L.w[0][i] * L.w[1][j] * L.w[2][k];
}

// f = -max_diag vol r (in place), e = 0
__global__ void __launch_bounds__(MG_THREADS)
k_mg_rhs(MgLevel L, float *r, float *e, float md, const KrylovState *st) {
    if (st->done) return;
    level_loop(L, [&](int i, int j, int k) {
        const long long c = L.at(i, j, k);
        r[c] = -md * cell_volume(L, i, j, k) * r[c];
        e[c] = 0.f;
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
    if (st->done) return;
    double acc = 0;
    level_loop(L, [&](int i, int j, int k) {
        const long long c = L.at(i, j, k);
        p[c] = z[c];
        acc += (double)r[c] * (double)z[c];
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
    if (st->done) return;
    double acc = 0;
    level_loop(L, [&](int i, int j, int k) {
        const long long c = L.at(i, j, k);
        const float v = mg_apply(L, p, i, j, k);
        q[c] = v;
        acc += (double)p[c] * (double)v;
    });
    double v[1] = {acc};
    if (grid_reduce<1>(v, 0u, part) && threadIdx.x == 0) {
        if (!(v[0] > 0.0) || !isfinite(v[0])) breakdown(st);
        else st->alpha = st->rho / v[0];
    }
}

// e += alpha p, r -= alpha q; err = RMS of r / (-max_diag vol); stop test
__global__ void __launch_bounds__(MG_THREADS)
k_mg_update(MgLevel L, float *e, float *r, const float *p, const float *q, float md,
            Partials<1> part, KrylovState *st) {
    if (st->done) return;
    const float a = (float)st->alpha;
    double acc = 0;
    level_loop(L, [&](int i, int j, int k) {
        const long long c = L.at(i, j, k);
        e[c] += a * p[c];
        const float rn = r[c] - a * q[c];
        r[c] = rn;
        const double ra = (double)rn / ((double)md * (double)cell_volume(L, i, j, k));
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
    if (st->done) return;
    double acc = 0;
    level_loop(L, [&](int i, int j, int k) {
        const long long c = L.at(i, j, k);
        acc += (double)r[c] * (double)z[c];
    });
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
    if (st->done) return;
    const float b = (float)st->beta;
    level_loop(L, [&](int i, int j, int k) {
        const long long c = L.at(i, j, k);
        p[c] = z[c] + b * p[c];
    });
}

int blocks_for(long long n, int cap) {
    long long b = (n + MG_THREADS - 1) / MG_THREADS;
    if (b < 1) b = 1;
    return (int)(b < cap ? b : cap);
}

// launches the V-cycle's steps (mg_vcycle's executor)
struct DeviceCycle {
    const LaunchCtx &L;
    const MgDev &M;
    const KrylovState *st;
    void smooth(int l, int color, bool zero) {
        L.pre(KK_MG_SMOOTH);
        zline_dispatch(L, M.L[l], M.x[l], M.f[l], color, zero ? 1 : 0, st);
        L.post(KK_MG_SMOOTH);
    }
    void restrict(int l) {
        L.pre(KK_MG_TRANSFER);
        k_mg_restrict<<<blocks_for(M.L[l + 1].cells(), L.blocks), MG_THREADS, 0, L.s>>>(
            M.L[l], M.L[l + 1], M.x[l], M.f[l], M.f[l + 1], st);
        L.post(KK_MG_TRANSFER);
    }
    void coarse() {
        const int l = M.levels - 1;
        L.pre(KK_MG_COARSE);
        k_mg_coarse<<<blocks_for((long long)M.ncoarse * 32, L.blocks), MG_THREADS, 0, L.s>>>(
            M.L[l], M.kinv, M.ncoarse, M.f[l], M.x[l], st);
        L.post(KK_MG_COARSE);
    }
    void prolong(int l) {
        L.pre(KK_MG_TRANSFER);
        k_mg_prolong<<<blocks_for(M.L[l].cells(), L.blocks), MG_THREADS, 0, L.s>>>(
            M.L[l], M.L[l + 1], M.x[l], M.x[l + 1], st);
        L.post(KK_MG_TRANSFER);
    }
};

}  // namespace

bool mg_prepare(const MgDev &M) {
    for (int l = 0; l < M.levels; l++)
        if (M.L[l].n[2] > 32 * ZL_MAX_R) return false;
    return true;
}

void launch_mg_vcycle(const LaunchCtx &L, const MgDev &M, const KrylovState *st) {
    DeviceCycle e{L, M, st};
    mg_vcycle(e, M.levels, MG_NU);
}

void launch_mg_begin(const LaunchCtx &L, const MgDev &M, const MgPcgBufs &B, double max_diag,
                     Partials<1> part, KrylovState *st) {
    const MgLevel &v = M.L[0];
    const int nb = blocks_for(v.cells(), L.blocks);
    L.pre(KK_MG_PCG);
    k_mg_rhs<<<nb, MG_THREADS, 0, L.s>>>(v, B.r, B.e, (float)max_diag, st);
    L.post(KK_MG_PCG);
    MgDev m = M;
    m.f[0] = B.r;
    m.x[0] = B.z;
    launch_mg_vcycle(L, m, st);
    L.pre(KK_MG_PCG);
    k_mg_first<<<L.blocks, MG_THREADS, 0, L.s>>>(v, B.r, B.z, B.p, part, st);
    L.post(KK_MG_PCG);
}

void launch_mg_iteration(const LaunchCtx &L, const MgDev &M, const MgPcgBufs &B,
                         double max_diag, Partials<1> part, KrylovState *st) {
    const MgLevel &v = M.L[0];
    L.pre(KK_MG_PCG);
    k_mg_spmv<<<L.blocks, MG_THREADS, 0, L.s>>>(v, B.p, B.q, part, st);
    L.post(KK_MG_PCG);
    L.pre(KK_MG_PCG);
    k_mg_update<<<L.blocks, MG_THREADS, 0, L.s>>>(v, B.e, B.r, B.p, B.q, (float)max_diag, part, st);
    L.post(KK_MG_PCG);
    MgDev m = M;
    m.f[0] = B.r;
    m.x[0] = B.z;
    launch_mg_vcycle(L, m, st);
    L.pre(KK_MG_PCG);
    k_mg_rz<<<L.blocks, MG_THREADS, 0, L.s>>>(v, B.r, B.z, part, st);
    L.post(KK_MG_PCG);
    L.pre(KK_MG_PCG);
    k_mg_pupdate<<<blocks_for(v.cells(), L.blocks), MG_THREADS, 0, L.s>>>(v, B.z, B.p, st);
    L.post(KK_MG_PCG);
}

}  // namespace dalm
