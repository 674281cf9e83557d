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

__global__ void __launch_bounds__(MG_THREADS)
k_mg_smooth(MgLevel L, float *x, const float *f, int color, int zero_start,
            const KrylovState *st) {
    if (st->done) return;
    const long long half = (long long)L.n[0] * L.n[1] * ((L.n[2] + 1) / 2);
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < half;
         n += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        if (mg_color_cell(L, n, color, i, j, k)) mg_smooth_cell(L, x, f, i, j, k, zero_start != 0);
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
        const MgLevel &v = M.L[l];
        const long long half = (long long)v.n[0] * v.n[1] * ((v.n[2] + 1) / 2);
        L.pre(KK_MG_SMOOTH);
        k_mg_smooth<<<blocks_for(half, L.blocks), MG_THREADS, 0, L.s>>>(v, M.x[l], M.f[l], color,
                                                                       zero ? 1 : 0, st);
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
