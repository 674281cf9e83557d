// Discrete-adjoint kernels (FP64).  Each kernel applies one transposed
// stage of the time step (adjoint_cell.cuh) as a gather: every output
// element is written by one thread, so the results do not depend on
// scheduling and need no atomics; the one sum over cells (the adjoint
// pressure right-hand side's norm) uses the deterministic grid reduction.
#include "adjoint.cuh"

namespace dalm {

namespace {

// grid-stride loop over the cells of a box, k fastest (coalesced rows)
template <typename F>
__device__ __forceinline__ void box_loop(const Box &b, F f) {
    const long long nk = b.hi[2] - b.lo[2], nj = b.hi[1] - b.lo[1], ni = b.hi[0] - b.lo[0];
    const long long tot = ni * nj * nk;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < tot;
         n += (long long)gridDim.x * blockDim.x) {
        int k = b.lo[2] + (int)(n % nk);
        long long r = n / nk;
        int j = b.lo[1] + (int)(r % nj);
        int i = b.lo[0] + (int)(r / nj);
        f(i, j, k);
    }
}

__global__ void __launch_bounds__(256) k_adj_velocity_bc(adj::AdjBcArgs A, long long n0, long long n1) {
    for (long long n = n0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; n < n1;
         n += (long long)gridDim.x * blockDim.x)
        adj::adj_velocity_bc_column(A, n);
}

__global__ void __launch_bounds__(256) k_adj_solid(StepParams P, Vec3<double> aU, Box box) {
    box_loop(box, [&](int i, int j, int k) { adj::adj_solid_cell(P, aU, i, j, k); });
}

__global__ void __launch_bounds__(256)
k_adj_project(adj::AdjProjectArgs A, Box box, Partials<1> part, double *sumsq) {
    double acc = 0;
    box_loop(box, [&](int i, int j, int k) { acc += adj::adj_project_cell(A, i, j, k); });
    double v[1] = {acc};
    if (grid_reduce<1>(v, 0u, part) && threadIdx.x == 0) *sumsq = v[0];
}

__global__ void __launch_bounds__(256) k_adj_faces(adj::AdjFacesArgs A, Box box) {
    box_loop(box, [&](int i, int j, int k) { adj::adj_faces_cell(A, i, j, k); });
}

__global__ void __launch_bounds__(256) k_adj_nut(adj::AdjNutArgs A, Box box) {
    box_loop(box, [&](int i, int j, int k) { adj::adj_nut_cell(A, i, j, k); });
}

__global__ void __launch_bounds__(256) k_adj_predict(adj::AdjPredictArgs A, Box box) {
    box_loop(box, [&](int i, int j, int k) { adj::adj_predict_cell(A, i, j, k); });
}

// one block per blade point: the six sums over its support, reduced in a
// fixed order
__global__ void __launch_bounds__(256)
k_adj_alm_gather(StepParams P, AlmDev A, Vec3<const double> af, double *out) {
    __shared__ double smem[32 * 6];
    const int a = blockIdx.x;
    int lo[3], hi[3];
    adj::alm_support_box(P, A, a, lo, hi);
    double acc[6] = {0, 0, 0, 0, 0, 0};
    Box b{{lo[0], lo[1], lo[2]}, {hi[0], hi[1], hi[2]}};
    if (!b.empty()) {
        const long long nk = b.hi[2] - b.lo[2], nj = b.hi[1] - b.lo[1], ni = b.hi[0] - b.lo[0];
        const long long tot = ni * nj * nk;
        for (long long n = threadIdx.x; n < tot; n += blockDim.x) {
            int k = b.lo[2] + (int)(n % nk);
            long long r = n / nk;
            int j = b.lo[1] + (int)(r % nj);
            int i = b.lo[0] + (int)(r / nj);
            adj::adj_alm_gather_term(P, A, af, a, i, j, k, acc);
        }
    }
    block_reduce<6>(acc, 0u, smem);
    if (threadIdx.x == 0)
        for (int m = 0; m < 6; m++) out[6 * (long long)a + m] = acc[m];
}

__global__ void k_adj_alm_point(adj::AdjAlmPointArgs X) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < X.A.ap_count) adj::adj_alm_point(X, a);
}

// adj::adj_alm_scatter in parallel without atomics: one thread per (point,
// corner) entry e.  The entries are streamed through shared memory in
// ascending order; the thread whose entry is the first one naming its cell
// sums every entry of that cell in that order, starting from the cell's
// value, and alone writes it: the serial loop's additions, in its order.
// Block 0's first threads add the per-turbine gradients.
constexpr int SCATTER_TILE = 256;

__global__ void __launch_bounds__(SCATTER_TILE)
k_adj_alm_scatter(adj::AdjAlmPointArgs X, Vec3<double> aU, double *grad) {
    __shared__ long long sid[SCATTER_TILE];
    __shared__ double sval[3][SCATTER_TILE];
    const long long ne = 8 * (long long)X.A.ap_count;
    if (blockIdx.x == 0)
        for (int t = threadIdx.x; t < X.A.wt_count; t += SCATTER_TILE)
            adj::adj_alm_turbine_grad(X.A, X.gth, X.torque, X.weight, t, grad);
    const long long e = blockIdx.x * (long long)SCATTER_TILE + threadIdx.x;
    const long long c = e < ne ? X.ids[e] : -1;
    bool owner = c >= 0;
    double acc[3] = {0, 0, 0};
    for (long long t0 = 0; t0 < ne; t0 += SCATTER_TILE) {
        const long long te = t0 + threadIdx.x;
        __syncthreads();
        if (te < ne) {
            sid[threadIdx.x] = X.ids[te];
            const double wq = X.w[te];
            for (int m = 0; m < 3; m++) sval[m][threadIdx.x] = wq * X.lU[3 * (te / 8) + m];
        } else {
            sid[threadIdx.x] = -1;
        }
        __syncthreads();
        if (!owner) continue;
        const int nt = ne - t0 < SCATTER_TILE ? (int)(ne - t0) : SCATTER_TILE;
        for (int u = 0; u < nt; u++) {
            if (sid[u] != c) continue;
            const long long eu = t0 + u;
            if (eu < e) {  // an earlier entry owns the cell
                owner = false;
                break;
            }
            if (eu == e)
                for (int m = 0; m < 3; m++) acc[m] = aU.c[m][c];
            for (int m = 0; m < 3; m++) acc[m] += sval[m][u];
        }
    }
    if (owner)
        for (int m = 0; m < 3; m++) aU.c[m][c] = acc[m];
}

__global__ void k_adj_scale(double *v, long long n, double s) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        v[i] *= s;
}

int grid_for(long long n, int cap) {
    long long b = (n + 255) / 256;
    if (b < 1) b = 1;
    return (int)(b < cap ? b : cap);
}

}  // namespace

void launch_adj_velocity_bc(const LaunchCtx &L, const adj::AdjBcArgs &A) {
    const Grid &g = A.P.g;
    long long nyz = (long long)g.nj() * g.nk(), nxz = (long long)g.ni() * g.nk(),
              nxy = (long long)g.ni() * g.nj();
    long long mid = 2 * (nyz + nxz), tot = mid + 2 * nxy;
    L.pre(KK_ADJ_BC);
    k_adj_velocity_bc<<<grid_for(mid, L.blocks), 256, 0, L.s>>>(A, 0, mid);
    L.post(KK_ADJ_BC);
    L.pre(KK_ADJ_BC);
    k_adj_velocity_bc<<<grid_for(tot - mid, L.blocks), 256, 0, L.s>>>(A, mid, tot);
    L.post(KK_ADJ_BC);
}

void launch_adj_project(const LaunchCtx &L, const adj::AdjProjectArgs &A, Partials<1> part,
                        double *sumsq) {
    const Grid &g = A.P.g;
    Box box{{g.gc, g.gc, g.gc}, {g.nx - g.gc, g.ny - g.gc, g.nz - g.gc}};
    if (A.P.solid) {  // the solid scaling sits between the projection and the BCs
        L.pre(KK_ADJ_PROJECT);
        k_adj_solid<<<L.blocks, 256, 0, L.s>>>(A.P, Vec3<double>{{const_cast<double *>(A.aU.c[0]),
                                                                  const_cast<double *>(A.aU.c[1]),
                                                                  const_cast<double *>(A.aU.c[2])}},
                                                box);
        L.post(KK_ADJ_PROJECT);
    }
    L.pre(KK_ADJ_PROJECT);
    k_adj_project<<<L.blocks, 256, 0, L.s>>>(A, box, part, sumsq);
    L.post(KK_ADJ_PROJECT);
}

void launch_adj_faces(const LaunchCtx &L, const adj::AdjFacesArgs &A) {
    const Grid &g = A.P.g;
    // the interior and the first outflow guide plane (the outlet face reads it)
    Box box{{g.gc, g.gc, g.gc}, {g.nx - g.gc + 1, g.ny - g.gc, g.nz - g.gc}};
    L.pre(KK_ADJ_FACES);
    k_adj_faces<<<L.blocks, 256, 0, L.s>>>(A, box);
    L.post(KK_ADJ_FACES);
}

void launch_adj_predict(const LaunchCtx &L, const adj::AdjNutArgs &N, const adj::AdjPredictArgs &A) {
    const Grid &g = A.P.g;
    Box inner{{g.gc, g.gc, g.gc}, {g.nx - g.gc, g.ny - g.gc, g.nz - g.gc}};
    Box all{{0, 0, 0}, {g.nx, g.ny, g.nz}};
    L.pre(KK_ADJ_NUT);
    k_adj_nut<<<L.blocks, 256, 0, L.s>>>(N, inner);
    L.post(KK_ADJ_NUT);
    L.pre(KK_ADJ_PREDICT);
    k_adj_predict<<<L.blocks, 256, 0, L.s>>>(A, all);
    L.post(KK_ADJ_PREDICT);
}

void launch_adj_scale(const LaunchCtx &L, double *v, long long n, double s) {
    L.pre(KK_ADJ_PROJECT);
    k_adj_scale<<<grid_for(n, L.blocks), 256, 0, L.s>>>(v, n, s);
    L.post(KK_ADJ_PROJECT);
}

void launch_adj_alm(const LaunchCtx &L, const StepParams &P, const AlmDev &A,
                    Vec3<const double> af, const adj::AdjAlmPointArgs &X, Vec3<double> aU,
                    double *grad) {
    if (A.ap_count <= 0) return;
    L.pre(KK_ADJ_ALM);
    k_adj_alm_gather<<<A.ap_count, 256, 0, L.s>>>(P, A, af, const_cast<double *>(X.gather));
    L.post(KK_ADJ_ALM);
    L.pre(KK_ADJ_ALM);
    k_adj_alm_point<<<(A.ap_count + 63) / 64, 64, 0, L.s>>>(X);
    L.post(KK_ADJ_ALM);
    L.pre(KK_ADJ_ALM);
    const long long ne = 8 * (long long)A.ap_count;
    k_adj_alm_scatter<<<(int)((ne + SCATTER_TILE - 1) / SCATTER_TILE), SCATTER_TILE, 0, L.s>>>(X, aU,
                                                                                            grad);
    L.post(KK_ADJ_ALM);
}

}  // namespace dalm
