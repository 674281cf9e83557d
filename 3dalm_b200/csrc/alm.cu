// Actuator-line kernels (FP64), compiled with --fmad=false so the blade-point
// arithmetic keeps the reference's rounding; only the libm calls (sin, cos,
// atan, exp) may differ from the host's by an ulp.
#include "alm_point.cuh"

namespace dalm {

namespace {

__device__ __forceinline__ double sq(double v) { return v * v; }

// update_ap_position + calc_ap_force (src/alm.h:233-370), one thread per
// blade point; the arithmetic is almpt's (alm_point.cuh), shared with the
// host path of the reference-order mode.
// T: storage type of the velocity field (double, or float for the mixed
// form's FP32 stencil fields); the point model is FP64 either way.
template <typename T>
__global__ void k_alm_points(StepParams P, AlmDev A, double t, Vec3<const T> U) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= A.ap_count) return;
    const TurbineDev &wt = A.wt[a / A.ap_per_wt];
    int bid = (a % A.ap_per_wt) / A.ap_per_blade;
    almpt::Pose q;
    almpt::point_pose(wt, A.r[a], bid, A.blades, t, q);
    long long id[8];
    double frac[3], f[3] = {0, 0, 0}, torque = 0, thrust = 0;
    if (almpt::point_cell(P.g, P.m.x, P.m.y, P.m.z, q.xyz, id, frac)) {
        double Uap[3];
        for (int m = 0; m < 3; m++) {
            const T *v = U.c[m];
            double c8[8];
            for (int n = 0; n < 8; n++) c8[n] = (double)v[id[n]];
            Uap[m] = almpt::trilinear(c8, frac);
        }
        almpt::point_force(wt, q, Uap, A.twist[a], A.chord[a], A.dr[a], A.atk, A.atk_count,
                           A.cd + (long long)a * A.atk_count, A.cl + (long long)a * A.atk_count,
                           f, torque, thrust);
    }
    for (int m = 0; m < 3; m++) {
        A.pt_xyz[a * 3 + m] = q.xyz[m];
        A.pt_f[a * 3 + m] = f[m];
    }
    A.pt_torque[a] = torque;
    A.pt_thrust[a] = thrust;
}

// Per-turbine torque / thrust in blade-point order (src/alm.h:384-398).
__global__ void k_alm_sums(AlmDev A) {
    int w = threadIdx.x;
    if (w >= A.wt_count) return;
    double torque = 0, thrust = 0;
    for (int a = w * A.ap_per_wt; a < (w + 1) * A.ap_per_wt; a++) {
        torque += A.pt_torque[a];
        thrust += A.pt_thrust[a];
    }
    A.wt_torque[w] = torque;
    A.wt_thrust[w] = thrust;
}

// distribute_ap_force (src/alm.h:416-448), support-confined: each block
// gathers, in blade-point order, the points whose truncated support reaches
// its tile, then every cell of the tile sums those points in that order
// (the reference's order with the negligible far terms left out).
template <typename FT>
__global__ void __launch_bounds__(TILE_THREADS)
k_alm_project(StepParams P, AlmDev A, Tiling T, Vec3<FT> F) {
    extern __shared__ int list[];
    __shared__ int warp_count[TILE_THREADS / 32];
    __shared__ int total;
    const Grid &g = P.g;
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (long long tile = blockIdx.x; tile < T.ntiles; tile += gridDim.x) {
        int i, j, k;
        bool valid = T.cell(tile, i, j, k);
        // tile bounding box in coordinates (cell-centre arrays are increasing)
        int tk = (int)(tile % T.ntk);
        int tj = (int)((tile / T.ntk) % T.ntj);
        int ti = (int)((tile / T.ntk) / T.ntj);
        int k0 = T.box.lo[2] + tk * TK, k1 = min(k0 + TK, T.box.hi[2]) - 1;
        int j0 = T.box.lo[1] + tj * TJ, j1 = min(j0 + TJ, T.box.hi[1]) - 1;
        int i0 = T.box.lo[0] + ti;
        double bx0 = P.m.x[i0], by0 = P.m.y[j0], by1 = P.m.y[j1], bz0 = P.m.z[k0],
               bz1 = P.m.z[k1];
        if (threadIdx.x == 0) total = 0;
        __syncthreads();
        for (int base = 0; base < A.ap_count; base += TILE_THREADS) {
            int a = base + threadIdx.x;
            bool near = false;
            if (a < A.ap_count) {
                double px = A.pt_xyz[a * 3], py = A.pt_xyz[a * 3 + 1], pz = A.pt_xyz[a * 3 + 2];
                double dx = px - bx0;
                double dy = py < by0 ? by0 - py : (py > by1 ? py - by1 : 0.0);
                double dz = pz < bz0 ? bz0 - pz : (pz > bz1 ? pz - bz1 : 0.0);
                near = dx * dx + dy * dy + dz * dz <= A.cutoff2;
            }
            unsigned mask = __ballot_sync(0xffffffffu, near);
            if (lane == 0) warp_count[warp] = __popc(mask);
            __syncthreads();
            int before = total;
            for (int w = 0; w < warp; w++) before += warp_count[w];
            if (near) list[before + __popc(mask & ((1u << lane) - 1u))] = a;
            __syncthreads();
            if (threadIdx.x == 0) {
                int s = 0;
                for (int w = 0; w < TILE_THREADS / 32; w++) s += warp_count[w];
                total += s;
            }
            __syncthreads();
        }
        int n = total;
        if (valid) {
            double fx = 0, fy = 0, fz = 0;
            double xc = P.m.x[i], yc = P.m.y[j], zc = P.m.z[k];
            for (int l = 0; l < n; l++) {
                int a = list[l];
                double r2 = sq(xc - A.pt_xyz[a * 3]) + sq(yc - A.pt_xyz[a * 3 + 1]) +
                            sq(zc - A.pt_xyz[a * 3 + 2]);
                if (r2 <= A.cutoff2) {
                    double wght = A.e_coef * exp(-r2 / A.pw2);
                    fx += wght * A.pt_f[a * 3];
                    fy += wght * A.pt_f[a * 3 + 1];
                    fz += wght * A.pt_f[a * 3 + 2];
                }
            }
            long long c = g.at(i, j, k);
            F.c[0][c] = (FT)fx;
            F.c[1][c] = (FT)fy;
            F.c[2][c] = (FT)fz;
        }
        __syncthreads();
    }
}

}  // namespace

template <typename T>
void launch_alm_points(const LaunchCtx &L, const StepParams &P, const AlmDev &A, double t,
                       Vec3<const T> u) {
    if (A.ap_count <= 0) return;
    L.pre(KK_ALM_POINTS);
    k_alm_points<T><<<(A.ap_count + 63) / 64, 64, 0, L.s>>>(P, A, t, u);
    L.post(KK_ALM_POINTS);
    L.pre(KK_ALM_SUMS);
    k_alm_sums<<<1, 32 * ((A.wt_count + 31) / 32), 0, L.s>>>(A);
    L.post(KK_ALM_SUMS);
}
template void launch_alm_points<double>(const LaunchCtx &, const StepParams &, const AlmDev &,
                                        double, Vec3<const double>);
template void launch_alm_points<float>(const LaunchCtx &, const StepParams &, const AlmDev &,
                                       double, Vec3<const float>);

template <typename FT>
void launch_alm_project(const LaunchCtx &L, const StepParams &P, const AlmDev &A,
                        const Box &box, Vec3<FT> f) {
    if (A.ap_count <= 0 || box.empty()) return;
    Tiling T = Tiling::make(box);
    long long blocks = T.ntiles < 4096 ? T.ntiles : 4096;
    size_t smem = sizeof(int) * (size_t)A.ap_count;
    L.pre(KK_ALM_PROJECT);
    k_alm_project<FT><<<(int)blocks, TILE_THREADS, smem, L.s>>>(P, A, T, f);
    L.post(KK_ALM_PROJECT);
}
template void launch_alm_project<double>(const LaunchCtx &, const StepParams &, const AlmDev &,
                                         const Box &, Vec3<double>);
template void launch_alm_project<float>(const LaunchCtx &, const StepParams &, const AlmDev &,
                                        const Box &, Vec3<float>);

}  // namespace dalm
