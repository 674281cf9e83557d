// Actuator-line kernels (FP64), compiled with --fmad=false so the blade-point
// arithmetic keeps the reference's rounding; only the libm calls (sin, cos,
// atan, exp) may differ from the host's by an ulp.
#include "alm.cuh"

namespace dalm {

namespace {

constexpr double PI_D = 3.14159265358979323846;  // M_PI (src/type.h:12)

__device__ __forceinline__ double sq(double v) { return v * v; }
__device__ __forceinline__ double sgn(double v) { return (double)((v > 0.) - (v < 0.)); }

// find_floor_index (src/util.h:119-146)
__device__ int floor_index(const double *a, double v, int n) {
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

// frame_transform (src/euler_angle.h:34-62)
__device__ void frame_transform(const double in[3], double out[3], double angle, int type) {
    double c = cos(angle), s = sin(angle);
    double x = in[0], y = in[1], z = in[2];
    switch (type) {
    case EULER_ROLL: out[0] = x; out[1] = c * y + s * z; out[2] = -s * y + c * z; break;
    case EULER_PITCH: out[0] = c * x - s * z; out[1] = y; out[2] = -s * x + c * z; break;
    case EULER_YAW: out[0] = c * x + s * y; out[1] = -s * x + c * y; out[2] = z; break;
    default: out[0] = x; out[1] = y; out[2] = z; break;
    }
}

// frame_transform_U (src/euler_angle.h:64-127), reproducing its two typos
// (roll: -s*v + v*w; yaw: ow*(-c*s - s*y)).
__device__ void frame_transform_U(const double p[3], const double U[3], double out[3],
                                  double angle, double ow, int type) {
    double c = cos(angle), s = sin(angle);
    double x = p[0], y = p[1], z = p[2], u = U[0], v = U[1], w = U[2];
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

__device__ double lin_interp(double v0, double v1, double x0, double x1, double xp) {
    double fx = (xp - x0) / (x1 - x0);  // src/util.h:166-174
    return v0 * (1 - fx) + v1 * fx;
}

__global__ void k_alm_points(StepParams P, AlmDev A, double t, Vec3<const double> U) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= A.ap_count) return;
    const Grid &g = P.g;
    const TurbineDev &wt = A.wt[a / A.ap_per_wt];
    // wt.angle, wt.ow (src/alm.h:236-244)
    double angle = wt.formula[0] * sin(wt.formula[1] * t + wt.formula[2]) + wt.formula[3];
    double ow = wt.formula[0] * wt.formula[1] * cos(wt.formula[1] * t + wt.formula[2]);
    // blade-point position (src/alm.h:250-266)
    int bid = (a % A.ap_per_wt) / A.ap_per_blade;
    double r = A.r[a];
    double theta = bid * (2 * PI_D / A.blades) + t * wt.rot_speed;
    double loc[3] = {wt.rot_center[0], wt.rot_center[1] + r * cos(theta),
                     wt.rot_center[2] + r * sin(theta)};
    double xyz[3];
    frame_transform(loc, xyz, -angle, wt.type);
    for (int m = 0; m < 3; m++) xyz[m] += wt.base[m];
    // force (src/alm.h:287-370)
    int i = floor_index(P.m.x, xyz[0], g.nx);
    int j = floor_index(P.m.y, xyz[1], g.ny);
    int k = floor_index(P.m.z, xyz[2], g.nz);
    double f[3] = {0, 0, 0}, torque = 0, thrust = 0;
    if (i >= g.gc && i < g.nx - g.gc && j >= g.gc && j < g.ny - g.gc && k >= g.gc &&
        k < g.nz - g.gc) {
        long long id[8] = {g.at(i, j, k),         g.at(i + 1, j, k),
                           g.at(i, j + 1, k),     g.at(i + 1, j + 1, k),
                           g.at(i, j, k + 1),     g.at(i + 1, j, k + 1),
                           g.at(i, j + 1, k + 1), g.at(i + 1, j + 1, k + 1)};
        double x0 = P.m.x[i], x1 = P.m.x[i + 1], y0 = P.m.y[j], y1 = P.m.y[j + 1];
        double z0 = P.m.z[k], z1 = P.m.z[k + 1];
        double fx = (xyz[0] - x0) / (x1 - x0), fy = (xyz[1] - y0) / (y1 - y0),
               fz = (xyz[2] - z0) / (z1 - z0);
        double Uap[3];
        for (int m = 0; m < 3; m++) {
            const double *v = U.c[m];
            // trilinear_interpolate (src/util.h:176-199)
            double v01 = v[id[0]] * (1 - fx) + v[id[1]] * fx;
            double v23 = v[id[2]] * (1 - fx) + v[id[3]] * fx;
            double v45 = v[id[4]] * (1 - fx) + v[id[5]] * fx;
            double v67 = v[id[6]] * (1 - fx) + v[id[7]] * fx;
            double v0123 = v01 * (1 - fy) + v23 * fy;
            double v4567 = v45 * (1 - fy) + v67 * fy;
            Uap[m] = v0123 * (1 - fz) + v4567 * fz;
        }
        double rel[3] = {xyz[0] - wt.base[0], xyz[1] - wt.base[1], xyz[2] - wt.base[2]};
        double Ur[3];
        frame_transform_U(rel, Uap, Ur, angle, ow, wt.type);
        double ux_ = Ur[0];
        double ut_ = r * wt.rot_speed + Ur[1] * sin(theta) - Ur[2] * cos(theta);
        double urel2 = ux_ * ux_ + ut_ * ut_;
        double phi = atan(ux_ / ut_);
        double atk = phi * 180 / PI_D - A.twist[a];
        // lookup_cdcl_table (src/alm.h:208-231)
        const double *cdt = A.cd + (long long)a * A.atk_count;
        const double *clt = A.cl + (long long)a * A.atk_count;
        int ti = floor_index(A.atk, atk, A.atk_count);
        double cd, cl;
        if (ti < 0) {
            cd = cdt[0]; cl = clt[0];
        } else if (ti >= A.atk_count - 1) {
            cd = cdt[A.atk_count - 1]; cl = clt[A.atk_count - 1];
        } else {
            cd = lin_interp(cdt[ti], cdt[ti + 1], A.atk[ti], A.atk[ti + 1], atk);
            cl = lin_interp(clt[ti], clt[ti + 1], A.atk[ti], A.atk[ti + 1], atk);
        }
        double fd = 0.5 * cd * urel2 * A.chord[a] * A.dr[a];
        double fl = 0.5 * cl * urel2 * A.chord[a] * A.dr[a];
        double fx_ = fl * cos(phi) + fd * sin(phi);
        double ft_ = fl * sin(phi) - fd * cos(phi);
        ft_ *= sgn(wt.rot_speed);
        double f_[3] = {-fx_, ft_ * sin(theta), -ft_ * cos(theta)};
        frame_transform(f_, f, -angle, wt.type);
        torque = fabs(ft_) * r;
        thrust = fx_;
    }
    for (int m = 0; m < 3; m++) {
        A.pt_xyz[a * 3 + m] = xyz[m];
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
__global__ void __launch_bounds__(TILE_THREADS)
k_alm_project(StepParams P, AlmDev A, Tiling T, Vec3<double> F) {
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
            F.c[0][c] = fx;
            F.c[1][c] = fy;
            F.c[2][c] = fz;
        }
        __syncthreads();
    }
}

}  // namespace

void launch_alm_points(const LaunchCtx &L, const StepParams &P, const AlmDev &A, double t,
                       Vec3<const double> u) {
    if (A.ap_count <= 0) return;
    L.pre(KK_ALM_POINTS);
    k_alm_points<<<(A.ap_count + 63) / 64, 64, 0, L.s>>>(P, A, t, u);
    L.post(KK_ALM_POINTS);
    L.pre(KK_ALM_SUMS);
    k_alm_sums<<<1, 32 * ((A.wt_count + 31) / 32), 0, L.s>>>(A);
    L.post(KK_ALM_SUMS);
}

void launch_alm_project(const LaunchCtx &L, const StepParams &P, const AlmDev &A,
                        const Box &box, Vec3<double> f) {
    if (A.ap_count <= 0 || box.empty()) return;
    Tiling T = Tiling::make(box);
    long long blocks = T.ntiles < 4096 ? T.ntiles : 4096;
    size_t smem = sizeof(int) * (size_t)A.ap_count;
    L.pre(KK_ALM_PROJECT);
    k_alm_project<<<(int)blocks, TILE_THREADS, smem, L.s>>>(P, A, T, f);
    L.post(KK_ALM_PROJECT);
}

}  // namespace dalm
