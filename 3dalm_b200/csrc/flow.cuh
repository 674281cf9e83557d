// Declarations shared by the host orchestrator and the CUDA translation units.
#pragma once

#include "common.cuh"

namespace dalm {

template <typename T>
struct Vec3 {
    T *c[3];
};

struct MeshDev {
    const double *x, *y, *z, *dx, *dy, *dz;  // stored-length 1-D arrays
};

// Matrix-free Poisson coefficients.  build_A (src/eq.h:701-798) makes A a
// function of 1-D mesh arrays only, so the seven coefficients of a cell are
// rebuilt from per-axis arrays:
//   ex[i] : 1/(dx (x_{i+1}-x_i)), or 2/(dx dx) at the x+ outlet   (unscaled)
//   ae[i], aw[i], an[j], as[j], at[k], ab[k]: unscaled, 0 at walls
//   ae_s .. ab_s : the same divided by max_diag (A[id][1..6] of the reference)
// and a_c = (((((0 - ex) - aw) - an) - as) - at) - ab) / max_diag, the exact
// operation sequence of the reference so a_c matches bit for bit.
struct PoissonCoef {
    const double *ex, *aw_u, *an_u, *as_u, *at_u, *ab_u;
    const double *ae, *aw, *an, *as, *at, *ab;
    const double *xpart;  // (0 - ex[i]) - aw_u[i]: the first two steps of a_c
    double max_diag;
    double inv_max_diag;  // 1 / max_diag (fast variant)
};

struct StepParams {
    Grid g;
    MeshDev m;
    double re, cs, dt, max_diag;
    double uin[3];
    const double *prof;  // inflow profile [ny][nz][3] on the device, or null
    Box fbox;            // cells where the ALM force may be non-zero
    // (Cs * cbrt(dx dy dz))^2 per interior cell, computed once on the host
    // with the same libm cbrt the reference calls (src/cfd.h:804, 823-824)
    const double *filter2;
    // 1: global sums in the reference's serial (i,j,k) order
    // (warp_serial_sums) instead of the parallel tree
    int reference_sums;
    int limiter;  // 0: the reference's b=4 limiter, 1: van Albada
    // turbulence-generating grid: solid volume fraction per cell (null: none);
    // set_solid_U scales the projected velocity by 1 - solid
    const double *solid;
    // retracted floor: the z- wall is slip for cell centres x < floor_start
    int retracted;
    double floor_start;
};

struct DiagState {
    double div2, max_cfl, avg_div;  // sum div^2, max cfl, ||div||/sqrt(N)
    double ncell;
};

// Sums in the reference's serial order.  The reference accumulates every
// global sum with one loop over interior cells, i outer, k inner
// (src/mv.h:8-55, src/cfd.h:1109-1141); a parallel tree sum rounds
// differently, and BiCGStab's iteration count and iterates are sensitive to
// that rounding.  This helper reproduces the serial order exactly and is run
// by a single warp: the warp loads 32 consecutive k values at a time, then
// folds them into the running sum one term at a time in lane order.  Every
// lane ends with the same total.
template <int N, typename Term>
__device__ inline void warp_serial_sums(const Grid &g, Term term, double (&total)[N]) {
    int lane = threadIdx.x & 31;
#pragma unroll
    for (int m = 0; m < N; m++) total[m] = 0;
    int kend = g.nz - g.gc;
    for (int i = g.gc; i < g.nx - g.gc; i++)
        for (int j = g.gc; j < g.ny - g.gc; j++)
            for (int k0 = g.gc; k0 < kend; k0 += 32) {
                int k = k0 + lane;
                double t[N];
                if (k < kend) {
                    term(g.at(i, j, k), t);
                } else {
#pragma unroll
                    for (int m = 0; m < N; m++) t[m] = 0;
                }
                int n = kend - k0 < 32 ? kend - k0 : 32;
                for (int l = 0; l < n; l++)
#pragma unroll
                    for (int m = 0; m < N; m++) total[m] = total[m] + __shfl_sync(0xffffffffu, t[m], l);
            }
}

// ---- flow kernels (flow_fp64.cu) ----
void launch_predict(const LaunchCtx &L, const StepParams &P, Vec3<const double> uold,
                    Vec3<double> unew, Vec3<const double> ju, Vec3<const double> f);
// The mixed-precision form's flow stages on FP32 stencil fields
// (flow_mixed.cu).  Mesh tables per axis, for stored index n:
//   ax    FP32 {1/d_n, 1/(x_{n+1} - x_n), 1/(x_n - x_{n-1}), 1/(x_{n+1} - x_{n-1})}
//   wd    FP32 {d_n, cbrt(d_n)^2}  (face areas; the Smagorinsky filter width
//         (Cs cbrt(dx dy dz))^2 = cs2 * wd_x.y * wd_y.y * wd_z.y)
//   inv64 FP64 {1/(x_{n+1} - x_n), 1/(x_{n+1} - x_{n-1})}  (the projection)
struct MixedGeom {
    const float4 *ax[3];
    const float2 *wd[3];
    const double2 *inv64[3];
    float cs2;
};
void launch_predict32(const LaunchCtx &L, const StepParams &P, const MixedGeom &geo,
                      Vec3<const float> uold, Vec3<float> unew, Vec3<const float> ju,
                      Vec3<const float> f);
// face fluxes and, with b non-null, the FP64 Poisson right-hand side
void launch_flux32(const LaunchCtx &L, const StepParams &P, const MixedGeom &geo,
                   Vec3<const float> u, Vec3<float> ju, double *b);
void launch_project32(const LaunchCtx &L, const StepParams &P, const MixedGeom &geo, Vec3<float> u,
                      Vec3<const float> ju_in, Vec3<float> ju_out, const double *p,
                      Partials<2> part, DiagState *diag);
void launch_flux_rhs(const LaunchCtx &L, const StepParams &P, Vec3<const double> u,
                     Vec3<double> ju, double *b);
void launch_flux_only(const LaunchCtx &L, const StepParams &P, Vec3<const double> u,
                      Vec3<double> ju);
void launch_pressure_bc(const LaunchCtx &L, const StepParams &P, double *p);
void launch_project(const LaunchCtx &L, const StepParams &P, Vec3<double> u,
                    Vec3<double> ju_in, Vec3<double> ju_out, const double *p, Partials<2> part,
                    DiagState *diag);
// apply_Ubc on FP64 (T = double) or FP32 (T = float, the mixed form's
// stencil fields) storage; FP64 arithmetic either way
template <typename T>
void launch_velocity_bc(const LaunchCtx &L, const StepParams &P, Vec3<T> u, Vec3<const T> uold);
void launch_diag(const LaunchCtx &L, const StepParams &P, Vec3<const double> u,
                 Vec3<const double> ju, Partials<2> part, DiagState *diag);
void launch_diag(const LaunchCtx &L, const StepParams &P, Vec3<const float> u,
                 Vec3<const float> ju, Partials<2> part, DiagState *diag);
void launch_nut_field(const LaunchCtx &L, const StepParams &P, Vec3<const double> u, double *nut);
void launch_div_field(const LaunchCtx &L, const StepParams &P, Vec3<const double> ju, double *div);
// Q-criterion of U on the interior (calc_q, src/cfd.h:949-1034)
void launch_q_field(const LaunchCtx &L, const StepParams &P, Vec3<const double> u, double *q);
template <typename T>
void launch_tavg(const LaunchCtx &L, const Grid &g, Vec3<double> tavg, Vec3<const T> u, double w);
// reference AoS/scalar layout <-> device SoA layout (ncomp = 1 or 3)
void launch_to_device_layout(const LaunchCtx &L, const Grid &g, const double *ref, int ncomp,
                             double *const *dst);
void launch_to_ref_layout(const LaunchCtx &L, const Grid &g, double *const *src, int ncomp,
                          double *ref);
void launch_fill(const LaunchCtx &L, double *p, long long n, double v);
// out[3 t + m] = U_m at device index idx[t] (probe sampling)
template <typename T>
void launch_gather_points(const LaunchCtx &L, Vec3<const T> u, const long long *idx, int n,
                          double *out);
// dst[x] = src[x] over n elements (FP32 <-> FP64 copies of a field)
void launch_widen(const LaunchCtx &L, const float *src, double *dst, long long n);
void launch_narrow(const LaunchCtx &L, const double *src, float *dst, long long n);

}  // namespace dalm
