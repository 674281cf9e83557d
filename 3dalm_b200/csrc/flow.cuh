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
    double max_diag;
};

struct StepParams {
    Grid g;
    MeshDev m;
    double re, cs, dt, max_diag;
    double uin[3];
    const double *prof;  // inflow profile [ny][nz][3] on the device, or null
    Box fbox;            // cells where the ALM force may be non-zero
};

struct DiagState {
    double div2, max_cfl, avg_div;  // sum div^2, max cfl, ||div||/sqrt(N)
    double ncell;
};

// ---- flow kernels (flow_fp64.cu) ----
void launch_predict(const LaunchCtx &L, const StepParams &P, Vec3<const double> uold,
                    Vec3<double> unew, Vec3<const double> ju, Vec3<const double> f);
void launch_flux_rhs(const LaunchCtx &L, const StepParams &P, Vec3<const double> u,
                     Vec3<double> ju, double *b);
void launch_flux_only(const LaunchCtx &L, const StepParams &P, Vec3<const double> u,
                      Vec3<double> ju);
void launch_pressure_bc(const LaunchCtx &L, const StepParams &P, double *p);
void launch_project(const LaunchCtx &L, const StepParams &P, Vec3<double> u,
                    Vec3<double> ju_in, Vec3<double> ju_out, const double *p, Partials<2> part,
                    DiagState *diag);
void launch_velocity_bc(const LaunchCtx &L, const StepParams &P, Vec3<double> u,
                        Vec3<const double> uold);
void launch_diag(const LaunchCtx &L, const StepParams &P, Vec3<const double> u,
                 Vec3<const double> ju, Partials<2> part, DiagState *diag);
void launch_nut_field(const LaunchCtx &L, const StepParams &P, Vec3<const double> u, double *nut);
void launch_div_field(const LaunchCtx &L, const StepParams &P, Vec3<const double> ju, double *div);
void launch_tavg(const LaunchCtx &L, const Grid &g, Vec3<double> tavg, Vec3<const double> u,
                 double w);
// reference AoS/scalar layout <-> device SoA layout (ncomp = 1 or 3)
void launch_to_device_layout(const LaunchCtx &L, const Grid &g, const double *ref, int ncomp,
                             double *const *dst);
void launch_to_ref_layout(const LaunchCtx &L, const Grid &g, double *const *src, int ncomp,
                          double *ref);
void launch_fill(const LaunchCtx &L, double *p, long long n, double v);

}  // namespace dalm
