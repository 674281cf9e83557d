// Launchers of the discrete-adjoint kernels (adjoint.cu).  The arithmetic
// of each kernel is in adjoint_cell.cuh.
#pragma once

#include "adjoint_cell.cuh"

namespace dalm {

// transposed apply_Ubc after the projection (two passes inside)
void launch_adj_velocity_bc(const LaunchCtx &L, const adj::AdjBcArgs &A);
// adjoint pressure right-hand side on the interior; writes sum(rhs^2) to *sumsq
void launch_adj_project(const LaunchCtx &L, const adj::AdjProjectArgs &A, Partials<1> part,
                        double *sumsq);
// v[0..n) *= s
void launch_adj_scale(const LaunchCtx &L, double *v, long long n, double s);
// transposed face interpolation + Poisson right-hand side, into A.aus
void launch_adj_faces(const LaunchCtx &L, const adj::AdjFacesArgs &A);
// transposed predictor: viscosity pass, then the stencil gather
void launch_adj_predict(const LaunchCtx &L, const adj::AdjNutArgs &N, const adj::AdjPredictArgs &A);
// actuator line at one time: gather over each point's support, the points'
// dual-number derivatives, and the ordered scatter onto aU and grad
void launch_adj_alm(const LaunchCtx &L, const StepParams &P, const AlmDev &A,
                    Vec3<const double> af, const adj::AdjAlmPointArgs &X, Vec3<double> aU,
                    double *grad);

}  // namespace dalm
