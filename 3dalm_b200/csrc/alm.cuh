// Actuator-line model on the device (src/alm.h, src/euler_angle.h).
#pragma once

#include "flow.cuh"

namespace dalm {

enum EulerAngleType { EULER_ROLL = 0, EULER_PITCH = 1, EULER_YAW = 2, EULER_NONE = 3 };

// WindTurbine (src/alm.h:23-33) without the per-step angle, which the
// blade-point kernel evaluates from `formula` at time t.
struct TurbineDev {
    double base[3], rot_center[3], formula[4], rot_speed;
    int type;
    int pad;
};

struct AlmDev {
    int wt_count, ap_count, ap_per_wt, ap_per_blade, blades, atk_count;
    double pw2;        // projection_width^2
    double e_coef;     // 1/(projection_width*sqrt(pi))^3
    double cutoff2;    // support radius^2 of the truncated Gaussian
    const TurbineDev *wt;
    const double *r, *dr, *chord, *twist;   // per point; twist includes pitch
    const double *cd, *cl, *atk;            // [ap][atk], [ap][atk], [atk]
    double *pt_xyz, *pt_f, *pt_torque, *pt_thrust;  // outputs per point
    double *wt_torque, *wt_thrust;                  // outputs per turbine
};

// update_ap_position + calc_ap_force (src/alm.h:233-414) and the per-turbine
// sums (src/alm.h:384-398).
// T: storage type of the sampled velocity (double, or float for the mixed
// form's FP32 stencil fields)
template <typename T>
void launch_alm_points(const LaunchCtx &L, const StepParams &P, const AlmDev &A, double t,
                       Vec3<const T> u);
// distribute_ap_force (src/alm.h:416-448) confined to each point's support,
// over `box` (cells outside every support get 0).
// FT: storage type of the force field
template <typename FT>
void launch_alm_project(const LaunchCtx &L, const StepParams &P, const AlmDev &A,
                        const Box &box, Vec3<FT> f);

}  // namespace dalm
