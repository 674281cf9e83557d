// The blade-point model of the actuator line in FP64: position, trilinear
// velocity sampling and force of one point (update_ap_position and
// calc_ap_force, reference src/alm.h:233-370, with find_floor_index,
// trilinear_interpolate and lookup_cdcl_table, src/util.h:119-199 and
// src/alm.h:208-231, and frame_transform / frame_transform_U,
// src/euler_angle.h:34-127).
//
// Everything is __host__ __device__ and written in the reference's
// operation order.  The device kernel (k_alm_points) and the host path of
// the reference-order mode run these same functions; the only difference
// between the two is the math library behind sin, cos and atan (the
// device's, or the host's libm, which is what the reference calls).
#pragma once

#include <cmath>

#include "alm.cuh"

#define DALM_PT_HD __host__ __device__ __forceinline__

namespace dalm {
namespace almpt {

constexpr double PI_D = 3.14159265358979323846;  // M_PI (src/type.h:12)

DALM_PT_HD double sgn(double v) { return (double)((v > 0.) - (v < 0.)); }

// find_floor_index (src/util.h:119-146)
DALM_PT_HD int floor_index(const double *a, double v, int n) {
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
DALM_PT_HD void frame_transform(const double in[3], double out[3], double angle, int type) {
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
DALM_PT_HD void frame_transform_U(const double p[3], const double U[3], double out[3],
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

DALM_PT_HD double lin_interp(double v0, double v1, double x0, double x1, double xp) {
    double fx = (xp - x0) / (x1 - x0);  // src/util.h:166-174
    return v0 * (1 - fx) + v1 * fx;
}

// A point's pose at time t: the turbine's angle and angular rate
// (src/alm.h:236-244), the blade azimuth and the position
// (src/alm.h:250-266).
struct Pose {
    double angle, ow, theta, r, xyz[3];
};

DALM_PT_HD void point_pose(const TurbineDev &wt, double r, int bid, int blades, double t, Pose &q) {
    q.angle = wt.formula[0] * sin(wt.formula[1] * t + wt.formula[2]) + wt.formula[3];
    q.ow = wt.formula[0] * wt.formula[1] * cos(wt.formula[1] * t + wt.formula[2]);
    q.r = r;
    q.theta = bid * (2 * PI_D / blades) + t * wt.rot_speed;
    double loc[3] = {wt.rot_center[0], wt.rot_center[1] + r * cos(q.theta),
                     wt.rot_center[2] + r * sin(q.theta)};
    frame_transform(loc, q.xyz, -q.angle, wt.type);
    for (int m = 0; m < 3; m++) q.xyz[m] += wt.base[m];
}

// The cell (i, j, k) whose upper corner neighbours enclose the point
// (src/alm.h:291-299), its 8 stored indices in the order of
// trilinear_interpolate and the fractions; false when the point lies outside
// the interior (its force is zero).
DALM_PT_HD bool point_cell(const Grid &g, const double *x, const double *y, const double *z,
                           const double xyz[3], long long id[8], double frac[3]) {
    int i = floor_index(x, xyz[0], g.nx);
    int j = floor_index(y, xyz[1], g.ny);
    int k = floor_index(z, xyz[2], g.nz);
    if (!(i >= g.gc && i < g.nx - g.gc && j >= g.gc && j < g.ny - g.gc && k >= g.gc &&
          k < g.nz - g.gc))
        return false;
    id[0] = g.at(i, j, k);
    id[1] = g.at(i + 1, j, k);
    id[2] = g.at(i, j + 1, k);
    id[3] = g.at(i + 1, j + 1, k);
    id[4] = g.at(i, j, k + 1);
    id[5] = g.at(i + 1, j, k + 1);
    id[6] = g.at(i, j + 1, k + 1);
    id[7] = g.at(i + 1, j + 1, k + 1);
    double x0 = x[i], x1 = x[i + 1], y0 = y[j], y1 = y[j + 1], z0 = z[k], z1 = z[k + 1];
    frac[0] = (xyz[0] - x0) / (x1 - x0);
    frac[1] = (xyz[1] - y0) / (y1 - y0);
    frac[2] = (xyz[2] - z0) / (z1 - z0);
    return true;
}

// trilinear_interpolate (src/util.h:176-199) of the 8 corner values
DALM_PT_HD double trilinear(const double v[8], const double frac[3]) {
    double fx = frac[0], fy = frac[1], fz = frac[2];
    double v01 = v[0] * (1 - fx) + v[1] * fx;
    double v23 = v[2] * (1 - fx) + v[3] * fx;
    double v45 = v[4] * (1 - fx) + v[5] * fx;
    double v67 = v[6] * (1 - fx) + v[7] * fx;
    double v0123 = v01 * (1 - fy) + v23 * fy;
    double v4567 = v45 * (1 - fy) + v67 * fy;
    return v0123 * (1 - fz) + v4567 * fz;
}

// Blade-element force, torque and thrust of a point from its sampled
// velocity (src/alm.h:335-363).  cdt / clt are the point's polar tables.
DALM_PT_HD void point_force(const TurbineDev &wt, const Pose &q, const double Uap[3],
                            double twist, double chord, double dr, const double *atk_lst,
                            int atk_count, const double *cdt, const double *clt, double f[3],
                            double &torque, double &thrust) {
    double rel[3] = {q.xyz[0] - wt.base[0], q.xyz[1] - wt.base[1], q.xyz[2] - wt.base[2]};
    double Ur[3];
    frame_transform_U(rel, Uap, Ur, q.angle, q.ow, wt.type);
    double ux_ = Ur[0];
    double ut_ = q.r * wt.rot_speed + Ur[1] * sin(q.theta) - Ur[2] * cos(q.theta);
    double urel2 = ux_ * ux_ + ut_ * ut_;
    double phi = atan(ux_ / ut_);
    double atk = phi * 180 / PI_D - twist;
    // lookup_cdcl_table (src/alm.h:208-231)
    int ti = floor_index(atk_lst, atk, atk_count);
    double cd, cl;
    if (ti < 0) {
        cd = cdt[0];
        cl = clt[0];
    } else if (ti >= atk_count - 1) {
        cd = cdt[atk_count - 1];
        cl = clt[atk_count - 1];
    } else {
        cd = lin_interp(cdt[ti], cdt[ti + 1], atk_lst[ti], atk_lst[ti + 1], atk);
        cl = lin_interp(clt[ti], clt[ti + 1], atk_lst[ti], atk_lst[ti + 1], atk);
    }
    double fd = 0.5 * cd * urel2 * chord * dr;
    double fl = 0.5 * cl * urel2 * chord * dr;
    double fx_ = fl * cos(phi) + fd * sin(phi);
    double ft_ = fl * sin(phi) - fd * cos(phi);
    ft_ *= sgn(wt.rot_speed);
    double f_[3] = {-fx_, ft_ * sin(q.theta), -ft_ * cos(q.theta)};
    frame_transform(f_, f, -q.angle, wt.type);
    torque = fabs(ft_) * q.r;
    thrust = fx_;
}

}  // namespace almpt
}  // namespace dalm
