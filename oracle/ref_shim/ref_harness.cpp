/*
 * ORACLE HARNESS (test infrastructure only — never shipped, never timed as the
 * product).  Compiles the reference solver's own headers (src/solver.h and
 * everything it includes) into a shared library with a flat C interface so
 * pytest can drive the reference FP64 path through ctypes and compare it with
 * both the C restatement in oracle/dalm_oracle.c and the CUDA product.
 *
 * Built by oracle/Makefile into oracle/_ref/libref3dalm.so from the sources
 * where they lie (read-only); nothing from the reference is copied here.
 *
 * Stage numbering is shared with include/dalm.h (enum dalm_stage) and
 * oracle/dalm_oracle.c:
 *   0 PREDICT  : cpy_array(Uold,U) + calc_intermediate_U      (src/solver.h:1042-1053)
 *   1 FLUX_RHS : interpolate_JU + apply_JUbc + calc_poisson_rhs (src/solver.h:1055-1077)
 *   2 POISSON  : SOR / BiCGStab dispatch                      (src/solver.h:1081-1106)
 *   3 PROJECT  : apply_pbc, project_p, set_solid_U, apply_Ubc, apply_JUbc,
 *                calc_nut, calc_divergence                    (src/solver.h:1112-1171)
 *   4 ALM      : run_alm(t = step*dt)                         (src/solver.h:1173-1180)
 *   5 DIAG     : avg_div, max_cfl                             (src/solver.h:1184-1186)
 *   6 TAVG     : running time average of U                    (src/solver.h:1194-1204)
 *
 * Two extensions that the reference lacks are applied here exactly as the
 * product applies them:
 *   - a per-(j,k) inflow profile (log-law inflow): after every apply_Ubc the
 *     x- ghost cells are overwritten with the profile, after every apply_JUbc
 *     the inflow face JU[gc-1][j][k][0] = (dy[j]*dz[k])*u_in(j,k);
 *   - per-turbine static yaw, collective pitch and rotor speed overrides:
 *     yaw sets angle_type = Yaw with formula {0,0,0,yaw}; pitch is added to the
 *     blade-point twist (alpha = deg(phi) - (twist + pitch)); omega replaces
 *     `rotation speed`.
 */
#include "solver.h"
#include "ref_stages.hpp"

#include <cstring>
#include <vector>

namespace {

using namespace refstages;

Real *field_ptr(Solver &s, int which, int *ncomp) {
    *ncomp = 1;
    switch (which) {
    case 0: *ncomp = 3; return s.cfd.U[0];
    case 1: *ncomp = 3; return s.cfd.Uold[0];
    case 2: *ncomp = 3; return s.cfd.JU[0];
    case 3: return s.cfd.p;
    case 4: return s.cfd.nut;
    case 5: return s.cfd.div;
    case 6: *ncomp = 3; return s.cfd.f[0];
    case 7: return s.eq.b;
    case 8: *ncomp = 3; return s.cfd.Utavg[0];
    default: return nullptr;
    }
}

}  // namespace

extern "C" {

void *ref_create(const char *case_dir) {
    RefCase *c = new RefCase();
    std::string prog = "solver";
    std::string dir = case_dir;
    char *argv[] = {&prog[0], &dir[0], nullptr};
    c->solver.initialize(2, argv);
    Solver &s = c->solver;
    for (Int i = 0; i < s.alm.ap_count; i++) c->base_twist.push_back(s.alm.ap_lst[i].twist);
    for (Int i = 0; i < s.alm.wt_count; i++) c->base_omega.push_back(s.alm.wt_lst[i].rot_speed);
    fflush(stdout);
    return c;
}

void ref_destroy(void *h) {
    RefCase *c = (RefCase *)h;
    c->solver.finalize();
    delete c;
}

void ref_size(void *h, int64_t out[4]) {
    Solver &s = ((RefCase *)h)->solver;
    out[0] = s.size[0]; out[1] = s.size[1]; out[2] = s.size[2]; out[3] = s.gc;
}

void ref_alm_counts(void *h, int64_t out[5]) {
    Solver &s = ((RefCase *)h)->solver;
    out[0] = s.alm.ap_count; out[1] = s.alm.wt_count; out[2] = s.alm.atk_count;
    out[3] = s.alm.ap_count > 0 ? s.alm.blade_per_wt : 0;
    out[4] = s.alm.ap_count > 0 ? s.alm.ap_per_blade : 0;
}

void ref_mesh(void *h, double *x, double *y, double *z, double *dx, double *dy, double *dz) {
    Solver &s = ((RefCase *)h)->solver;
    memcpy(x, s.mesh.x, s.size[0] * sizeof(double));
    memcpy(y, s.mesh.y, s.size[1] * sizeof(double));
    memcpy(z, s.mesh.z, s.size[2] * sizeof(double));
    memcpy(dx, s.mesh.dx, s.size[0] * sizeof(double));
    memcpy(dy, s.mesh.dy, s.size[1] * sizeof(double));
    memcpy(dz, s.mesh.dz, s.size[2] * sizeof(double));
}

double ref_max_diag(void *h) { return ((RefCase *)h)->solver.eq.max_diag; }

/* Coefficient matrix A[len][7] as assembled by build_A (src/eq.h:701-798). */
void ref_matrix(void *h, double *A) {
    Solver &s = ((RefCase *)h)->solver;
    memcpy(A, s.eq.A[0], cell_count(s) * 7 * sizeof(double));
}

void ref_set_inflow_profile(void *h, const double *prof) {
    RefCase *c = (RefCase *)h;
    Solver &s = c->solver;
    if (!prof) { c->has_profile = false; return; }
    c->profile.assign(prof, prof + s.size[1] * s.size[2] * 3);
    c->has_profile = true;
}

void ref_set_turbine_params(void *h, const double *yaw_deg, const double *pitch_deg,
                            const double *omega) {
    RefCase *c = (RefCase *)h;
    Solver &s = c->solver;
    Int ap_per_wt = s.alm.ap_count > 0 ? s.alm.ap_count / s.alm.wt_count : 0;
    for (Int w = 0; w < s.alm.wt_count; w++) {
        WindTurbine &wt = s.alm.wt_lst[w];
        if (yaw_deg) {
            wt.angle_type = EulerAngle::Yaw;
            wt.formula[0] = 0; wt.formula[1] = 0; wt.formula[2] = 0;
            wt.formula[3] = deg_to_rad(yaw_deg[w]);
        }
        if (omega) wt.rot_speed = omega[w];
        if (pitch_deg) {
            for (Int a = w * ap_per_wt; a < (w + 1) * ap_per_wt; a++)
                s.alm.ap_lst[a].twist = c->base_twist[a] + pitch_deg[w];
        }
    }
}

void ref_get_field(void *h, int which, double *out) {
    Solver &s = ((RefCase *)h)->solver;
    int nc;
    Real *p = field_ptr(s, which, &nc);
    if (p) memcpy(out, p, cell_count(s) * nc * sizeof(double));
}

void ref_set_field(void *h, int which, const double *in) {
    Solver &s = ((RefCase *)h)->solver;
    int nc;
    Real *p = field_ptr(s, which, &nc);
    if (p) memcpy(p, in, cell_count(s) * nc * sizeof(double));
}

/* flags bit0: apply the velocity BCs to U (with Uold := U);
 * flags bit1: recompute JU from U (interpolate_JU + apply_JUbc), else take JU.
 * Derived fields (nut, div, ALM force at t = step*dt, diagnostics) are always
 * recomputed, mirroring src/solver.h:767-833. */
void ref_set_state(void *h, const double *U, const double *JU, const double *p, int flags) {
    RefCase *c = (RefCase *)h;
    Solver &s = c->solver;
    Int len = cell_count(s);
    memcpy(s.cfd.U[0], U, len * 3 * sizeof(double));
    if (p) memcpy(s.cfd.p, p, len * sizeof(double));
    if (JU && !(flags & 2)) memcpy(s.cfd.JU[0], JU, len * 3 * sizeof(double));
    derive_state(c, flags | (JU ? 0 : 2));
}

void ref_step(void *h, int n) {
    for (int i = 0; i < n; i++) do_step((RefCase *)h);
}

void ref_stage(void *h, int stage) { do_stage((RefCase *)h, stage); }

void ref_advance_clock(void *h) { ((RefCase *)h)->solver.rt.step++; }

void ref_stats(void *h, int64_t *ints, double *reals) {
    Solver &s = ((RefCase *)h)->solver;
    ints[0] = s.rt.step;
    ints[1] = s.eq.it;
    ints[2] = s.rt.max_step;
    ints[3] = s.rt.tavg_step_count;
    reals[0] = s.eq.err;
    reals[1] = s.cfd.avg_div;
    reals[2] = s.cfd.max_cfl;
    reals[3] = s.rt.dt;
}

void ref_set_poisson(void *h, int64_t max_it, double tol) {
    Solver &s = ((RefCase *)h)->solver;
    s.eq.max_it = max_it;
    s.eq.tol = tol;
}

void ref_turbines(void *h, double *torque, double *thrust) {
    Solver &s = ((RefCase *)h)->solver;
    for (Int w = 0; w < s.alm.wt_count; w++) {
        torque[w] = s.alm.wt_lst[w].torque;
        thrust[w] = s.alm.wt_lst[w].thrust;
    }
}

void ref_points(void *h, double *xyz, double *f, double *torque, double *thrust) {
    Solver &s = ((RefCase *)h)->solver;
    for (Int a = 0; a < s.alm.ap_count; a++) {
        ActuatorPoint &ap = s.alm.ap_lst[a];
        for (int m = 0; m < 3; m++) {
            xyz[a * 3 + m] = ap.xyz[m];
            f[a * 3 + m] = ap.f[m];
        }
        torque[a] = ap.torque;
        thrust[a] = ap.thrust;
    }
}

/* Blade-point tables after build_ap_props (src/alm.h:35-142). */
void ref_point_tables(void *h, double *r, double *dr, double *chord, double *twist,
                      double *cd, double *cl, double *atk) {
    Solver &s = ((RefCase *)h)->solver;
    for (Int a = 0; a < s.alm.ap_count; a++) {
        r[a] = s.alm.ap_lst[a].r;
        dr[a] = s.alm.ap_lst[a].dr;
        chord[a] = s.alm.ap_lst[a].chord;
        twist[a] = s.alm.ap_lst[a].twist;
        for (Int j = 0; j < s.alm.atk_count; j++) {
            cd[a * s.alm.atk_count + j] = s.alm.cd_tbl[a][j];
            cl[a * s.alm.atk_count + j] = s.alm.cl_tbl[a][j];
        }
    }
    for (Int j = 0; j < s.alm.atk_count; j++) atk[j] = s.alm.atk_lst[j];
}

}  // extern "C"
