/*
 * Stage sequencing of the reference solver's time step, shared by the
 * single-rank oracle library (ref_harness.cpp) and the multi-rank CPU
 * baseline launcher (ref_mpirun.cpp).  TEST / BASELINE INFRASTRUCTURE ONLY.
 *
 * Include after "solver.h".  Stage numbering (shared with include/dalm.h,
 * enum dalm_stage, and oracle/dalm_oracle.c):
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
 * product applies them (only on the rank that owns the x- boundary, like the
 * reference's own inflow condition):
 *   - a per-(j,k) inflow profile (log-law inflow): after every apply_Ubc the
 *     x- ghost cells are overwritten with the profile, after every apply_JUbc
 *     the inflow face JU[gc-1][j][k][0] = (dy[j]*dz[k])*u_in(j,k);
 *   - per-turbine static yaw, collective pitch and rotor speed overrides
 *     (ref_harness.cpp, ref_set_turbine_params).
 */
#pragma once

#include <vector>

namespace refstages {

struct RefCase {
    Solver solver;
    bool has_profile = false;
    std::vector<Real> profile;      // [NY][NZ][3]
    std::vector<Real> base_twist;   // per actuator point
    std::vector<Real> base_omega;   // per turbine
};

inline Int cell_count(Solver &s) { return s.size[0] * s.size[1] * s.size[2]; }

inline void inflow_override_U(RefCase *c) {
    if (!c->has_profile) return;
    Solver &s = c->solver;
    if (s.mpi.rank != 0) return;  // the x- boundary belongs to rank 0 (src/bc.h:17)
    for (Int i = 0; i < s.gc; i++)
        for (Int j = s.gc; j < s.size[1] - s.gc; j++)
            for (Int k = s.gc; k < s.size[2] - s.gc; k++) {
                Int id = index(i, j, k, s.size);
                const Real *pr = &c->profile[(j * s.size[2] + k) * 3];
                s.cfd.U[id][0] = pr[0];
                s.cfd.U[id][1] = pr[1];
                s.cfd.U[id][2] = pr[2];
            }
}

inline void inflow_override_JU(RefCase *c) {
    if (!c->has_profile) return;
    Solver &s = c->solver;
    if (s.mpi.rank != 0) return;  // src/bc.h:244
    Int i = s.gc - 1;
    for (Int j = s.gc; j < s.size[1] - s.gc; j++)
        for (Int k = s.gc; k < s.size[2] - s.gc; k++) {
            Int id = index(i, j, k, s.size);
            Real yz = s.mesh.dy[j] * s.mesh.dz[k];
            s.cfd.JU[id][0] = yz * c->profile[(j * s.size[2] + k) * 3 + 0];
        }
}

inline void do_Ubc(RefCase *c) {
    Solver &s = c->solver;
    apply_Ubc(s.cfd.U, s.cfd.Uold, s.cfd.Uin, s.mesh.x, s.mesh.y, s.mesh.z,
              s.mesh.dx, s.mesh.dy, s.mesh.dz, s.rt.dt, s.size, s.gc, &s.mpi,
              s.cfd.retracted_floor, s.cfd.floor_start_x);
    inflow_override_U(c);
}

inline void do_JUbc(RefCase *c) {
    Solver &s = c->solver;
    apply_JUbc(s.cfd.JU, s.cfd.Uin, s.mesh.dy, s.mesh.dz, s.size, s.gc, &s.mpi);
    inflow_override_JU(c);
}

inline void do_alm(RefCase *c) {
    Solver &s = c->solver;
    run_alm(s.cfd.U, s.cfd.f, s.alm.projection_width, s.mesh.x, s.mesh.y, s.mesh.z,
            s.alm.wt_lst, s.alm.wt_count, s.alm.ap_lst, s.alm.ap_count,
            s.alm.blade_per_wt, s.alm.ap_per_blade, s.alm.cd_tbl, s.alm.cl_tbl,
            s.alm.atk_lst, s.alm.atk_count, s.rt.get_time(), s.size, s.gc, &s.mpi);
}

inline void do_diag(RefCase *c) {
    Solver &s = c->solver;
    Int n = (s.gsize[0] - 2 * s.gc) * (s.gsize[1] - 2 * s.gc) * (s.gsize[2] - 2 * s.gc);
    s.cfd.avg_div = calc_l2_norm(s.cfd.div, s.size, s.gc, &s.mpi) / sqrt(n);
    s.cfd.max_cfl = calc_max_cfl(s.cfd.U, s.mesh.dx, s.mesh.dy, s.mesh.dz, s.rt.dt,
                                 s.size, s.gc, &s.mpi);
}

inline void do_stage(RefCase *c, int stage) {
    Solver &s = c->solver;
    Int len = cell_count(s);
    switch (stage) {
    case 0:
        cpy_array(s.cfd.Uold, s.cfd.U, len);
        calc_intermediate_U(s.cfd.U, s.cfd.Uold, s.cfd.JU, s.cfd.nut, s.cfd.f,
                            s.mesh.x, s.mesh.y, s.mesh.z, s.mesh.dx, s.mesh.dy, s.mesh.dz,
                            s.cfd.Re, s.rt.dt, s.size, s.gc, &s.mpi);
        break;
    case 1:
        interpolate_JU(s.cfd.U, s.cfd.JU, s.mesh.dx, s.mesh.dy, s.mesh.dz, s.size, s.gc, &s.mpi);
        do_JUbc(c);
        calc_poisson_rhs(s.cfd.JU, s.eq.b, s.mesh.dx, s.mesh.dy, s.mesh.dz, s.rt.dt,
                         s.eq.max_diag, s.size, s.gc, &s.mpi);
        break;
    case 2:
        if (s.eq.method == "BiCG") {
            if (s.eq.pc_method == "SOR") {
                run_pbicgstab(s.eq.A, s.cfd.p, s.eq.b, s.eq.r, s.eq.r0, s.eq.p, s.eq.pp, s.eq.q,
                              s.eq.s, s.eq.ss, s.eq.t, s.eq.it, s.eq.max_it, s.eq.err, s.eq.tol,
                              s.eq.pc_relax_rate, s.eq.pc_max_it, s.gsize, s.size, s.offset,
                              s.gc, &s.mpi);
            } else if (s.eq.pc_method == "Jacobi") {
                run_pbicgstab(s.eq.A, s.cfd.p, s.eq.b, s.eq.r, s.eq.r0, s.eq.p, s.eq.pp, s.eq.q,
                              s.eq.s, s.eq.ss, s.eq.t, s.eq.tmp, s.eq.it, s.eq.max_it, s.eq.err,
                              s.eq.tol, s.eq.pc_max_it, s.gsize, s.size, s.gc, &s.mpi);
            }
        } else if (s.eq.method == "SOR") {
            run_sor(s.eq.A, s.cfd.p, s.eq.b, s.eq.r, s.eq.relax_rate, s.eq.it, s.eq.max_it,
                    s.eq.err, s.eq.tol, s.gsize, s.size, s.offset, s.gc, &s.mpi);
        }
        break;
    case 3:
        apply_pbc(s.cfd.Uold, s.cfd.p, s.cfd.nut, s.mesh.z, s.mesh.dx, s.mesh.dy, s.mesh.dz,
                  s.cfd.Re, s.size, s.gc, &s.mpi);
        project_p(s.cfd.U, s.cfd.JU, s.cfd.p, s.mesh.x, s.mesh.y, s.mesh.z, s.mesh.dx,
                  s.mesh.dy, s.mesh.dz, s.rt.dt, s.size, s.gc, &s.mpi);
        set_solid_U(s.cfd.U, s.cfd.solid, s.size, s.gc);
        do_Ubc(c);
        do_JUbc(c);
        calc_nut(s.cfd.U, s.cfd.nut, s.mesh.x, s.mesh.y, s.mesh.z, s.mesh.dx, s.mesh.dy,
                 s.mesh.dz, s.cfd.Cs, s.size, s.gc, &s.mpi);
        calc_divergence(s.cfd.JU, s.cfd.div, s.mesh.dx, s.mesh.dy, s.mesh.dz, s.size, s.gc, &s.mpi);
        break;
    case 4:
        do_alm(c);
        break;
    case 5:
        do_diag(c);
        break;
    case 6: {
        const Real curr_time = s.rt.get_time();
        if (curr_time >= s.rt.tavg_start_time) {
            s.rt.tavg_step_count++;
            Real weight = 1. / s.rt.tavg_step_count;
            calc_ax_plus_by(1. - weight, s.cfd.Utavg, weight, s.cfd.U, s.cfd.Utavg, len);
        }
        break;
    }
    default:
        break;
    }
}

/* src/solver.h:1034-1306 without field output and probes (out of scope). */
inline void do_step(RefCase *c) {
    Solver &s = c->solver;
    if (s.rt.step != 0) {
        for (int st = 0; st <= 5; st++) do_stage(c, st);
    }
    do_stage(c, 6);
    s.rt.step++;
}

/* After U (and p, JU) have been written: the state derivation of
 * src/solver.h:767-833.  flags bit0: apply the velocity BCs to U (with
 * Uold := U); bit1: recompute JU from U (interpolate_JU + apply_JUbc).  nut,
 * div, the ALM force at t = step*dt and the diagnostics are always
 * recomputed. */
inline void derive_state(RefCase *c, int flags) {
    Solver &s = c->solver;
    Int len = cell_count(s);
    if (flags & 1) {
        cpy_array(s.cfd.Uold, s.cfd.U, len);
        do_Ubc(c);
    }
    if (flags & 2) {
        interpolate_JU(s.cfd.U, s.cfd.JU, s.mesh.dx, s.mesh.dy, s.mesh.dz, s.size, s.gc, &s.mpi);
        do_JUbc(c);
    }
    calc_nut(s.cfd.U, s.cfd.nut, s.mesh.x, s.mesh.y, s.mesh.z, s.mesh.dx, s.mesh.dy, s.mesh.dz,
             s.cfd.Cs, s.size, s.gc, &s.mpi);
    calc_divergence(s.cfd.JU, s.cfd.div, s.mesh.dx, s.mesh.dy, s.mesh.dz, s.size, s.gc, &s.mpi);
    do_alm(c);
    do_diag(c);
}

}  // namespace refstages
