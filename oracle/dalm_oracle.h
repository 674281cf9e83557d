/*
 * ORACLE — CPU restatement of the 3dalm per-time-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load this library, and only as the checker
 * (or as the timed CPU baseline); the product never links or calls it.
 *
 * Plain C, FP64, serial, reference field layout:
 *   linear index  (i*NY + j)*NZ + k, k contiguous          (src/util.h:11-13)
 *   vector fields AoS [len][3]                             (src/solver.h:287-290)
 * Every function cites the reference file:line it restates.  The arithmetic
 * follows the reference's operation order so that, built with
 * -ffp-contract=off, it agrees bit for bit with the reference compiled the
 * same way (oracle/_ref), which the CPU tests check.
 */
#ifndef DALM_ORACLE_H
#define DALM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_EULER_ROLL = 0, OR_EULER_PITCH = 1, OR_EULER_YAW = 2, OR_EULER_NONE = 3 };
enum { OR_SOLVER_SOR = 0, OR_SOLVER_BICG = 1, OR_SOLVER_JACOBI = 2 };
enum { OR_PC_JACOBI = 0, OR_PC_SOR = 1 };

/* Everything the reference reads from setup.json / mesh.json /
 * windturbine.json, already parsed (JSON parsing is done by oracle.py). */
typedef struct {
    int64_t size[3];          /* stored sizes incl. guide cells */
    int64_t gc;
    const double *x, *y, *z;  /* cell centres incl. guide cells (mesh.json) */
    double uin[3];
    double re, cs, dt;
    int64_t max_step;
    double tavg_start_time;
    int solver;               /* OR_SOLVER_* */
    int pc;                   /* OR_PC_*      */
    int64_t max_it, pc_max_it;
    double tol, relax, pc_relax;
    /* actuator line (turbine_count == 0: no turbines) */
    int64_t turbine_count, blades, points_per_blade;
    double projection_width, rotor_r, hub_r, tower, overhang;
    const double *base;       /* [T][3] */
    const int *angle_type;    /* [T] */
    const double *formula;    /* [T][4] */
    const double *rot_speed;  /* [T] */
    int64_t station_count, atk_count;
    const double *station_r, *station_chord, *station_twist; /* [S] */
    const double *station_cd, *station_cl;                   /* [S][atk] */
    const double *atk;                                       /* [atk] */
    /* turbulence-generating grid (has_grid != 0): bar width, mesh spacing,
     * thickness, placement (src/solver.h:599-611) */
    int has_grid;
    double grid_bar, grid_mesh, grid_thick, grid_at[3];
    /* retracted floor: slip z- wall for x < floor_start (src/solver.h:618-625) */
    int retracted_floor;
    double floor_start;
} oracle_params;

typedef struct dalm_oracle dalm_oracle;

dalm_oracle *oracle_create(const oracle_params *prm);
void oracle_destroy(dalm_oracle *o);

void oracle_size(const dalm_oracle *o, int64_t out[4]);
void oracle_mesh(const dalm_oracle *o, double *x, double *y, double *z,
                 double *dx, double *dy, double *dz);
double oracle_max_diag(const dalm_oracle *o);
void oracle_matrix(const dalm_oracle *o, double *A);

void oracle_set_inflow_profile(dalm_oracle *o, const double *prof);
void oracle_set_turbine_params(dalm_oracle *o, const double *yaw_deg,
                               const double *pitch_deg, const double *omega);
void oracle_set_state(dalm_oracle *o, const double *U, const double *JU,
                      const double *p, int flags);
void oracle_stage(dalm_oracle *o, int stage);
void oracle_step(dalm_oracle *o, int n);
void oracle_advance_clock(dalm_oracle *o);
void oracle_get_field(const dalm_oracle *o, int which, double *out);
void oracle_set_field(dalm_oracle *o, int which, const double *in);
void oracle_stats(const dalm_oracle *o, int64_t *ints, double *reals);
void oracle_set_poisson(dalm_oracle *o, int64_t max_it, double tol);
/* Test-only: 1 sums dot products pairwise instead of serially (measures the
 * solver's sensitivity to summation order); 0 (default) is the reference. */
void oracle_set_sum_order(dalm_oracle *o, int mode);
/* 0: the reference's b=4 limiter (default), 1: the smooth van Albada limiter */
void oracle_set_limiter(dalm_oracle *o, int limiter);
void oracle_turbines(const dalm_oracle *o, double *torque, double *thrust);
void oracle_points(const dalm_oracle *o, double *xyz, double *f, double *torque,
                   double *thrust);
void oracle_point_tables(const dalm_oracle *o, double *r, double *dr, double *chord,
                         double *twist, double *cd, double *cl, double *atk);

#ifdef __cplusplus
}
#endif
#endif
