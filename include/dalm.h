/*
 * dalm.h — C ABI of the B200-native 3dalm time-step hot path.
 *
 * The reference (ki2098/3dalm) has no plugin or operator API: its hot path
 * is the sequence of free `static` functions that Solver::main_loop_once()
 * calls (src/solver.h:1034-1306), each taking raw host pointers that are
 * mirrored on the device by OpenACC data regions.  This header replaces that
 * sequence with an opaque handle that owns device-resident state on one GPU.
 * Every entry point names the reference code it stands in for.
 *
 * Conventions
 *   - C linkage, plain pointers and sizes, no exceptions cross the ABI.
 *   - Every function returns DALM_OK (0) or a DALM_ERR_* code; the message
 *     is available from dalm_last_error(handle) (or dalm_last_error(NULL)
 *     for failures that occur before a handle exists).
 *   - Host arrays use the reference's field layout: linear cell index
 *     (i*NY + j)*NZ + k with k contiguous, guide cells included
 *     (src/util.h:11-13); vector fields are AoS [len][3]
 *     (src/solver.h:287-290).  NX, NY, NZ are the stored sizes from
 *     mesh.json (interior + 2*gc).
 *   - One CUDA stream per handle; a handle is not thread safe.
 */
#ifndef DALM_H
#define DALM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define DALM_OK 0
#define DALM_ERR_ARG 1          /* bad argument (NULL handle, size, enum)     */
#define DALM_ERR_CASE 2         /* unreadable / inconsistent case JSON        */
#define DALM_ERR_CUDA 3         /* CUDA runtime error or no usable GPU        */
#define DALM_ERR_NONFINITE 4    /* NaN/Inf detected in the state              */
#define DALM_ERR_DEVICE_WAIT 5  /* a capped device-side wait ran out          */
#define DALM_ERR_UNSUPPORTED 6  /* option combination not implemented         */

/* ---- enums ------------------------------------------------------------ */
enum dalm_precision {
    DALM_FP64 = 0,        /* every stage in FP64, the reference's arithmetic */
    DALM_MIXED = 1        /* BiCGStab cases: the stencil fields U, JU and
                             f stored and computed in FP32 (predictor,
                             face fluxes, projection, velocity BCs), the
                             pressure solve by FP64 iterative refinement
                             with FP32 inner passes (dalm_options.
                             mixed_inner: multigrid-preconditioned CG by
                             default, or the case's BiCGStab); the
                             pressure, the Poisson right-hand side, the
                             pressure-gradient corrections, residuals,
                             norms, dots and the blade-point model in
                             FP64, the stop test on the FP64 residual; a
                             pass that stalls or breaks down hands the
                             rest of the solve to the FP64 solver.  With
                             reference_sums the stencil fields stay FP64;
                             SOR / Jacobi cases run in FP64.  The ABI
                             reads and writes the fields in FP64 (values
                             are rounded to FP32 on the way in).          */
};

enum dalm_limiter {
    DALM_LIMITER_MINMOD = 0,    /* the reference's b=4 minmod-type limiter,
                                   src/cfd.h:37-54                           */
    DALM_LIMITER_VAN_ALBADA = 1 /* smooth van Albada limiter (extension: not in
                                   the reference), kappa-MUSCL form:
                                   s = (2ab+eps)/(a^2+b^2+eps), eps 1e-12  */
};

/* Fields addressable by dalm_get_field / dalm_set_field (reference arrays). */
enum dalm_field {
    DALM_FIELD_U = 0,      /* Cfd::U     [len][3]  src/solver.h:287 */
    DALM_FIELD_UOLD = 1,   /* Cfd::Uold  [len][3]                   */
    DALM_FIELD_JU = 2,     /* Cfd::JU    [len][3]  face fluxes      */
    DALM_FIELD_P = 3,      /* Cfd::p     [len]                      */
    DALM_FIELD_NUT = 4,    /* Cfd::nut   [len]  (from the current U) */
    DALM_FIELD_DIV = 5,    /* Cfd::div   [len]  (from the current JU)*/
    DALM_FIELD_F = 6,      /* Cfd::f     [len][3]  ALM body force   */
    DALM_FIELD_B = 7,      /* Eq::b      [len]  Poisson RHS         */
    DALM_FIELD_UTAVG = 8   /* Cfd::Utavg [len][3]                   */
};

/* Stages of one time step (Solver::main_loop_once, src/solver.h:1034-1306). */
enum dalm_stage {
    DALM_STAGE_PREDICT = 0,  /* cpy_array(Uold,U) + calc_intermediate_U  :1042-1053 */
    DALM_STAGE_FLUX_RHS = 1, /* interpolate_JU + apply_JUbc + calc_poisson_rhs :1055-1077 */
    DALM_STAGE_POISSON = 2,  /* run_sor / run_pbicgstab                   :1081-1106 */
    DALM_STAGE_PROJECT = 3,  /* apply_pbc, project_p, apply_Ubc, apply_JUbc,
                                calc_nut, calc_divergence               :1112-1171 */
    DALM_STAGE_ALM = 4,      /* run_alm(t = step*dt)                      :1173-1180 */
    DALM_STAGE_DIAG = 5,     /* avg_div, max_cfl                          :1184-1186 */
    DALM_STAGE_TAVG = 6      /* running time average of U                 :1194-1204 */
};

/* dalm_set_state flags */
#define DALM_SET_APPLY_UBC 1     /* apply the velocity BCs to U (Uold := U)   */
#define DALM_SET_RECOMPUTE_JU 2  /* JU := interpolate_JU(U) + apply_JUbc      */

typedef struct dalm_handle dalm_handle;

/* FP32 inner solves of DALM_MIXED (extension: the reference has FP64 only).
 * Both stop at the same residual reduction and feed the same FP64
 * refinement, whose stop test is the reference's. */
enum dalm_mixed_inner {
    DALM_INNER_MULTIGRID = 0, /* conjugate gradients preconditioned by a
                                 geometric multigrid V-cycle (zebra z-line
                                 relaxation with x-y semi-coarsening,
                                 piecewise-constant transfers, exact
                                 coarsest solve); falls back to
                                 DALM_INNER_BICGSTAB when the coarsest level
                                 would exceed 1024 cells or a z-column 256 */
    DALM_INNER_BICGSTAB = 1   /* the case's Jacobi(k)-preconditioned BiCGStab
                                 (src/eq.h:333-402) in FP32 vectors        */
};

typedef struct {
    int precision;        /* enum dalm_precision                         */
    int limiter;          /* enum dalm_limiter                           */
    int device;           /* CUDA device ordinal                         */
    int time_average;     /* 1: maintain Utavg from "time avg start time" */
    int check_finite;     /* 1: fail a step with DALM_ERR_NONFINITE      */
    int poisson_batch;    /* Krylov iterations enqueued between host
                             convergence checks (0: automatic)           */
    int use_graphs;       /* 1: replay iteration batches as CUDA graphs  */
    int profile;          /* 1: time every kernel launch with CUDA events
                             (dalm_get_kernel_timings)                   */
    int reference_sums;   /* 1: every global sum (Krylov dots, norms,
                             divergence norm) in the reference's serial
                             cell order instead of a parallel tree, and
                             the actuator line (blade points and the dense
                             Gaussian projection) evaluated on the host
                             with the host's libm; with it the FP64 step
                             reproduces the reference's rounding, turbines
                             included (slow: for parity checks)          */
    int fused_krylov;     /* 1: each half of a Jacobi(3)-BiCGStab
                             iteration (update, preconditioner, SpMV, dot
                             products) as one kernel, 20 instead of 35
                             vectors per cell per iteration; 0 (default):
                             one kernel per reference loop, which is as
                             fast on B200 today (the fused kernels are
                             latency-bound).  Ignored with reference_sums
                             and other preconditioners.                 */
    int refine_inner_it;  /* DALM_MIXED: FP32 iterations per refinement
                             pass before the FP64 residual is recomputed
                             (0: automatic, 100)                         */
    int write_output;     /* 1: dalm_step writes the reference's output
                             files into <case_dir>/output at the case's
                             output times (inst_/tavg_ binaries with U, p,
                             div, q, f / U, snapshot.json, partition.json)
                             and a per-turbine turbines.csv every step   */
    int mixed_inner;      /* DALM_MIXED: the FP32 inner solver of each
                             refinement pass, enum dalm_mixed_inner      */
    int fused_jacobi;     /* 1: the FP64 Jacobi(3) preconditioner's last
                             two sweeps in one pass over HBM (3 instead of
                             6 vectors per cell; same results bit for
                             bit); 0 (default): one kernel per sweep,
                             which is as fast under the power cap (the
                             fused pair is instruction-bound)            */
    int reserved[2];
} dalm_options;

/* Fills *opt with the defaults (FP64, minmod, device 0, time average on,
 * finite check on, automatic batch, graphs on). */
void dalm_default_options(dalm_options *opt);

/* Solver::initialize (src/solver.h:542-1020): reads <case_dir>/setup.json,
 * mesh.json and (when "windturbine array" is present) windturbine.json,
 * builds the mesh (src/io.h:98-164), the Poisson scaling max_diag
 * (build_A, src/eq.h:701-798), the turbines and blade-point tables
 * (src/alm.h:35-206), fills U = Uold = Uin, p = 0 and runs the initial
 * BCs, face fluxes, eddy viscosity, divergence and ALM force
 * (src/solver.h:737-833).  opt may be NULL for the defaults. */
int dalm_create(const char *case_dir, const dalm_options *opt, dalm_handle **out);

/* Solver::finalize (src/solver.h:1022-1032): releases device memory. */
void dalm_destroy(dalm_handle *h);

/* Message for the last failure on h (or the last handle-less failure). */
const char *dalm_last_error(const dalm_handle *h);

/* Stored sizes (incl. guide cells) and guide-cell count (Solver::size, gc). */
int dalm_get_size(dalm_handle *h, int64_t size[3], int64_t *gc);

/* Mesh arrays x,y,z (cell centres) and dx,dy,dz (src/io.h:112-163);
 * each NULL-able, lengths NX, NY, NZ. */
int dalm_get_mesh(dalm_handle *h, double *x, double *y, double *z,
                  double *dx, double *dy, double *dz);

/* Time step and last step index: runtime.dt and max_step = (Int)(time/dt)
 * (src/solver.h:589-597, 193-199); the reference runs steps 0..max_step. */
int dalm_get_runtime(dalm_handle *h, double *dt, int64_t *max_step);

/* Poisson scaling factor max|a_c| (Eq::max_diag, src/eq.h:775-797). */
int dalm_get_max_diag(dalm_handle *h, double *max_diag);

/* Replace the state (U incl. guide cells; JU and p NULL-able) and recompute
 * the derived fields (nut, div, ALM force at t = step*dt, diagnostics) the
 * way Solver::initialize does (src/solver.h:767-833). */
int dalm_set_state(dalm_handle *h, const double *U, const double *JU,
                   const double *p, int flags);

/* Copy one reference array to / from the host (enum dalm_field). */
int dalm_get_field(dalm_handle *h, int field, double *out);
int dalm_set_field(dalm_handle *h, int field, const double *in);

/* Log-law (or any) inflow extension: per-(j,k) inflow ghost values
 * prof[NY][NZ][3] replace the uniform Uin of apply_Ubc/apply_JUbc
 * (src/bc.h:16-30, 243-257).  NULL restores the uniform Uin. */
int dalm_set_inflow_profile(dalm_handle *h, const double *prof);

/* Per-turbine overrides (arrays of length turbine_count, each NULL-able):
 * static yaw in degrees (angle type Yaw, src/alm.h:182-199), collective
 * pitch in degrees added to every blade point's twist (alpha = deg(phi) -
 * (twist + pitch), extends src/alm.h:344) and rotor speed in rad/s
 * (`rotation speed`, src/alm.h:161). */
int dalm_set_turbine_params(dalm_handle *h, const double *yaw_deg,
                            const double *pitch_deg, const double *omega);

/* The current per-turbine parameters in the units of
 * dalm_set_turbine_params (yaw: the angle offset in degrees). */
int dalm_get_turbine_params(dalm_handle *h, double *yaw_deg, double *pitch_deg,
                            double *omega);

/* Discrete adjoint of the time stepping (no reference counterpart; the
 * reference has no differentiation).  From the current state, runs the
 * forward steps through step t1 exactly as dalm_step does (the handle ends
 * at step t1 + 1), storing a restart point every ckpt_every steps, then the
 * transposed steps backwards with checkpoint-every-k recomputation.
 *   *J                 = mean over steps t0..t1 of sum_w torque_w |omega_w|
 *   grad[3 w + 0, 1, 2] = dJ / d(yaw_deg, pitch_deg, omega) of turbine w
 * The forces the first step reads are re-evaluated from the current velocity
 * and parameters first (the same forces unless the parameters changed since
 * the last actuator-line evaluation).  Requires turbines with a yaw-type
 * angle (dalm_set_turbine_params sets it) and max(step, 1) <= t0 <= t1.
 * The adjoint pressure solves reuse the case's solver; derivatives at the
 * kinks (the b=4 limiter, |JU| in the upwind flux, |ft| in the torque, the
 * polar table, trilinear cell switches) are those of the branch taken. */
int dalm_adjoint_power_grad(dalm_handle *h, int t0, int t1, int ckpt_every,
                            double *grad, double *J);

/* Statistics of the last dalm_adjoint_power_grad: adjoint pressure solves,
 * their total iterations, the largest final residual relative to its
 * right-hand side, and the forward steps recomputed from restart points. */
int dalm_get_adjoint_stats(dalm_handle *h, int64_t *solves, int64_t *iterations,
                           double *max_rel_residual, int64_t *recomputed_steps);

/* Solver::main_loop_once() x nsteps (src/solver.h:1034-1306) without field
 * output and probes; step 0 is integration-free as in the reference. */
int dalm_step(dalm_handle *h, int nsteps);

/* Run one stage of the current step (enum dalm_stage); does not advance the
 * step counter.  Used for stage-by-stage parity checks. */
int dalm_run_stage(dalm_handle *h, int stage);

/* Advance the step counter without integrating (the step-0 path). */
int dalm_advance_clock(dalm_handle *h);

/* Per-step stdout line of the reference, src/solver.h:1188-1190:
 * step, Poisson iterations and residual (Eq::it, Eq::err), avg_div, max_cfl.
 * Any pointer may be NULL. */
int dalm_get_step_stats(dalm_handle *h, int64_t *step, int64_t *poisson_it,
                        double *poisson_err, double *avg_div, double *max_cfl);

/* Poisson stop rule overrides (eq."max iteration", eq."tolerance"). */
int dalm_set_poisson(dalm_handle *h, int64_t max_it, double tol);

/* counts[0] = turbines, [1] = blade points, [2] = blades per turbine,
 * [3] = points per blade, [4] = attack-angle table length. */
int dalm_get_counts(dalm_handle *h, int64_t counts[5]);

/* Per-turbine thrust and torque summed over blade points
 * (src/alm.h:384-398) and power = torque*|omega| (extension).  NULL-able. */
int dalm_get_turbines(dalm_handle *h, double *thrust, double *torque, double *power);

/* Per-blade-point position, force, torque and thrust (ActuatorPoint,
 * src/alm.h:10-21).  NULL-able. */
int dalm_get_points(dalm_handle *h, double *xyz, double *f, double *torque,
                    double *thrust);

/* Wait for all work queued on the handle's stream. */
int dalm_synchronize(dalm_handle *h);

/* The handle's CUDA stream (a cudaStream_t), for callers that order their
 * own work or CUDA events against the solver's. */
int dalm_get_stream(dalm_handle *h, void **stream);

/* Device time in milliseconds accumulated per stage since the last reset
 * (ms[7], indexed by enum dalm_stage) and the number of kernel launches
 * issued.  Stage times are measured with CUDA events on the handle's stream
 * when opt.profile = 1 (else ms[] stays 0). */
int dalm_get_timings(dalm_handle *h, double ms[7], int64_t *launches, int reset);

/* Per-kernel launch statistics (opt.profile = 1): for kernel kind
 * index < dalm_kernel_kinds(), its name, launches, summed device time in ms
 * and algorithmic DRAM bytes per launch (the roofline numerator). */
int dalm_kernel_kinds(void);
int dalm_get_kernel_timing(dalm_handle *h, int index, const char **name,
                           int64_t *launches, double *ms, double *bytes_per_launch);

/* No counterpart in the reference (its diagnostics run inside its own
 * OpenACC data region).  For callers that cannot let a library allocate
 * device memory -- an OpenACC program that keeps U and JU in its own data
 * region and passes device pointers via `host_data use_device`, a caller
 * whose memory pool already owns the device, or code that must not
 * allocate in the middle of a time step -- this computes the step
 * diagnostics of a state already in device memory without any allocation:
 * out[0] = ||div(JU)||_2 / sqrt(N) (calc_divergence + calc_l2_norm) and
 * out[1] = max CFL (calc_max_cfl), written to the device array `out`.
 * U and JU are device arrays in the reference layout ([len][3] with guide
 * cells), dx, dy, dz device arrays of the stored lengths, stream a
 * cudaStream_t (NULL: the default stream); the work is asynchronous.
 * Limit: the reduction keeps one partial per 32 x 8 x 16 block of interior
 * cells in a fixed 256 KiB device array, so at most 16384 such blocks
 * (512 x 256 x 128 interior cells need 4096); larger grids return
 * DALM_ERR_UNSUPPORTED.  The first call on a device looks up that array's
 * address and must come before any stream capture; calls that overlap on
 * the GPU share the array and race. */
int dalm_diagnostics_noalloc(const double *U, const double *JU, const double *dx,
                             const double *dy, const double *dz, const int64_t size[3],
                             int64_t gc, double dt, double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* DALM_H */
