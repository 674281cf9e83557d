// Pressure Poisson solvers on the device (src/eq.h, src/mv.h).
#pragma once

#include "flow.cuh"
#include "tma.cuh"

namespace dalm {

// Iteration state kept in device memory so the whole Krylov / SOR loop runs
// without a host round trip per dot product; the host only polls `done`
// between batches of enqueued iterations.
struct KrylovState {
    double rho, rho_old, alpha, omega, beta, err;
    double ncell;     // interior cell count (effective_count)
    double tol;
    long long it, max_it;
    int done;         // 1 once the reference loop would have exited
    int wait_error;   // non-zero: a bounded device-side wait ran out
    // iterative refinement (DALM_MIXED): the outer state's pass count and
    // limits, and the inner state's breakdown guard
    long long outer_it, max_outer;
    double inner_rtol;     // inner solves stop at inner_rtol * |outer residual|
    long long inner_cap;   // ... or after inner_cap iterations
    int guard;             // 1: a non-finite Krylov scalar ends the solve as a breakdown
    int breakdown;
};

// Vectors of one solve A x = b in precision T: FP64 (Cfd::p and the
// reference's Eq members) or FP32 (the inner solves A e = r of iterative
// refinement, x = e).
template <typename T>
struct PoissonBufsT {
    T *x;              // pressure (Cfd::p), or the refinement correction e
    const T *b;        // right-hand side (Eq::b), or the refinement residual
    T *r, *r0, *pk, *q, *s, *t;   // Eq::r, r0, p, q, s, t
    T *pp, *ss;        // preconditioned directions (Eq::pp, Eq::ss)
    T *tp, *ts;        // Jacobi ping-pong partners of pp and ss
};
using PoissonBufs = PoissonBufsT<double>;

// TMA maps of every Poisson buffer, looked up by device pointer.
struct MapTable {
    static constexpr int MAX = 32;
    int n = 0;
    const void *ptr[MAX];
    FieldMaps maps[MAX];
    void add(const Grid &g, const void *p, int elem_bytes = 8) {
        if (n >= MAX) throw std::logic_error("MapTable full");
        ptr[n] = p;
        maps[n] = make_field_maps(g, p, elem_bytes);
        n++;
    }
    const FieldMaps &of(const void *p) const {
        for (int m = 0; m < n; m++)
            if (ptr[m] == p) return maps[m];
        throw std::invalid_argument("no TMA map for this buffer");
    }
};

enum PoissonMethod { PM_SOR = 0, PM_BICG = 1, PM_JACOBI = 2 };
enum PreconMethod { PC_JACOBI = 0, PC_SOR = 1 };

struct PoissonConfig {
    int method, pc;
    double relax, pc_relax;
    int pc_sweeps;
    int reference_sums;  // 1: global sums in the reference's serial order
    int jacobi2;         // 1: FP64 Jacobi(3): the last two sweeps in one pass
    Segments seg;        // column segments of the interior (one per block)
    const MapTable *maps;
};

// The interior's column segments, sized to fill the GPU.
Segments poisson_segments(const Grid &g, int sm_count);

// Resets a solve's state.  Iterative refinement: max_outer, inner_rtol and
// inner_cap set up the outer state; guard = 1 marks the inner state.
void launch_poisson_begin(const LaunchCtx &L, KrylovState *st, long long max_it, double tol,
                          double ncell, long long max_outer = 0, double inner_rtol = 0,
                          long long inner_cap = 0, int guard = 0);
// red-black SOR (src/eq.h:291-306): one iteration = red, black, residual norm
void launch_sor_iteration(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                          const PoissonBufs &B, const PoissonConfig &cfg, Partials<1> part,
                          KrylovState *st);
// standalone Jacobi: one sweep + residual norm
void launch_jacobi_iteration(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                             const PoissonBufs &B, const PoissonConfig &cfg, Partials<1> part,
                             KrylovState *st);
// BiCGStab (src/eq.h:333-473), in FP64 or, for the inner solves of
// iterative refinement, FP32 (global sums and scalars stay FP64)
void launch_bicg_init(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                      const PoissonBufs &B, const PoissonConfig &cfg, Partials<1> part,
                      KrylovState *st);
template <typename T>
void launch_bicg_iteration(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                           const PoissonBufsT<T> &B, const PoissonConfig &cfg, Partials<2> part,
                           KrylovState *st);

// Iterative refinement: the FP64 residual r = b - A x of the pressure x and
// its FP64 norm; unless that meets the tolerance, seeds the FP32 inner solve
// A e = r (inner r = r0 = fp32(r), q = 0, rho = <r, r>; e restarts from 0 at
// the inner solve's first x update).
void launch_refine_residual(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                            const PoissonConfig &cfg, const double *x, const double *b,
                            const PoissonBufsT<float> &inner, Partials<2> part,
                            KrylovState *outer, KrylovState *inner_st);
// x += sign * e: the FP64 accumulation of an FP32 correction (sign -1 takes
// a rejected correction back)
void launch_refine_update(const LaunchCtx &L, const Grid &g, const PoissonConfig &cfg, double *x,
                          const float *e, double sign);
// x += alpha ppf + omega ssf; r = s - omega t; <r0,r>, <r,r> (fast arithmetic)
void launch_bicg_xr(const LaunchCtx &L, const Grid &g, const PoissonBufs &B, const double *ppf,
                    const double *ssf, const PoissonConfig &cfg, Partials<2> part,
                    KrylovState *st);

// Ping-pong partners of p and q for the fused iteration: iteration n reads
// pk[n % 2], q[n % 2] and writes pk[(n + 1) % 2], q[(n + 1) % 2].
struct FusedBufs {
    double *pk[2], *q[2];
};
// true when the fused kernels implement this configuration: BiCGStab with
// 3 Jacobi sweeps, tree sums (not the reference-order mode)
bool fused_bicg_available(const PoissonConfig &cfg);
// BiCGStab iteration n (from 0) as two fused half-iteration kernels + the
// x / r update (poisson_fused.cu)
void launch_bicg_iteration_fused(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                                 const PoissonBufs &B, const FusedBufs &F, long long n,
                                 const PoissonConfig &cfg, Partials<2> part, KrylovState *st);

}  // namespace dalm
