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
};

struct PoissonBufs {
    double *x;             // pressure (Cfd::p)
    const double *b;       // right-hand side (Eq::b)
    double *r, *r0, *pk, *q, *s, *t;   // Eq::r, r0, p, q, s, t
    double *pp, *ss;       // preconditioned directions (Eq::pp, Eq::ss)
    double *tp, *ts;       // Jacobi ping-pong partners of pp and ss
};

// TMA maps of every Poisson buffer, looked up by device pointer.
struct MapTable {
    static constexpr int MAX = 16;
    int n = 0;
    const void *ptr[MAX];
    FieldMaps maps[MAX];
    void add(const Grid &g, const void *p) {
        ptr[n] = p;
        maps[n] = make_field_maps(g, p, 8);
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
    Segments seg;        // column segments of the interior (one per block)
    const MapTable *maps;
};

// The interior's column segments, sized to fill the GPU.
Segments poisson_segments(const Grid &g, int sm_count);
// Dynamic shared memory of the TMA stencil kernels (one ring per block).
size_t poisson_stencil_smem();

void launch_poisson_begin(const LaunchCtx &L, KrylovState *st, long long max_it, double tol,
                          double ncell);
// red-black SOR (src/eq.h:291-306): one iteration = red, black, residual norm
void launch_sor_iteration(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                          const PoissonBufs &B, const PoissonConfig &cfg, Partials<1> part,
                          KrylovState *st);
// standalone Jacobi: one sweep + residual norm
void launch_jacobi_iteration(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                             const PoissonBufs &B, const PoissonConfig &cfg, Partials<1> part,
                             KrylovState *st);
// BiCGStab (src/eq.h:333-473)
void launch_bicg_init(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                      const PoissonBufs &B, const PoissonConfig &cfg, Partials<1> part,
                      KrylovState *st);
void launch_bicg_iteration(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                           const PoissonBufs &B, const PoissonConfig &cfg, Partials<2> part,
                           KrylovState *st);

}  // namespace dalm
