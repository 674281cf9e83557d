// Pressure Poisson solvers (src/eq.h, src/mv.h) with matrix-free
// coefficients and on-device loop control.
//
// Compiled with --fmad=false: each cell update keeps the reference's
// operation order, so red-black SOR sweeps and Jacobi sweeps reproduce the
// reference bit for bit.  Global dot products and norms are summed either
// by a deterministic parallel tree (default) or, in reference-order-sum
// mode, serially in the reference's cell order (k_seq).
//
// Kernels walk column segments (Segments): a block owns 32 (k) x 8 (j)
// cells of a column and marches through a chunk of i-planes, rotating the
// west / centre / east values of the stencil operand through registers, so
// each plane of the operand is read once from DRAM per sweep.
#include <cfloat>

#include "poisson.cuh"

namespace dalm {

namespace {

// Per-thread (fixed j, k) part of the coefficients: everything except the
// i-dependent terms, hoisted out of the i march.
struct ColumnCoef {
    double an, as, at, ab;          // scaled (A[id][3..6] of the reference)
    double an_u, as_u, at_u, ab_u;  // unscaled, for the diagonal
};

__device__ __forceinline__ ColumnCoef column_coef(const PoissonCoef &C, int j, int k) {
    ColumnCoef cc;
    cc.an = C.an[j]; cc.as = C.as[j]; cc.at = C.at[k]; cc.ab = C.ab[k];
    cc.an_u = C.an_u[j]; cc.as_u = C.as_u[j]; cc.at_u = C.at_u[k]; cc.ab_u = C.ab_u[k];
    return cc;
}

// a_c of cell (i, j, k) exactly as build_A assembles and scales it
// (src/eq.h:720-794): ((((((0 - ex) - aw) - an) - as) - at) - ab) / max_diag,
// the first two subtractions precomputed per i in C.xpart.
__device__ __forceinline__ double diag(const PoissonCoef &C, const ColumnCoef &cc, int i) {
    double acu = C.xpart[i] - cc.an_u;
    acu = acu - cc.as_u;
    acu = acu - cc.at_u;
    acu = acu - cc.ab_u;
    return acu / C.max_diag;
}

// ac*xc + ae*xe + aw*xw + an*xn + as*xs + at*xt + ab*xb, left to right
// (src/mv.h:87, 214; src/eq.h:36, 177); xw, xc, xe come from registers.
__device__ __forceinline__ double apply_a(const Grid &g, double ac, double ae, double aw,
                                          const ColumnCoef &cc, double xw, double xc, double xe,
                                          const double *v, long long c) {
    return ac * xc + ae * xe + aw * xw + cc.an * v[c + g.sy] + cc.as * v[c - g.sy] +
           cc.at * v[c + 1] + cc.ab * v[c - 1];
}

#define SEGMENT_LOOP(S)                                                   \
    for (int u = blockIdx.x; u < (S).count; u += gridDim.x) {             \
        int i0, i1, j, k;                                                 \
        if (!(S).column(u, i0, i1, j, k)) continue;                       \
        long long c0 = g.at(i0, j, k);

#define SEGMENT_END }

__global__ void k_begin(KrylovState *st, long long max_it, double tol, double ncell) {
    st->rho = 0; st->rho_old = 1; st->alpha = 1; st->omega = 1; st->beta = 0; st->err = 0;
    st->ncell = ncell; st->tol = tol; st->it = 0; st->max_it = max_it; st->done = 0;
}

// Residual norm at the end of a SOR / Jacobi iteration and the stop rule
// `while (it < max_it && err > tol)` (src/eq.h:297-305).
__device__ __forceinline__ void finish_iteration(KrylovState *st, double sum_r2) {
    st->err = sqrt(sum_r2) / sqrt(st->ncell);
    st->it += 1;
    if (!(st->it < st->max_it && st->err > st->tol)) st->done = 1;
}

// ---------------------------------------------------------------- SOR

// sweep_sor_at_cell (src/eq.h:145-181), colour (i+j+k)%2 (offsets 0).
// The colour's cells are updated in place; their neighbours all have the
// other colour, so the registers rotated along i are never stale.
__global__ void __launch_bounds__(TILE_THREADS)
k_sor_sweep(Grid g, PoissonCoef C, Segments S, double *x, const double *b, double w, int color,
            const KrylovState *st) {
    if (st->done) return;
    SEGMENT_LOOP(S)
    ColumnCoef cc = column_coef(C, j, k);
    long long c = c0;
    double xw = x[c - g.sx], xc = x[c];
    for (int i = i0; i < i1; i++, c += g.sx) {
        double xe = x[c + g.sx];
        if (((i + j + k) & 1) == color) {
            double ac = diag(C, cc, i);
            double rel = (b[c] - apply_a(g, ac, C.ae[i], C.aw[i], cc, xw, xc, xe, x, c)) / ac;
            xc = xc + w * rel;
            x[c] = xc;
        }
        xw = xc;
        xc = xe;
    }
    SEGMENT_END
}

// calc_residual + calc_l2_norm (src/mv.h:33-182) fused; when `copy_from`
// is set the iterate lives there (Jacobi ping-pong) and is copied into x.
// With `rstore` the residual is stored (reference-order sums read it back).
__global__ void __launch_bounds__(TILE_THREADS)
k_residual_norm(Grid g, PoissonCoef C, Segments S, double *x, const double *copy_from,
                const double *b, double *rstore, Partials<1> part, KrylovState *st) {
    if (st->done) return;
    const double *v = copy_from ? copy_from : x;
    double acc = 0;
    SEGMENT_LOOP(S)
    ColumnCoef cc = column_coef(C, j, k);
    long long c = c0;
    double xw = v[c - g.sx], xc = v[c];
    for (int i = i0; i < i1; i++, c += g.sx) {
        double xe = v[c + g.sx];
        double r = b[c] - apply_a(g, diag(C, cc, i), C.ae[i], C.aw[i], cc, xw, xc, xe, v, c);
        acc += r * r;
        if (rstore) rstore[c] = r;
        if (copy_from) x[c] = xc;
        xw = xc;
        xc = xe;
    }
    SEGMENT_END
    if (rstore) return;
    double vals[1] = {acc};
    if (grid_reduce<1>(vals, 0u, part) && threadIdx.x == 0) finish_iteration(st, vals[0]);
}

// sweep_jacobi_at_cell (src/eq.h:6-39): out = in + (rhs - A in)/ac.
__global__ void __launch_bounds__(TILE_THREADS)
k_jacobi_sweep(Grid g, PoissonCoef C, Segments S, double *out, const double *in, const double *rhs,
               const KrylovState *st) {
    if (st->done) return;
    SEGMENT_LOOP(S)
    ColumnCoef cc = column_coef(C, j, k);
    long long c = c0;
    double xw = in[c - g.sx], xc = in[c];
    for (int i = i0; i < i1; i++, c += g.sx) {
        double xe = in[c + g.sx];
        double ac = diag(C, cc, i);
        double rel = (rhs[c] - apply_a(g, ac, C.ae[i], C.aw[i], cc, xw, xc, xe, in, c)) / ac;
        out[c] = xc + rel;
        xw = xc;
        xc = xe;
    }
    SEGMENT_END
}

// ------------------------------------------------------------ BiCGStab
//
// run_pbicgstab (src/eq.h:333-473).  One iteration is
//   p-update (+ first Jacobi sweep from zero) -> PC sweeps -> q = A pp, <r0,q>
//   -> s-update (+ first sweep) -> PC sweeps -> t = A ss, <t,s>, <t,t>
//   -> x, r update, <r0,r>, <r,r>
// Each reduction's last block computes the next scalar (alpha, omega, err,
// rho, beta) on the device.

// ---- finishers: the scalar updates after each global sum -----------------

// rho = <r0, r> and the breakdown test (src/eq.h:349-353)
__device__ __forceinline__ void fin_init(KrylovState *st, double r0r) {
    st->rho = r0r;
    if (fabs(st->rho) < FLT_MIN) {
        st->err = st->rho;
        st->done = 1;
    }
}
// alpha = rho / <r0, q> (src/eq.h:371)
__device__ __forceinline__ void fin_q(KrylovState *st, double r0q) { st->alpha = st->rho / r0q; }
// omega = <t, s> / <t, t> (src/eq.h:383)
__device__ __forceinline__ void fin_t(KrylovState *st, double ts, double tt) { st->omega = ts / tt; }
// rhoold = rho; err = ||r||/sqrt(N); it++; loop test; next rho, breakdown
// test and beta (src/eq.h:397-401, 349-358)
__device__ __forceinline__ void fin_xr(KrylovState *st, double r0r, double rr) {
    st->rho_old = st->rho;
    st->err = sqrt(rr) / sqrt(st->ncell);
    st->it += 1;
    if (!(st->it < st->max_it && st->err > st->tol)) {
        st->done = 1;
    } else {
        st->rho = r0r;
        if (fabs(r0r) < FLT_MIN) {
            st->err = r0r;
            st->done = 1;
        } else {
            st->beta = (r0r / st->rho_old) * (st->alpha / st->omega);
        }
    }
}

enum SeqSite { SEQ_RESIDUAL = 0, SEQ_INIT = 1, SEQ_Q = 2, SEQ_T = 3, SEQ_XR = 4 };

// One warp: the sums of one site in the reference's serial order, then its
// finisher (reference-order-sum mode).
__global__ void k_seq(Grid g, int site, const double *a0, const double *b0, const double *a1,
                      const double *b1, KrylovState *st) {
    if (site != SEQ_INIT && st->done) return;
    double tot[2];
    if (a1) {
        warp_serial_sums<2>(g, [&](long long c, double (&t)[2]) {
            t[0] = a0[c] * b0[c];
            t[1] = a1[c] * b1[c];
        }, tot);
    } else {
        double one[1];
        warp_serial_sums<1>(g, [&](long long c, double (&t)[1]) { t[0] = a0[c] * b0[c]; }, one);
        tot[0] = one[0];
        tot[1] = 0;
    }
    if (threadIdx.x != 0) return;
    switch (site) {
    case SEQ_RESIDUAL: finish_iteration(st, tot[0]); break;
    case SEQ_INIT: fin_init(st, tot[0]); break;
    case SEQ_Q: fin_q(st, tot[0]); break;
    case SEQ_T: fin_t(st, tot[0], tot[1]); break;
    case SEQ_XR: fin_xr(st, tot[0], tot[1]); break;
    }
}

// calc_residual, cpy_array(r0, r), fill(q, 0) and the first rho = <r0, r>
// (src/eq.h:342-353).
__global__ void __launch_bounds__(TILE_THREADS)
k_bicg_init(Grid g, PoissonCoef C, Segments S, PoissonBufs B, int seq, Partials<1> part,
            KrylovState *st) {
    double acc = 0;
    SEGMENT_LOOP(S)
    ColumnCoef cc = column_coef(C, j, k);
    long long c = c0;
    double xw = B.x[c - g.sx], xc = B.x[c];
    for (int i = i0; i < i1; i++, c += g.sx) {
        double xe = B.x[c + g.sx];
        double r = B.b[c] - apply_a(g, diag(C, cc, i), C.ae[i], C.aw[i], cc, xw, xc, xe, B.x, c);
        B.r[c] = r;
        B.r0[c] = r;
        B.q[c] = 0;
        acc += r * r;
        xw = xc;
        xc = xe;
    }
    SEGMENT_END
    if (seq) return;
    double vals[1] = {acc};
    if (grid_reduce<1>(vals, 0u, part) && threadIdx.x == 0) fin_init(st, vals[0]);
}

// p = r (it 0) or r + beta (p - omega q) (src/eq.h:355-365); with the
// Jacobi preconditioner also the first sweep of run_jacobi_pc from a zero
// guess, which is exactly 0 + (p - 0)/ac (src/eq.h:367-368); with SOR
// the zero guess itself (src/eq.h:438).
__global__ void __launch_bounds__(TILE_THREADS)
k_bicg_p(Grid g, PoissonCoef C, Segments S, PoissonBufs B, int first_sweep, const KrylovState *st) {
    if (st->done) return;
    const bool first = (st->it == 0);
    const double beta = st->beta, omega = st->omega;
    SEGMENT_LOOP(S)
    ColumnCoef cc = column_coef(C, j, k);
    long long c = c0;
    for (int i = i0; i < i1; i++, c += g.sx) {
        double pv = first ? B.r[c] : B.r[c] + beta * (B.pk[c] - omega * B.q[c]);
        B.pk[c] = pv;
        B.pp[c] = first_sweep ? 0.0 + (pv - 0.0) / diag(C, cc, i) : 0.0;
    }
    SEGMENT_END
}

// s = r - alpha q (src/eq.h:373-377) with the same first-sweep fusion.
__global__ void __launch_bounds__(TILE_THREADS)
k_bicg_s(Grid g, PoissonCoef C, Segments S, PoissonBufs B, int first_sweep, const KrylovState *st) {
    if (st->done) return;
    const double alpha = st->alpha;
    SEGMENT_LOOP(S)
    ColumnCoef cc = column_coef(C, j, k);
    long long c = c0;
    for (int i = i0; i < i1; i++, c += g.sx) {
        double sv = B.r[c] - alpha * B.q[c];
        B.s[c] = sv;
        B.ss[c] = first_sweep ? 0.0 + (sv - 0.0) / diag(C, cc, i) : 0.0;
    }
    SEGMENT_END
}

// q = A pp and <r0, q>; alpha = rho / <r0, q> (src/eq.h:369-371).
__global__ void __launch_bounds__(TILE_THREADS)
k_bicg_q(Grid g, PoissonCoef C, Segments S, PoissonBufs B, const double *ppf, int seq,
         Partials<1> part, KrylovState *st) {
    if (st->done) return;
    double acc = 0;
    SEGMENT_LOOP(S)
    ColumnCoef cc = column_coef(C, j, k);
    long long c = c0;
    double xw = ppf[c - g.sx], xc = ppf[c];
    for (int i = i0; i < i1; i++, c += g.sx) {
        double xe = ppf[c + g.sx];
        double qv = apply_a(g, diag(C, cc, i), C.ae[i], C.aw[i], cc, xw, xc, xe, ppf, c);
        B.q[c] = qv;
        acc += B.r0[c] * qv;
        xw = xc;
        xc = xe;
    }
    SEGMENT_END
    if (seq) return;
    double vals[1] = {acc};
    if (grid_reduce<1>(vals, 0u, part) && threadIdx.x == 0) fin_q(st, vals[0]);
}

// t = A ss, <t, s>, <t, t>; omega = <t,s>/<t,t> (src/eq.h:381-383).
__global__ void __launch_bounds__(TILE_THREADS)
k_bicg_t(Grid g, PoissonCoef C, Segments S, PoissonBufs B, const double *ssf, int seq,
         Partials<2> part, KrylovState *st) {
    if (st->done) return;
    double ts = 0, tt = 0;
    SEGMENT_LOOP(S)
    ColumnCoef cc = column_coef(C, j, k);
    long long c = c0;
    double xw = ssf[c - g.sx], xc = ssf[c];
    for (int i = i0; i < i1; i++, c += g.sx) {
        double xe = ssf[c + g.sx];
        double tv = apply_a(g, diag(C, cc, i), C.ae[i], C.aw[i], cc, xw, xc, xe, ssf, c);
        B.t[c] = tv;
        ts += tv * B.s[c];
        tt += tv * tv;
        xw = xc;
        xc = xe;
    }
    SEGMENT_END
    if (seq) return;
    double vals[2] = {ts, tt};
    if (grid_reduce<2>(vals, 0u, part) && threadIdx.x == 0) fin_t(st, vals[0], vals[1]);
}

// x += alpha pp + omega ss; r = s - omega t (src/eq.h:385-395) with
// <r0, r> and <r, r> for the finisher.
__global__ void __launch_bounds__(TILE_THREADS)
k_bicg_xr(Grid g, Segments S, PoissonBufs B, const double *ppf, const double *ssf, int seq,
          Partials<2> part, KrylovState *st) {
    if (st->done) return;
    const double alpha = st->alpha, omega = st->omega;
    double r0r = 0, rr = 0;
    SEGMENT_LOOP(S)
    long long c = c0;
    for (int i = i0; i < i1; i++, c += g.sx) {
        B.x[c] = B.x[c] + alpha * ppf[c] + omega * ssf[c];
        double rv = B.s[c] - omega * B.t[c];
        B.r[c] = rv;
        r0r += B.r0[c] * rv;
        rr += rv * rv;
    }
    SEGMENT_END
    if (seq) return;
    double vals[2] = {r0r, rr};
    if (grid_reduce<2>(vals, 0u, part) && threadIdx.x == 0) fin_xr(st, vals[0], vals[1]);
}

Box interior_box(const Grid &g) {
    return Box{{g.gc, g.gc, g.gc}, {g.nx - g.gc, g.ny - g.gc, g.nz - g.gc}};
}

void seq_launch(const LaunchCtx &L, const Grid &g, int site, const double *a0, const double *b0,
                const double *a1, const double *b1, KrylovState *st) {
    L.pre(KK_SEQ_SUM);
    k_seq<<<1, 32, 0, L.s>>>(g, site, a0, b0, a1, b1, st);
    L.post(KK_SEQ_SUM);
}

}  // namespace

Segments poisson_segments(const Grid &g, int sm_count) {
    return Segments::make(interior_box(g), sm_count * 8);
}

void launch_poisson_begin(const LaunchCtx &L, KrylovState *st, long long max_it, double tol,
                          double ncell) {
    L.pre(KK_POISSON_BEGIN);
    k_begin<<<1, 1, 0, L.s>>>(st, max_it, tol, ncell);
    L.post(KK_POISSON_BEGIN);
}

void launch_sor_iteration(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                          const PoissonBufs &B, const PoissonConfig &cfg, Partials<1> part,
                          KrylovState *st) {
    const Segments &S = cfg.seg;
    for (int color = 0; color < 2; color++) {
        L.pre(KK_SOR_SWEEP);
        k_sor_sweep<<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, B.x, B.b, cfg.relax, color, st);
        L.post(KK_SOR_SWEEP);
    }
    double *rs = cfg.reference_sums ? B.r : nullptr;
    L.pre(KK_RESIDUAL_NORM);
    k_residual_norm<<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, B.x, nullptr, B.b, rs, part, st);
    L.post(KK_RESIDUAL_NORM);
    if (rs) seq_launch(L, g, SEQ_RESIDUAL, B.r, B.r, nullptr, nullptr, st);
}

void launch_jacobi_iteration(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                             const PoissonBufs &B, const PoissonConfig &cfg, Partials<1> part,
                             KrylovState *st) {
    const Segments &S = cfg.seg;
    L.pre(KK_JACOBI_SWEEP);
    k_jacobi_sweep<<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, B.tp, B.x, B.b, st);
    L.post(KK_JACOBI_SWEEP);
    double *rs = cfg.reference_sums ? B.r : nullptr;
    L.pre(KK_RESIDUAL_NORM);
    k_residual_norm<<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, B.x, B.tp, B.b, rs, part, st);
    L.post(KK_RESIDUAL_NORM);
    if (rs) seq_launch(L, g, SEQ_RESIDUAL, B.r, B.r, nullptr, nullptr, st);
}

void launch_bicg_init(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                      const PoissonBufs &B, const PoissonConfig &cfg, Partials<1> part,
                      KrylovState *st) {
    const Segments &S = cfg.seg;
    L.pre(KK_BICG_INIT);
    k_bicg_init<<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, B, cfg.reference_sums, part, st);
    L.post(KK_BICG_INIT);
    if (cfg.reference_sums) seq_launch(L, g, SEQ_INIT, B.r0, B.r, nullptr, nullptr, st);
}

// Applies the preconditioner to `rhs` with the first sweep already done
// into `x` (Jacobi) or `x` zeroed (SOR); returns the buffer holding M^-1 rhs.
static double *precondition(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                            const PoissonConfig &cfg, double *x, double *tmp, const double *rhs,
                            const KrylovState *st) {
    const Segments &S = cfg.seg;
    if (cfg.pc == PC_SOR) {
        for (int n = 0; n < cfg.pc_sweeps; n++) {
            for (int color = 0; color < 2; color++) {
                L.pre(KK_SOR_SWEEP);
                k_sor_sweep<<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, x, rhs, cfg.pc_relax,
                                                                color, st);
                L.post(KK_SOR_SWEEP);
            }
        }
        return x;
    }
    double *cur = x, *nxt = tmp;
    for (int n = 1; n < cfg.pc_sweeps; n++) {
        L.pre(KK_JACOBI_SWEEP);
        k_jacobi_sweep<<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, nxt, cur, rhs, st);
        L.post(KK_JACOBI_SWEEP);
        double *t = cur;
        cur = nxt;
        nxt = t;
    }
    return cur;
}

void launch_bicg_iteration(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                           const PoissonBufs &B, const PoissonConfig &cfg, Partials<2> part,
                           KrylovState *st) {
    const Segments &S = cfg.seg;
    int first = (cfg.pc == PC_JACOBI && cfg.pc_sweeps >= 1) ? 1 : 0;
    int seq = cfg.reference_sums;
    Partials<1> part1{part.buf, part.ticket};
    L.pre(KK_BICG_P);
    k_bicg_p<<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, B, first, st);
    L.post(KK_BICG_P);
    double *ppf = precondition(L, g, C, cfg, B.pp, B.tp, B.pk, st);
    L.pre(KK_BICG_Q);
    k_bicg_q<<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, B, ppf, seq, part1, st);
    L.post(KK_BICG_Q);
    if (seq) seq_launch(L, g, SEQ_Q, B.r0, B.q, nullptr, nullptr, st);
    L.pre(KK_BICG_S);
    k_bicg_s<<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, B, first, st);
    L.post(KK_BICG_S);
    double *ssf = precondition(L, g, C, cfg, B.ss, B.ts, B.s, st);
    L.pre(KK_BICG_T);
    k_bicg_t<<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, B, ssf, seq, part, st);
    L.post(KK_BICG_T);
    if (seq) seq_launch(L, g, SEQ_T, B.t, B.s, B.t, B.t, st);
    L.pre(KK_BICG_XR);
    k_bicg_xr<<<S.count, TILE_THREADS, 0, L.s>>>(g, S, B, ppf, ssf, seq, part, st);
    L.post(KK_BICG_XR);
    if (seq) seq_launch(L, g, SEQ_XR, B.r0, B.r, B.r, B.r, st);
}

}  // namespace dalm
