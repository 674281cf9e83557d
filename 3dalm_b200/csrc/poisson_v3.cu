// Pressure Poisson solvers (src/eq.h, src/mv.h) with matrix-free
// coefficients and on-device loop control.
//
// Two arithmetic variants of every kernel (template flag EXACT):
//   EXACT = true   the reference's operation order and rounding: separate
//                  multiplies and adds (this file is compiled with
//                  --fmad=false), true divisions by a_c.  Used together with
//                  reference-order sums, the solve reproduces the reference
//                  bit for bit.
//   EXACT = false  fused multiply-adds and a Newton-refined reciprocal of a_c
//                  (the fast default); results differ from the reference in
//                  the last bits, like any other summation order.
//
// Kernels walk column segments (Segments): a block owns 32 (k) x 8 (j)
// cells of a column and marches through a chunk of i-planes.  The stencil
// kernels stage each plane of their operand (one-cell halo in j, two in k)
// and of their point-wise input in shared memory with TMA
// (cp.async.bulk.tensor), NSTAGE planes deep, and compute two planes per
// pass, so the loads of the next planes are in flight while the current
// ones are computed.
#include <cfloat>

#include "poisson.cuh"

namespace dalm {

namespace {

// Per-thread (fixed j, k) part of the coefficients, hoisted out of the march.
struct ColumnCoef {
    double an, as, at, ab;          // scaled (A[id][3..6] of the reference)
    double an_u, as_u, at_u, ab_u;  // unscaled, for the diagonal
    double colsum;                  // an_u + as_u + at_u + ab_u (fast variant)
};

__device__ __forceinline__ ColumnCoef column_coef(const PoissonCoef &C, int j, int k) {
    ColumnCoef cc;
    cc.an = C.an[j]; cc.as = C.as[j]; cc.at = C.at[k]; cc.ab = C.ab[k];
    cc.an_u = C.an_u[j]; cc.as_u = C.as_u[j]; cc.at_u = C.at_u[k]; cc.ab_u = C.ab_u[k];
    cc.colsum = cc.an_u + cc.as_u + cc.at_u + cc.ab_u;
    return cc;
}

// a_c exactly as build_A assembles and scales it (src/eq.h:720-794):
// ((((((0 - ex) - aw) - an) - as) - at) - ab) / max_diag, the first two
// subtractions precomputed per i in xpart.
template <bool EXACT>
__device__ __forceinline__ double diag(double xpart, const ColumnCoef &cc, const PoissonCoef &C) {
    if (EXACT) {
        double acu = xpart - cc.an_u;
        acu = acu - cc.as_u;
        acu = acu - cc.at_u;
        acu = acu - cc.ab_u;
        return acu / C.max_diag;
    }
    return (xpart - cc.colsum) * C.inv_max_diag;
}

// 1/a with a Newton-Raphson refinement (two steps, quadratic convergence)
// of the hardware's approximate reciprocal; a is a diagonal entry, never
// near zero or subnormal.
__device__ __forceinline__ double fast_rcp(double a) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
    double e = __fma_rn(-a, y, 1.0);
    y = __fma_rn(y, e, y);
    e = __fma_rn(-a, y, 1.0);
    return __fma_rn(y, e, y);
}

// A x at one cell: ac*xc + ae*xe + aw*xw + an*xn + as*xs + at*xt + ab*xb,
// left to right (src/mv.h:87, 214; src/eq.h:36, 177).
template <bool EXACT>
__device__ __forceinline__ double apply_a(double ac, double ae, double aw, const ColumnCoef &cc,
                                          double xc, double xe, double xw, double xn, double xs,
                                          double xt, double xb) {
    if (EXACT)
        return ac * xc + ae * xe + aw * xw + cc.an * xn + cc.as * xs + cc.at * xt + cc.ab * xb;
    double v = ac * xc;
    v = __fma_rn(ae, xe, v);
    v = __fma_rn(aw, xw, v);
    v = __fma_rn(cc.an, xn, v);
    v = __fma_rn(cc.as, xs, v);
    v = __fma_rn(cc.at, xt, v);
    return __fma_rn(cc.ab, xb, v);
}

// (b - ax)/ac, the Jacobi / SOR relaxation (src/eq.h:36, 177)
template <bool EXACT>
__device__ __forceinline__ double relax(double b, double ax, double ac) {
    if (EXACT) return (b - ax) / ac;
    return (b - ax) * fast_rcp(ac);
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
    st->wait_error = 0;
}

// ---- finishers: the scalar updates after each global sum -----------------

// residual norm of a SOR / Jacobi iteration and the stop rule
// `while (it < max_it && err > tol)` (src/eq.h:297-305)
__device__ __forceinline__ void finish_iteration(KrylovState *st, double sum_r2) {
    st->err = sqrt(sum_r2) / sqrt(st->ncell);
    st->it += 1;
    if (!(st->it < st->max_it && st->err > st->tol)) st->done = 1;
}
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

// ---- point-wise BiCGStab kernels -------------------------------------------
//
// run_pbicgstab (src/eq.h:333-473).  One iteration is
//   p-update (+ first Jacobi sweep from zero) -> PC sweeps -> q = A pp, <r0,q>
//   -> s-update (+ first sweep) -> PC sweeps -> t = A ss, <t,s>, <t,t>
//   -> x, r update, <r0,r>, <r,r>
// Each reduction's last block computes the next scalar (alpha, omega, err,
// rho, beta) on the device.

// p = r (it 0) or r + beta (p - omega q) (src/eq.h:355-365); with the
// Jacobi preconditioner also the first sweep of run_jacobi_pc from a zero
// guess, which is exactly 0 + (p - 0)/ac (src/eq.h:367-368); with SOR
// the zero guess itself (src/eq.h:438).
template <bool EXACT>
__global__ void __launch_bounds__(TILE_THREADS)
k_bicg_p(Grid g, PoissonCoef C, Segments S, PoissonBufs B, int first_sweep, const KrylovState *st) {
    if (st->done) return;
    const bool first = (st->it == 0);
    const double beta = st->beta, omega = st->omega;
    SEGMENT_LOOP(S)
    ColumnCoef cc = column_coef(C, j, k);
    long long c = c0;
    for (int i = i0; i < i1; i++, c += g.sx) {
        double pv = first ? B.r[c]
                          : (EXACT ? B.r[c] + beta * (B.pk[c] - omega * B.q[c])
                                   : __fma_rn(beta, __fma_rn(-omega, B.q[c], B.pk[c]), B.r[c]));
        B.pk[c] = pv;
        if (!first_sweep) {
            B.pp[c] = 0.0;
        } else {
            double ac = diag<EXACT>(C.xpart[i], cc, C);
            B.pp[c] = EXACT ? 0.0 + (pv - 0.0) / ac : pv * fast_rcp(ac);
        }
    }
    SEGMENT_END
}

// s = r - alpha q (src/eq.h:373-377) with the same first-sweep fusion.
template <bool EXACT>
__global__ void __launch_bounds__(TILE_THREADS)
k_bicg_s(Grid g, PoissonCoef C, Segments S, PoissonBufs B, int first_sweep, const KrylovState *st) {
    if (st->done) return;
    const double alpha = st->alpha;
    SEGMENT_LOOP(S)
    ColumnCoef cc = column_coef(C, j, k);
    long long c = c0;
    for (int i = i0; i < i1; i++, c += g.sx) {
        double sv = EXACT ? B.r[c] - alpha * B.q[c] : __fma_rn(-alpha, B.q[c], B.r[c]);
        B.s[c] = sv;
        if (!first_sweep) {
            B.ss[c] = 0.0;
        } else {
            double ac = diag<EXACT>(C.xpart[i], cc, C);
            B.ss[c] = EXACT ? 0.0 + (sv - 0.0) / ac : sv * fast_rcp(ac);
        }
    }
    SEGMENT_END
}

// x += alpha pp + omega ss; r = s - omega t (src/eq.h:385-395) with
// <r0, r> and <r, r> for the finisher.
template <bool EXACT>
__global__ void __launch_bounds__(TILE_THREADS)
k_bicg_xr(Grid g, Segments S, PoissonBufs B, const double *ppf, const double *ssf, int seq,
          Partials<2> part, KrylovState *st) {
    if (st->done) return;
    const double alpha = st->alpha, omega = st->omega;
    double r0r = 0, rr = 0;
    SEGMENT_LOOP(S)
    long long c = c0;
    for (int i = i0; i < i1; i++, c += g.sx) {
        double rv;
        if (EXACT) {
            B.x[c] = B.x[c] + alpha * ppf[c] + omega * ssf[c];
            rv = B.s[c] - omega * B.t[c];
        } else {
            B.x[c] = __fma_rn(omega, ssf[c], __fma_rn(alpha, ppf[c], B.x[c]));
            rv = __fma_rn(-omega, B.t[c], B.s[c]);
        }
        B.r[c] = rv;
        r0r += B.r0[c] * rv;
        rr += rv * rv;
    }
    SEGMENT_END
    if (seq) return;
    double vals[2] = {r0r, rr};
    if (grid_reduce<2>(vals, 0u, part) && threadIdx.x == 0) fin_xr(st, vals[0], vals[1]);
}

// ------------------------------------------------------- TMA stencil sweeps

constexpr int NSTAGE = 8;
constexpr int MAXCHUNK = 32;                  // Segments caps a chunk at 32 planes
constexpr int HK = 2;                         // halo in k: 16 bytes of FP64
constexpr int TKW = TK + 2 * HK;              // 36
constexpr int TJW = TJ + 2;                   // 10
constexpr int OP_ELEMS = TKW * TJW;
constexpr int OP_BYTES = OP_ELEMS * 8;        // 2880
constexpr int OP_BYTES_PAD = ((OP_BYTES + 127) / 128) * 128;
constexpr int PW_BYTES = TK * TJ * 8;         // 2048
constexpr int STAGE_BYTES = OP_BYTES_PAD + PW_BYTES;

enum StencilKind {
    SK_JACOBI = 0,    // out = x + (rhs - A x)/ac          sweep_jacobi_at_cell, src/eq.h:6-39
    SK_RESIDUAL = 1,  // sum (b - A x)^2 [, r stored] [, x copied]   src/mv.h:33-182
    SK_INIT = 2,      // r = r0 = b - A x, q = 0, sum r*r         src/eq.h:342-353
    SK_Q = 3,         // q = A pp, sum r0*q                       src/eq.h:369-371
    SK_T = 4,         // t = A ss, sum t*s, sum t*t               src/eq.h:381-383
    SK_SOR = 5        // red-black update in place                src/eq.h:145-181
};

struct StencilArgs {
    double *out;    // JACOBI out, RESIDUAL r (or null), INIT r, Q q, T t, SOR x
    double *out2;   // RESIDUAL copy target (or null), INIT r0
    double *out3;   // INIT q
    double w;       // SOR relaxation
    int color;      // SOR colour
    int reduce;     // 0: no tree reduction (the reference-order path sums)
};

// One block = one column segment.  Load L (0 <= L < nplanes + 2) brings
// plane i0 - 1 + L of the operand (halo box) and, for the planes the block
// computes, of the point-wise input (plain box) into ring stage L % NSTAGE.
// Plane i0 + n is computed from loads n, n + 1, n + 2.  Each pass computes
// two planes and then refills the two stages it released.
template <int KIND, bool EXACT>
__global__ void __launch_bounds__(TILE_THREADS)
k_stencil(Grid g, PoissonCoef C, Segments S, const __grid_constant__ CUtensorMap m_op,
          const __grid_constant__ CUtensorMap m_pw, StencilArgs A, Partials<2> part,
          KrylovState *st) {
    if (KIND != SK_INIT && st->done) return;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) unsigned long long bar[NSTAGE];
    __shared__ double s_ae[MAXCHUNK], s_aw[MAXCHUNK], s_xp[MAXCHUNK];
    const int u = blockIdx.x;
    int i0, i1, j, k;
    const bool active = S.column(u, i0, i1, j, k);
    const int col = u % S.ncol;
    const int k0 = S.box.lo[2] + (col % S.ntk) * TK, j0 = S.box.lo[1] + (col / S.ntk) * TJ;
    const int nplanes = i1 - i0, nload = nplanes + 2;
    const int xo = k0 - HK + (int)g.off, xp = k0 + (int)g.off;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    if (threadIdx.x == 0) {
        for (int s = 0; s < NSTAGE; s++) mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    if (threadIdx.x < nplanes) {
        s_ae[threadIdx.x] = C.ae[i0 + threadIdx.x];
        s_aw[threadIdx.x] = C.aw[i0 + threadIdx.x];
        s_xp[threadIdx.x] = C.xpart[i0 + threadIdx.x];
    }
    __syncthreads();
    auto issue = [&](int L) {
        int s = L % NSTAGE;
        unsigned char *base = smem + s * STAGE_BYTES;
        bool pw = (L >= 1 && L <= nplanes);
        mbar_expect_tx(&bar[s], OP_BYTES + (pw ? PW_BYTES : 0));
        tma_load_3d(base, &m_op, xo, j0 - 1, i0 - 1 + L, &bar[s]);
        if (pw) tma_load_3d(base + OP_BYTES_PAD, &m_pw, xp, j0, i0 - 1 + L, &bar[s]);
    };
    int issued = 0;
    if (threadIdx.x == 0)
        for (; issued < NSTAGE && issued < nload; issued++) issue(issued);

    ColumnCoef cc;
    if (active) cc = column_coef(C, j, k);
    const int idx = (warp + 1) * TKW + lane + HK;
    const int sx = (int)g.sx;
    const int cbase = active ? (int)g.at(i0, j, k) : 0;
    double acc0 = 0, acc1 = 0;

    // one cell of plane i0 + nn
    auto cell = [&](int nn) {
        const double *W = (const double *)(smem + (nn % NSTAGE) * STAGE_BYTES);
        const double *Cp = (const double *)(smem + ((nn + 1) % NSTAGE) * STAGE_BYTES);
        const double *E = (const double *)(smem + ((nn + 2) % NSTAGE) * STAGE_BYTES);
        const double pw = ((const double *)((const unsigned char *)Cp + OP_BYTES_PAD))[warp * TK + lane];
        const int c = cbase + nn * sx;
        const double xc = Cp[idx];
        const double ac = diag<EXACT>(s_xp[nn], cc, C);
        const double ax = apply_a<EXACT>(ac, s_ae[nn], s_aw[nn], cc, xc, E[idx], W[idx],
                                         Cp[idx + TKW], Cp[idx - TKW], Cp[idx + 1], Cp[idx - 1]);
        if (KIND == SK_JACOBI) {
            A.out[c] = xc + relax<EXACT>(pw, ax, ac);
        } else if (KIND == SK_RESIDUAL) {
            double r = pw - ax;
            acc0 += r * r;
            if (A.out) A.out[c] = r;
            if (A.out2) A.out2[c] = xc;
        } else if (KIND == SK_INIT) {
            double r = pw - ax;
            A.out[c] = r;
            A.out2[c] = r;
            A.out3[c] = 0;
            acc0 += r * r;
        } else if (KIND == SK_Q) {
            A.out[c] = ax;
            acc0 += pw * ax;
        } else if (KIND == SK_T) {
            A.out[c] = ax;
            acc0 += ax * pw;
            acc1 += ax * ax;
        } else if (KIND == SK_SOR) {
            const int i = i0 + nn;
            if (((i + j + k) & 1) == A.color) {
                double rel = relax<EXACT>(pw, ax, ac);
                A.out[c] = EXACT ? xc + A.w * rel : __fma_rn(A.w, rel, xc);
            }
        }
    };

    int waited = 0;
    bool fail = false;
    for (int n = 0; n < nplanes; n += 2) {
        const int m = nplanes - n < 2 ? nplanes - n : 2;
        while (!fail && waited <= n + m + 1) {
            fail = !mbar_wait(&bar[waited % NSTAGE], (unsigned)((waited / NSTAGE) & 1));
            if (!fail) waited++;
        }
        if (!fail && active) {
            cell(n);
            if (m == 2) cell(n + 1);
        }
        if (__syncthreads_or(fail)) break;
        if (threadIdx.x == 0) {
            fence_proxy_async();  // the released stages were read through the generic proxy
            for (int q = 0; q < m && issued < nload; q++) issue(issued++);
        }
    }
    if (__syncthreads_or(fail)) {
        // a bounded wait ran out: report, drain what is still in flight, stop
        if (threadIdx.x == 0) {
            st->wait_error = 1;
            st->done = 1;
            for (int L = waited; L < issued; L++)
                mbar_wait(&bar[L % NSTAGE], (unsigned)((L / NSTAGE) & 1));
        }
        return;
    }
    if (KIND == SK_JACOBI || KIND == SK_SOR || !A.reduce) return;
    double vals[2] = {acc0, acc1};
    if (grid_reduce<2>(vals, 0u, part) && threadIdx.x == 0) {
        if (KIND == SK_RESIDUAL) finish_iteration(st, vals[0]);
        if (KIND == SK_INIT) fin_init(st, vals[0]);
        if (KIND == SK_Q) fin_q(st, vals[0]);
        if (KIND == SK_T) fin_t(st, vals[0], vals[1]);
    }
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

template <int KIND>
void stencil_launch(const LaunchCtx &L, int kind_tag, const Grid &g, const PoissonCoef &C,
                    const PoissonConfig &cfg, const double *op, const double *pw,
                    const StencilArgs &A, Partials<2> part, KrylovState *st) {
    const Segments &S = cfg.seg;
    const CUtensorMap &mo = cfg.maps->of(op).halo, &mp = cfg.maps->of(pw).plain;
    L.pre(kind_tag);
    if (cfg.reference_sums)
        k_stencil<KIND, true><<<S.count, TILE_THREADS, NSTAGE * STAGE_BYTES, L.s>>>(g, C, S, mo, mp,
                                                                                 A, part, st);
    else
        k_stencil<KIND, false><<<S.count, TILE_THREADS, NSTAGE * STAGE_BYTES, L.s>>>(g, C, S, mo, mp,
                                                                                  A, part, st);
    L.post(kind_tag);
}

}  // namespace

Segments poisson_segments(const Grid &g, int sm_count) {
    Segments s = Segments::make(interior_box(g), sm_count * 8);
    if (s.ich > MAXCHUNK) throw std::logic_error("segment chunk exceeds MAXCHUNK");
    if (g.total >= (1LL << 31)) throw std::invalid_argument("grid too large for 32-bit cell offsets");
    return s;
}

size_t poisson_stencil_smem() { return (size_t)NSTAGE * STAGE_BYTES; }

void launch_poisson_begin(const LaunchCtx &L, KrylovState *st, long long max_it, double tol,
                          double ncell) {
    L.pre(KK_POISSON_BEGIN);
    k_begin<<<1, 1, 0, L.s>>>(st, max_it, tol, ncell);
    L.post(KK_POISSON_BEGIN);
}

static void sor_sweep(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                      const PoissonConfig &cfg, double *x, const double *rhs, double w, int color,
                      KrylovState *st) {
    StencilArgs A{x, nullptr, nullptr, w, color, 0};
    stencil_launch<SK_SOR>(L, KK_SOR_SWEEP, g, C, cfg, x, rhs, A, Partials<2>{nullptr, nullptr}, st);
}

static void jacobi_sweep(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                         const PoissonConfig &cfg, double *out, const double *in,
                         const double *rhs, KrylovState *st) {
    StencilArgs A{out, nullptr, nullptr, 0, 0, 0};
    stencil_launch<SK_JACOBI>(L, KK_JACOBI_SWEEP, g, C, cfg, in, rhs, A,
                              Partials<2>{nullptr, nullptr}, st);
}

void launch_sor_iteration(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                          const PoissonBufs &B, const PoissonConfig &cfg, Partials<1> part,
                          KrylovState *st) {
    for (int color = 0; color < 2; color++)
        sor_sweep(L, g, C, cfg, B.x, B.b, cfg.relax, color, st);
    double *rs = cfg.reference_sums ? B.r : nullptr;
    StencilArgs A{rs, nullptr, nullptr, 0, 0, !cfg.reference_sums};
    stencil_launch<SK_RESIDUAL>(L, KK_RESIDUAL_NORM, g, C, cfg, B.x, B.b, A,
                                Partials<2>{part.buf, part.ticket}, st);
    if (rs) seq_launch(L, g, SEQ_RESIDUAL, B.r, B.r, nullptr, nullptr, st);
}

void launch_jacobi_iteration(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                             const PoissonBufs &B, const PoissonConfig &cfg, Partials<1> part,
                             KrylovState *st) {
    jacobi_sweep(L, g, C, cfg, B.tp, B.x, B.b, st);
    double *rs = cfg.reference_sums ? B.r : nullptr;
    StencilArgs A{rs, B.x, nullptr, 0, 0, !cfg.reference_sums};
    stencil_launch<SK_RESIDUAL>(L, KK_RESIDUAL_NORM, g, C, cfg, B.tp, B.b, A,
                                Partials<2>{part.buf, part.ticket}, st);
    if (rs) seq_launch(L, g, SEQ_RESIDUAL, B.r, B.r, nullptr, nullptr, st);
}

void launch_bicg_init(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                      const PoissonBufs &B, const PoissonConfig &cfg, Partials<1> part,
                      KrylovState *st) {
    StencilArgs A{B.r, B.r0, B.q, 0, 0, !cfg.reference_sums};
    stencil_launch<SK_INIT>(L, KK_BICG_INIT, g, C, cfg, B.x, B.b, A,
                            Partials<2>{part.buf, part.ticket}, st);
    if (cfg.reference_sums) seq_launch(L, g, SEQ_INIT, B.r0, B.r, nullptr, nullptr, st);
}

// Applies the preconditioner to `rhs` with the first sweep already done
// into `x` (Jacobi) or `x` zeroed (SOR); returns the buffer holding M^-1 rhs.
static double *precondition(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                            const PoissonConfig &cfg, double *x, double *tmp, const double *rhs,
                            KrylovState *st) {
    if (cfg.pc == PC_SOR) {
        for (int n = 0; n < cfg.pc_sweeps; n++)
            for (int color = 0; color < 2; color++)
                sor_sweep(L, g, C, cfg, x, rhs, cfg.pc_relax, color, st);
        return x;
    }
    double *cur = x, *nxt = tmp;
    for (int n = 1; n < cfg.pc_sweeps; n++) {
        jacobi_sweep(L, g, C, cfg, nxt, cur, rhs, st);
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
    L.pre(KK_BICG_P);
    if (seq) k_bicg_p<true><<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, B, first, st);
    else k_bicg_p<false><<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, B, first, st);
    L.post(KK_BICG_P);
    double *ppf = precondition(L, g, C, cfg, B.pp, B.tp, B.pk, st);
    StencilArgs Aq{B.q, nullptr, nullptr, 0, 0, !seq};
    stencil_launch<SK_Q>(L, KK_BICG_Q, g, C, cfg, ppf, B.r0, Aq, part, st);
    if (seq) seq_launch(L, g, SEQ_Q, B.r0, B.q, nullptr, nullptr, st);
    L.pre(KK_BICG_S);
    if (seq) k_bicg_s<true><<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, B, first, st);
    else k_bicg_s<false><<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, B, first, st);
    L.post(KK_BICG_S);
    double *ssf = precondition(L, g, C, cfg, B.ss, B.ts, B.s, st);
    StencilArgs At{B.t, nullptr, nullptr, 0, 0, !seq};
    stencil_launch<SK_T>(L, KK_BICG_T, g, C, cfg, ssf, B.s, At, part, st);
    if (seq) seq_launch(L, g, SEQ_T, B.t, B.s, B.t, B.t, st);
    L.pre(KK_BICG_XR);
    if (seq) k_bicg_xr<true><<<S.count, TILE_THREADS, 0, L.s>>>(g, S, B, ppf, ssf, seq, part, st);
    else k_bicg_xr<false><<<S.count, TILE_THREADS, 0, L.s>>>(g, S, B, ppf, ssf, seq, part, st);
    L.post(KK_BICG_XR);
    if (seq) seq_launch(L, g, SEQ_XR, B.r0, B.r, B.r, B.r, st);
}

}  // namespace dalm
