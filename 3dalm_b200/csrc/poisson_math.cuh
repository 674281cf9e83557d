// Per-cell arithmetic and the Krylov scalar updates shared by the Poisson
// kernels (poisson_v3.cu: one kernel per reference loop, in FP64 or FP32;
// poisson_fused.cu: fused FP64 BiCGStab half-iterations), so that every
// path computes a cell value with the same operations in the same order.
#pragma once

#include <cfloat>

#include "poisson.cuh"

namespace dalm {
namespace {

// Per-thread (fixed j, k) part of the coefficients, hoisted out of the march.
template <typename T>
struct ColumnCoef {
    T an, as, at, ab;                  // scaled (A[id][3..6] of the reference)
    double an_u, as_u, at_u, ab_u;     // unscaled, for the exact diagonal
    T colsum;                          // an_u + as_u + at_u + ab_u (fast variant)
};

template <typename T>
__device__ __forceinline__ ColumnCoef<T> column_coef(const PoissonCoef &C, int j, int k) {
    ColumnCoef<T> cc;
    cc.an = (T)C.an[j]; cc.as = (T)C.as[j]; cc.at = (T)C.at[k]; cc.ab = (T)C.ab[k];
    cc.an_u = C.an_u[j]; cc.as_u = C.as_u[j]; cc.at_u = C.at_u[k]; cc.ab_u = C.ab_u[k];
    cc.colsum = (T)(cc.an_u + cc.as_u + cc.at_u + cc.ab_u);
    return cc;
}

// a_c exactly as build_A assembles and scales it (src/eq.h:720-794):
// ((((((0 - ex) - aw) - an) - as) - at) - ab) / max_diag, the first two
// subtractions precomputed per i in xpart.
template <bool EXACT, typename T>
__device__ __forceinline__ T diag(T xpart, const ColumnCoef<T> &cc, const PoissonCoef &C) {
    if (EXACT) {
        double acu = (double)xpart - cc.an_u;
        acu = acu - cc.as_u;
        acu = acu - cc.at_u;
        acu = acu - cc.ab_u;
        return (T)(acu / C.max_diag);
    }
    return (xpart - cc.colsum) * (T)C.inv_max_diag;
}

// 1/a: in FP64 the hardware's approximate reciprocal refined by two
// Newton-Raphson steps (quadratic convergence); in FP32 the IEEE
// reciprocal.  a is a diagonal entry, never near zero or subnormal.
__device__ __forceinline__ double fast_rcp(double a) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
    double e = __fma_rn(-a, y, 1.0);
    y = __fma_rn(y, e, y);
    e = __fma_rn(-a, y, 1.0);
    return __fma_rn(y, e, y);
}
__device__ __forceinline__ float fast_rcp(float a) { return __frcp_rn(a); }

// A x at one cell: ac*xc + ae*xe + aw*xw + an*xn + as*xs + at*xt + ab*xb,
// left to right (src/mv.h:87, 214; src/eq.h:36, 177).
template <bool EXACT, typename T>
__device__ __forceinline__ T apply_a(T ac, T ae, T aw, const ColumnCoef<T> &cc, T xc, T xe, T xw,
                                     T xn, T xs, T xt, T xb) {
    if (EXACT)
        return ac * xc + ae * xe + aw * xw + cc.an * xn + cc.as * xs + cc.at * xt + cc.ab * xb;
    T v = ac * xc;
    v = fma(ae, xe, v);
    v = fma(aw, xw, v);
    v = fma(cc.an, xn, v);
    v = fma(cc.as, xs, v);
    v = fma(cc.at, xt, v);
    return fma(cc.ab, xb, v);
}

// (b - ax)/ac, the Jacobi / SOR relaxation (src/eq.h:36, 177)
template <bool EXACT, typename T>
__device__ __forceinline__ T relax(T b, T ax, T ac) {
    if (EXACT) return (b - ax) / ac;
    return (b - ax) * fast_rcp(ac);
}

// ---- finishers: the scalar updates after each global sum -----------------

// Inner solves of iterative refinement (guard set) only: a non-finite (for
// omega also a zero) scalar ends the solve as a breakdown, and its
// correction is discarded.
__device__ __forceinline__ bool broke_down(KrylovState *st, double v, bool zero_too = false) {
    if (!st->guard || (isfinite(v) && !(zero_too && v == 0.0))) return false;
    st->breakdown = 1;
    st->done = 1;
    return true;
}

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
__device__ __forceinline__ void fin_q(KrylovState *st, double r0q) {
    st->alpha = st->rho / r0q;
    broke_down(st, st->alpha);
}
// omega = <t, s> / <t, t> (src/eq.h:383)
__device__ __forceinline__ void fin_t(KrylovState *st, double ts, double tt) {
    st->omega = ts / tt;
    broke_down(st, st->omega, true);
}
// rhoold = rho; err = ||r||/sqrt(N); it++; loop test; next rho, breakdown
// test and beta (src/eq.h:397-401, 349-358)
__device__ __forceinline__ void fin_xr(KrylovState *st, double r0r, double rr) {
    st->rho_old = st->rho;
    st->err = sqrt(rr) / sqrt(st->ncell);
    st->it += 1;
    if (broke_down(st, st->err)) return;
    if (!(st->it < st->max_it && st->err > st->tol)) {
        st->done = 1;
    } else {
        st->rho = r0r;
        if (fabs(r0r) < FLT_MIN) {
            st->err = r0r;
            st->done = 1;
        } else {
            st->beta = (r0r / st->rho_old) * (st->alpha / st->omega);
            broke_down(st, st->beta);
        }
    }
}
// Iterative refinement: the FP64 residual r = b - A x decides whether the
// solve is done; otherwise the next inner solve A e = r starts from e = 0
// with rho = <r, r> (of the FP32 r) and a tolerance relative to |r|.
__device__ __forceinline__ void fin_refine(KrylovState *outer, KrylovState *inner, double r2,
                                           double rr32) {
    outer->err = sqrt(r2) / sqrt(outer->ncell);
    outer->it += inner->it;
    inner->it = 0;
    if (!(outer->err > outer->tol) || outer->outer_it >= outer->max_outer ||
        outer->it >= outer->max_it) {
        outer->done = 1;
        inner->done = 1;
        return;
    }
    inner->rho = rr32;
    inner->rho_old = 1;
    inner->alpha = 1;
    inner->omega = 1;
    inner->beta = 0;
    inner->err = 0;
    inner->tol = fmax(outer->inner_rtol * outer->err, 0.3 * outer->tol);
    // the case's iteration cap counts every inner iteration
    inner->max_it = min(outer->max_it - outer->it, outer->inner_cap);
    inner->ncell = outer->ncell;
    inner->done = fabs(rr32) < FLT_MIN ? 1 : 0;
}

}  // namespace
}  // namespace dalm
