// Pressure Poisson solvers (src/eq.h, src/mv.h) with matrix-free
// coefficients and on-device loop control, one kernel per reference loop.
// Vectors are FP64 (the reference's precision) or, for the inner solves of
// iterative refinement, FP32; global sums and Krylov scalars are always
// FP64.
//
// Two arithmetic variants of every FP64 kernel (template flag EXACT):
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
// kernels stage each plane of their operand (one-cell halo in j, 16 bytes of
// halo in k) and of their point-wise input in shared memory with TMA
// (cp.async.bulk.tensor), NSTAGE planes deep, and compute PPP planes per
// pass, so the loads of the next planes are in flight while the current
// ones are computed.
#include <cfloat>
#include <type_traits>

#include "poisson.cuh"
#include "poisson_math.cuh"

namespace dalm {

namespace {

template <typename T>
constexpr bool kF64 = std::is_same<T, double>::value;

// Calls f(std::true_type) for the exact variant (FP64 with reference-order
// sums), else f(std::false_type); FP32 never instantiates the exact one.
template <typename T, typename F>
void with_exact(bool exact, F &&f) {
    if constexpr (kF64<T>) {
        if (exact) {
            f(std::true_type{});
            return;
        }
    }
    f(std::false_type{});
}

// the profiling kind of an FP64 kernel kind for element type T
template <typename T>
int kk(int k) {
    if constexpr (kF64<T>) return k;
    switch (k) {
    case KK_SOR_SWEEP: return KK_SOR_SWEEP32;
    case KK_JACOBI_SWEEP: return KK_JACOBI_SWEEP32;
    case KK_BICG_P: return KK_BICG_P32;
    case KK_BICG_Q: return KK_BICG_Q32;
    case KK_BICG_S: return KK_BICG_S32;
    case KK_BICG_T: return KK_BICG_T32;
    case KK_BICG_XR: return KK_BICG_XR32;
    default: return k;
    }
}

#define SEGMENT_LOOP(S)                                                   \
    for (int u = blockIdx.x; u < (S).count; u += gridDim.x) {             \
        int i0, i1, j, k;                                                 \
        if (!(S).column(u, i0, i1, j, k)) continue;                       \
        long long c0 = g.at(i0, j, k);

#define SEGMENT_END }

__global__ void k_begin(KrylovState *st, long long max_it, double tol, double ncell,
                        long long max_outer, double inner_rtol, long long inner_cap, int guard) {
    st->rho = 0; st->rho_old = 1; st->alpha = 1; st->omega = 1; st->beta = 0; st->err = 0;
    st->ncell = ncell; st->tol = tol; st->it = 0; st->max_it = max_it; st->done = 0;
    st->wait_error = 0; st->outer_it = 0; st->max_outer = max_outer; st->inner_rtol = inner_rtol;
    st->inner_cap = inner_cap; st->guard = guard; st->breakdown = 0;
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
template <bool EXACT, typename T>
__global__ void __launch_bounds__(TILE_THREADS)
k_bicg_p(Grid g, PoissonCoef C, Segments S, PoissonBufsT<T> B, int first_sweep,
         const KrylovState *st) {
    if (st->done) return;
    const bool first = (st->it == 0);
    const T beta = (T)st->beta, omega = (T)st->omega;
    SEGMENT_LOOP(S)
    ColumnCoef<T> cc = column_coef<T>(C, j, k);
    long long c = c0;
    for (int i = i0; i < i1; i++, c += g.sx) {
        T pv = first ? B.r[c]
                     : (EXACT ? B.r[c] + beta * (B.pk[c] - omega * B.q[c])
                              : fma(beta, fma(-omega, B.q[c], B.pk[c]), B.r[c]));
        B.pk[c] = pv;
        if (!first_sweep) {
            B.pp[c] = (T)0;
        } else {
            T ac = diag<EXACT, T>((T)C.xpart[i], cc, C);
            B.pp[c] = EXACT ? (T)0 + (pv - (T)0) / ac : pv * fast_rcp(ac);
        }
    }
    SEGMENT_END
}

// s = r - alpha q (src/eq.h:373-377) with the same first-sweep fusion.
template <bool EXACT, typename T>
__global__ void __launch_bounds__(TILE_THREADS)
k_bicg_s(Grid g, PoissonCoef C, Segments S, PoissonBufsT<T> B, int first_sweep,
         const KrylovState *st) {
    if (st->done) return;
    const T alpha = (T)st->alpha;
    // distinct vectors, so the march may batch loads across planes (C4:
    // 11.0 against 11.4 ms per step; the same form measured slower for
    // k_bicg_p and k_bicg_xr, which keep the plain loop)
    const T *__restrict__ r = B.r, *__restrict__ q = B.q;
    T *__restrict__ sp = B.s, *__restrict__ ssp = B.ss;
    SEGMENT_LOOP(S)
    ColumnCoef<T> cc = column_coef<T>(C, j, k);
    long long c = c0;
#pragma unroll 4
    for (int i = i0; i < i1; i++, c += g.sx) {
        T sv = EXACT ? r[c] - alpha * q[c] : fma(-alpha, q[c], r[c]);
        sp[c] = sv;
        if (!first_sweep) {
            ssp[c] = (T)0;
        } else {
            T ac = diag<EXACT, T>((T)C.xpart[i], cc, C);
            ssp[c] = EXACT ? (T)0 + (sv - (T)0) / ac : sv * fast_rcp(ac);
        }
    }
    SEGMENT_END
}

// x += alpha pp + omega ss; r = s - omega t (src/eq.h:385-395) with
// <r0, r> and <r, r> (FP64 sums) for the finisher.  An inner solve of
// iterative refinement (guard set) starts from x = 0: its first update
// ignores the x left by the previous solve.
template <bool EXACT, typename T>
__global__ void __launch_bounds__(TILE_THREADS)
k_bicg_xr(Grid g, Segments S, PoissonBufsT<T> B, const T *ppf, const T *ssf, int seq,
          Partials<2> part, KrylovState *st) {
    if (st->done) return;
    const T alpha = (T)st->alpha, omega = (T)st->omega;
    const bool restart = st->guard && st->it == 0;
    double r0r = 0, rr = 0;
    SEGMENT_LOOP(S)
    long long c = c0;
    for (int i = i0; i < i1; i++, c += g.sx) {
        const T x0 = restart ? (T)0 : B.x[c];
        T rv;
        if (EXACT) {
            B.x[c] = x0 + alpha * ppf[c] + omega * ssf[c];
            rv = B.s[c] - omega * B.t[c];
        } else {
            B.x[c] = fma(omega, ssf[c], fma(alpha, ppf[c], x0));
            rv = fma(-omega, B.t[c], B.s[c]);
        }
        B.r[c] = rv;
        r0r += (double)B.r0[c] * (double)rv;
        rr += (double)rv * (double)rv;
    }
    SEGMENT_END
    if (seq) return;
    double vals[2] = {r0r, rr};
    if (grid_reduce<2>(vals, 0u, part) && threadIdx.x == 0) fin_xr(st, vals[0], vals[1]);
}

// x += sign * e (FP64 accumulation of the FP32 refinement correction)
__global__ void __launch_bounds__(TILE_THREADS)
k_refine_update(Grid g, Segments S, double *x, const float *e, double sign) {
    SEGMENT_LOOP(S)
    long long c = c0;
    for (int i = i0; i < i1; i++, c += g.sx) x[c] = fma(sign, (double)e[c], x[c]);
    SEGMENT_END
}

// ------------------------------------------------------- TMA stencil sweeps

constexpr int NSTAGE = 8;  // TMA ring depth (planes)
constexpr int PPP = 3;     // planes computed per pass (one block barrier each);
                           // 3 measured ~1 % faster over the C4 step than 2, and
                           // 4 with a 10-stage ring slower (3 blocks per SM)
constexpr int MAXCHUNK = 32;  // Segments caps a chunk at 32 planes

// shared-memory geometry of one ring stage for element type T
template <typename T>
struct Geo {
    static constexpr int HK = 16 / (int)sizeof(T);   // halo in k: 16 bytes
    static constexpr int TKW = TK + 2 * HK;
    static constexpr int TJW = TJ + 2;
    static constexpr int OP_BYTES = TKW * TJW * (int)sizeof(T);
    static constexpr int OP_PAD = ((OP_BYTES + 127) / 128) * 128;
    static constexpr int PW_BYTES = TK * TJ * (int)sizeof(T);
    static constexpr int STAGE = OP_PAD + PW_BYTES;
};

enum StencilKind {
    SK_JACOBI = 0,    // out = x + (rhs - A x)/ac          sweep_jacobi_at_cell, src/eq.h:6-39
    SK_RESIDUAL = 1,  // sum (b - A x)^2 [, r stored] [, x copied]   src/mv.h:33-182
    SK_INIT = 2,      // r = r0 = b - A x, q = 0, sum r*r         src/eq.h:342-353
    SK_Q = 3,         // q = A pp, sum r0*q                       src/eq.h:369-371
    SK_T = 4,         // t = A ss, sum t*s, sum t*t               src/eq.h:381-383
    SK_SOR = 5,       // red-black update in place                src/eq.h:145-181
    SK_REFINE = 6     // FP64 r = b - A x; FP32 inner r [= r0, q = 0]; sums r*r
};

struct StencilArgs {
    void *out;      // JACOBI out, RESIDUAL r (or null), INIT r, Q q, T t, SOR x, REFINE r32
    void *out2;     // RESIDUAL copy target (or null), INIT r0, REFINE r0_32
    void *out3;     // INIT q, REFINE q32
    double w;       // SOR relaxation
    int color;      // SOR colour
    int reduce;     // 0: no tree reduction (the reference-order path sums)
    KrylovState *st2;  // REFINE: the inner solve's state
};

// One block = one column segment.  Load L (0 <= L < nplanes + 2) brings
// plane i0 - 1 + L of the operand (halo box) and, for the planes the block
// computes, of the point-wise input (plain box) into ring stage L % NSTAGE.
// Plane i0 + n is computed from loads n, n + 1, n + 2.  Each pass computes
// PPP planes and then refills the PPP stages it released.
template <int KIND, bool EXACT, typename T>
__global__ void __launch_bounds__(TILE_THREADS)
k_stencil(Grid g, PoissonCoef C, Segments S, const __grid_constant__ CUtensorMap m_op,
          const __grid_constant__ CUtensorMap m_pw, StencilArgs A, Partials<2> part,
          KrylovState *st) {
    using G = Geo<T>;
    if (KIND != SK_INIT && st->done) return;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) unsigned long long bar[NSTAGE];
    __shared__ T s_ae[MAXCHUNK], s_aw[MAXCHUNK], s_xp[MAXCHUNK];
    const int u = blockIdx.x;
    int i0, i1, j, k;
    const bool active = S.column(u, i0, i1, j, k);
    const int col = u % S.ncol;
    const int k0 = S.box.lo[2] + (col % S.ntk) * TK, j0 = S.box.lo[1] + (col / S.ntk) * TJ;
    const int nplanes = i1 - i0, nload = nplanes + 2;
    const int xo = k0 - G::HK + (int)g.off, xp = k0 + (int)g.off;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    if (threadIdx.x == 0) {
        for (int s = 0; s < NSTAGE; s++) mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    if (threadIdx.x < nplanes) {
        s_ae[threadIdx.x] = (T)C.ae[i0 + threadIdx.x];
        s_aw[threadIdx.x] = (T)C.aw[i0 + threadIdx.x];
        s_xp[threadIdx.x] = (T)C.xpart[i0 + threadIdx.x];
    }
    __syncthreads();
    auto issue = [&](int L) {
        int s = L % NSTAGE;
        unsigned char *base = smem + s * G::STAGE;
        bool pw = (L >= 1 && L <= nplanes);
        mbar_expect_tx(&bar[s], G::OP_BYTES + (pw ? G::PW_BYTES : 0));
        tma_load_3d(base, &m_op, xo, j0 - 1, i0 - 1 + L, &bar[s]);
        if (pw) tma_load_3d(base + G::OP_PAD, &m_pw, xp, j0, i0 - 1 + L, &bar[s]);
    };
    int issued = 0;
    if (threadIdx.x == 0)
        for (; issued < NSTAGE && issued < nload; issued++) issue(issued);

    ColumnCoef<T> cc;
    if (active) cc = column_coef<T>(C, j, k);
    const int idx = (warp + 1) * G::TKW + lane + G::HK;
    const int sx = (int)g.sx;
    const int cbase = active ? (int)g.at(i0, j, k) : 0;
    double acc0 = 0, acc1 = 0;

    // one cell of plane i0 + nn
    auto cell = [&](int nn) {
        const T *W = (const T *)(smem + (nn % NSTAGE) * G::STAGE);
        const T *Cp = (const T *)(smem + ((nn + 1) % NSTAGE) * G::STAGE);
        const T *E = (const T *)(smem + ((nn + 2) % NSTAGE) * G::STAGE);
        const T pw = ((const T *)((const unsigned char *)Cp + G::OP_PAD))[warp * TK + lane];
        const int c = cbase + nn * sx;
        const T xc = Cp[idx];
        const T ac = diag<EXACT, T>(s_xp[nn], cc, C);
        const T ax = apply_a<EXACT, T>(ac, s_ae[nn], s_aw[nn], cc, xc, E[idx], W[idx],
                                       Cp[idx + G::TKW], Cp[idx - G::TKW], Cp[idx + 1], Cp[idx - 1]);
        if (KIND == SK_JACOBI) {
            ((T *)A.out)[c] = xc + relax<EXACT, T>(pw, ax, ac);
        } else if (KIND == SK_RESIDUAL) {
            T r = pw - ax;
            acc0 += (double)r * (double)r;
            if (A.out) ((T *)A.out)[c] = r;
            if (A.out2) ((T *)A.out2)[c] = xc;
        } else if (KIND == SK_INIT) {
            T r = pw - ax;
            ((T *)A.out)[c] = r;
            ((T *)A.out2)[c] = r;
            ((T *)A.out3)[c] = (T)0;
            acc0 += (double)r * (double)r;
        } else if (KIND == SK_Q) {
            ((T *)A.out)[c] = ax;
            acc0 += (double)pw * (double)ax;
        } else if (KIND == SK_T) {
            ((T *)A.out)[c] = ax;
            acc0 += (double)ax * (double)pw;
            acc1 += (double)ax * (double)ax;
        } else if (KIND == SK_SOR) {
            const int i = i0 + nn;
            if (((i + j + k) & 1) == A.color) {
                T rel = relax<EXACT, T>(pw, ax, ac);
                ((T *)A.out)[c] = EXACT ? xc + (T)A.w * rel : fma((T)A.w, rel, xc);
            }
        } else if (KIND == SK_REFINE) {
            const double r = (double)pw - (double)ax;
            const float r32 = (float)r;
            ((float *)A.out)[c] = r32;
            if (A.out2) ((float *)A.out2)[c] = r32;  // BiCGStab inner solves only
            if (A.out3) ((float *)A.out3)[c] = 0.f;
            acc0 += r * r;
            acc1 += (double)r32 * (double)r32;
        }
    };

    int waited = 0;
    bool fail = false;
    for (int n = 0; n < nplanes; n += PPP) {
        const int m = nplanes - n < PPP ? nplanes - n : PPP;
        while (!fail && waited <= n + m + 1) {
            fail = !mbar_wait(&bar[waited % NSTAGE], (unsigned)((waited / NSTAGE) & 1));
            if (!fail) waited++;
        }
        if (!fail && active) {
#pragma unroll
            for (int q = 0; q < PPP; q++)
                if (q < m) cell(n + q);
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
        if (KIND == SK_REFINE) fin_refine(st, A.st2, vals[0], vals[1]);
    }
}

// Two Jacobi sweeps in one pass over HBM (FP64): out = J(J(x)), J the
// sweep of k_stencil<SK_JACOBI> with right-hand side rhs.  A block marches
// its column segment through i; per plane it computes the first sweep on
// the tile and a one-cell ring around it (34 x 10 cells, from x staged by
// TMA in the wide box, 40 x 14, and rhs in the halo box, 36 x 10) into a
// four-plane shared ring, and the second sweep on the tile one plane
// behind.  The ring cells of the first sweep are recomputed by each block
// that needs them (the unfused pair writes and re-reads the whole
// intermediate vector instead): 3 vectors per cell instead of 6.  The
// intermediate is zero outside the interior, as the unfused pair's scratch
// vector is (its guide cells are never written), and every cell value comes
// from the same diag / apply_a / relax as k_stencil's, so the result is the
// unfused pair's bit for bit, in both arithmetic variants.
//
// Load L (0 <= L < nplanes + 4) brings x plane i0 - 2 + L and, for
// 1 <= L <= nplanes + 2, rhs plane i0 - 2 + L into stage L % J2_STAGES.
// First sweep at plane i0 - 1 + a reads x loads a .. a + 2 and rhs load
// a + 1; the second sweep at plane i0 + b reads first-sweep planes b .. b + 2
// and rhs load b + 2.  Iteration a computes first-sweep plane a, then (one
// barrier later) second-sweep plane a - 2, and refills the stage of load
// a - 1, whose last reader ran before that barrier.
constexpr int J2_STAGES = 6;
constexpr int J2_WK = TK + 2 * WIDE_HK, J2_WJ = TJ + 2 * WIDE_HJ;  // x box: 40 x 14
constexpr int J2_HK = 2, J2_HKW = TK + 2 * J2_HK, J2_HJW = TJ + 2;  // rhs / ring: 36 x 10
constexpr int J2_XB = J2_WK * J2_WJ * 8, J2_RB = J2_HKW * J2_HJW * 8;
constexpr int J2_RBP = ((J2_RB + 127) / 128) * 128;  // stages stay 128-byte aligned
constexpr int J2_STAGE = J2_XB + J2_RBP;
constexpr int J2_RING = 2 * (TK + 2) + 2 * TJ;  // 84 cells around the tile
constexpr int J2_SMEM = J2_STAGES * J2_STAGE + 4 * J2_RB;
static_assert(J2_XB % 128 == 0 && J2_STAGE % 128 == 0, "TMA destinations 128-byte aligned");
static_assert(J2_RING <= TILE_THREADS, "one ring cell per thread at most");

// the q-th ring cell (0 <= q < 84) relative to the tile origin: rows -1 and
// 8 over columns -1 .. 32, then columns -1 and 32 of rows 0 .. 7
__device__ __forceinline__ void j2_ring_cell(int q, int &jj, int &kk) {
    if (q < 2 * (TK + 2)) {
        jj = q < TK + 2 ? -1 : TJ;
        kk = (q < TK + 2 ? q : q - (TK + 2)) - 1;
    } else {
        const int t = q - 2 * (TK + 2);
        jj = t >> 1;
        kk = (t & 1) ? TK : -1;
    }
}

template <bool EXACT>
__global__ void __launch_bounds__(TILE_THREADS)
k_jacobi2(Grid g, PoissonCoef C, Segments S, const __grid_constant__ CUtensorMap m_x,
          const __grid_constant__ CUtensorMap m_rhs, double *out, KrylovState *st) {
    using T = double;
    if (st->done) return;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) unsigned long long bar[J2_STAGES];
    const int u = blockIdx.x;
    int i0, i1, j, k;
    const bool active = S.column(u, i0, i1, j, k);
    const int col = u % S.ncol;
    const int k0 = S.box.lo[2] + (col % S.ntk) * TK, j0 = S.box.lo[1] + (col / S.ntk) * TJ;
    const int nplanes = i1 - i0, nload = nplanes + 4;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gc = g.gc;
    T *ring = (T *)(smem + J2_STAGES * J2_STAGE);  // four first-sweep planes, 36 x 10 each
    // per-plane coefficients of planes i0 - 1 .. i1 (index a = plane - i0 + 1)
    __shared__ T s_xp[MAXCHUNK + 2], s_ae[MAXCHUNK + 2], s_aw[MAXCHUNK + 2];

    if (threadIdx.x == 0) {
        for (int s = 0; s < J2_STAGES; s++) mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    if (threadIdx.x < nplanes + 2) {
        const int ip = i0 - 1 + threadIdx.x;
        const bool in = ip >= gc && ip < g.nx - gc;
        s_xp[threadIdx.x] = in ? (T)C.xpart[ip] : (T)0;
        s_ae[threadIdx.x] = in ? (T)C.ae[ip] : (T)0;
        s_aw[threadIdx.x] = in ? (T)C.aw[ip] : (T)0;
    }
    __syncthreads();
    auto issue = [&](int L) {
        const int s = L % J2_STAGES;
        unsigned char *base = smem + s * J2_STAGE;
        const bool rhs = L >= 1 && L <= nplanes + 2;
        mbar_expect_tx(&bar[s], J2_XB + (rhs ? J2_RB : 0));
        tma_load_3d(base, &m_x, k0 - WIDE_HK + (int)g.off, j0 - WIDE_HJ, i0 - 2 + L, &bar[s]);
        if (rhs)
            tma_load_3d(base + J2_XB, &m_rhs, k0 - J2_HK + (int)g.off, j0 - 1, i0 - 2 + L, &bar[s]);
    };
    int issued = 0;
    if (threadIdx.x == 0)
        for (; issued < J2_STAGES && issued < nload; issued++) issue(issued);

    // this thread's cells of the first sweep: the tile cell and at most one
    // ring cell, relative to (j0, k0)
    int rj = 0, rk = 0;
    const bool has_ring = threadIdx.x < J2_RING;
    if (has_ring) j2_ring_cell(threadIdx.x, rj, rk);
    auto interior_jk = [&](int jj, int kk) {
        const int jg = j0 + jj, kg = k0 + kk;
        return jg >= gc && jg < g.ny - gc && kg >= gc && kg < g.nz - gc;
    };
    const bool tile_in = interior_jk(warp, lane), ring_in = has_ring && interior_jk(rj, rk);
    ColumnCoef<T> cc{}, cr{};
    if (tile_in) cc = column_coef<T>(C, j0 + warp, k0 + lane);
    if (ring_in) cr = column_coef<T>(C, j0 + rj, k0 + rk);
    const int sx = (int)g.sx;
    const int cbase = active ? (int)g.at(i0, j, k) : 0;

    // one cell of a sweep at plane index a (plane i0 - 1 + a) with diagonal
    // ac: x values from the planes W, Cp, E at index xi (row stride rs), rhs
    // at rh[ri]; relax<EXACT>'s arithmetic, with 1/ac (fast variant) given
    auto sweep = [&](int a, T ac, T rac, const ColumnCoef<T> &c, const T *W, const T *Cp,
                     const T *E, int xi, int rs, const T *rh, int ri) {
        const T xc = Cp[xi];
        const T ax = apply_a<EXACT, T>(ac, s_ae[a], s_aw[a], c, xc, E[xi], W[xi], Cp[xi + rs],
                                       Cp[xi - rs], Cp[xi + 1], Cp[xi - 1]);
        return xc + (EXACT ? relax<true, T>(rh[ri], ax, ac) : (rh[ri] - ax) * rac);
    };
    auto inv = [](T ac) { return EXACT ? (T)0 : fast_rcp(ac); };
    T ac_prev = 0, rac_prev = 0;  // the tile cell's diagonal at the previous iteration's plane
    auto xplane = [&](int L) { return (const T *)(smem + (L % J2_STAGES) * J2_STAGE); };
    auto rplane = [&](int L) { return (const T *)(smem + (L % J2_STAGES) * J2_STAGE + J2_XB); };
    auto xidx = [](int jj, int kk) { return (jj + WIDE_HJ) * J2_WK + kk + WIDE_HK; };
    auto hidx = [](int jj, int kk) { return (jj + 1) * J2_HKW + kk + J2_HK; };

    int waited = 0;
    bool fail = false;
    for (int a = 0; a < nplanes + 2; a++) {
        while (!fail && waited <= a + 2) {
            fail = !mbar_wait(&bar[waited % J2_STAGES], (unsigned)((waited / J2_STAGES) & 1));
            if (!fail) waited++;
        }
        // the tile cell's diagonal at first-sweep plane a (the second sweep
        // reaches this plane in the next iteration)
        const T ac = diag<EXACT, T>(s_xp[a], cc, C), rac = inv(ac);
        if (!fail) {
            // first sweep at plane i0 - 1 + a into ring slot a % 4
            const int ip = i0 - 1 + a;
            const bool plane_in = ip >= gc && ip < g.nx - gc;
            T *R = ring + (a & 3) * (J2_HKW * J2_HJW);
            const T *W = xplane(a), *Cp = xplane(a + 1), *E = xplane(a + 2), *rh = rplane(a + 1);
            R[hidx(warp, lane)] = (plane_in && tile_in)
                                      ? sweep(a, ac, rac, cc, W, Cp, E, xidx(warp, lane), J2_WK, rh,
                                              hidx(warp, lane))
                                      : (T)0;
            if (has_ring) {
                T v = (T)0;
                if (plane_in && ring_in) {
                    const T acr = diag<EXACT, T>(s_xp[a], cr, C);
                    v = sweep(a, acr, inv(acr), cr, W, Cp, E, xidx(rj, rk), J2_WK, rh, hidx(rj, rk));
                }
                R[hidx(rj, rk)] = v;
            }
        }
        if (__syncthreads_or(fail)) break;
        if (a >= 2 && active) {
            // second sweep at plane i0 + b, b = a - 2 (first-sweep plane index b + 1)
            const int b = a - 2;
            const T *Aw = ring + (b & 3) * (J2_HKW * J2_HJW);
            const T *Ac = ring + ((b + 1) & 3) * (J2_HKW * J2_HJW);
            const T *Ae = ring + ((b + 2) & 3) * (J2_HKW * J2_HJW);
            out[cbase + b * sx] = sweep(b + 1, ac_prev, rac_prev, cc, Aw, Ac, Ae, hidx(warp, lane),
                                        J2_HKW, rplane(b + 2), hidx(warp, lane));
        }
        ac_prev = ac;
        rac_prev = rac;
        if (threadIdx.x == 0 && a >= 1 && issued < nload) {
            fence_proxy_async();  // the released stage was read through the generic proxy
            issue(issued++);
        }
    }
    if (__syncthreads_or(fail)) {
        // a bounded wait ran out: report, drain what is still in flight, stop
        if (threadIdx.x == 0) {
            st->wait_error = 1;
            st->done = 1;
            for (int L = waited; L < issued; L++)
                mbar_wait(&bar[L % J2_STAGES], (unsigned)((L / J2_STAGES) & 1));
        }
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

template <int KIND, typename T>
void stencil_launch(const LaunchCtx &L, int kind_tag, const Grid &g, const PoissonCoef &C,
                    const PoissonConfig &cfg, const T *op, const T *pw, const StencilArgs &A,
                    Partials<2> part, KrylovState *st) {
    const Segments &S = cfg.seg;
    const CUtensorMap &mo = cfg.maps->of(op).halo, &mp = cfg.maps->of(pw).plain;
    const size_t smem = (size_t)NSTAGE * Geo<T>::STAGE;
    L.pre(kind_tag);
    with_exact<T>(cfg.reference_sums != 0, [&](auto ex) {
        auto kern = k_stencil<KIND, decltype(ex)::value, T>;
        if (smem > 48 * 1024)
            DALM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<S.count, TILE_THREADS, smem, L.s>>>(g, C, S, mo, mp, A, part, st);
    });
    L.post(kind_tag);
}

template <typename T>
void sor_sweep(const LaunchCtx &L, const Grid &g, const PoissonCoef &C, const PoissonConfig &cfg,
               T *x, const T *rhs, double w, int color, KrylovState *st) {
    StencilArgs A{x, nullptr, nullptr, w, color, 0, nullptr};
    stencil_launch<SK_SOR, T>(L, kk<T>(KK_SOR_SWEEP), g, C, cfg, x, rhs, A,
                              Partials<2>{nullptr, nullptr}, st);
}

template <typename T>
void jacobi_sweep(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                  const PoissonConfig &cfg, T *out, const T *in, const T *rhs, KrylovState *st) {
    StencilArgs A{out, nullptr, nullptr, 0, 0, 0, nullptr};
    stencil_launch<SK_JACOBI, T>(L, kk<T>(KK_JACOBI_SWEEP), g, C, cfg, in, rhs, A,
                                 Partials<2>{nullptr, nullptr}, st);
}

// Applies the preconditioner to `rhs` with the first sweep already done
// into `x` (Jacobi) or `x` zeroed (SOR); returns the buffer holding M^-1 rhs.
template <typename T>
T *precondition(const LaunchCtx &L, const Grid &g, const PoissonCoef &C, const PoissonConfig &cfg,
                T *x, T *tmp, const T *rhs, KrylovState *st) {
    if (cfg.pc == PC_SOR) {
        for (int n = 0; n < cfg.pc_sweeps; n++)
            for (int color = 0; color < 2; color++)
                sor_sweep<T>(L, g, C, cfg, x, rhs, cfg.pc_relax, color, st);
        return x;
    }
    if constexpr (kF64<T>) {
        if (cfg.jacobi2 && cfg.pc_sweeps == 3) {  // the last two sweeps in one pass: M^-1 rhs into tmp
            const Segments &S = cfg.seg;
            const CUtensorMap &mx = cfg.maps->of(x).wide, &mr = cfg.maps->of(rhs).halo;
            L.pre(KK_JACOBI_SWEEP2);
            with_exact<T>(cfg.reference_sums != 0, [&](auto ex) {
                auto kern = k_jacobi2<decltype(ex)::value>;
                DALM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, J2_SMEM));
                kern<<<S.count, TILE_THREADS, J2_SMEM, L.s>>>(g, C, S, mx, mr, tmp, st);
            });
            L.post(KK_JACOBI_SWEEP2);
            return tmp;
        }
    }
    T *cur = x, *nxt = tmp;
    for (int n = 1; n < cfg.pc_sweeps; n++) {
        jacobi_sweep<T>(L, g, C, cfg, nxt, cur, rhs, st);
        T *t = cur;
        cur = nxt;
        nxt = t;
    }
    return cur;
}

}  // namespace

Segments poisson_segments(const Grid &g, int sm_count) {
    Segments s = Segments::make(interior_box(g), sm_count * 8);
    if (s.ich > MAXCHUNK) throw std::logic_error("segment chunk exceeds MAXCHUNK");
    if (g.total >= (1LL << 31)) throw std::invalid_argument("grid too large for 32-bit cell offsets");
    return s;
}

void launch_poisson_begin(const LaunchCtx &L, KrylovState *st, long long max_it, double tol,
                          double ncell, long long max_outer, double inner_rtol,
                          long long inner_cap, int guard) {
    L.pre(KK_POISSON_BEGIN);
    k_begin<<<1, 1, 0, L.s>>>(st, max_it, tol, ncell, max_outer, inner_rtol, inner_cap, guard);
    L.post(KK_POISSON_BEGIN);
}

void launch_sor_iteration(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                          const PoissonBufs &B, const PoissonConfig &cfg, Partials<1> part,
                          KrylovState *st) {
    for (int color = 0; color < 2; color++)
        sor_sweep<double>(L, g, C, cfg, B.x, B.b, cfg.relax, color, st);
    double *rs = cfg.reference_sums ? B.r : nullptr;
    StencilArgs A{rs, nullptr, nullptr, 0, 0, !cfg.reference_sums, nullptr};
    stencil_launch<SK_RESIDUAL, double>(L, KK_RESIDUAL_NORM, g, C, cfg, B.x, B.b, A,
                                        Partials<2>{part.buf, part.ticket}, st);
    if (rs) seq_launch(L, g, SEQ_RESIDUAL, B.r, B.r, nullptr, nullptr, st);
}

void launch_jacobi_iteration(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                             const PoissonBufs &B, const PoissonConfig &cfg, Partials<1> part,
                             KrylovState *st) {
    jacobi_sweep<double>(L, g, C, cfg, B.tp, B.x, B.b, st);
    double *rs = cfg.reference_sums ? B.r : nullptr;
    StencilArgs A{rs, B.x, nullptr, 0, 0, !cfg.reference_sums, nullptr};
    stencil_launch<SK_RESIDUAL, double>(L, KK_RESIDUAL_NORM, g, C, cfg, B.tp, B.b, A,
                                        Partials<2>{part.buf, part.ticket}, st);
    if (rs) seq_launch(L, g, SEQ_RESIDUAL, B.r, B.r, nullptr, nullptr, st);
}

void launch_bicg_init(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                      const PoissonBufs &B, const PoissonConfig &cfg, Partials<1> part,
                      KrylovState *st) {
    StencilArgs A{B.r, B.r0, B.q, 0, 0, !cfg.reference_sums, nullptr};
    stencil_launch<SK_INIT, double>(L, KK_BICG_INIT, g, C, cfg, B.x, B.b, A,
                                    Partials<2>{part.buf, part.ticket}, st);
    if (cfg.reference_sums) seq_launch(L, g, SEQ_INIT, B.r0, B.r, nullptr, nullptr, st);
}

template <typename T>
void launch_bicg_iteration(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                           const PoissonBufsT<T> &B, const PoissonConfig &cfg, Partials<2> part,
                           KrylovState *st) {
    const Segments &S = cfg.seg;
    const int first = (cfg.pc == PC_JACOBI && cfg.pc_sweeps >= 1) ? 1 : 0;
    const bool exact = kF64<T> && cfg.reference_sums;
    const int seq = exact ? 1 : 0;
    L.pre(kk<T>(KK_BICG_P));
    with_exact<T>(exact, [&](auto ex) {
        k_bicg_p<decltype(ex)::value, T><<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, B, first, st);
    });
    L.post(kk<T>(KK_BICG_P));
    T *ppf = precondition<T>(L, g, C, cfg, B.pp, B.tp, B.pk, st);
    StencilArgs Aq{B.q, nullptr, nullptr, 0, 0, !seq, nullptr};
    stencil_launch<SK_Q, T>(L, kk<T>(KK_BICG_Q), g, C, cfg, ppf, B.r0, Aq, part, st);
    if (seq) seq_launch(L, g, SEQ_Q, (const double *)B.r0, (const double *)B.q, nullptr, nullptr, st);
    L.pre(kk<T>(KK_BICG_S));
    with_exact<T>(exact, [&](auto ex) {
        k_bicg_s<decltype(ex)::value, T><<<S.count, TILE_THREADS, 0, L.s>>>(g, C, S, B, first, st);
    });
    L.post(kk<T>(KK_BICG_S));
    T *ssf = precondition<T>(L, g, C, cfg, B.ss, B.ts, B.s, st);
    StencilArgs At{B.t, nullptr, nullptr, 0, 0, !seq, nullptr};
    stencil_launch<SK_T, T>(L, kk<T>(KK_BICG_T), g, C, cfg, ssf, B.s, At, part, st);
    if (seq)
        seq_launch(L, g, SEQ_T, (const double *)B.t, (const double *)B.s, (const double *)B.t,
                   (const double *)B.t, st);
    L.pre(kk<T>(KK_BICG_XR));
    with_exact<T>(exact, [&](auto ex) {
        k_bicg_xr<decltype(ex)::value, T>
            <<<S.count, TILE_THREADS, 0, L.s>>>(g, S, B, ppf, ssf, seq, part, st);
    });
    L.post(kk<T>(KK_BICG_XR));
    if (seq)
        seq_launch(L, g, SEQ_XR, (const double *)B.r0, (const double *)B.r, (const double *)B.r,
                   (const double *)B.r, st);
}

template void launch_bicg_iteration<double>(const LaunchCtx &, const Grid &, const PoissonCoef &,
                                            const PoissonBufsT<double> &, const PoissonConfig &,
                                            Partials<2>, KrylovState *);
template void launch_bicg_iteration<float>(const LaunchCtx &, const Grid &, const PoissonCoef &,
                                           const PoissonBufsT<float> &, const PoissonConfig &,
                                           Partials<2>, KrylovState *);

void launch_bicg_xr(const LaunchCtx &L, const Grid &g, const PoissonBufs &B, const double *ppf,
                    const double *ssf, const PoissonConfig &cfg, Partials<2> part,
                    KrylovState *st) {
    L.pre(KK_BICG_XR);
    k_bicg_xr<false, double>
        <<<cfg.seg.count, TILE_THREADS, 0, L.s>>>(g, cfg.seg, B, ppf, ssf, 0, part, st);
    L.post(KK_BICG_XR);
}

void launch_refine_residual(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                            const PoissonConfig &cfg, const double *x, const double *b,
                            const PoissonBufsT<float> &inner, Partials<2> part,
                            KrylovState *outer, KrylovState *inner_st) {
    StencilArgs A{inner.r, inner.r0, inner.q, 0, 0, 1, inner_st};
    PoissonConfig fast = cfg;
    fast.reference_sums = 0;
    stencil_launch<SK_REFINE, double>(L, KK_REFINE_RESIDUAL, g, C, fast, x, b, A, part, outer);
}

void launch_refine_update(const LaunchCtx &L, const Grid &g, const PoissonConfig &cfg, double *x,
                          const float *e, double sign) {
    L.pre(KK_REFINE_UPDATE);
    k_refine_update<<<cfg.seg.count, TILE_THREADS, 0, L.s>>>(g, cfg.seg, x, e, sign);
    L.post(KK_REFINE_UPDATE);
}

}  // namespace dalm
