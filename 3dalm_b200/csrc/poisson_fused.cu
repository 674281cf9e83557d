// Fused half-iterations of the Jacobi(3)-preconditioned BiCGStab
// (run_pbicgstab, src/eq.h:333-473, fast arithmetic).
//
// One reference iteration is, per half,
//   P half: p = r + beta (p - omega q)            (src/eq.h:355-365)
//           pp = M^-1 p: Jacobi from zero, 3 sweeps (src/eq.h:367-368)
//           q = A pp, <r0, q> -> alpha            (src/eq.h:369-371)
//   S half: s = r - alpha q                       (src/eq.h:373-377)
//           ss = M^-1 s                           (src/eq.h:379-380)
//           t = A ss, <t, s>, <t, t> -> omega     (src/eq.h:381-383)
// and the unfused kernels run each statement as its own pass over HBM (5
// passes, 13-14 vectors per cell per half).  Here each half is ONE kernel:
// a block marches its column segment through i and, per plane, computes the
// point-wise update and the first sweep on a 40 x 14 box (the 32 x 8 tile
// plus a 3-cell halo in j and k), the second sweep on 36 x 12 (halo 2), the
// third on 34 x 10 (halo 1) and A pp on the tile, from shared-memory rings
// of planes; neighbours' halos are recomputed instead of being written and
// re-read.  HBM traffic per half: P reads r, p, q, r0 and writes p', pp, q'
// (7 vectors); S reads r, q and writes s, ss, t (5).  p and q are
// ping-pong buffers, because a block reads its neighbours' old p and q as
// its halo while it writes its own new ones.
//
// Every cell value is computed with the same operations in the same order
// as the unfused fast kernels (shared helpers in poisson_math.cuh); only
// the order of the global sums differs.
#include "poisson.cuh"
#include "poisson_math.cuh"

namespace dalm {

namespace {

enum FusedKind { FK_P = 0, FK_S = 1 };

constexpr int FH = 3;                     // halo: 2 stencil sweeps + the SpMV
constexpr int WK = TK + 2 * WIDE_HK;      // 40: k0 - 4 .. k0 + 35
constexpr int WJ = TJ + 2 * WIDE_HJ;      // 14: j0 - 3 .. j0 + 10
constexpr int WN = WK * WJ;               // doubles per plane buffer
constexpr int PB = WN * 8;                // bytes per plane buffer
constexpr int TB = TK * TJ * 8;           // bytes per tile plane (r0)
constexpr int NSF = 4;                    // TMA ring depth
constexpr int MAXP = 32 + 2 * FH;         // planes a block loads at most (chunks <= 32)
constexpr int NRING_A = 84, NRING_B = 92, NRING_C = 128;  // halo rings, see ring_cell
constexpr int NEXTRA = NRING_A + NRING_B + NRING_C - TILE_THREADS;  // second ring cells: 48
static_assert(WIDE_HJ == FH && WIDE_HK == 4, "the wide box must carry the halo");
static_assert((WK - 4) * (WJ - 2) - (WK - 6) * (WJ - 4) == NRING_B, "ring sizes");

template <int KIND>
struct FusedGeo {
    static constexpr int NIN = KIND == FK_P ? 3 : 2;   // wide inputs per plane
    static constexpr int STAGE = NIN * PB + (KIND == FK_P ? TB : 0);
    // + w1, w2, w3 planes (two each) and 1/ac planes (three)
    static constexpr int SMEM = NSF * STAGE + (3 * 2 + 3) * PB;
};

struct FusedArgs {
    double *v_out;   // P: new p;  S: s
    double *w_out;   // P: pp;     S: ss
    double *av_out;  // P: new q;  S: t
};

// The q-th cell (0 <= q < 304) of the halo rings around the 32 x 8 tile in
// the 40 x 14 box, ordered by how many phases need it: ring A (the border
// of the 34 x 10 box: phases 1-3), ring B (border of 36 x 12: phases 1-2),
// ring C (the rest: phase 1).  Returns (row, column) and the ring (0-2).
__device__ __forceinline__ void ring_cell(int q, int &r, int &c, int &ring) {
    if (q < NRING_A) {             // rows 2, 11 (34 wide from column 3); columns 3, 36
        ring = 0;
        if (q < 68) { r = q < 34 ? 2 : 11; c = 3 + (q < 34 ? q : q - 34); }
        else { const int s = q - 68; r = 3 + (s >> 1); c = (s & 1) ? 36 : 3; }
    } else if (q < NRING_A + NRING_B) {   // rows 1, 12 (36 wide from column 2); columns 2, 37
        ring = 1;
        const int s = q - NRING_A;
        if (s < 72) { r = s < 36 ? 1 : 12; c = 2 + (s < 36 ? s : s - 36); }
        else { const int t = s - 72; r = 2 + (t >> 1); c = (t & 1) ? 37 : 2; }
    } else {                       // rows 0, 13 (all 40); columns 0, 1, 38, 39 of rows 1-12
        ring = 2;
        const int s = q - NRING_A - NRING_B;
        if (s < 80) { r = s < 40 ? 0 : 13; c = s < 40 ? s : s - 40; }
        else { const int t = s - 80, m = t & 3; r = 1 + (t >> 2); c = m < 2 ? m : 36 + m; }
    }
}

// Constants of one cell of the box a thread owns for the whole march.
struct OwnCell {
    int idx;            // r * WK + c
    bool in;            // (j, k) inside the interior
    double cs;          // an_u + as_u + at_u + ab_u (the diagonal's column part)
    double an, as, at, ab;
};

// One block = one column segment: tile (k0, j0), planes [i0, i1).  Load L
// (0 <= L < np + 6) stages plane ib + L (ib = i0 - 3) of the inputs in wide
// boxes, and (P half) the r0 tile of plane ib + L - 3.  Step L computes
//   phase 1: v, w1 = v / ac        on plane ib + L     (40 x 14)
//   phase 2: w2 = sweep(w1)        on plane ib + L - 1 (36 x 12)
//   phase 3: w3 = sweep(w2)        on plane ib + L - 2 (34 x 10)
//   phase 4: A w3 and the sums     on plane ib + L - 3 (32 x 8)
// Every thread owns the same cells in every phase: one tile cell (all four
// phases) and one or two halo-ring cells.  The values of an owned cell on
// the planes a sweep needs (i - 1, i, i + 1) and its right-hand side stay
// in the thread's registers; only the j +- 1, k +- 1 neighbours are read
// from the shared-memory planes.  Cells outside the interior hold 0, as the
// ghost cells of the unfused kernels' buffers do.
template <int KIND>
__global__ void __launch_bounds__(TILE_THREADS, 2)
k_fused(Grid g, PoissonCoef C, Segments S, const __grid_constant__ CUtensorMap m_a,
        const __grid_constant__ CUtensorMap m_b, const __grid_constant__ CUtensorMap m_c,
        const __grid_constant__ CUtensorMap m_r0, FusedArgs A, Partials<2> part,
        KrylovState *st) {
    using G = FusedGeo<KIND>;
    if (st->done) return;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) unsigned long long bar[NSF];
    __shared__ double s_ae[MAXP], s_aw[MAXP], s_xp[MAXP];

    const int tid = threadIdx.x;
    const int u = blockIdx.x;
    const int col = u % S.ncol, chunk = u / S.ncol;
    const int k0 = S.box.lo[2] + (col % S.ntk) * TK, j0 = S.box.lo[1] + (col / S.ntk) * TJ;
    int i0, i1;
    S.chunk_range(chunk, i0, i1);
    const int np = i1 - i0, nload = np + 2 * FH;
    const int kb = k0 - WIDE_HK, jb = j0 - WIDE_HJ, ib = i0 - FH;
    const int off = (int)g.off;
    const double alpha = st->alpha, beta = st->beta, omega = st->omega;
    const bool first = (st->it == 0);
    const double inv_md = C.inv_max_diag;
    const Box bx = S.box;

    if (tid == 0) {
        for (int s = 0; s < NSF; s++) mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    if (tid < nload) {
        const int i = ib + tid;
        const bool ok = i >= 0 && i < g.nx;
        s_ae[tid] = ok ? C.ae[i] : 0.0;
        s_aw[tid] = ok ? C.aw[i] : 0.0;
        s_xp[tid] = ok ? C.xpart[i] : 0.0;
    }
    auto own = [&](int r, int c) {
        OwnCell o;
        const int j = jb + r, k = kb + c;
        o.idx = r * WK + c;
        o.in = j >= bx.lo[1] && j < bx.hi[1] && k >= bx.lo[2] && k < bx.hi[2];
        const bool jok = j >= 0 && j < g.ny, kok = k >= 0 && k < g.nz;
        o.an = jok ? C.an[j] : 0.0;
        o.as = jok ? C.as[j] : 0.0;
        o.at = kok ? C.at[k] : 0.0;
        o.ab = kok ? C.ab[k] : 0.0;
        o.cs = (jok && kok) ? C.an_u[j] + C.as_u[j] + C.at_u[k] + C.ab_u[k] : 0.0;
        return o;
    };
    const int tr = tid >> 5, tc = tid & 31;
    const OwnCell cT = own(WIDE_HJ + tr, WIDE_HK + tc);   // tile cell
    int rr, rc, ring1;
    ring_cell(tid, rr, rc, ring1);
    const OwnCell cR = own(rr, rc);                        // first ring cell
    const bool has_x = tid < NEXTRA;
    int xr = 0, xc = 0, ringx = 2;
    if (has_x) ring_cell(TILE_THREADS + tid, xr, xc, ringx);
    const OwnCell cX = own(xr, xc);                        // second ring cell (ring C)
    const long long sy = g.sy;
    const long long toff = (long long)(j0 + tr) * sy + k0 + tc + off;  // tile cell in its plane
    __syncthreads();

    auto plane_in = [&](int m) { const int i = ib + m; return i >= bx.lo[0] && i < bx.hi[0]; };
    auto issue = [&](int L) {
        const int s = L % NSF;
        unsigned char *base = smem + s * G::STAGE;
        const bool r0p = KIND == FK_P && L >= 2 * FH;  // r0 of output plane ib + L - 3
        mbar_expect_tx(&bar[s], G::NIN * PB + (r0p ? TB : 0));
        tma_load_3d(base, &m_a, kb + off, jb, ib + L, &bar[s]);
        if (KIND == FK_P) {
            tma_load_3d(base + PB, &m_b, kb + off, jb, ib + L, &bar[s]);
            tma_load_3d(base + 2 * PB, &m_c, kb + off, jb, ib + L, &bar[s]);
            if (r0p) tma_load_3d(base + 3 * PB, &m_r0, k0 + off, j0, ib + L - FH, &bar[s]);
        } else {
            tma_load_3d(base + PB, &m_c, kb + off, jb, ib + L, &bar[s]);
        }
    };
    int issued = 0;
    if (tid == 0)
        for (; issued < NSF && issued < nload; issued++) issue(issued);

    double *wpl = (double *)(smem + NSF * G::STAGE);   // w1, w2, w3 planes, two of each
    auto W1s = [&](int m) { return wpl + (0 + (m & 1)) * WN; };
    auto W2s = [&](int m) { return wpl + (2 + (m & 1)) * WN; };
    auto W3s = [&](int m) { return wpl + (4 + (m & 1)) * WN; };
    auto Rs = [&](int m) { return wpl + (6 + m % 3) * WN; };   // 1/ac, computed in phase 1

    // phase 1 at one owned cell: v, 1/ac and w1 = v / ac (the first sweep
    // from zero)
    auto point = [&](const OwnCell &o, const double *in_a, const double *in_b, const double *in_c,
                     bool pin, double xp, double &v, double &w, double &rc) {
        const int e = o.idx;
        if (KIND == FK_P)
            v = first ? in_a[e] : __fma_rn(beta, __fma_rn(-omega, in_c[e], in_b[e]), in_a[e]);
        else
            v = __fma_rn(-alpha, in_c[e], in_a[e]);
        rc = fast_rcp((xp - o.cs) * inv_md);
        w = v * rc;
        const bool in = pin && o.in;
        v = in ? v : 0.0;
        w = in ? w : 0.0;
    };
    // A x at an owned cell of plane m (apply_a<false>: same operations, same
    // order): centre, east (i + 1) and west (i - 1) from registers, the
    // in-plane neighbours from the shared plane P
    auto ax_at = [&](const OwnCell &o, const double *P, int m, double ac, double xc, double xe,
                     double xw) {
        double v = ac * xc;
        v = __fma_rn(s_ae[m], xe, v);
        v = __fma_rn(s_aw[m], xw, v);
        v = __fma_rn(o.an, P[o.idx + WK], v);
        v = __fma_rn(o.as, P[o.idx - WK], v);
        v = __fma_rn(o.at, P[o.idx + 1], v);
        return __fma_rn(o.ab, P[o.idx - 1], v);
    };
    // sweep_jacobi_at_cell (relax<false>) at an owned cell of plane m; 1/ac
    // from the plane's ring (the same fast_rcp value phase 1 computed)
    auto sweep = [&](const OwnCell &o, const double *P, int m, bool pin, double xc, double xe,
                     double xw, double rhs) {
        const double ac = (s_xp[m] - o.cs) * inv_md;
        const double ax = ax_at(o, P, m, ac, xc, xe, xw);
        const double w = xc + (rhs - ax) * Rs(m)[o.idx];
        return (pin && o.in) ? w : 0.0;
    };

    // register histories: suffix n = the value n planes behind the newest
    double tv0 = 0, tv1 = 0, tv2 = 0, tv3 = 0;      // tile cell: v
    double t10 = 0, t11 = 0, t12 = 0;               //            w1
    double t20 = 0, t21 = 0, t22 = 0;               //            w2
    double t30 = 0, t31 = 0, t32 = 0;               //            w3
    double rv0 = 0, rv1 = 0, rv2 = 0;               // ring cell: v
    double r10 = 0, r11 = 0, r12 = 0;               //            w1
    double r20 = 0, r21 = 0, r22 = 0;               //            w2

    double acc0 = 0.0, acc1 = 0.0;
    bool fail = false;
    int L = 0;
    for (; L < nload; L++) {
        tv3 = tv2; tv2 = tv1; tv1 = tv0;
        t12 = t11; t11 = t10;
        t22 = t21; t21 = t20;
        t32 = t31; t31 = t30;
        rv2 = rv1; rv1 = rv0;
        r12 = r11; r11 = r10;
        r22 = r21; r21 = r20;
        // Three barriers per step (after phases 1, 2 and 3): phase 4 of step
        // L and phase 1 of step L + 1 touch disjoint buffers (W3 / stage L
        // against W1, 1/ac and stage L + 1), and a failed wait is caught at
        // the first barrier, before any shared plane it touched is read.
        if (!fail) fail = !mbar_wait(&bar[L % NSF], (unsigned)((L / NSF) & 1));
        const unsigned char *stg = smem + (L % NSF) * G::STAGE;
        const double *in_a = (const double *)stg;
        const double *in_b = (const double *)(stg + PB);
        const double *in_c = (const double *)(stg + (KIND == FK_P ? 2 : 1) * PB);
        // Each phase computes all its cells before it stores any: a store to
        // a shared plane would otherwise order the next cell's loads after it.
        {   // phase 1, plane L
            const bool pin = plane_in(L);
            const double xp = s_xp[L];
            double *P1 = W1s(L), *R1 = Rs(L);
            double xv = 0.0, xw = 0.0, rc_t = 0.0, rc_r = 0.0, rc_x = 0.0;
            point(cT, in_a, in_b, in_c, pin, xp, tv0, t10, rc_t);
            point(cR, in_a, in_b, in_c, pin, xp, rv0, r10, rc_r);
            if (has_x) point(cX, in_a, in_b, in_c, pin, xp, xv, xw, rc_x);
            P1[cT.idx] = t10;
            P1[cR.idx] = r10;
            R1[cT.idx] = rc_t;
            R1[cR.idx] = rc_r;
            if (has_x) {
                P1[cX.idx] = xw;
                R1[cX.idx] = rc_x;
            }
            if (!fail && cT.in && L >= FH && L < FH + np)
                A.v_out[(long long)(ib + L) * g.sx + toff] = tv0;
        }
        if (__syncthreads_or(fail)) break;
        // every thread is past step L - 1: its stage is free for load L - 1 + NSF
        if (tid == 0 && L >= 1 && issued < nload) {
            fence_proxy_async();  // the released stage was read through the generic proxy
            issue(issued++);
        }
        if (L >= 2) {   // phase 2, plane L - 1
            const int m = L - 1;
            const bool pin = plane_in(m);
            const double *P1 = W1s(m);
            double *P2 = W2s(m);
            t20 = sweep(cT, P1, m, pin, t11, t10, t12, tv1);
            if (ring1 <= 1) r20 = sweep(cR, P1, m, pin, r11, r10, r12, rv1);
            P2[cT.idx] = t20;
            if (ring1 <= 1) P2[cR.idx] = r20;
        }
        __syncthreads();
        if (L >= 4) {   // phase 3, plane L - 2
            const int m = L - 2;
            const bool pin = plane_in(m);
            const double *P2 = W2s(m);
            double *P3 = W3s(m);
            t30 = sweep(cT, P2, m, pin, t21, t20, t22, tv2);
            const double r30 = ring1 == 0 ? sweep(cR, P2, m, pin, r21, r20, r22, rv2) : 0.0;
            P3[cT.idx] = t30;
            if (ring1 == 0) P3[cR.idx] = r30;
            if (cT.in && m >= FH && m < FH + np) A.w_out[(long long)(ib + m) * g.sx + toff] = t30;
        }
        __syncthreads();
        if (L >= 2 * FH && cT.in) {
            // phase 4: A w3 on the tile of plane L - 3, which lies in [i0, i1)
            const int m = L - FH;
            const double ac = (s_xp[m] - cT.cs) * inv_md;
            const double ax = ax_at(cT, W3s(m), m, ac, t31, t30, t32);
            A.av_out[(long long)(ib + m) * g.sx + toff] = ax;
            if (KIND == FK_P) {
                const double *r0 = (const double *)(stg + 3 * PB);
                acc0 += r0[tid] * ax;
            } else {
                acc0 += ax * tv3;
                acc1 += ax * ax;
            }
        }
    }
    if (fail) {
        // a bounded wait ran out: report, drain what is still in flight, stop
        if (tid == 0) {
            st->wait_error = 1;
            st->done = 1;
            for (int q = L; q < issued; q++) mbar_wait(&bar[q % NSF], (unsigned)((q / NSF) & 1));
        }
        return;
    }
    double vals[2] = {acc0, acc1};
    if (grid_reduce<2>(vals, 0u, part) && tid == 0) {
        if (KIND == FK_P) fin_q(st, vals[0]);
        else fin_t(st, vals[0], vals[1]);
    }
}

template <int KIND>
void fused_launch(const LaunchCtx &L, int kind_tag, const Grid &g, const PoissonCoef &C,
                  const PoissonConfig &cfg, const CUtensorMap &ma, const CUtensorMap &mb,
                  const CUtensorMap &mc, const CUtensorMap &mr0, const FusedArgs &A,
                  Partials<2> part, KrylovState *st) {
    // The shared-memory limit is an attribute of the function in the current
    // device's context: set it on every launch (a host-side call of about a
    // microsecond), so handles on several devices or threads need no shared
    // flag.
    DALM_CUDA(cudaFuncSetAttribute(k_fused<KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   FusedGeo<KIND>::SMEM));
    L.pre(kind_tag);
    k_fused<KIND><<<cfg.seg.count, TILE_THREADS, FusedGeo<KIND>::SMEM, L.s>>>(
        g, C, cfg.seg, ma, mb, mc, mr0, A, part, st);
    L.post(kind_tag);
}

}  // namespace

bool fused_bicg_available(const PoissonConfig &cfg) {
    return cfg.method == PM_BICG && cfg.pc == PC_JACOBI && cfg.pc_sweeps == FH &&
           !cfg.reference_sums && cfg.seg.ich <= 32;
}

void launch_bicg_iteration_fused(const LaunchCtx &L, const Grid &g, const PoissonCoef &C,
                                 const PoissonBufs &B, const FusedBufs &F, long long n,
                                 const PoissonConfig &cfg, Partials<2> part, KrylovState *st) {
    const int a = (int)(n & 1), b = 1 - a;
    const MapTable &M = *cfg.maps;
    FusedArgs Ap{F.pk[b], B.pp, F.q[b]};
    fused_launch<FK_P>(L, KK_BICG_PF, g, C, cfg, M.of(B.r).wide, M.of(F.pk[a]).wide,
                       M.of(F.q[a]).wide, M.of(B.r0).plain, Ap, part, st);
    FusedArgs As{B.s, B.ss, B.t};
    const CUtensorMap &mq = M.of(F.q[b]).wide;
    fused_launch<FK_S>(L, KK_BICG_SF, g, C, cfg, M.of(B.r).wide, mq, mq, mq, As, part, st);
    launch_bicg_xr(L, g, B, B.pp, B.ss, cfg, part, st);
}

}  // namespace dalm
