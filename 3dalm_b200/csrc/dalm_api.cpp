// C ABI (include/dalm.h) and the host orchestration of one time step.
//
// The handle owns all device state of one case on one GPU and one stream.
// A step enqueues the stage kernels in the order of Solver::main_loop_once
// (src/solver.h:1034-1306); the only host synchronisation inside a step is
// the Poisson loop's convergence poll, once per batch of iterations.
#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dalm.h"
#include "adjoint.cuh"
#include "alm_point.cuh"
#include "case_io.hpp"
#include "multigrid.cuh"
#include "multigrid_setup.hpp"
#include "output_io.hpp"
#include "poisson.cuh"

using namespace dalm;

namespace {

thread_local std::string g_last_error;

constexpr double PI_D = 3.14159265358979323846;
// Truncation radius of the Gaussian projection: r^2 <= 40 eps^2, where the
// dropped weight exp(-40) ~ 4e-18 of the peak is below FP64 resolution of f.
constexpr double ALM_CUTOFF_EPS2 = 40.0;
// iterations per captured CUDA graph of the Poisson loop
constexpr int GRAPH_UNIT = 8;
// Iterative refinement (DALM_MIXED): an FP32 inner solve stops at
// max(INNER_RTOL x the FP64 residual, 0.3 x the solve's tolerance) or after
// the pass cap (refine_inner_it, default INNER_CAP iterations); a pass that
// shrinks the FP64 residual by less than 1/STALL hands the rest of the solve
// to the FP64 solver.  With 1e-4 (a reduction FP32 multigrid-CG reaches in
// two iterations) one pass usually meets the tolerance; with 1e-3 the pass
// stopped just above it and a second pass (and its V-cycle) followed
// (measured on the 512x256x128 case: 5.6 against 6.4 ms per step).
constexpr double INNER_RTOL = 1e-4;
constexpr long long INNER_CAP = 100;
constexpr double STALL = 0.85;
constexpr long long MAX_REFINE = 1000;
// Adjoint pressure solves stop at this RMS residual relative to the RMS of
// their right-hand side.
constexpr double ADJ_RTOL = 1e-10;

const char *kKindNames[KK_COUNT] = {
    "predict", "flux_rhs", "pressure_bc", "project", "velocity_bc", "diag", "tavg",
    "alm_points", "alm_sums", "alm_project",
    "sor_sweep", "residual_norm", "jacobi_sweep",
    "bicg_init", "bicg_p", "bicg_q", "bicg_s", "bicg_t", "bicg_xr",
    "poisson_begin", "layout", "seq_sum", "bicg_p_fused", "bicg_s_fused", "refine_residual",
    "refine_update", "sor_sweep32", "jacobi_sweep32", "bicg_p32", "bicg_q32", "bicg_s32",
    "bicg_t32", "bicg_xr32", "adj_velocity_bc", "adj_project", "adj_faces", "adj_nut",
    "adj_predict", "adj_alm", "mg_smooth", "mg_transfer", "mg_coarse", "mg_pcg",
    "jacobi_sweep2"};

}  // namespace

// Message for dalm_last_error(NULL) from translation units without a handle.
void dalm::set_last_error(const std::string &msg) { g_last_error = msg; }

namespace {

struct EventPair {
    cudaEvent_t a, b;
    int kind;
};

}  // namespace

struct dalm_handle {
    CaseData cs;
    dalm_options opt;
    Grid g;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    LaunchCtx L;
    std::string err;
    std::vector<void *> allocs;

    // mesh and coefficients
    MeshDev mesh{};
    PoissonCoef coef{};
    StepParams P{};
    // fields
    double *U[2][3] = {};
    int ucur = 0;
    double *JU[2][3] = {};
    int jcur = 0;
    double *F[3] = {};
    double *Pp = nullptr, *B = nullptr;
    double *Utavg[3] = {};
    double *scratch = nullptr;   // one scalar field for nut / div output
    double *staging = nullptr;   // reference-layout staging buffer (3*len)
    PoissonBufs pb{};
    PoissonBufsT<float> pbf{};  // inner solves A e = r of iterative refinement (DALM_MIXED)
    bool mixed = false;
    long long refine_fp32_it = 0, refine_fp64_it = 0, refine_passes = 0;  // last solve
    std::vector<long long> last_inner;  // inner iterations per refinement pass, last solve
    // multigrid-preconditioned CG inner solves (DALM_INNER_MULTIGRID)
    bool mg_on = false;
    MgDev mgd;
    MgPcgBufs mgb{};
    MixedGeom geo{};  // mesh tables of the FP32 flow stages
    // DALM_MIXED stencil fields in FP32 (not with reference-order sums): the
    // stages run on these; U, JU and F above are FP64 views of them,
    // refreshed (widen) when the ABI reads the state and written back
    // (narrow) when it sets it.
    bool f32 = false;
    bool f64_stale = false;
    float *U32[2][3] = {}, *JU32[2][3] = {}, *F32[3] = {};
    FusedBufs fb{};
    bool fused = false;  // BiCGStab iterations as fused half-iteration kernels
    PoissonConfig pcfg{};
    MapTable maps;
    double *partial = nullptr;
    unsigned int *ticket = nullptr;
    KrylovState *d_kst = nullptr, *h_kst = nullptr;
    struct GraphUnit {
        cudaGraphExec_t exec = nullptr;
        long long kernels = 0;
    } graph_unit[2];  // per solve (FP64, FP32 inner)
    // output in the reference's formats (opt.write_output)
    std::string out_dir;
    double next_output_time = 0;
    std::vector<SnapshotEntry> snapshots;
    std::ofstream turbine_log;
    bool trace = false;          // DALM_TRACE_POISSON=1: one stderr line per pressure solve
    bool trace_batches = false;  // DALM_TRACE_POISSON=2: also one per batch of iterations
    DiagState *d_diag = nullptr, *h_diag = nullptr;
    double *d_prof = nullptr;
    // actuator line
    AlmDev alm{};
    std::vector<TurbineDev> h_wt;
    std::vector<double> base_twist, twist;
    double *h_wt_out = nullptr;  // pinned: torque[T], thrust[T]
    Box fbox{{0, 0, 0}, {0, 0, 0}};
    std::vector<double> pitch_deg;  // collective pitch per turbine (dalm_set_turbine_params)
    double last_alm_time = 0;       // time of the last actuator-line evaluation
    // reference-order mode: blade points evaluated on the host (alm_points_host)
    long long *d_alm_ids = nullptr;  // [ap][8] stored indices of the sampling corners
    double *d_alm_corner = nullptr;  // [ap][8][3] velocity at those corners
    std::vector<double> h_pt_xyz, h_pt_f;  // [ap][3] positions and forces of the last evaluation
    // runtime
    int64_t step = 0, tavg_count = 0, last_it = 0;
    int64_t max_it = 0;
    double tol = 0;
    long long launch_count = 0;
    // profiling
    std::vector<cudaEvent_t> ev_pool;
    std::vector<EventPair> ev_pending;
    cudaEvent_t ev_open = nullptr;
    double kind_ms[KK_COUNT] = {};
    double kind_bytes[KK_COUNT] = {};  // launch-dependent algorithmic bytes (LaunchCtx::bytes)
    int64_t kind_launches[KK_COUNT] = {};
    double stage_ms[7] = {};
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> stage_pending;

    ~dalm_handle() { release(); }

    void release() {
        if (stream) cudaStreamSynchronize(stream);
        for (auto &p : probe_list)
            if (!p.recs.empty()) flush_probe(p);
        probe_list.clear();
        for (auto &gu : graph_unit) {
            if (gu.exec) cudaGraphExecDestroy(gu.exec);
            gu.exec = nullptr;
        }
        for (void *p : allocs) cudaFree(p);
        allocs.clear();
        if (h_kst) cudaFreeHost(h_kst);
        if (h_diag) cudaFreeHost(h_diag);
        if (h_wt_out) cudaFreeHost(h_wt_out);
        h_kst = nullptr; h_diag = nullptr; h_wt_out = nullptr;
        for (auto e : ev_pool) cudaEventDestroy(e);
        for (auto &p : ev_pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
        for (auto &p : stage_pending) { cudaEventDestroy(p.second.first); cudaEventDestroy(p.second.second); }
        ev_pool.clear(); ev_pending.clear(); stage_pending.clear();
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
    }

    template <typename T>
    T *dalloc(size_t n) {
        void *p = nullptr;
        DALM_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
        DALM_CUDA(cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(T)));
        allocs.push_back(p);
        return (T *)p;
    }
    template <typename T>
    T *upload(const std::vector<T> &v) {
        T *p = dalloc<T>(v.size());
        if (!v.empty())
            DALM_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
        return p;
    }

    // ---- profiling -------------------------------------------------------
    cudaEvent_t take_event() {
        if (ev_pool.empty()) {
            cudaEvent_t e;
            DALM_CUDA(cudaEventCreate(&e));
            return e;
        }
        cudaEvent_t e = ev_pool.back();
        ev_pool.pop_back();
        return e;
    }
    static void hook(void *self, int kind, int phase) {
        dalm_handle *h = (dalm_handle *)self;
        cudaEvent_t e = h->take_event();
        DALM_CUDA(cudaEventRecord(e, h->stream));
        if (phase == 0) {
            h->ev_open = e;
        } else {
            h->ev_pending.push_back({h->ev_open, e, kind});
            h->ev_open = nullptr;
        }
    }
    void harvest() {
        for (auto &p : ev_pending) {
            DALM_CUDA(cudaEventSynchronize(p.b));
            float ms = 0;
            DALM_CUDA(cudaEventElapsedTime(&ms, p.a, p.b));
            kind_ms[p.kind] += ms;
            kind_launches[p.kind] += 1;
            ev_pool.push_back(p.a);
            ev_pool.push_back(p.b);
        }
        ev_pending.clear();
        for (auto &p : stage_pending) {
            DALM_CUDA(cudaEventSynchronize(p.second.second));
            float ms = 0;
            DALM_CUDA(cudaEventElapsedTime(&ms, p.second.first, p.second.second));
            stage_ms[p.first] += ms;
            ev_pool.push_back(p.second.first);
            ev_pool.push_back(p.second.second);
        }
        stage_pending.clear();
    }
    struct StageTimer {
        dalm_handle *h;
        int stage;
        cudaEvent_t a = nullptr;
        StageTimer(dalm_handle *h_, int s) : h(h_), stage(s) {
            if (h->opt.profile) {
                a = h->take_event();
                DALM_CUDA(cudaEventRecord(a, h->stream));
            }
        }
        ~StageTimer() noexcept(false) {
            if (a) {
                cudaEvent_t b = h->take_event();
                DALM_CUDA(cudaEventRecord(b, h->stream));
                h->stage_pending.push_back({stage, {a, b}});
            }
        }
    };

    // ---- construction ----------------------------------------------------
    void init(const std::string &dir, const dalm_options &o) {
        opt = o;
        if (opt.precision != DALM_FP64 && opt.precision != DALM_MIXED)
            throw std::invalid_argument("unknown precision");
        if (opt.limiter != DALM_LIMITER_MINMOD && opt.limiter != DALM_LIMITER_VAN_ALBADA)
            throw std::invalid_argument("unknown limiter");
        if (opt.mixed_inner != DALM_INNER_MULTIGRID && opt.mixed_inner != DALM_INNER_BICGSTAB)
            throw std::invalid_argument("unknown mixed_inner");
        const char *tr = std::getenv("DALM_TRACE_POISSON");
        trace = tr && (tr[0] == '1' || tr[0] == '2');
        trace_batches = tr && tr[0] == '2';
        cs = load_case(dir);
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
            throw CudaError("no CUDA device is available");
        if (opt.device < 0 || opt.device >= ndev) throw std::invalid_argument("bad device ordinal");
        DALM_CUDA(cudaSetDevice(opt.device));
        DALM_CUDA(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, opt.device));
        DALM_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        g = Grid::make((int)cs.size[0], (int)cs.size[1], (int)cs.size[2], (int)cs.gc);
        L.s = stream;
        L.blocks = reduction_blocks(sm_count);
        L.launches = &launch_count;
        if (opt.profile) {
            L.hook = &dalm_handle::hook;
            L.self = this;
            L.kind_bytes = kind_bytes;
        }
        max_it = cs.max_it;
        tol = cs.tol;

        // mesh
        mesh.x = upload(cs.x); mesh.y = upload(cs.y); mesh.z = upload(cs.z);
        mesh.dx = upload(cs.dx); mesh.dy = upload(cs.dy); mesh.dz = upload(cs.dz);
        build_coefficients();
        {
            const std::vector<double> *ctr[3] = {&cs.x, &cs.y, &cs.z}, *wid[3] = {&cs.dx, &cs.dy, &cs.dz};
            for (int a = 0; a < 3; a++) {
                const std::vector<double> &x = *ctr[a], &d = *wid[a];
                std::vector<float4> t(x.size(), make_float4(0.f, 0.f, 0.f, 0.f));
                std::vector<float2> w(x.size());
                std::vector<double2> r(x.size(), make_double2(0.0, 0.0));
                for (size_t n = 0; n < x.size(); n++) {
                    const double cb = std::cbrt(d[n]);
                    w[n] = make_float2((float)d[n], (float)(cb * cb));
                    if (n + 1 < x.size()) r[n].x = 1.0 / (x[n + 1] - x[n]);
                    if (n >= 1 && n + 1 < x.size()) r[n].y = 1.0 / (x[n + 1] - x[n - 1]);
                }
                for (size_t n = 1; n + 1 < x.size(); n++)
                    t[n] = make_float4((float)(1.0 / d[n]), (float)(1.0 / (x[n + 1] - x[n])),
                                       (float)(1.0 / (x[n] - x[n - 1])),
                                       (float)(1.0 / (x[n + 1] - x[n - 1])));
                geo.ax[a] = upload(t);
                geo.wd[a] = upload(w);
                geo.inv64[a] = upload(r);
            }
            geo.cs2 = (float)(cs.cs * cs.cs);
        }

        size_t n = (size_t)g.total;
        for (int b = 0; b < 2; b++)
            for (int m = 0; m < 3; m++) {
                U[b][m] = dalloc<double>(n);
                JU[b][m] = dalloc<double>(n);
            }
        for (int m = 0; m < 3; m++) {
            F[m] = dalloc<double>(n);
            Utavg[m] = dalloc<double>(n);
        }
        Pp = dalloc<double>(n);
        B = dalloc<double>(n);
        double **kv[] = {&pb.r, &pb.r0, &pb.pk, &pb.q, &pb.s, &pb.t, &pb.pp, &pb.ss, &pb.tp, &pb.ts};
        for (auto v : kv) *v = dalloc<double>(n);
        pb.x = Pp;
        pb.b = B;
        pcfg.method = cs.method == "BiCG" ? PM_BICG : (cs.method == "SOR" ? PM_SOR : PM_JACOBI);
        pcfg.pc = cs.pc_method == "SOR" ? PC_SOR : PC_JACOBI;
        pcfg.relax = cs.relax;
        pcfg.pc_relax = cs.pc_relax;
        pcfg.pc_sweeps = (int)cs.pc_max_it;
        pcfg.reference_sums = opt.reference_sums ? 1 : 0;
        pcfg.jacobi2 = opt.fused_jacobi ? 1 : 0;
        pcfg.seg = poisson_segments(g, sm_count);
        fused = opt.fused_krylov && fused_bicg_available(pcfg);
        // FP32 inner solves exist for BiCGStab only; SOR and Jacobi solves
        // stay FP64 under DALM_MIXED
        mixed = opt.precision == DALM_MIXED && pcfg.method == PM_BICG;
        f32 = mixed && !opt.reference_sums;
        if (f32) {
            for (int b = 0; b < 2; b++)
                for (int m = 0; m < 3; m++) {
                    U32[b][m] = dalloc<float>(n);
                    JU32[b][m] = dalloc<float>(n);
                }
            for (int m = 0; m < 3; m++) {
                F32[m] = dalloc<float>(n);
                DALM_CUDA(cudaMemset(F32[m], 0, sizeof(float) * n));
            }
        }
        if (mixed) {
            float **kv32[] = {&pbf.x, &pbf.r, &pbf.r0, &pbf.pk, &pbf.q, &pbf.s, &pbf.t,
                              &pbf.pp, &pbf.ss, &pbf.tp, &pbf.ts};
            for (auto v : kv32) *v = dalloc<float>(n);
            pbf.b = pbf.r0;  // e starts at 0, so the inner r0 = r = b
            if (opt.mixed_inner == DALM_INNER_MULTIGRID) setup_multigrid();
        }
        fb = FusedBufs{{pb.pk, nullptr}, {pb.q, nullptr}};
        if (fused) {
            fb.pk[1] = dalloc<double>(n);
            fb.q[1] = dalloc<double>(n);
        }
        const double *tma_fields[] = {pb.x, pb.b, pb.r, pb.r0, pb.pk, pb.q,
                                      pb.s, pb.t, pb.pp, pb.ss, pb.tp, pb.ts};
        for (const double *v : tma_fields) maps.add(g, v);
        if (fused) {
            maps.add(g, fb.pk[1]);
            maps.add(g, fb.q[1]);
        }
        if (mixed) {
            const float *tma32[] = {pbf.x, pbf.r, pbf.r0, pbf.pk, pbf.q, pbf.s,
                                    pbf.t, pbf.pp, pbf.ss, pbf.tp, pbf.ts};
            for (const float *v : tma32) maps.add(g, v, 4);
        }
        pcfg.maps = &maps;
        partial = dalloc<double>((size_t)std::max(L.blocks, pcfg.seg.count) * 4);
        ticket = dalloc<unsigned int>(1);
        d_kst = dalloc<KrylovState>(2);  // [0] the solve (refinement: outer), [1] inner
        d_diag = dalloc<DiagState>(1);
        DALM_CUDA(cudaHostAlloc((void **)&h_kst, 2 * sizeof(KrylovState), cudaHostAllocDefault));
        DALM_CUDA(cudaHostAlloc((void **)&h_diag, sizeof(DiagState), cudaHostAllocDefault));
        memset(h_kst, 0, 2 * sizeof(KrylovState));
        memset(h_diag, 0, sizeof(DiagState));
        DiagState d0{};
        d0.ncell = (double)g.ni() * g.nj() * g.nk();
        DALM_CUDA(cudaMemcpy(d_diag, &d0, sizeof(d0), cudaMemcpyHostToDevice));

        P.g = g;
        P.m = mesh;
        P.re = cs.re; P.cs = cs.cs; P.dt = cs.dt; P.max_diag = cs.max_diag;
        for (int m = 0; m < 3; m++) P.uin[m] = cs.uin[m];
        P.prof = nullptr;
        P.fbox = fbox;
        P.reference_sums = opt.reference_sums ? 1 : 0;
        P.limiter = opt.limiter == DALM_LIMITER_VAN_ALBADA ? 1 : 0;
        P.filter2 = build_filter();
        P.solid = nullptr;
        P.retracted = cs.retracted_floor ? 1 : 0;
        P.floor_start = cs.floor_start;
        if (cs.has_grid) {
            solid_host = build_solid();
            P.solid = upload(solid_host);
        }

        init_alm();

        // Solver::initialize tail (src/solver.h:737-833): U = Uold = Uin,
        // p = 0, BCs, flux, nut/div (on demand here), ALM force, diagnostics.
        for (int b = 0; b < 2; b++)
            for (int m = 0; m < 3; m++) launch_fill(L, U[b][m], g.total, cs.uin[m]);
        if (cs.has_grid) {  // set_solid_U on the initial field (src/solver.h:767-770)
            std::vector<double> u((size_t)g.total);
            for (int m = 0; m < 3; m++) {
                for (size_t c = 0; c < u.size(); c++) u[c] = (1. - solid_host[c]) * cs.uin[m];
                DALM_CUDA(cudaMemcpy(U[ucur][m], u.data(), sizeof(double) * u.size(),
                                     cudaMemcpyHostToDevice));
            }
        }
        narrow_state(false);
        refresh_after_state(DALM_SET_APPLY_UBC | DALM_SET_RECOMPUTE_JU, nullptr);
        DALM_CUDA(cudaStreamSynchronize(stream));
        if (opt.write_output) init_output();
    }

    // The multigrid levels of the inner solves (multigrid.cuh): merged-cell
    // geometry from the interior centres and widths, FP32 conductances and
    // widths, level vectors with zero guide cells, the coarsest operator's
    // inverse.  A coarsest level above MG_MAX_COARSE cells (interior counts
    // with large odd factors) leaves the BiCGStab inner solves in place.
    void setup_multigrid() {
        const int gc = (int)cs.gc;
        const std::vector<double> *c[3] = {&cs.x, &cs.y, &cs.z}, *d[3] = {&cs.dx, &cs.dy, &cs.dz};
        std::vector<double> cen[3], w[3];
        for (int a = 0; a < 3; a++) {
            cen[a].assign(c[a]->begin() + gc, c[a]->end() - gc);
            w[a].assign(d[a]->begin() + gc, d[a]->end() - gc);
        }
        std::vector<MgGeometry> geo = mg_build_levels(cen, w, MG_MAX_LEVELS, MG_COARSE_TARGET);
        const MgGeometry &C = geo.back();
        if (C.cells() > MG_MAX_COARSE) {
            if (trace)
                std::fprintf(stderr, "[dalm] multigrid: coarsest level %lld cells > %d, "
                             "BiCGStab inner solves\n", C.cells(), MG_MAX_COARSE);
            return;
        }
        mgd.levels = (int)geo.size();
        for (int l = 0; l < mgd.levels; l++) {
            const MgGeometry &G = geo[l];
            MgLevel &v = mgd.L[l];
            v.g = l == 0 ? g : Grid::make(G.n[0] + 2, G.n[1] + 2, G.n[2] + 2, 1);
            std::vector<float> fcf[3], fw[3];
            for (int a = 0; a < 3; a++) {
                v.n[a] = G.n[a];
                v.fac[a] = G.fac[a];
                fcf[a].assign(G.cf[a].begin(), G.cf[a].end());
                fw[a].assign(G.w[a].begin(), G.w[a].end());
                v.cf[a] = upload(fcf[a]);
                v.w[a] = upload(fw[a]);
            }
            // the smoother's z-line factors on the two finest levels, when the
            // mesh allows (on the coarser, latency-bound levels the table's
            // loads cost more than the elimination they save: measured on C4)
            MgLineTable T;
            if (l < 2 && mg_line_table(v.n, fcf, fw, T)) {
                v.lcls[0] = upload(T.cls[0]);
                v.lcls[1] = upload(T.cls[1]);
                v.lky = T.ky;
                v.ltab = upload(T.tab);
            }
            if (l > 0) {
                mgd.x[l] = dalloc<float>((size_t)v.g.total);
                mgd.f[l] = dalloc<float>((size_t)v.g.total);
            }
        }
        if (!mg_prepare(mgd)) {
            if (trace) std::fprintf(stderr, "[dalm] multigrid: z-columns too long, BiCGStab inner solves\n");
            return;
        }
        std::vector<double> inv = mg_spd_inverse(mg_dense_operator(C), C.cells());
        mgd.kinv = upload(std::vector<float>(inv.begin(), inv.end()));
        mgd.ncoarse = (int)C.cells();
        const size_t n = (size_t)g.total;
        mgb = MgPcgBufs{pbf.r, pbf.x, dalloc<float>(n), dalloc<float>(n), dalloc<float>(n)};
        mg_on = true;
    }

    // Solid volume fraction of the turbulence-generating grid per interior
    // cell (set_turbulence_generating_grid, src/solver.h:52-159): a vertical
    // bar layer of thickness `thick` ending at x = placement_x, with bars of
    // width `bar` every `mesh` in y, and a horizontal bar layer just upstream
    // with bars every `mesh` in z; same operation order as the reference.
    std::vector<double> solid_host;
    static double intersection(double h1, double t1, double h2, double t2) {
        double l1 = t1 - h1, l2 = t2 - h2, x1 = t1 - h2, x2 = t2 - h1;  // src/util.h:84-90
        return std::fmax(0., std::fmin(l1, std::fmin(l2, std::fmin(x1, x2))));
    }
    std::vector<double> build_solid() const {
        std::vector<double> s((size_t)g.total, 0.0);
        const double thick = cs.grid_thick, mesh_w = cs.grid_mesh, bar = cs.grid_bar;
        const double gx = cs.grid_at[0], gy = cs.grid_at[1], gz = cs.grid_at[2];
        for (int i = g.gc; i < g.nx - g.gc; i++)
            for (int j = g.gc; j < g.ny - g.gc; j++)
                for (int k = g.gc; k < g.nz - g.gc; k++) {
                    double xc = cs.x[i], yc = cs.y[j], zc = cs.z[k];
                    double dxc = cs.dx[i], dyc = cs.dy[j], dzc = cs.dz[k];
                    double xv = intersection(xc - 0.5 * dxc, xc + 0.5 * dxc, gx - thick, gx);
                    int64_t bj = (int64_t)std::round((yc - gy) / mesh_w);
                    double by = bj * mesh_w + gy;
                    double yi = intersection(yc - 0.5 * dyc, yc + 0.5 * dyc, by - 0.5 * bar,
                                             by + 0.5 * bar);
                    double xh = intersection(xc - 0.5 * dxc, xc + 0.5 * dxc, gx - 2 * thick,
                                             gx - thick);
                    int64_t bk = (int64_t)std::round((zc - gz) / mesh_w);
                    double bz = bk * mesh_w + gz;
                    double zi = intersection(zc - 0.5 * dzc, zc + 0.5 * dzc, bz - 0.5 * bar,
                                             bz + 0.5 * bar);
                    double occupied = xv * yi * dzc + xh * zi * dyc;
                    s[(size_t)g.at(i, j, k)] = occupied / (dxc * dyc * dzc);
                }
        return s;
    }

    // (Cs * cbrt(dx dy dz))^2 per interior cell with the host libm's cbrt,
    // the factor calc_nut_at_cell applies (src/cfd.h:804, 823-824).
    const double *build_filter() {
        std::vector<double> f((size_t)g.total, 0.0);
        for (int i = g.gc; i < g.nx - g.gc; i++)
            for (int j = g.gc; j < g.ny - g.gc; j++)
                for (int k = g.gc; k < g.nz - g.gc; k++) {
                    double volume = cs.dx[i] * cs.dy[j] * cs.dz[k];
                    double filter = cbrt(volume);
                    double v = cs.cs * filter;
                    f[(size_t)g.at(i, j, k)] = v * v;
                }
        return upload(f);
    }

    // build_A (src/eq.h:701-798) as per-axis arrays; see PoissonCoef.
    void build_coefficients() {
        int64_t gc = cs.gc, NX = cs.size[0], NY = cs.size[1], NZ = cs.size[2];
        double md = cs.max_diag;
        std::vector<double> ex(NX, 0), awu(NX, 0), ae(NX, 0), aw(NX, 0);
        std::vector<double> anu(NY, 0), asu(NY, 0), an(NY, 0), as(NY, 0);
        std::vector<double> atu(NZ, 0), abu(NZ, 0), at(NZ, 0), ab(NZ, 0);
        for (int64_t i = gc; i < NX - gc; i++) {
            if (i < NX - gc - 1) {
                double v = 1 / (cs.dx[i] * (cs.x[i + 1] - cs.x[i]));
                ex[i] = v;
                ae[i] = v / md;
            } else {
                ex[i] = 2 / (cs.dx[i] * cs.dx[i]);
            }
            if (i > gc) {
                awu[i] = 1 / (cs.dx[i] * (cs.x[i] - cs.x[i - 1]));
                aw[i] = awu[i] / md;
            }
        }
        for (int64_t j = gc; j < NY - gc; j++) {
            if (j < NY - gc - 1) { anu[j] = 1 / (cs.dy[j] * (cs.y[j + 1] - cs.y[j])); an[j] = anu[j] / md; }
            if (j > gc) { asu[j] = 1 / (cs.dy[j] * (cs.y[j] - cs.y[j - 1])); as[j] = asu[j] / md; }
        }
        for (int64_t k = gc; k < NZ - gc; k++) {
            if (k < NZ - gc - 1) { atu[k] = 1 / (cs.dz[k] * (cs.z[k + 1] - cs.z[k])); at[k] = atu[k] / md; }
            if (k > gc) { abu[k] = 1 / (cs.dz[k] * (cs.z[k] - cs.z[k - 1])); ab[k] = abu[k] / md; }
        }
        coef.ex = upload(ex); coef.aw_u = upload(awu);
        coef.an_u = upload(anu); coef.as_u = upload(asu);
        coef.at_u = upload(atu); coef.ab_u = upload(abu);
        coef.ae = upload(ae); coef.aw = upload(aw);
        coef.an = upload(an); coef.as = upload(as);
        coef.at = upload(at); coef.ab = upload(ab);
        coef.max_diag = md;
        coef.inv_max_diag = 1.0 / md;
        std::vector<double> xpart(NX, 0);
        for (int64_t i = 0; i < NX; i++) xpart[i] = (0.0 - ex[i]) - awu[i];
        coef.xpart = upload(xpart);
    }

    void init_alm() {
        int64_t T = (int64_t)cs.turbines.size();
        alm.wt_count = (int)T;
        alm.ap_count = (int)cs.ap_count();
        if (alm.ap_count == 0) return;
        alm.ap_per_blade = (int)cs.ap_per_blade;
        alm.blades = (int)cs.blades;
        alm.ap_per_wt = (int)(cs.blades * cs.ap_per_blade);
        alm.atk_count = (int)cs.atk_count;
        double pw = cs.projection_width;
        alm.pw2 = pw * pw;
        double c = pw * sqrt(PI_D);
        alm.e_coef = 1 / (c * c * c);  // 1/cubic(pw*sqrt(Pi)), src/alm.h:433
        alm.cutoff2 = ALM_CUTOFF_EPS2 * alm.pw2;
        for (auto &t : cs.turbines) {
            TurbineDev d{};
            for (int m = 0; m < 3; m++) { d.base[m] = t.base[m]; d.rot_center[m] = t.rot_center[m]; }
            for (int m = 0; m < 4; m++) d.formula[m] = t.formula[m];
            d.rot_speed = t.rot_speed;
            d.type = t.angle_type;
            h_wt.push_back(d);
        }
        base_twist = cs.ap_twist;
        twist = cs.ap_twist;
        pitch_deg.assign((size_t)T, 0.0);
        alm.wt = upload(h_wt);
        alm.r = upload(cs.ap_r);
        alm.dr = upload(cs.ap_dr);
        alm.chord = upload(cs.ap_chord);
        alm.twist = upload(twist);
        alm.cd = upload(cs.ap_cd);
        alm.cl = upload(cs.ap_cl);
        alm.atk = upload(cs.atk);
        alm.pt_xyz = dalloc<double>(3 * alm.ap_count);
        alm.pt_f = dalloc<double>(3 * alm.ap_count);
        alm.pt_torque = dalloc<double>(alm.ap_count);
        alm.pt_thrust = dalloc<double>(alm.ap_count);
        alm.wt_torque = dalloc<double>(T);
        alm.wt_thrust = dalloc<double>(T);
        DALM_CUDA(cudaHostAlloc((void **)&h_wt_out, sizeof(double) * 2 * T, cudaHostAllocDefault));
        memset(h_wt_out, 0, sizeof(double) * 2 * T);
    }

    // ---- views -----------------------------------------------------------
    Vec3<double> u_cur() { return {{U[ucur][0], U[ucur][1], U[ucur][2]}}; }
    Vec3<double> u_old() { return {{U[1 - ucur][0], U[1 - ucur][1], U[1 - ucur][2]}}; }
    Vec3<double> ju_cur() { return {{JU[jcur][0], JU[jcur][1], JU[jcur][2]}}; }
    Vec3<double> ju_other() { return {{JU[1 - jcur][0], JU[1 - jcur][1], JU[1 - jcur][2]}}; }
    static Vec3<const double> c(Vec3<double> v) { return {{v.c[0], v.c[1], v.c[2]}}; }
    Vec3<double> f3() { return {{F[0], F[1], F[2]}}; }
    Vec3<float> u32_cur() { return {{U32[ucur][0], U32[ucur][1], U32[ucur][2]}}; }
    Vec3<float> u32_old() { return {{U32[1 - ucur][0], U32[1 - ucur][1], U32[1 - ucur][2]}}; }
    Vec3<float> ju32_cur() { return {{JU32[jcur][0], JU32[jcur][1], JU32[jcur][2]}}; }
    Vec3<float> ju32_other() { return {{JU32[1 - jcur][0], JU32[1 - jcur][1], JU32[1 - jcur][2]}}; }
    Vec3<float> f32v() { return {{F32[0], F32[1], F32[2]}}; }
    static Vec3<const float> c(Vec3<float> v) { return {{v.c[0], v.c[1], v.c[2]}}; }

    // FP64 views of the FP32 stencil fields (DALM_MIXED): widen before the
    // ABI or an FP64 kernel reads U, Uold, JU or f; narrow after the ABI
    // wrote them (with_ju: JU too, else it is recomputed from U)
    void widen_state() {
        if (!f32 || !f64_stale) return;
        const long long n = g.total;
        for (int b = 0; b < 2; b++)
            for (int m = 0; m < 3; m++) launch_widen(L, U32[b][m], U[b][m], n);
        for (int m = 0; m < 3; m++) {
            launch_widen(L, JU32[jcur][m], JU[jcur][m], n);
            launch_widen(L, F32[m], F[m], n);
        }
        f64_stale = false;
    }
    void narrow_state(bool with_ju) {
        if (!f32) return;
        const long long n = g.total;
        for (int b = 0; b < 2; b++)
            for (int m = 0; m < 3; m++) launch_narrow(L, U[b][m], U32[b][m], n);
        for (int m = 0; m < 3; m++) {
            if (with_ju) {
                launch_narrow(L, JU[jcur][m], JU32[jcur][m], n);
                launch_narrow(L, JU[jcur][m], JU32[1 - jcur][m], n);
            }
            launch_narrow(L, F[m], F32[m], n);
        }
    }

    // ---- stages ----------------------------------------------------------
    void stage_predict() {
        StageTimer t(this, DALM_STAGE_PREDICT);
        P.fbox = fbox;
        if (f32) {
            launch_predict32(L, P, geo, c(u32_cur()), u32_old(), c(ju32_cur()), c(f32v()));
            f64_stale = true;
        } else {
            launch_predict(L, P, c(u_cur()), u_old(), c(ju_cur()), c(f3()));
        }
        ucur = 1 - ucur;  // the old buffer is now Uold
    }
    void stage_flux_rhs() {
        StageTimer t(this, DALM_STAGE_FLUX_RHS);
        if (f32) {
            launch_flux32(L, P, geo, c(u32_cur()), ju32_cur(), B);
            f64_stale = true;
        } else {
            launch_flux_rhs(L, P, c(u_cur()), ju_cur(), B);
        }
    }
    // iteration n (from 0) of the current solve
    void enqueue_poisson_iteration(long long n) {
        if (fused) {
            launch_bicg_iteration_fused(L, g, coef, pb, fb, n, pcfg, Partials<2>{partial, ticket}, d_kst);
        } else if (pcfg.method == PM_BICG) {
            launch_bicg_iteration<double>(L, g, coef, pb, pcfg, Partials<2>{partial, ticket}, d_kst);
        } else if (pcfg.method == PM_SOR) {
            launch_sor_iteration(L, g, coef, pb, pcfg, Partials<1>{partial, ticket}, d_kst);
        } else {
            launch_jacobi_iteration(L, g, coef, pb, pcfg, Partials<1>{partial, ticket}, d_kst);
        }
    }
    void fetch_states() {
        DALM_CUDA(cudaMemcpyAsync(h_kst, d_kst, 2 * sizeof(KrylovState), cudaMemcpyDeviceToHost, stream));
        DALM_CUDA(cudaStreamSynchronize(stream));
        if (h_kst[0].wait_error || h_kst[1].wait_error)
            throw DeviceWaitError("a TMA stage wait in the Poisson solver ran out");
    }
    // Enqueues iterations of solve `which` in batches and polls the device's
    // `done` flag in between.  The first batch stops a little short of
    // `hint` (the previous comparable solve's count); later batches grow
    // with the count so far.  Kernels enqueued after convergence return at
    // once.  Returns the iterations the solve took.
    // one iteration n of solve `which` (0: the FP64 solve, 1: the FP32
    // inner solve of the mixed form)
    void enqueue_one(int which, long long n, KrylovState *st) {
        if (which == 1 && mg_on)
            launch_mg_iteration(L, mgd, mgb, coef.max_diag, Partials<1>{partial, ticket}, st);
        else if (which == 1)
            launch_bicg_iteration<float>(L, g, coef, pbf, pcfg, Partials<2>{partial, ticket}, st);
        else
            enqueue_poisson_iteration(n);
    }
    // CUDA graphs (opt.use_graphs, not with per-kernel profiling): a unit of
    // GRAPH_UNIT iterations of a solve is captured once per handle and
    // replayed.  Kernel arguments are fixed per handle (the Krylov scalars
    // live in device memory); the fused kernels' ping-pong depends only on
    // the iteration's parity, and units start at even iterations.
    bool use_graphs() const { return opt.use_graphs && !opt.profile; }
    // Iterations per graph unit: one for the multigrid inner solves, whose
    // few (~90-kernel) iterations per pass are enqueued one at a time past
    // the previous pass's count; GRAPH_UNIT for the Krylov solves.
    bool mg_inner(int which) const { return which == 1 && mg_on; }
    int unit_of(int which) const { return mg_inner(which) ? 1 : GRAPH_UNIT; }
    void enqueue_unit(int which, long long n0) {
        GraphUnit &gu = graph_unit[which];
        if (!gu.exec) {
            const long long before = launch_count;
            cudaGraph_t graph = nullptr;
            DALM_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            try {
                for (int n = 0; n < unit_of(which); n++) enqueue_one(which, n0 + n, d_kst + which);
            } catch (...) {
                cudaStreamEndCapture(stream, &graph);
                if (graph) cudaGraphDestroy(graph);
                launch_count = before;
                throw;
            }
            DALM_CUDA(cudaStreamEndCapture(stream, &graph));
            cudaError_t e = cudaGraphInstantiate(&gu.exec, graph, 0);
            cudaGraphDestroy(graph);
            DALM_CUDA(e);
            gu.kernels = launch_count - before;
            launch_count = before;  // capturing launched nothing
        }
        DALM_CUDA(cudaGraphLaunch(gu.exec, stream));
        launch_count += gu.kernels;
    }
    long long run_batches(int which, long long hint, long long cap) {
        KrylovState *st = d_kst + which;
        long long issued = 0;
        const bool mg = mg_inner(which);
        long long batch = opt.poisson_batch > 0 ? opt.poisson_batch
                          : mg                  ? std::max<long long>(1, hint)
                                                : std::min<long long>(256, hint > 12 ? hint / 2 : 4);
        const bool graphs = use_graphs();
        const int unit = unit_of(which);
        while (true) {
            batch = std::min<long long>(batch, std::max<long long>(1, cap - issued));
            if (graphs) {
                // whole units; iterations past the stop return at once
                const long long units = (batch + unit - 1) / unit;
                for (long long u = 0; u < units; u++) enqueue_unit(which, issued + u * unit);
                batch = units * unit;
            } else {
                for (long long n = 0; n < batch; n++) enqueue_one(which, issued + n, st);
            }
            issued += batch;
            fetch_states();
            if (trace_batches)
                std::fprintf(stderr, "[dalm]     solve %d: %lld iterations, residual %.3e\n", which,
                             (long long)h_kst[which].it, h_kst[which].err);
            if (h_kst[which].done) break;
            if (issued > cap + GRAPH_UNIT)
                throw std::runtime_error("Poisson loop did not stop at its iteration limit");
            batch = opt.poisson_batch > 0 ? opt.poisson_batch
                    : mg                  ? 1
                                          : std::max<long long>(8, std::min<long long>(96, issued / 8));
        }
        return h_kst[which].it;
    }
    // The reference's solve (FP64) from the current p; `used` iterations of
    // the case's cap are already spent.
    void solve_fp64(long long used) {
        double ncell = (double)g.ni() * g.nj() * g.nk();
        launch_poisson_begin(L, d_kst, max_it - used, tol, ncell);
        if (pcfg.method == PM_BICG)
            launch_bicg_init(L, g, coef, pb, pcfg, Partials<1>{partial, ticket}, d_kst);
        long long hint = mixed ? refine_fp64_it : last_it;
        long long n = run_batches(0, hint, max_it - used);
        refine_fp64_it = n;
        h_kst[0].it = used + n;
    }
    void stage_poisson() {
        StageTimer t(this, DALM_STAGE_POISSON);
        if (!mixed) {
            solve_fp64(0);
        } else {
            solve_mixed();
        }
        last_it = h_kst[0].it;
        if (trace)
            std::fprintf(stderr, "[dalm] step %lld poisson it %lld err %.3e (FP32 %lld in %lld passes, FP64 %lld)\n",
                         (long long)step, (long long)last_it, h_kst[0].err, refine_fp32_it,
                         refine_passes, mixed ? refine_fp64_it : last_it);
    }
    // Iterative refinement (DALM_MIXED): r = b - A p and its norm in FP64;
    // an FP32 BiCGStab solve of A e = r from e = 0, capped at the pass cap;
    // p += e; repeat until the FP64 residual meets the tolerance.  A pass
    // that makes the residual worse is taken back; a pass that breaks down,
    // or gains less than 1/STALL, ends the refinement and the reference's
    // FP64 solve finishes from the current p.
    // FP64 residual of the pressure, its norm and the stop test; the next
    // inner solve's right-hand side in FP32
    void refine_residual() {
        PoissonBufsT<float> in = pbf;
        if (mg_on) in.r0 = in.q = nullptr;  // multigrid-CG reads the residual alone
        launch_refine_residual(L, g, coef, pcfg, Pp, B, in, Partials<2>{partial, ticket}, d_kst,
                               d_kst + 1);
    }
    void solve_mixed() {
        const double ncell = (double)g.ni() * g.nj() * g.nk();
        const long long cap = opt.refine_inner_it > 0 ? opt.refine_inner_it : INNER_CAP;
        launch_poisson_begin(L, d_kst, max_it, tol, ncell, MAX_REFINE, INNER_RTOL, cap);
        launch_poisson_begin(L, d_kst + 1, max_it, tol, ncell, 0, 0, 0, 1);
        refine_residual();
        // The first pass's inner solve is enqueued before the residual is
        // read back (one host round trip fewer per solve): when the residual
        // already meets the tolerance, the finisher has marked the inner
        // solve done, its kernels return at once and the pass is dropped.
        bool first = true;
        double prev = 0;
        refine_fp32_it = 0;
        refine_fp64_it = 0;
        refine_passes = 0;
        bool fallback = false;
        long long used = 0;
        size_t pass = 0;
        while (first || !h_kst[0].done) {
            if (last_inner.size() <= pass) last_inner.push_back(0);
            // multigrid-CG: scaled right-hand side, e = 0, first direction
            // (here, not with the residual, so that a rejected pass can
            // still take its correction back)
            if (mg_on) launch_mg_begin(L, mgd, mgb, coef.max_diag, Partials<1>{partial, ticket}, d_kst + 1);
            last_inner[pass] = run_batches(1, last_inner[pass], cap);
            if (first) {
                first = false;
                prev = h_kst[0].err;
                if (h_kst[0].done) break;  // met before any inner iteration
            }
            refine_fp32_it += h_kst[1].it;
            refine_passes = (long long)pass + 1;
            if (h_kst[1].breakdown) {  // the correction is discarded, p unchanged
                used = h_kst[0].it + h_kst[1].it;
                fallback = true;
                break;
            }
            launch_refine_update(L, g, pcfg, Pp, pbf.x, 1.0);
            refine_residual();
            fetch_states();
            const double now = h_kst[0].err;
            if (trace)
                std::fprintf(stderr, "[dalm]   pass %zu FP32 it %lld -> residual %.3e\n", pass,
                             last_inner[pass], now);
            if (!(now < prev)) {  // worse (or not finite): take the correction back
                launch_refine_update(L, g, pcfg, Pp, pbf.x, -1.0);
                used = h_kst[0].it;
                fallback = true;
                break;
            }
            if (!h_kst[0].done && now > STALL * prev) {
                used = h_kst[0].it;
                fallback = true;
                break;
            }
            prev = now;
            pass++;
        }
        if (fallback && used < max_it) solve_fp64(used);
    }
    void stage_project() {
        StageTimer t(this, DALM_STAGE_PROJECT);
        launch_pressure_bc(L, P, Pp);
        if (f32) {
            launch_project32(L, P, geo, u32_cur(), c(ju32_cur()), ju32_other(), Pp,
                             Partials<2>{partial, ticket}, d_diag);
            jcur = 1 - jcur;
            launch_velocity_bc(L, P, u32_cur(), c(u32_old()));
            f64_stale = true;
        } else {
            launch_project(L, P, u_cur(), ju_cur(), ju_other(), Pp, Partials<2>{partial, ticket},
                           d_diag);
            jcur = 1 - jcur;
            launch_velocity_bc(L, P, u_cur(), c(u_old()));
        }
    }

    // Blade-point positions on the host (same formulas as the device) to
    // bound the cells the truncated Gaussians can reach.
    Box force_box(double tm) {
        Box b{{0, 0, 0}, {0, 0, 0}};
        if (alm.ap_count == 0) return b;
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int a = 0; a < alm.ap_count; a++) {
            const TurbineDev &wt = h_wt[a / alm.ap_per_wt];
            double angle = wt.formula[0] * sin(wt.formula[1] * tm + wt.formula[2]) + wt.formula[3];
            int bid = (a % alm.ap_per_wt) / alm.ap_per_blade;
            double r = cs.ap_r[a];
            double th = bid * (2 * PI_D / alm.blades) + tm * wt.rot_speed;
            double in[3] = {wt.rot_center[0], wt.rot_center[1] + r * cos(th), wt.rot_center[2] + r * sin(th)};
            double cc = cos(-angle), ss = sin(-angle), out[3];
            switch (wt.type) {
            case EULER_ROLL: out[0] = in[0]; out[1] = cc * in[1] + ss * in[2]; out[2] = -ss * in[1] + cc * in[2]; break;
            case EULER_PITCH: out[0] = cc * in[0] - ss * in[2]; out[1] = in[1]; out[2] = -ss * in[0] + cc * in[2]; break;
            case EULER_YAW: out[0] = cc * in[0] + ss * in[1]; out[1] = -ss * in[0] + cc * in[1]; out[2] = in[2]; break;
            default: out[0] = in[0]; out[1] = in[1]; out[2] = in[2]; break;
            }
            for (int m = 0; m < 3; m++) {
                double v = out[m] + wt.base[m];
                lo[m] = std::min(lo[m], v);
                hi[m] = std::max(hi[m], v);
            }
        }
        double R = sqrt(alm.cutoff2);
        const std::vector<double> *ax[3] = {&cs.x, &cs.y, &cs.z};
        for (int m = 0; m < 3; m++) {
            const std::vector<double> &c = *ax[m];
            int n = (int)c.size(), gc = (int)cs.gc;
            int l = (int)(std::lower_bound(c.begin(), c.end(), lo[m] - R) - c.begin()) - 1;
            int h = (int)(std::upper_bound(c.begin(), c.end(), hi[m] + R) - c.begin()) + 1;
            b.lo[m] = std::max(gc, l);
            b.hi[m] = std::min(n - gc, h);
        }
        if (b.empty()) b = Box{{0, 0, 0}, {0, 0, 0}};
        return b;
    }

    static Box unite(const Box &a, const Box &b) {
        if (a.empty()) return b;
        if (b.empty()) return a;
        Box u;
        for (int m = 0; m < 3; m++) {
            u.lo[m] = std::min(a.lo[m], b.lo[m]);
            u.hi[m] = std::max(a.hi[m], b.hi[m]);
        }
        return u;
    }

    // The blade-point model (update_ap_position + calc_ap_force,
    // src/alm.h:233-414) on the host, for the reference-order mode: the
    // same almpt functions as k_alm_points, with the host's libm sin, cos
    // and atan (the reference's), so positions, angles and loads are the
    // reference's bit for bit.  The velocity at the 8 sampling corners of
    // every point is gathered on the device and read back (one synchronising
    // round trip per evaluation); the results go to the device arrays the
    // projection and the statistics read.
    void alm_points_host(double tm, Vec3<const double> u) {
        const int n = alm.ap_count;
        if (!d_alm_ids) {
            d_alm_ids = dalloc<long long>(8 * (size_t)n);
            d_alm_corner = dalloc<double>(24 * (size_t)n);
        }
        std::vector<almpt::Pose> pose((size_t)n);
        std::vector<long long> ids(8 * (size_t)n, g.at(g.gc, g.gc, g.gc));
        std::vector<double> frac(3 * (size_t)n, 0.0);
        std::vector<char> inside((size_t)n, 0);
        for (int a = 0; a < n; a++) {
            const TurbineDev &wt = h_wt[a / alm.ap_per_wt];
            int bid = (a % alm.ap_per_wt) / alm.ap_per_blade;
            almpt::point_pose(wt, cs.ap_r[a], bid, alm.blades, tm, pose[a]);
            inside[a] = almpt::point_cell(g, cs.x.data(), cs.y.data(), cs.z.data(), pose[a].xyz,
                                          &ids[8 * (size_t)a], &frac[3 * (size_t)a]);
        }
        DALM_CUDA(cudaMemcpyAsync(d_alm_ids, ids.data(), sizeof(long long) * ids.size(),
                                  cudaMemcpyHostToDevice, stream));
        launch_gather_points(L, u, d_alm_ids, 8 * n, d_alm_corner);
        std::vector<double> corner(24 * (size_t)n);
        DALM_CUDA(cudaMemcpyAsync(corner.data(), d_alm_corner, sizeof(double) * corner.size(),
                                  cudaMemcpyDeviceToHost, stream));
        DALM_CUDA(cudaStreamSynchronize(stream));
        std::vector<double> &xyz = h_pt_xyz, &f = h_pt_f;
        xyz.assign(3 * (size_t)n, 0.0);
        f.assign(3 * (size_t)n, 0.0);
        std::vector<double> tq((size_t)n, 0.0), th((size_t)n, 0.0), sums(2 * (size_t)alm.wt_count, 0.0);
        const int na = alm.atk_count;
        for (int a = 0; a < n; a++) {
            for (int m = 0; m < 3; m++) xyz[3 * (size_t)a + m] = pose[a].xyz[m];
            if (!inside[a]) continue;
            double Uap[3];
            for (int m = 0; m < 3; m++) {
                double c8[8];
                for (int q = 0; q < 8; q++) c8[q] = corner[(8 * (size_t)a + q) * 3 + m];
                Uap[m] = almpt::trilinear(c8, &frac[3 * (size_t)a]);
            }
            almpt::point_force(h_wt[a / alm.ap_per_wt], pose[a], Uap, twist[a], cs.ap_chord[a],
                               cs.ap_dr[a], cs.atk.data(), na, &cs.ap_cd[(size_t)a * na],
                               &cs.ap_cl[(size_t)a * na], &f[3 * (size_t)a], tq[a], th[a]);
        }
        // per-turbine sums in blade-point order (src/alm.h:384-398)
        for (int w = 0; w < alm.wt_count; w++) {
            double torque = 0, thrust = 0;
            for (int a = w * alm.ap_per_wt; a < (w + 1) * alm.ap_per_wt; a++) {
                torque += tq[a];
                thrust += th[a];
            }
            sums[w] = torque;
            sums[alm.wt_count + w] = thrust;
        }
        const size_t b3 = sizeof(double) * 3 * (size_t)n, b1 = sizeof(double) * (size_t)n,
                     bw = sizeof(double) * (size_t)alm.wt_count;
        DALM_CUDA(cudaMemcpyAsync(alm.pt_xyz, xyz.data(), b3, cudaMemcpyHostToDevice, stream));
        DALM_CUDA(cudaMemcpyAsync(alm.pt_f, f.data(), b3, cudaMemcpyHostToDevice, stream));
        DALM_CUDA(cudaMemcpyAsync(alm.pt_torque, tq.data(), b1, cudaMemcpyHostToDevice, stream));
        DALM_CUDA(cudaMemcpyAsync(alm.pt_thrust, th.data(), b1, cudaMemcpyHostToDevice, stream));
        DALM_CUDA(cudaMemcpyAsync(alm.wt_torque, sums.data(), bw, cudaMemcpyHostToDevice, stream));
        DALM_CUDA(cudaMemcpyAsync(alm.wt_thrust, sums.data() + alm.wt_count, bw,
                                  cudaMemcpyHostToDevice, stream));
        // the host vectors go out of scope at return: wait for the copies
        DALM_CUDA(cudaStreamSynchronize(stream));
    }

    // distribute_ap_force (src/alm.h:416-448) on the host for the
    // reference-order mode: every interior cell sums every blade point in
    // point order with the host's exp, untruncated, exactly the reference's
    // loop; the whole field is uploaded and the predictor reads it on the
    // whole interior.  Cells are independent, so host threads split the
    // i-planes without changing any result.
    void alm_project_host() {
        const int n = alm.ap_count, gc = (int)cs.gc;
        const double pw = cs.projection_width;
        const double c = pw * sqrt(PI_D);
        const double e = 1 / (c * c * c);  // 1/cubic(projection_width*sqrt(Pi))
        std::vector<double> fh[3];
        for (auto &v : fh) v.assign((size_t)g.total, 0.0);
        auto planes = [&](int i0, int i1) {
            for (int i = i0; i < i1; i++)
                for (int j = gc; j < g.ny - gc; j++)
                    for (int k = gc; k < g.nz - gc; k++) {
                        double fx = 0, fy = 0, fz = 0;
                        const double xc = cs.x[i], yc = cs.y[j], zc = cs.z[k];
                        for (int a = 0; a < n; a++) {
                            const double *p = &h_pt_xyz[3 * (size_t)a];
                            const double dx = xc - p[0], dy = yc - p[1], dz = zc - p[2];
                            const double r2 = dx * dx + dy * dy + dz * dz;
                            const double wght = e * exp(-r2 / (pw * pw));
                            fx += wght * h_pt_f[3 * (size_t)a];
                            fy += wght * h_pt_f[3 * (size_t)a + 1];
                            fz += wght * h_pt_f[3 * (size_t)a + 2];
                        }
                        const long long id = g.at(i, j, k);
                        fh[0][id] = fx;
                        fh[1][id] = fy;
                        fh[2][id] = fz;
                    }
        };
        const int ni = g.nx - 2 * gc;
        int nt = (int)std::min<unsigned>(std::max(1u, std::thread::hardware_concurrency()), 32u);
        nt = std::max(1, std::min(nt, ni));
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; t++)
            pool.emplace_back(planes, gc + (int)((long long)ni * t / nt), gc + (int)((long long)ni * (t + 1) / nt));
        for (auto &th : pool) th.join();
        for (int m = 0; m < 3; m++)
            DALM_CUDA(cudaMemcpyAsync(F[m], fh[m].data(), sizeof(double) * (size_t)g.total,
                                      cudaMemcpyHostToDevice, stream));
        DALM_CUDA(cudaStreamSynchronize(stream));
        fbox = Box{{gc, gc, gc}, {g.nx - gc, g.ny - gc, g.nz - gc}};
    }

    void stage_alm() { alm_at(cs.dt * (double)step); }  // rt.get_time(), src/solver.h:189-191
    void alm_at(double tm) {
        if (alm.ap_count == 0) return;
        StageTimer t(this, DALM_STAGE_ALM);
        last_alm_time = tm;
        if (opt.reference_sums) {
            alm_points_host(tm, c(u_cur()));
            alm_project_host();
        } else if (f32) {
            launch_alm_points(L, P, alm, tm, c(u32_cur()));
            Box cur = force_box(tm);
            launch_alm_project(L, P, alm, unite(fbox, cur), f32v());
            fbox = cur;
            f64_stale = true;
        } else {
            launch_alm_points(L, P, alm, tm, c(u_cur()));
            Box cur = force_box(tm);
            launch_alm_project(L, P, alm, unite(fbox, cur), f3());
            fbox = cur;
        }
    }
    void stage_diag() {
        StageTimer t(this, DALM_STAGE_DIAG);
        if (f32)
            launch_diag(L, P, c(u32_cur()), c(ju32_cur()), Partials<2>{partial, ticket}, d_diag);
        else
            launch_diag(L, P, c(u_cur()), c(ju_cur()), Partials<2>{partial, ticket}, d_diag);
        DALM_CUDA(cudaMemcpyAsync(h_diag, d_diag, sizeof(DiagState), cudaMemcpyDeviceToHost, stream));
    }
    void stage_tavg() {
        if (!opt.time_average) return;
        double tm = cs.dt * (double)step;
        if (!(tm >= cs.tavg_start_time)) return;
        StageTimer t(this, DALM_STAGE_TAVG);
        tavg_count++;
        double w = 1. / tavg_count;
        if (f32)
            launch_tavg(L, g, {{Utavg[0], Utavg[1], Utavg[2]}}, c(u32_cur()), w);
        else
            launch_tavg(L, g, {{Utavg[0], Utavg[1], Utavg[2]}}, c(u_cur()), w);
    }

    void run_stage(int s) {
        switch (s) {
        case DALM_STAGE_PREDICT: stage_predict(); break;
        case DALM_STAGE_FLUX_RHS: stage_flux_rhs(); break;
        case DALM_STAGE_POISSON: stage_poisson(); break;
        case DALM_STAGE_PROJECT: stage_project(); break;
        case DALM_STAGE_ALM: stage_alm(); break;
        case DALM_STAGE_DIAG: stage_diag(); break;
        case DALM_STAGE_TAVG: stage_tavg(); break;
        default: throw std::invalid_argument("unknown stage");
        }
    }

    // Solver::main_loop_once (src/solver.h:1034-1306)
    void step_once() {
        if (step != 0) {
            stage_predict();
            stage_flux_rhs();
            stage_poisson();
            stage_project();
            stage_alm();
        }
        stage_tavg();
        if (opt.write_output) write_outputs();
        step++;
    }

    // ---- output in the reference's formats -------------------------------
    // output/ beside the case files like the reference's solver
    // (src/solver.h:569-588), partition.json (src/solver.h:980-998), and a
    // per-turbine load time series turbines.csv (no reference counterpart).
    void init_output() {
        out_dir = (std::filesystem::path(cs.dir) / "output").string();
        std::filesystem::create_directories(out_dir);
        write_partition_json(out_dir + "/partition.json", cs.size, cs.gc);
        next_output_time = cs.output_start_time;
        if (alm.ap_count > 0)  // the blade-point tables at set-up (src/solver.h:949-974)
            write_ap_info(out_dir + "/ap_info.log", alm.ap_count, alm.atk_count, cs.ap_r,
                          cs.ap_dr, cs.ap_chord, base_twist, cs.ap_cd, cs.ap_cl, cs.atk);
        if (alm.wt_count > 0) {
            turbine_log.open(out_dir + "/turbines.csv");
            if (!turbine_log) throw std::runtime_error("cannot write " + out_dir + "/turbines.csv");
            turbine_log << "step,time";
            for (int w = 0; w < alm.wt_count; w++)
                turbine_log << ",thrust" << w << ",torque" << w << ",power" << w;
            turbine_log << "\n";
        }
        if (cs.has_grid) {  // the grid's solid fraction at set-up (src/solver.h:747-762)
            std::vector<double> ref((size_t)cs.size[0] * cs.size[1] * cs.size[2], 0.0);
            for (int i = 0; i < g.nx; i++)
                for (int j = 0; j < g.ny; j++)
                    for (int k = 0; k < g.nz; k++)
                        ref[((size_t)i * g.ny + j) * g.nz + k] = solid_host[(size_t)g.at(i, j, k)];
            write_field_binary(out_dir + "/" + binary_filename("solid", 0, step), cs.size, cs.gc,
                               cs.x, cs.y, cs.z, {{"solid", 1, ref.data()}});
        }
        init_probes();
    }

    // ---- probes (struct Probe, src/solver.h:406-465) ----------------------
    // Each requested point is snapped to the nearest cell centre among the
    // interior and the first guide layer (find_nearest_index, src/util.h:
    // 92-106); points that land in the guide layer stay inactive.  Active
    // probes record (t, u, v, w) in FP32 every step once t >= output start
    // time, buffered and appended to probe<m>.csv every 10000 records and
    // when the handle is destroyed, in the reference's text format.
    struct Probe {
        std::string path;
        long long cell;  // device index
        std::vector<std::array<float, 4>> recs;
    };
    std::vector<Probe> probe_list;
    long long *d_probe_idx = nullptr;
    double *d_probe_val = nullptr;
    static int64_t nearest_index(const double *x, double y, int64_t len) {
        if (y < x[0]) return 0;
        if (y >= x[len - 1]) return len - 1;
        for (int64_t i = 0; i < len - 1; i++)
            if (x[i] <= y && y < x[i + 1]) return (y - x[i] < x[i + 1] - y) ? i : i + 1;
        return -1;
    }
    void init_probes() {
        const int64_t gc = cs.gc;
        std::vector<long long> idx;
        for (size_t m = 0; 3 * m + 2 < cs.probes.size(); m++) {
            const double px = cs.probes[3 * m], py = cs.probes[3 * m + 1], pz = cs.probes[3 * m + 2];
            int64_t ni = nearest_index(cs.x.data() + gc - 1, px, cs.size[0] - 2 * gc + 2) + gc - 1;
            int64_t nj = nearest_index(cs.y.data() + gc - 1, py, cs.size[1] - 2 * gc + 2) + gc - 1;
            int64_t nk = nearest_index(cs.z.data() + gc - 1, pz, cs.size[2] - 2 * gc + 2) + gc - 1;
            if (!(ni >= gc && ni < cs.size[0] - gc && nj >= gc && nj < cs.size[1] - gc && nk >= gc &&
                  nk < cs.size[2] - gc))
                continue;
            Probe p;
            p.path = out_dir + "/probe" + std::to_string(m) + ".csv";
            p.cell = g.at((int)ni, (int)nj, (int)nk);
            std::ofstream ofs(p.path);
            if (!ofs) throw std::runtime_error("cannot write " + p.path);
            ofs << "# " << cs.x[ni] << " " << cs.y[nj] << " " << cs.z[nk] << std::endl;
            ofs << "t,u,v,w" << std::endl;
            idx.push_back(p.cell);
            probe_list.push_back(std::move(p));
        }
        if (!idx.empty()) {
            d_probe_idx = upload(idx);
            d_probe_val = dalloc<double>(3 * idx.size());
        }
    }
    void record_probes(double t) {
        if (probe_list.empty() || !(t >= cs.output_start_time)) return;
        const int n = (int)probe_list.size();
        std::vector<double> v(3 * (size_t)n);
        if (f32)
            launch_gather_points(L, c(u32_cur()), d_probe_idx, n, d_probe_val);
        else
            launch_gather_points(L, c(u_cur()), d_probe_idx, n, d_probe_val);
        DALM_CUDA(cudaMemcpyAsync(v.data(), d_probe_val, sizeof(double) * v.size(),
                                  cudaMemcpyDeviceToHost, stream));
        DALM_CUDA(cudaStreamSynchronize(stream));
        for (int m = 0; m < n; m++) {
            Probe &p = probe_list[m];
            p.recs.push_back({(float)t, (float)v[3 * m], (float)v[3 * m + 1], (float)v[3 * m + 2]});
            if (p.recs.size() == 10000) flush_probe(p);
        }
    }
    static void flush_probe(Probe &p) {
        std::ofstream ofs(p.path, std::ios::app);
        for (const auto &r : p.recs) ofs << r[0] << "," << r[1] << "," << r[2] << "," << r[3] << std::endl;
        p.recs.clear();
    }
    // The end of main_loop_once (src/solver.h:1194-1253): the turbine loads,
    // and at the output times the inst_ file (U, p, div, q, f), the tavg_
    // file (time-averaged U) once averaging has started, and snapshot.json.
    void write_outputs() {
        const double t = cs.dt * (double)step;
        record_probes(t);
        if (turbine_log.is_open() && step != 0) {
            sync_stats();
            char buf[96];
            std::snprintf(buf, sizeof buf, "%lld,%.17g", (long long)step, t);
            turbine_log << buf;
            for (int w = 0; w < alm.wt_count; w++) {
                const double tq = h_wt_out[w], th = h_wt_out[alm.wt_count + w];
                std::snprintf(buf, sizeof buf, ",%.17g,%.17g,%.17g", th, tq,
                              tq * std::fabs(h_wt[w].rot_speed));
                turbine_log << buf;
            }
            turbine_log << "\n";
            turbine_log.flush();
        }
        if (!(t - 0.5 * cs.dt < next_output_time && next_output_time <= t + 0.5 * cs.dt)) return;
        next_output_time += cs.output_interval_time;
        widen_state();
        const size_t cells = (size_t)g.nx * g.ny * g.nz;
        std::vector<double> u(3 * cells), p(cells), dv(cells), q(cells), f(3 * cells);
        get_field(DALM_FIELD_U, u.data());
        get_field(DALM_FIELD_P, p.data());
        get_field(DALM_FIELD_DIV, dv.data());
        double *s = scratch_field();
        launch_q_field(L, P, c(u_cur()), s);
        download_field(&s, 1, q.data());
        get_field(DALM_FIELD_F, f.data());
        write_field_binary(out_dir + "/" + binary_filename("inst", 0, step), cs.size, cs.gc, cs.x,
                           cs.y, cs.z,
                           {{"U", 3, u.data()}, {"p", 1, p.data()}, {"div", 1, dv.data()},
                            {"q", 1, q.data()}, {"f", 3, f.data()}});
        const bool tavg = t >= cs.tavg_start_time;
        if (tavg) {
            get_field(DALM_FIELD_UTAVG, u.data());
            write_field_binary(out_dir + "/" + binary_filename("tavg", 0, step), cs.size, cs.gc,
                               cs.x, cs.y, cs.z, {{"U", 3, u.data()}});
        }
        snapshots.push_back({step, t, tavg});
        write_snapshot_json(out_dir + "/snapshot.json", snapshots);
    }

    // derived quantities after a state change (src/solver.h:767-833)
    void refresh_after_state(int flags, const double *JU_host) {
        if (f32) {
            // U (and p) were written to the FP64 views: narrow U, then derive
            // on the FP32 fields
            for (int m = 0; m < 3; m++) launch_narrow(L, U[ucur][m], U32[ucur][m], g.total);
            if (flags & DALM_SET_APPLY_UBC) {
                for (int m = 0; m < 3; m++)
                    DALM_CUDA(cudaMemcpyAsync(U32[1 - ucur][m], U32[ucur][m], sizeof(float) * g.total,
                                              cudaMemcpyDeviceToDevice, stream));
                launch_velocity_bc(L, P, u32_cur(), c(u32_old()));
            }
            if ((flags & DALM_SET_RECOMPUTE_JU) || !JU_host) {
                launch_flux32(L, P, geo, c(u32_cur()), ju32_cur(), nullptr);
            } else {
                upload_field(JU_host, 3, JU[jcur]);
                for (int m = 0; m < 3; m++) {
                    launch_narrow(L, JU[jcur][m], JU32[jcur][m], g.total);
                    launch_narrow(L, JU[jcur][m], JU32[1 - jcur][m], g.total);
                }
            }
            f64_stale = true;
            stage_alm();
            stage_diag();
            return;
        }
        if (flags & DALM_SET_APPLY_UBC) {
            for (int m = 0; m < 3; m++)
                DALM_CUDA(cudaMemcpyAsync(U[1 - ucur][m], U[ucur][m], sizeof(double) * g.total,
                                          cudaMemcpyDeviceToDevice, stream));
            launch_velocity_bc(L, P, u_cur(), c(u_old()));
        }
        if ((flags & DALM_SET_RECOMPUTE_JU) || !JU_host) {
            launch_flux_only(L, P, c(u_cur()), ju_cur());
        } else {
            upload_field(JU_host, 3, JU[jcur]);
            upload_field(JU_host, 3, JU[1 - jcur]);
        }
        stage_alm();
        stage_diag();
    }

    // ---- host <-> device layout -----------------------------------------
    double *stage_buffer() {
        if (!staging) staging = dalloc<double>((size_t)3 * g.nx * g.ny * g.nz);
        return staging;
    }
    void upload_field(const double *host, int nc, double *const *dst) {
        double *s = stage_buffer();
        size_t bytes = sizeof(double) * (size_t)nc * g.nx * g.ny * g.nz;
        DALM_CUDA(cudaMemcpyAsync(s, host, bytes, cudaMemcpyHostToDevice, stream));
        launch_to_device_layout(L, g, s, nc, dst);
        DALM_CUDA(cudaStreamSynchronize(stream));
    }
    void download_field(double *const *src, int nc, double *host) {
        double *s = stage_buffer();
        size_t bytes = sizeof(double) * (size_t)nc * g.nx * g.ny * g.nz;
        launch_to_ref_layout(L, g, src, nc, s);
        DALM_CUDA(cudaMemcpyAsync(host, s, bytes, cudaMemcpyDeviceToHost, stream));
        DALM_CUDA(cudaStreamSynchronize(stream));
    }
    double *scratch_field() {
        if (!scratch) scratch = dalloc<double>((size_t)g.total);
        DALM_CUDA(cudaMemsetAsync(scratch, 0, sizeof(double) * g.total, stream));
        return scratch;
    }

    void get_field(int which, double *out) {
        widen_state();
        switch (which) {
        case DALM_FIELD_U: download_field(U[ucur], 3, out); break;
        case DALM_FIELD_UOLD: download_field(U[1 - ucur], 3, out); break;
        case DALM_FIELD_JU: download_field(JU[jcur], 3, out); break;
        case DALM_FIELD_P: download_field(&Pp, 1, out); break;
        case DALM_FIELD_NUT: {
            double *s = scratch_field();
            launch_nut_field(L, P, c(u_cur()), s);
            download_field(&s, 1, out);
            break;
        }
        case DALM_FIELD_DIV: {
            double *s = scratch_field();
            launch_div_field(L, P, c(ju_cur()), s);
            download_field(&s, 1, out);
            break;
        }
        case DALM_FIELD_F: download_field(F, 3, out); break;
        case DALM_FIELD_B: download_field(&B, 1, out); break;
        case DALM_FIELD_UTAVG: download_field(Utavg, 3, out); break;
        default: throw std::invalid_argument("unknown field");
        }
    }
    void set_field(int which, const double *in) {
        // with FP32 stencil fields the FP64 copy is written, then rounded
        // into the FP32 field the stages use
        auto narrow3 = [&](double *const *src, float *const *dst) {
            if (!f32) return;
            for (int m = 0; m < 3; m++) launch_narrow(L, src[m], dst[m], g.total);
            f64_stale = true;
        };
        widen_state();
        switch (which) {
        case DALM_FIELD_U: upload_field(in, 3, U[ucur]); narrow3(U[ucur], U32[ucur]); break;
        case DALM_FIELD_UOLD: upload_field(in, 3, U[1 - ucur]); narrow3(U[1 - ucur], U32[1 - ucur]); break;
        case DALM_FIELD_JU:
            upload_field(in, 3, JU[jcur]);
            upload_field(in, 3, JU[1 - jcur]);
            narrow3(JU[jcur], JU32[jcur]);
            narrow3(JU[jcur], JU32[1 - jcur]);
            break;
        case DALM_FIELD_P: upload_field(in, 1, &Pp); break;
        case DALM_FIELD_F:
            upload_field(in, 3, F);
            narrow3(F, F32);
            fbox = Box{{(int)cs.gc, (int)cs.gc, (int)cs.gc},
                       {g.nx - (int)cs.gc, g.ny - (int)cs.gc, g.nz - (int)cs.gc}};
            break;
        case DALM_FIELD_B: upload_field(in, 1, &B); break;
        case DALM_FIELD_UTAVG: upload_field(in, 3, Utavg); break;
        default: throw std::invalid_argument("field is derived and cannot be set");
        }
        if (f32) DALM_CUDA(cudaStreamSynchronize(stream));
    }

    // ---- discrete adjoint of the time stepping ------------------------------
    //
    // J = mean over steps t0..t1 of the total turbine power; its gradient with
    // respect to every turbine's yaw (deg), collective pitch (deg) and rotor
    // speed (rad/s).  The forward run from the current state stores a
    // restart point every k steps; the reverse sweep takes the segments last
    // to first, recomputes each from its restart point while recording the
    // velocity and face fluxes of every step, then runs the transposed steps
    // (adjoint_cell.cuh) backwards through it.  The adjoint pressure solve
    // reuses the forward solver: A^T = M A M^-1 with M the cell volumes.
    struct AdjointStats {
        long long solves = 0, iterations = 0, recomputed_steps = 0;
        double max_rel_residual = 0;
    } adj_stats;
    long long adj_hint = 0;

    // device buffers of one gradient run, freed when it ends
    struct Scratch {
        std::vector<void *> ptrs;
        ~Scratch() {
            for (void *p : ptrs) cudaFree(p);
        }
        template <typename T>
        T *get(size_t n) {
            void *p = nullptr;
            DALM_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
            ptrs.push_back(p);
            return (T *)p;
        }
    };
    // a restart point: the fields a step reads and the host-side step state
    struct Snapshot {
        double *U[3], *JU[3], *F[3], *p;
        int64_t step, last_it;
        Box fbox;
        double alm_time;
    };
    void alloc_snapshot(Scratch &S, Snapshot &c) {
        for (int m = 0; m < 3; m++) {
            c.U[m] = S.get<double>(g.total);
            c.JU[m] = S.get<double>(g.total);
            c.F[m] = S.get<double>(g.total);
        }
        c.p = S.get<double>(g.total);
    }
    void d2d(double *dst, const double *src, size_t n = 0) {
        DALM_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * (n ? n : (size_t)g.total),
                                  cudaMemcpyDeviceToDevice, stream));
    }
    void zero(double *p, size_t n = 0) {
        DALM_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * (n ? n : (size_t)g.total), stream));
    }
    void save(Snapshot &c) {
        for (int m = 0; m < 3; m++) {
            d2d(c.U[m], U[ucur][m]);
            d2d(c.JU[m], JU[jcur][m]);
            d2d(c.F[m], F[m]);
        }
        d2d(c.p, Pp);
        c.step = step;
        c.last_it = last_it;
        c.fbox = fbox;
        c.alm_time = last_alm_time;
    }
    void load(const Snapshot &c) {
        for (int m = 0; m < 3; m++) {
            d2d(U[ucur][m], c.U[m]);
            d2d(JU[jcur][m], c.JU[m]);
            d2d(F[m], c.F[m]);
        }
        d2d(Pp, c.p);
        step = c.step;
        last_it = c.last_it;
        fbox = c.fbox;
        last_alm_time = c.alm_time;
    }
    // one time step without time averaging or output (recomputation)
    void integrate_step() {
        stage_predict();
        stage_flux_rhs();
        stage_poisson();
        stage_project();
        stage_alm();
        step++;
    }
    // The adjoint pressure solves use FP64 iterative refinement with the
    // multigrid-CG inner solves when the case's solver is BiCGStab and the
    // multigrid levels can be built (set up on first use in FP64 handles;
    // a mixed handle whose inner solver is BiCGStab keeps it); the result
    // meets the same FP64 residual test either way.
    bool mg_tried = false;
    bool adjoint_refinement() {
        if (pcfg.method != PM_BICG) return false;
        if (mixed && opt.mixed_inner != DALM_INNER_MULTIGRID) return false;
        if (!mg_on && !mg_tried) {
            mg_tried = true;
            const size_t n = (size_t)g.total;
            if (!pbf.x) {  // the refinement's FP32 vectors (multigrid path only)
                pbf.x = dalloc<float>(n);
                pbf.r = dalloc<float>(n);
                pbf.r0 = dalloc<float>(n);
                pbf.q = dalloc<float>(n);
                pbf.b = pbf.r0;
            }
            setup_multigrid();
        }
        return mg_on;
    }
    // A y = rhs (in B) from the guess in Pp, to an absolute RMS residual
    long long adjoint_solve(double tol_abs) {
        double ncell = (double)g.ni() * g.nj() * g.nk();
        launch_poisson_begin(L, d_kst, max_it, tol_abs, ncell);
        if (pcfg.method == PM_BICG)
            launch_bicg_init(L, g, coef, pb, pcfg, Partials<1>{partial, ticket}, d_kst);
        long long n = run_batches(0, adj_hint > 0 ? adj_hint : last_it, max_it);
        adj_hint = n;
        return n;
    }

    struct AdjBuffers {
        double *aU[3], *aV[3], *aJU[3], *af[3], *nu, *s6[6], *y, *grad, *sumsq;
        double *gather, *w, *lU, *gth, *torque;
        long long *ids;
    };

    // the transposed actuator line at time t on velocity u (the adjoint of the
    // force it projected is B.af), with the objective weight of its power
    void adjoint_alm(AdjBuffers &A, double t, Vec3<const double> u, double weight) {
        launch_alm_points(L, P, alm, t, u);
        adj::AdjAlmPointArgs X{P, alm, u, t, weight, A.gather, A.ids, A.w, A.lU, A.gth, A.torque};
        launch_adj_alm(L, P, alm, Vec3<const double>{{A.af[0], A.af[1], A.af[2]}}, X,
                       Vec3<double>{{A.aU[0], A.aU[1], A.aU[2]}}, A.grad);
    }

    // one transposed time step n: V = U^n, JUn = JU^n, U1 = U^{n+1}; on entry
    // A.aU, A.aJU, A.af hold the adjoints of U^{n+1}, JU^{n+1}, f^{n+1}, on
    // exit those of U^n, JU^n, f^n
    void adjoint_step(AdjBuffers &A, int64_t n, double *const *V, double *const *JUn,
                      double *const *U1, double weight) {
        const Vec3<const double> v{{V[0], V[1], V[2]}}, ju{{JUn[0], JUn[1], JUn[2]}},
            u1{{U1[0], U1[1], U1[2]}};
        Vec3<double> aU{{A.aU[0], A.aU[1], A.aU[2]}}, aV{{A.aV[0], A.aV[1], A.aV[2]}},
            aJU{{A.aJU[0], A.aJU[1], A.aJU[2]}}, af{{A.af[0], A.af[1], A.af[2]}};
        adjoint_alm(A, cs.dt * (double)n, u1, weight);
        launch_adj_velocity_bc(L, adj::AdjBcArgs{P, v, aU, aV});
        launch_adj_project(L, adj::AdjProjectArgs{P, c(aU), c(aJU), B}, Partials<1>{partial, ticket},
                           A.sumsq);
        double sumsq = 0;
        DALM_CUDA(cudaMemcpyAsync(&sumsq, A.sumsq, sizeof(double), cudaMemcpyDeviceToHost, stream));
        DALM_CUDA(cudaStreamSynchronize(stream));
        if (!std::isfinite(sumsq)) throw std::runtime_error("non-finite adjoint pressure right-hand side");
        if (sumsq > 0) {
            const double ncell = (double)g.ni() * g.nj() * g.nk();
            const double rms = std::sqrt(sumsq / ncell);
            // solved at unit RMS right-hand side (the breakdown test of the
            // Krylov solver is absolute); the previous step's solution,
            // scaled alike, is the guess
            d2d(Pp, A.y);
            launch_adj_scale(L, Pp, g.total, 1.0 / rms);
            launch_adj_scale(L, B, g.total, 1.0 / rms);
            long long it;
            if (adjoint_refinement()) {
                const double saved = tol;
                tol = ADJ_RTOL;
                solve_mixed();
                tol = saved;
                it = h_kst[0].it;
            } else {
                it = adjoint_solve(ADJ_RTOL);
            }
            d2d(A.y, Pp);
            launch_adj_scale(L, A.y, g.total, rms);
            adj_stats.solves++;
            adj_stats.iterations += it;
            adj_stats.max_rel_residual = std::max(adj_stats.max_rel_residual, h_kst[0].err);
        } else {
            zero(A.y);
        }
        launch_adj_faces(L, adj::AdjFacesArgs{P, c(aJU), A.y, aU});
        adj::AdjNutArgs N{P, v, c(aU), A.nu, {}};
        adj::AdjPredictArgs Q{P, v, ju, c(aU), A.nu, {}, aV, aJU, af};
        for (int m = 0; m < 6; m++) {
            N.s6[m] = A.s6[m];
            Q.s6[m] = A.s6[m];
        }
        launch_adj_predict(L, N, Q);
        for (int m = 0; m < 3; m++) {
            std::swap(A.aU[m], A.aV[m]);
            zero(A.aV[m]);
        }
    }

    void power_gradient(int64_t t0, int64_t t1, int64_t k, double *grad_out, double *J_out) {
        if (f32)
            throw Unsupported("the discrete adjoint differentiates the FP64 form "
                              "(DALM_FP64, or DALM_MIXED with reference_sums)");
        const int T = alm.wt_count;
        if (T == 0) throw Unsupported("the case has no turbines");
        if (k < 1) throw std::invalid_argument("ckpt_every must be at least 1");
        const int64_t n_first = std::max<int64_t>(step, 1);
        if (t0 < n_first || t1 < t0)
            throw std::invalid_argument("need max(current step, 1) <= t0 <= t1");
        for (const TurbineDev &w : h_wt)
            if (w.type != EULER_YAW)
                throw Unsupported("the gradient needs yaw-type turbine angles "
                                  "(dalm_set_turbine_params sets them)");
        adj_stats = AdjointStats{};
        // the forces the first step reads, from the current velocity and
        // parameters at the time of the last actuator-line evaluation
        const double t_init = last_alm_time;
        alm_at(t_init);

        Scratch S;
        const int64_t nsteps = t1 - n_first + 1, nseg = (nsteps + k - 1) / k;
        const int64_t last0 = n_first + (nseg - 1) * k;  // first step of the last segment
        std::vector<Snapshot> ck((size_t)nseg);
        for (auto &c : ck) alloc_snapshot(S, c);
        Snapshot fin;
        alloc_snapshot(S, fin);
        double *fin_uold[3];
        for (int m = 0; m < 3; m++) fin_uold[m] = S.get<double>(g.total);
        // tape of one segment: U^n for k+1 steps, JU^n for k
        std::vector<std::array<double *, 3>> tU((size_t)k + 1), tJU((size_t)k);
        for (auto &a : tU)
            for (int m = 0; m < 3; m++) a[m] = S.get<double>(g.total);
        for (auto &a : tJU)
            for (int m = 0; m < 3; m++) a[m] = S.get<double>(g.total);
        auto record = [&](int64_t slot, bool with_flux) {
            for (int m = 0; m < 3; m++) {
                d2d(tU[(size_t)slot][m], U[ucur][m]);
                if (with_flux) d2d(tJU[(size_t)slot][m], JU[jcur][m]);
            }
        };

        // forward run
        double J = 0;
        if (step == 0) step_once();  // step 0: no integration (time average, output)
        for (int64_t n = n_first; n <= t1; n++) {
            if ((n - n_first) % k == 0) save(ck[(size_t)((n - n_first) / k)]);
            if (n >= last0) record(n - last0, true);
            step_once();
            if (n >= t0) {
                fetch_step_outputs();
                DALM_CUDA(cudaStreamSynchronize(stream));
                for (int w = 0; w < T; w++) J += h_wt_out[w] * std::fabs(h_wt[w].rot_speed);
            }
        }
        record(t1 - last0 + 1, false);
        J /= (double)(t1 - t0 + 1);
        if (!std::isfinite(J)) throw std::runtime_error("non-finite power in the forward run");
        save(fin);
        for (int m = 0; m < 3; m++) d2d(fin_uold[m], U[1 - ucur][m]);
        DiagState *fin_diag = S.get<DiagState>(1);
        KrylovState *fin_kst = S.get<KrylovState>(2);
        DALM_CUDA(cudaMemcpyAsync(fin_diag, d_diag, sizeof(DiagState), cudaMemcpyDeviceToDevice, stream));
        DALM_CUDA(cudaMemcpyAsync(fin_kst, d_kst, 2 * sizeof(KrylovState), cudaMemcpyDeviceToDevice, stream));
        fetch_step_outputs();
        DALM_CUDA(cudaStreamSynchronize(stream));
        KrylovState fin_hkst[2] = {h_kst[0], h_kst[1]};
        DiagState fin_hdiag = *h_diag;
        std::vector<double> fin_wt(h_wt_out, h_wt_out + 2 * T);
        const int64_t fin_last_it = last_it;

        // reverse sweep
        AdjBuffers A{};
        for (int m = 0; m < 3; m++) {
            A.aU[m] = S.get<double>(g.total);
            A.aV[m] = S.get<double>(g.total);
            A.aJU[m] = S.get<double>(g.total);
            A.af[m] = S.get<double>(g.total);
            zero(A.aU[m]); zero(A.aV[m]); zero(A.aJU[m]); zero(A.af[m]);
        }
        A.nu = S.get<double>(g.total);
        for (int m = 0; m < 6; m++) A.s6[m] = S.get<double>(g.total);
        A.y = S.get<double>(g.total);
        zero(A.y);
        A.grad = S.get<double>(3 * (size_t)T);
        zero(A.grad, 3 * (size_t)T);
        A.sumsq = S.get<double>(1);
        const size_t ap = (size_t)alm.ap_count;
        A.gather = S.get<double>(6 * ap);
        A.ids = S.get<long long>(8 * ap);
        A.w = S.get<double>(8 * ap);
        A.lU = S.get<double>(3 * ap);
        A.gth = S.get<double>(3 * ap);
        A.torque = S.get<double>(ap);
        const double weight = 1.0 / (double)(t1 - t0 + 1);
        for (int64_t s = nseg - 1; s >= 0; s--) {
            const int64_t n0 = n_first + s * k, n1 = std::min(n0 + k - 1, t1);
            if (s != nseg - 1) {  // the last segment was recorded by the forward run
                load(ck[(size_t)s]);
                for (int64_t n = n0; n <= n1; n++) {
                    record(n - n0, true);
                    integrate_step();
                    adj_stats.recomputed_steps++;
                }
                record(n1 - n0 + 1, false);
            }
            for (int64_t n = n1; n >= n0; n--)
                adjoint_step(A, n, tU[(size_t)(n - n0)].data(), tJU[(size_t)(n - n0)].data(),
                             tU[(size_t)(n - n0 + 1)].data(), n >= t0 ? weight : 0.0);
        }
        // the first step's forces: the actuator line at t_init on U^{n_first}
        adjoint_alm(A, t_init, Vec3<const double>{{tU[0][0], tU[0][1], tU[0][2]}}, 0.0);

        // back to the end of the forward run
        load(fin);
        last_it = fin_last_it;
        for (int m = 0; m < 3; m++) d2d(U[1 - ucur][m], fin_uold[m]);
        DALM_CUDA(cudaMemcpyAsync(d_diag, fin_diag, sizeof(DiagState), cudaMemcpyDeviceToDevice, stream));
        DALM_CUDA(cudaMemcpyAsync(d_kst, fin_kst, 2 * sizeof(KrylovState), cudaMemcpyDeviceToDevice, stream));
        launch_alm_points(L, P, alm, fin.alm_time, c(u_cur()));
        std::vector<double> g_dev(3 * (size_t)T);
        DALM_CUDA(cudaMemcpyAsync(g_dev.data(), A.grad, sizeof(double) * 3 * T, cudaMemcpyDeviceToHost, stream));
        DALM_CUDA(cudaStreamSynchronize(stream));
        h_kst[0] = fin_hkst[0];
        h_kst[1] = fin_hkst[1];
        *h_diag = fin_hdiag;
        std::copy(fin_wt.begin(), fin_wt.end(), h_wt_out);
        for (size_t i = 0; i < g_dev.size(); i++)
            if (!std::isfinite(g_dev[i])) throw std::runtime_error("non-finite adjoint gradient");
        if (grad_out) std::copy(g_dev.begin(), g_dev.end(), grad_out);
        if (J_out) *J_out = J;
    }

    // The last step's diagnostics and turbine loads into their pinned host
    // copies, enqueued where a reader is about to synchronise rather than
    // every step (each small copy costs the stream a few microseconds).
    void fetch_step_outputs() {
        DALM_CUDA(cudaMemcpyAsync(h_diag, d_diag, sizeof(DiagState), cudaMemcpyDeviceToHost, stream));
        if (alm.ap_count > 0) {
            DALM_CUDA(cudaMemcpyAsync(h_wt_out, alm.wt_torque, sizeof(double) * alm.wt_count,
                                      cudaMemcpyDeviceToHost, stream));
            DALM_CUDA(cudaMemcpyAsync(h_wt_out + alm.wt_count, alm.wt_thrust,
                                      sizeof(double) * alm.wt_count, cudaMemcpyDeviceToHost, stream));
        }
    }
    void sync_stats() {
        fetch_step_outputs();
        DALM_CUDA(cudaStreamSynchronize(stream));
        if (opt.profile) harvest();
    }
};

// ---------------------------------------------------------------- C ABI

#define API_BEGIN(h)                                   \
    if (!(h)) {                                        \
        g_last_error = "null handle";                  \
        return DALM_ERR_ARG;                           \
    }                                                  \
    try {
#define API_END(h)                                     \
    }                                                  \
    catch (const CudaError &e) {                       \
        (h)->err = e.what();                           \
        return DALM_ERR_CUDA;                          \
    }                                                  \
    catch (const DeviceWaitError &e) {                 \
        (h)->err = e.what();                           \
        return DALM_ERR_DEVICE_WAIT;                   \
    }                                                  \
    catch (const Unsupported &e) {                     \
        (h)->err = e.what();                           \
        return DALM_ERR_UNSUPPORTED;                   \
    }                                                  \
    catch (const std::invalid_argument &e) {           \
        (h)->err = e.what();                           \
        return DALM_ERR_ARG;                           \
    }                                                  \
    catch (const std::exception &e) {                  \
        (h)->err = e.what();                           \
        return DALM_ERR_CASE;                          \
    }                                                  \
    return DALM_OK;

extern "C" {

void dalm_default_options(dalm_options *opt) {
    if (!opt) return;
    memset(opt, 0, sizeof(*opt));
    opt->precision = DALM_FP64;
    opt->limiter = DALM_LIMITER_MINMOD;
    opt->device = 0;
    opt->time_average = 1;
    opt->check_finite = 1;
    opt->poisson_batch = 0;
    opt->use_graphs = 1;
    opt->profile = 0;
    opt->reference_sums = 0;
    opt->fused_krylov = 0;
    opt->write_output = 0;
    opt->refine_inner_it = 0;
}

int dalm_create(const char *case_dir, const dalm_options *opt, dalm_handle **out) {
    if (!case_dir || !out) {
        g_last_error = "null argument";
        return DALM_ERR_ARG;
    }
    *out = nullptr;
    dalm_options o;
    if (opt) o = *opt;
    else dalm_default_options(&o);
    std::unique_ptr<dalm_handle> h(new dalm_handle());
    try {
        h->init(case_dir, o);
    } catch (const CudaError &e) {
        g_last_error = e.what();
        return DALM_ERR_CUDA;
    } catch (const Unsupported &e) {
        g_last_error = e.what();
        return DALM_ERR_UNSUPPORTED;
    } catch (const std::invalid_argument &e) {
        g_last_error = e.what();
        return DALM_ERR_ARG;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return DALM_ERR_CASE;
    }
    *out = h.release();
    return DALM_OK;
}

void dalm_destroy(dalm_handle *h) { delete h; }

const char *dalm_last_error(const dalm_handle *h) {
    return h ? h->err.c_str() : g_last_error.c_str();
}

int dalm_get_size(dalm_handle *h, int64_t size[3], int64_t *gc) {
    API_BEGIN(h)
    if (size)
        for (int m = 0; m < 3; m++) size[m] = h->cs.size[m];
    if (gc) *gc = h->cs.gc;
    API_END(h)
}

int dalm_get_mesh(dalm_handle *h, double *x, double *y, double *z, double *dx, double *dy,
                  double *dz) {
    API_BEGIN(h)
    auto cp = [](double *d, const std::vector<double> &v) {
        if (d) memcpy(d, v.data(), v.size() * sizeof(double));
    };
    cp(x, h->cs.x); cp(y, h->cs.y); cp(z, h->cs.z);
    cp(dx, h->cs.dx); cp(dy, h->cs.dy); cp(dz, h->cs.dz);
    API_END(h)
}

int dalm_get_runtime(dalm_handle *h, double *dt, int64_t *max_step) {
    API_BEGIN(h)
    if (dt) *dt = h->cs.dt;
    if (max_step) *max_step = h->cs.max_step;
    API_END(h)
}

int dalm_get_max_diag(dalm_handle *h, double *md) {
    API_BEGIN(h)
    if (!md) throw std::invalid_argument("null pointer");
    *md = h->cs.max_diag;
    API_END(h)
}

int dalm_set_state(dalm_handle *h, const double *U, const double *JU, const double *p, int flags) {
    API_BEGIN(h)
    if (!U) throw std::invalid_argument("U must not be null");
    h->upload_field(U, 3, h->U[h->ucur]);
    if (p) h->upload_field(p, 1, &h->Pp);
    h->refresh_after_state(flags, JU);
    h->sync_stats();
    API_END(h)
}

int dalm_get_field(dalm_handle *h, int field, double *out) {
    API_BEGIN(h)
    if (!out) throw std::invalid_argument("null output");
    h->get_field(field, out);
    API_END(h)
}

int dalm_set_field(dalm_handle *h, int field, const double *in) {
    API_BEGIN(h)
    if (!in) throw std::invalid_argument("null input");
    h->set_field(field, in);
    API_END(h)
}

int dalm_set_inflow_profile(dalm_handle *h, const double *prof) {
    API_BEGIN(h)
    DALM_CUDA(cudaStreamSynchronize(h->stream));
    if (!prof) {
        h->P.prof = nullptr;
    } else {
        if (!h->d_prof) h->d_prof = h->dalloc<double>((size_t)3 * h->g.ny * h->g.nz);
        DALM_CUDA(cudaMemcpy(h->d_prof, prof, sizeof(double) * 3 * h->g.ny * h->g.nz,
                             cudaMemcpyHostToDevice));
        h->P.prof = h->d_prof;
    }
    API_END(h)
}

int dalm_set_turbine_params(dalm_handle *h, const double *yaw_deg, const double *pitch_deg,
                            const double *omega) {
    API_BEGIN(h)
    if (h->alm.ap_count == 0) return DALM_OK;
    DALM_CUDA(cudaStreamSynchronize(h->stream));
    int T = h->alm.wt_count, per = h->alm.ap_per_wt;
    for (int w = 0; w < T; w++) {
        TurbineDev &d = h->h_wt[w];
        if (yaw_deg) {
            d.type = EULER_YAW;
            d.formula[0] = d.formula[1] = d.formula[2] = 0;
            d.formula[3] = yaw_deg[w] * PI_D / 180;  // deg_to_rad, src/util.h:214-216
        }
        if (omega) d.rot_speed = omega[w];
        if (pitch_deg) {
            h->pitch_deg[w] = pitch_deg[w];
            for (int a = w * per; a < (w + 1) * per; a++) h->twist[a] = h->base_twist[a] + pitch_deg[w];
        }
    }
    DALM_CUDA(cudaMemcpy((void *)h->alm.wt, h->h_wt.data(), sizeof(TurbineDev) * T,
                         cudaMemcpyHostToDevice));
    DALM_CUDA(cudaMemcpy((void *)h->alm.twist, h->twist.data(), sizeof(double) * h->twist.size(),
                         cudaMemcpyHostToDevice));
    API_END(h)
}

int dalm_get_turbine_params(dalm_handle *h, double *yaw_deg, double *pitch_deg, double *omega) {
    API_BEGIN(h)
    for (int w = 0; w < h->alm.wt_count; w++) {
        const TurbineDev &d = h->h_wt[w];
        if (yaw_deg) yaw_deg[w] = d.formula[3] * 180 / PI_D;
        if (pitch_deg) pitch_deg[w] = h->pitch_deg[w];
        if (omega) omega[w] = d.rot_speed;
    }
    API_END(h)
}

int dalm_adjoint_power_grad(dalm_handle *h, int t0, int t1, int ckpt_every, double *grad,
                            double *J) {
    API_BEGIN(h)
    h->power_gradient(t0, t1, ckpt_every, grad, J);
    API_END(h)
}

int dalm_get_adjoint_stats(dalm_handle *h, int64_t *solves, int64_t *iterations,
                           double *max_rel_residual, int64_t *recomputed_steps) {
    API_BEGIN(h)
    if (solves) *solves = h->adj_stats.solves;
    if (iterations) *iterations = h->adj_stats.iterations;
    if (max_rel_residual) *max_rel_residual = h->adj_stats.max_rel_residual;
    if (recomputed_steps) *recomputed_steps = h->adj_stats.recomputed_steps;
    API_END(h)
}

int dalm_step(dalm_handle *h, int nsteps) {
    API_BEGIN(h)
    if (nsteps < 0) throw std::invalid_argument("nsteps < 0");
    for (int n = 0; n < nsteps; n++) h->step_once();
    h->sync_stats();
    if (h->opt.check_finite && h->step > 1) {
        if (!std::isfinite(h->h_diag->avg_div) || !std::isfinite(h->h_kst->err)) {
            h->err = "non-finite state after step " + std::to_string(h->step - 1);
            return DALM_ERR_NONFINITE;
        }
    }
    API_END(h)
}

int dalm_run_stage(dalm_handle *h, int stage) {
    API_BEGIN(h)
    h->run_stage(stage);
    h->sync_stats();
    API_END(h)
}

int dalm_advance_clock(dalm_handle *h) {
    API_BEGIN(h)
    h->step++;
    API_END(h)
}

int dalm_get_step_stats(dalm_handle *h, int64_t *step, int64_t *poisson_it, double *poisson_err,
                        double *avg_div, double *max_cfl) {
    API_BEGIN(h)
    h->sync_stats();
    if (step) *step = h->step;
    if (poisson_it) *poisson_it = h->h_kst->it;
    if (poisson_err) *poisson_err = h->h_kst->err;
    if (avg_div) *avg_div = h->h_diag->avg_div;
    if (max_cfl) *max_cfl = h->h_diag->max_cfl;
    API_END(h)
}

int dalm_set_poisson(dalm_handle *h, int64_t max_it, double tol) {
    API_BEGIN(h)
    h->max_it = max_it;
    h->tol = tol;
    API_END(h)
}

int dalm_get_counts(dalm_handle *h, int64_t counts[5]) {
    API_BEGIN(h)
    if (!counts) throw std::invalid_argument("null output");
    counts[0] = h->alm.wt_count;
    counts[1] = h->alm.ap_count;
    counts[2] = h->alm.blades;
    counts[3] = h->alm.ap_per_blade;
    counts[4] = h->alm.atk_count;
    API_END(h)
}

int dalm_get_turbines(dalm_handle *h, double *thrust, double *torque, double *power) {
    API_BEGIN(h)
    h->sync_stats();
    int T = h->alm.wt_count;
    for (int w = 0; w < T; w++) {
        double tq = h->h_wt_out[w], th = h->h_wt_out[T + w];
        if (thrust) thrust[w] = th;
        if (torque) torque[w] = tq;
        if (power) power[w] = tq * fabs(h->h_wt[w].rot_speed);
    }
    API_END(h)
}

int dalm_get_points(dalm_handle *h, double *xyz, double *f, double *torque, double *thrust) {
    API_BEGIN(h)
    h->sync_stats();
    int n = h->alm.ap_count;
    if (n == 0) return DALM_OK;
    if (xyz) DALM_CUDA(cudaMemcpy(xyz, h->alm.pt_xyz, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
    if (f) DALM_CUDA(cudaMemcpy(f, h->alm.pt_f, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
    if (torque) DALM_CUDA(cudaMemcpy(torque, h->alm.pt_torque, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (thrust) DALM_CUDA(cudaMemcpy(thrust, h->alm.pt_thrust, sizeof(double) * n, cudaMemcpyDeviceToHost));
    API_END(h)
}

int dalm_synchronize(dalm_handle *h) {
    API_BEGIN(h)
    h->sync_stats();
    API_END(h)
}

int dalm_get_stream(dalm_handle *h, void **stream) {
    API_BEGIN(h)
    if (!stream) throw std::invalid_argument("null output");
    *stream = (void *)h->stream;
    API_END(h)
}

int dalm_get_timings(dalm_handle *h, double ms[7], int64_t *launches, int reset) {
    API_BEGIN(h)
    h->sync_stats();
    if (ms)
        for (int s = 0; s < 7; s++) ms[s] = h->stage_ms[s];
    if (launches) *launches = h->launch_count;
    if (reset) {
        for (int s = 0; s < 7; s++) h->stage_ms[s] = 0;
        for (int k = 0; k < KK_COUNT; k++) {
            h->kind_ms[k] = 0;
            h->kind_launches[k] = 0;
            h->kind_bytes[k] = 0;
        }
        h->launch_count = 0;
    }
    API_END(h)
}

int dalm_kernel_kinds(void) { return KK_COUNT; }

int dalm_get_kernel_timing(dalm_handle *h, int index, const char **name, int64_t *launches,
                           double *ms, double *bytes_per_launch) {
    API_BEGIN(h)
    if (index < 0 || index >= KK_COUNT) throw std::invalid_argument("kernel index out of range");
    h->sync_stats();
    if (name) *name = kKindNames[index];
    if (launches) *launches = h->kind_launches[index];
    if (ms) *ms = h->kind_ms[index];
    if (bytes_per_launch) {
        // algorithmic DRAM bytes: each persistent array read or written once
        // per launch over interior cells (8-byte scalars)
        double n = (double)h->g.ni() * h->g.nj() * h->g.nk();
        double stored = (double)h->g.nx * h->g.ny * h->g.nz;
        double fcells = h->fbox.empty() ? 0.0
                        : (double)(h->fbox.hi[0] - h->fbox.lo[0]) * (h->fbox.hi[1] - h->fbox.lo[1]) *
                              (h->fbox.hi[2] - h->fbox.lo[2]);
        double s = 0;
        // the stencil fields U, JU, f: 8 bytes, or 4 as the mixed form's FP32 fields
        const double v = h->f32 ? 0.5 : 1.0;
        switch (index) {
        case KK_PREDICT: s = h->f32 ? v * (9 * n + 3 * fcells) : 9 * n + 3 * fcells + 6 * (stored - n); break;
        case KK_FLUX_RHS: s = 6 * v * n + n; break;       // R U; W JU (stencil fields), b (FP64)
        case KK_PROJECT: s = 12 * v * n + n; break;       // R U, JU, p; W U, JU
        case KK_DIAG: s = 6 * v * n; break;
        case KK_TAVG: s = (6 + 3 * v) * stored; break;    // R Utavg, U; W Utavg
        case KK_ALM_PROJECT: s = 3 * v * fcells; break;
        case KK_SOR_SWEEP: s = 2 * n; break;
        case KK_RESIDUAL_NORM: s = (h->pcfg.method == PM_JACOBI ? 3 : 2) * n; break;
        case KK_JACOBI_SWEEP: s = 3 * n; break;
        case KK_JACOBI_SWEEP2: s = 3 * n; break;  // R x, rhs; W out: the pair's bytes
        case KK_BICG_INIT: s = 5 * n; break;
        case KK_BICG_P: s = 5 * n; break;
        case KK_BICG_Q: s = 3 * n; break;
        case KK_BICG_S: s = 4 * n; break;
        case KK_BICG_T: s = 3 * n; break;
        case KK_BICG_XR: s = 8 * n; break;
        case KK_BICG_PF: s = 7 * n; break;
        case KK_BICG_SF: s = 5 * n; break;
        case KK_REFINE_RESIDUAL:  // R x, b (FP64); W r (FP32) [, r0, q for BiCGStab inner solves]
            s = (h->mg_on ? 2.5 : 3.5) * n;
            break;
        case KK_REFINE_UPDATE: s = 2.5 * n; break;    // R x, e; W x
        // FP32 vectors: half the scalars' bytes
        case KK_SOR_SWEEP32: s = 2 * n / 2.0; break;
        case KK_JACOBI_SWEEP32: s = 3 * n / 2.0; break;
        case KK_BICG_P32: s = 5 * n / 2.0; break;
        case KK_BICG_Q32: s = 3 * n / 2.0; break;
        case KK_BICG_S32: s = 4 * n / 2.0; break;
        case KK_BICG_T32: s = 3 * n / 2.0; break;
        case KK_BICG_XR32: s = 8 * n / 2.0; break;
        default: s = 0; break;
        }
        *bytes_per_launch = 8.0 * s;
        // kinds whose launches differ in size (the multigrid levels) count
        // their bytes at launch time
        if (h->kind_bytes[index] > 0 && h->kind_launches[index] > 0)
            *bytes_per_launch = h->kind_bytes[index] / (double)h->kind_launches[index];
    }
    API_END(h)
}

}  // extern "C"
