// Host-side driver of the adjoint building blocks (test infrastructure).
//
// Compiled by tests/test_adjoint_math.py with nvcc as host code only (no
// kernel is launched): it runs the same __host__ __device__ functions the
// CUDA kernels call (3dalm_b200/csrc/adjoint_cell.cuh) over a small grid in
// plain loops, so the CPU test suite can check the transposed stages
// against finite differences of the oracle's forward step.  Fields are host
// arrays in the product's padded SoA layout (Grid::make).
#include <cstring>
#include <vector>

#include "../3dalm_b200/csrc/adjoint_cell.cuh"

using namespace dalm;

namespace {

struct Ctx {
    StepParams P{};
    AlmDev A{};
    std::vector<TurbineDev> wt;
    std::vector<double> pt_xyz, pt_f, pt_torque, pt_thrust, wt_torque, wt_thrust;
};

Vec3<double> v3(double **p) { return {{p[0], p[1], p[2]}}; }
Vec3<const double> c3(double **p) { return {{p[0], p[1], p[2]}}; }

}  // namespace

extern "C" {

void *hx_create(int nx, int ny, int nz, int gc, const double *x, const double *y,
                const double *z, const double *dx, const double *dy, const double *dz,
                double re, double dt, double max_diag, int limiter, const double *filter2) {
    Ctx *c = new Ctx();
    c->P.g = Grid::make(nx, ny, nz, gc);
    c->P.m = MeshDev{x, y, z, dx, dy, dz};
    c->P.re = re;
    c->P.dt = dt;
    c->P.max_diag = max_diag;
    c->P.limiter = limiter;
    c->P.filter2 = filter2;
    return c;
}

void hx_destroy(void *ctx) { delete (Ctx *)ctx; }

long long hx_total(void *ctx) { return ((Ctx *)ctx)->P.g.total; }

void hx_set_alm(void *ctx, int wt_count, int ap_per_wt, int ap_per_blade, int blades,
                int atk_count, double pw2, double e_coef, double cutoff2, const double *base,
                const double *rot_center, const double *formula, const double *rot_speed,
                const int *type, const double *r, const double *dr, const double *chord,
                const double *twist, const double *cd, const double *cl, const double *atk) {
    Ctx *c = (Ctx *)ctx;
    c->wt.assign(wt_count, TurbineDev{});
    for (int w = 0; w < wt_count; w++) {
        for (int m = 0; m < 3; m++) {
            c->wt[w].base[m] = base[3 * w + m];
            c->wt[w].rot_center[m] = rot_center[3 * w + m];
        }
        for (int m = 0; m < 4; m++) c->wt[w].formula[m] = formula[4 * w + m];
        c->wt[w].rot_speed = rot_speed[w];
        c->wt[w].type = type[w];
    }
    int ap = wt_count * ap_per_wt;
    c->pt_xyz.assign(3 * ap, 0);
    c->pt_f.assign(3 * ap, 0);
    c->pt_torque.assign(ap, 0);
    c->pt_thrust.assign(ap, 0);
    AlmDev &A = c->A;
    A.wt_count = wt_count;
    A.ap_count = ap;
    A.ap_per_wt = ap_per_wt;
    A.ap_per_blade = ap_per_blade;
    A.blades = blades;
    A.atk_count = atk_count;
    A.pw2 = pw2;
    A.e_coef = e_coef;
    A.cutoff2 = cutoff2;
    A.wt = c->wt.data();
    A.r = r; A.dr = dr; A.chord = chord; A.twist = twist;
    A.cd = cd; A.cl = cl; A.atk = atk;
    A.pt_xyz = c->pt_xyz.data();
    A.pt_f = c->pt_f.data();
    A.pt_torque = c->pt_torque.data();
    A.pt_thrust = c->pt_thrust.data();
}

// The forward blade points (generic point model with plain doubles): fills
// xyz[ap][3], f[ap][3], torque[ap], thrust[ap].
void hx_alm_points(void *ctx, double **U, double t, double *xyz, double *f, double *torque,
                   double *thrust) {
    Ctx *c = (Ctx *)ctx;
    const double z3[3] = {0, 0, 0};
    for (int a = 0; a < c->A.ap_count; a++) {
        const TurbineDev &wt = c->wt[a / c->A.ap_per_wt];
        adj::PointEval<double> e;
        adj::alm_point_eval<double>(c->P, c->A, wt, a, t, c3(U), wt.formula[3], 0.0, wt.rot_speed,
                                    z3, e);
        for (int m = 0; m < 3; m++) {
            xyz[3 * a + m] = e.xyz[m];
            f[3 * a + m] = e.f[m];
        }
        torque[a] = e.torque;
        thrust[a] = e.thrust;
    }
}

// Adjoint of the actuator line at time t on velocity U: af is the adjoint of
// the projected force, weight the objective's weight of this step's power.
void hx_adj_alm(void *ctx, double **U, double **af, double t, double weight, double **aU,
                double *grad) {
    Ctx *c = (Ctx *)ctx;
    int n = c->A.ap_count;
    hx_alm_points(ctx, U, t, c->pt_xyz.data(), c->pt_f.data(), c->pt_torque.data(),
                  c->pt_thrust.data());
    std::vector<double> gather(6 * n, 0.0), lU(3 * n), gth(3 * n), w(8 * n), tq(n);
    std::vector<long long> ids(8 * n);
    for (int a = 0; a < n; a++) {
        int lo[3], hi[3];
        adj::alm_support_box(c->P, c->A, a, lo, hi);
        double acc[6] = {0, 0, 0, 0, 0, 0};
        for (int i = lo[0]; i < hi[0]; i++)
            for (int j = lo[1]; j < hi[1]; j++)
                for (int k = lo[2]; k < hi[2]; k++)
                    adj::adj_alm_gather_term(c->P, c->A, c3(af), a, i, j, k, acc);
        for (int m = 0; m < 6; m++) gather[6 * a + m] = acc[m];
    }
    adj::AdjAlmPointArgs X{c->P, c->A, c3(U), t, weight, gather.data(), ids.data(),
                           w.data(), lU.data(), gth.data(), tq.data()};
    for (int a = 0; a < n; a++) adj::adj_alm_point(X, a);
    adj::adj_alm_scatter(c->A, ids.data(), w.data(), lU.data(), gth.data(), tq.data(), weight,
                         v3(aU), grad);
}

void hx_adj_velocity_bc(void *ctx, double **V, double **aU, double **aV) {
    Ctx *c = (Ctx *)ctx;
    const Grid &g = c->P.g;
    long long tot = 2 * ((long long)g.nj() * g.nk() + (long long)g.ni() * g.nk() +
                         (long long)g.ni() * g.nj());
    adj::AdjBcArgs A{c->P, c3(V), v3(aU), v3(aV)};
    for (long long n = 0; n < tot; n++) adj::adj_velocity_bc_column(A, n);
}

double hx_adj_project(void *ctx, double **aU, double **aJU, double *rhs) {
    Ctx *c = (Ctx *)ctx;
    const Grid &g = c->P.g;
    adj::AdjProjectArgs A{c->P, c3(aU), c3(aJU), rhs};
    double s = 0;
    for (int i = g.gc; i < g.nx - g.gc; i++)
        for (int j = g.gc; j < g.ny - g.gc; j++)
            for (int k = g.gc; k < g.nz - g.gc; k++) s += adj::adj_project_cell(A, i, j, k);
    return s;
}

void hx_adj_faces(void *ctx, double **aJU, const double *y, double **aus) {
    Ctx *c = (Ctx *)ctx;
    const Grid &g = c->P.g;
    adj::AdjFacesArgs A{c->P, c3(aJU), y, v3(aus)};
    for (int i = g.gc; i <= g.nx - g.gc; i++)
        for (int j = g.gc; j < g.ny - g.gc; j++)
            for (int k = g.gc; k < g.nz - g.gc; k++) adj::adj_faces_cell(A, i, j, k);
}

void hx_adj_predict(void *ctx, double **V, double **JU, double **aus, double **aV, double **aJU,
                    double **af) {
    Ctx *c = (Ctx *)ctx;
    const Grid &g = c->P.g;
    std::vector<double> nu(g.total, 0.0);
    std::vector<std::vector<double>> s6(6, std::vector<double>(g.total, 0.0));
    adj::AdjNutArgs N{c->P, c3(V), c3(aus), nu.data(), {}};
    for (int m = 0; m < 6; m++) N.s6[m] = s6[m].data();
    for (int i = g.gc; i < g.nx - g.gc; i++)
        for (int j = g.gc; j < g.ny - g.gc; j++)
            for (int k = g.gc; k < g.nz - g.gc; k++) adj::adj_nut_cell(N, i, j, k);
    adj::AdjPredictArgs A{c->P, c3(V), c3(JU), c3(aus), nu.data(), {}, v3(aV), v3(aJU), v3(af)};
    for (int m = 0; m < 6; m++) A.s6[m] = s6[m].data();
    for (int i = 0; i < g.nx; i++)
        for (int j = 0; j < g.ny; j++)
            for (int k = 0; k < g.nz; k++) adj::adj_predict_cell(A, i, j, k);
}

}  // extern "C"
