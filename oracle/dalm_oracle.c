/*
 * ORACLE — CPU restatement of the 3dalm per-time-step hot path (FP64, serial).
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py as the checker; never by the product.
 *
 * Pinned against the reference itself: tests/test_oracle_pin.py drives this
 * file and the reference solver compiled from its own sources
 * (oracle/_ref/libref3dalm.so, recipe in oracle/Makefile) on identical
 * inputs and requires bit-identical fields; tests/golden/ holds fixtures
 * produced by the reference for when oracle/_ref is not built.
 *
 * Citations are path:line in the reference project (ki2098/3dalm).
 */
#include "dalm_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_PI 3.14159265358979323846 /* M_PI, src/type.h:12 */

typedef struct {
    double base[3], rot_center[3];
    int angle_type;
    double angle, ow, formula[4], rot_speed, torque, thrust;
} or_turbine; /* WindTurbine, src/alm.h:23-33 */

typedef struct {
    double xyz[3], r, chord, twist, theta, dr, f[3], torque, thrust;
} or_point; /* ActuatorPoint, src/alm.h:10-21 (velocity slot unused) */

struct dalm_oracle {
    int64_t nx, ny, nz, gc, len;
    double *x, *y, *z, *dx, *dy, *dz;
    double uin[3], re, cs, dt;
    /* fields (Cfd, src/solver.h:286-344) */
    double *U, *Uold, *Utavg, *JU, *p, *nut, *div, *f;
    /* Poisson (Eq, src/solver.h:346-404) */
    double *A, *b, *r, *r0, *pk, *pp, *q, *s, *ss, *t, *tmp;
    double max_diag;
    int solver, pc;
    int64_t it, max_it, pc_max_it;
    double err, tol, relax, pc_relax;
    double avg_div, max_cfl;
    int sum_order; /* 0: the reference's serial sums; 1: pairwise (test only) */
    int limiter;   /* 0: the reference's b=4 limiter, 1: van Albada (extension) */
    double *solid; /* turbulence-generating grid's solid fraction, or NULL */
    int retracted; /* retracted floor */
    double floor_start;
    /* runtime (src/solver.h:176-205) */
    int64_t step, max_step, tavg_count;
    double tavg_start_time;
    /* inflow profile extension */
    int has_profile;
    double *profile; /* [NY][NZ][3] */
    /* actuator line (Alm, src/solver.h:467-517) */
    int64_t wt_count, ap_count, blades, ap_per_blade, atk_count;
    double projection_width;
    or_turbine *wt;
    or_point *ap;
    double *base_twist;
    double *cd, *cl, *atk; /* [ap][atk], [ap][atk], [atk] */
};

static inline int64_t ID(const dalm_oracle *o, int64_t i, int64_t j, int64_t k) {
    return (i * o->ny + j) * o->nz + k; /* index(), src/util.h:11-13 */
}
static inline double sq(double v) { return v * v; }
static inline double cube(double v) { return v * v * v; }
static inline double sgn(double v) { return (double)((v > 0.) - (v < 0.)); } /* src/util.h:83-85 */

/* find_floor_index, src/util.h:119-146 (binary search, -1 below range) */
static int64_t floor_index(const double *a, double v, int64_t n) {
    if (v < a[0]) return -1;
    if (v >= a[n - 1]) return n - 1;
    int64_t lo = 0, hi = n - 1, found = -1;
    while (lo <= hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (a[mid] <= v) {
            found = mid;
            lo = mid + 1;
        } else {
            hi = mid - 1;
        }
    }
    return found;
}

/* Lagrange extrapolation through three points, src/util.h:201-212 */
static double quad_poly(double x0, double x1, double x2, double f0, double f1, double f2,
                        double x3) {
    double l0 = ((x3 - x1) * (x3 - x2)) / ((x0 - x1) * (x0 - x2));
    double l1 = ((x3 - x0) * (x3 - x2)) / ((x1 - x0) * (x1 - x2));
    double l2 = ((x3 - x0) * (x3 - x1)) / ((x2 - x0) * (x2 - x1));
    return f0 * l0 + f1 * l1 + f2 * l2;
}

/* ------------------------------------------------------------------ setup */

/* dx[i] = (x[i+1]-x[i-1])/2 with one-sided ends, src/io.h:112-125 */
static void build_spacing(const double *c, double *d, int64_t n) {
    for (int64_t i = 1; i < n - 1; i++) d[i] = 0.5 * (c[i + 1] - c[i - 1]);
    d[0] = -1.5 * c[0] + 2.0 * c[1] - 0.5 * c[2];
    d[n - 1] = 1.5 * c[n - 1] - 2.0 * c[n - 2] + 0.5 * c[n - 3];
}

/* get_intersection, src/util.h:84-90 */
static double intersection(double h1, double t1, double h2, double t2) {
    double l1 = t1 - h1, l2 = t2 - h2, x1 = t1 - h2, x2 = t2 - h1;
    return fmax(0., fmin(l1, fmin(l2, fmin(x1, x2))));
}

/* set_turbulence_generating_grid, src/solver.h:52-159 */
static void build_solid(dalm_oracle *o, const oracle_params *prm) {
    o->solid = calloc(o->len, sizeof(double));
    double thick = prm->grid_thick, mesh = prm->grid_mesh, bar = prm->grid_bar;
    double gx = prm->grid_at[0], gy = prm->grid_at[1], gz = prm->grid_at[2];
    for (int64_t i = o->gc; i < o->nx - o->gc; i++)
        for (int64_t j = o->gc; j < o->ny - o->gc; j++)
            for (int64_t k = o->gc; k < o->nz - o->gc; k++) {
                double xc = o->x[i], yc = o->y[j], zc = o->z[k];
                double dxc = o->dx[i], dyc = o->dy[j], dzc = o->dz[k];
                double xv = intersection(xc - 0.5 * dxc, xc + 0.5 * dxc, gx - thick, gx);
                int64_t bj = (int64_t)round((yc - gy) / mesh);
                double by = bj * mesh + gy;
                double yi = intersection(yc - 0.5 * dyc, yc + 0.5 * dyc, by - 0.5 * bar, by + 0.5 * bar);
                double xh = intersection(xc - 0.5 * dxc, xc + 0.5 * dxc, gx - 2 * thick, gx - thick);
                int64_t bk = (int64_t)round((zc - gz) / mesh);
                double bz = bk * mesh + gz;
                double zi = intersection(zc - 0.5 * dzc, zc + 0.5 * dzc, bz - 0.5 * bar, bz + 0.5 * bar);
                double occupied = xv * yi * dzc + xh * zi * dyc;
                o->solid[ID(o, i, j, k)] = occupied / (dxc * dyc * dzc);
            }
}

/* set_solid_U, src/cfd.h:1143-1160 */
static void solid_velocity(dalm_oracle *o) {
    if (!o->solid) return;
    for (int64_t i = o->gc; i < o->nx - o->gc; i++)
        for (int64_t j = o->gc; j < o->ny - o->gc; j++)
            for (int64_t k = o->gc; k < o->nz - o->gc; k++) {
                int64_t id = ID(o, i, j, k);
                for (int m = 0; m < 3; m++) o->U[id * 3 + m] = (1. - o->solid[id]) * o->U[id * 3 + m];
            }
}

/* build_A, src/eq.h:701-798 (single domain, offset 0) */
static void build_matrix(dalm_oracle *o) {
    double max_diag = 0;
    int64_t gc = o->gc;
    for (int64_t i = gc; i < o->nx - gc; i++)
        for (int64_t j = gc; j < o->ny - gc; j++)
            for (int64_t k = gc; k < o->nz - gc; k++) {
                double *a = &o->A[ID(o, i, j, k) * 7];
                double dxc = o->dx[i], dyc = o->dy[j], dzc = o->dz[k];
                double dxec = o->x[i + 1] - o->x[i], dxcw = o->x[i] - o->x[i - 1];
                double dync = o->y[j + 1] - o->y[j], dycs = o->y[j] - o->y[j - 1];
                double dztc = o->z[k + 1] - o->z[k], dzcb = o->z[k] - o->z[k - 1];
                double ae = 0, aw = 0, an = 0, as = 0, at = 0, ab = 0, ac = 0;
                if (i < o->nx - gc - 1) {
                    ae = 1 / (dxc * dxec);
                    ac -= ae;
                } else {
                    ac -= 2 / (dxc * dxc); /* x+ outlet: Dirichlet p = 0 */
                }
                if (i > gc) { aw = 1 / (dxc * dxcw); ac -= aw; }
                if (j < o->ny - gc - 1) { an = 1 / (dyc * dync); ac -= an; }
                if (j > gc) { as = 1 / (dyc * dycs); ac -= as; }
                if (k < o->nz - gc - 1) { at = 1 / (dzc * dztc); ac -= at; }
                if (k > gc) { ab = 1 / (dzc * dzcb); ac -= ab; }
                a[0] = ac; a[1] = ae; a[2] = aw; a[3] = an; a[4] = as; a[5] = at; a[6] = ab;
                if (fabs(ac) > max_diag) max_diag = fabs(ac);
            }
    for (int64_t i = gc; i < o->nx - gc; i++)
        for (int64_t j = gc; j < o->ny - gc; j++)
            for (int64_t k = gc; k < o->nz - gc; k++) {
                double *a = &o->A[ID(o, i, j, k) * 7];
                for (int m = 0; m < 7; m++) a[m] /= max_diag;
            }
    o->max_diag = max_diag;
}

/* build_ap_props (JSON form, then array form), src/alm.h:35-142 */
static void build_points(dalm_oracle *o, const oracle_params *prm) {
    int64_t S = prm->station_count, NA = prm->atk_count;
    int64_t ap_per_wt = prm->blades * prm->points_per_blade;
    o->ap_count = prm->turbine_count * ap_per_wt;
    o->atk_count = NA;
    o->ap = calloc(o->ap_count ? o->ap_count : 1, sizeof(or_point));
    o->base_twist = calloc(o->ap_count ? o->ap_count : 1, sizeof(double));
    o->cd = calloc(o->ap_count * NA + 1, sizeof(double));
    o->cl = calloc(o->ap_count * NA + 1, sizeof(double));
    o->atk = calloc(NA + 1, sizeof(double));
    for (int64_t j = 0; j < NA; j++) o->atk[j] = prm->atk[j];
    double dr = (prm->rotor_r - prm->hub_r) / prm->points_per_blade;
    for (int64_t a = 0; a < o->ap_count; a++) {
        or_point *pt = &o->ap[a];
        double r = prm->hub_r + (a % prm->points_per_blade + 0.5) * dr;
        pt->r = r;
        pt->dr = dr;
        int64_t af = floor_index(prm->station_r, r, S);
        double *cd = &o->cd[a * NA], *cl = &o->cl[a * NA];
        if (af < 0 || af >= S - 1) {
            int64_t s = af < 0 ? 0 : S - 1;
            pt->chord = prm->station_chord[s];
            pt->twist = prm->station_twist[s];
            for (int64_t j = 0; j < NA; j++) {
                cd[j] = prm->station_cd[s * NA + j];
                cl[j] = prm->station_cl[s * NA + j];
            }
        } else {
            double a1 = (r - prm->station_r[af]) / (prm->station_r[af + 1] - prm->station_r[af]);
            double a0 = 1 - a1;
            pt->chord = a0 * prm->station_chord[af] + a1 * prm->station_chord[af + 1];
            pt->twist = a0 * prm->station_twist[af] + a1 * prm->station_twist[af + 1];
            for (int64_t j = 0; j < NA; j++) {
                cd[j] = a0 * prm->station_cd[af * NA + j] + a1 * prm->station_cd[(af + 1) * NA + j];
                cl[j] = a0 * prm->station_cl[af * NA + j] + a1 * prm->station_cl[(af + 1) * NA + j];
            }
        }
        o->base_twist[a] = pt->twist;
    }
}

dalm_oracle *oracle_create(const oracle_params *prm) {
    dalm_oracle *o = calloc(1, sizeof(dalm_oracle));
    o->nx = prm->size[0]; o->ny = prm->size[1]; o->nz = prm->size[2];
    o->gc = prm->gc;
    o->len = o->nx * o->ny * o->nz;
    int64_t n[3] = {o->nx, o->ny, o->nz};
    const double *src[3] = {prm->x, prm->y, prm->z};
    double **c[3] = {&o->x, &o->y, &o->z}, **d[3] = {&o->dx, &o->dy, &o->dz};
    for (int a = 0; a < 3; a++) {
        *c[a] = malloc(n[a] * sizeof(double));
        *d[a] = malloc(n[a] * sizeof(double));
        memcpy(*c[a], src[a], n[a] * sizeof(double));
        build_spacing(*c[a], *d[a], n[a]);
    }
    memcpy(o->uin, prm->uin, sizeof(o->uin));
    o->re = prm->re; o->cs = prm->cs; o->dt = prm->dt;
    o->max_step = prm->max_step;
    o->tavg_start_time = prm->tavg_start_time;
    o->solver = prm->solver; o->pc = prm->pc;
    o->max_it = prm->max_it; o->pc_max_it = prm->pc_max_it;
    o->tol = prm->tol; o->relax = prm->relax; o->pc_relax = prm->pc_relax;
    int64_t L = o->len;
    double **vec3[] = {&o->U, &o->Uold, &o->Utavg, &o->JU, &o->f};
    for (int a = 0; a < 5; a++) *vec3[a] = calloc(3 * L, sizeof(double));
    double **vec1[] = {&o->p, &o->nut, &o->div, &o->b, &o->r, &o->r0, &o->pk, &o->pp,
                       &o->q, &o->s, &o->ss, &o->t, &o->tmp};
    for (int a = 0; a < 13; a++) *vec1[a] = calloc(L, sizeof(double));
    o->A = calloc(7 * L, sizeof(double));
    build_matrix(o);
    /* fill U, Uold with Uin, p = 0: src/solver.h:737-740 */
    for (int64_t id = 0; id < L; id++)
        for (int m = 0; m < 3; m++) o->U[id * 3 + m] = o->Uold[id * 3 + m] = o->uin[m];
    o->retracted = prm->retracted_floor;
    o->floor_start = prm->floor_start;
    if (prm->has_grid) {  /* src/solver.h:742-770 */
        build_solid(o, prm);
        solid_velocity(o);
    }
    /* turbines: build_wt_props, src/alm.h:144-206 (angle slots parsed by caller) */
    o->wt_count = prm->turbine_count;
    o->blades = prm->blades;
    o->ap_per_blade = prm->points_per_blade;
    o->projection_width = prm->projection_width;
    o->wt = calloc(o->wt_count ? o->wt_count : 1, sizeof(or_turbine));
    for (int64_t w = 0; w < o->wt_count; w++) {
        or_turbine *t = &o->wt[w];
        for (int m = 0; m < 3; m++) t->base[m] = prm->base[w * 3 + m];
        t->rot_speed = prm->rot_speed[w];
        t->rot_center[0] = -prm->overhang;
        t->rot_center[1] = 0;
        t->rot_center[2] = prm->tower;
        t->angle_type = prm->angle_type[w];
        for (int m = 0; m < 4; m++) t->formula[m] = prm->formula[w * 4 + m];
    }
    if (o->wt_count > 0) build_points(o, prm);
    return o;
}

void oracle_destroy(dalm_oracle *o) {
    if (!o) return;
    double *all[] = {o->x, o->y, o->z, o->dx, o->dy, o->dz, o->U, o->Uold, o->Utavg, o->JU,
                     o->p, o->nut, o->div, o->f, o->A, o->b, o->r, o->r0, o->pk, o->pp,
                     o->q, o->s, o->ss, o->t, o->tmp, o->profile, o->base_twist, o->cd,
                     o->cl, o->atk, o->solid};
    for (size_t a = 0; a < sizeof(all) / sizeof(all[0]); a++) free(all[a]);
    free(o->wt);
    free(o->ap);
    free(o);
}

/* ------------------------------------------------------ momentum predictor */

/* The smooth van Albada limiter (an extension: the reference has only the
 * b=4 limiter): face value f +- (s/4)[(1 - k s) a + (1 + k s) b] with the
 * switch s = (2ab + eps)/(a^2 + b^2 + eps), eps = 1e-12 (van Albada, van
 * Leer & Roberts 1982, kappa-MUSCL form); the GPU uses the same operations. */
static double va_switch(double a, double b) {
    const double eps = 1e-12;
    return (2. * a * b + eps) / (a * a + b * b + eps);
}

/* κ=1/3 MUSCL face reconstruction with the b=(3-κ)/(1-κ) limiter (or van
 * Albada, limiter 1) and upwind flux along one axis, src/cfd.h:37-60 */
static void muscl_axis(double fmm, double fm, double fc, double fp, double fpp, double Jp,
                       double Jm, double *flux_p, double *flux_m, int limiter) {
    const double kap = 1. / 3.;
    const double bb = (3. - kap) / (1. - kap);
    const double e = 1.;
    double d4 = fpp - fp, d3 = fp - fc, d2 = fc - fm, d1 = fm - fmm;
    if (limiter == 1) {
        const double sp = va_switch(d4, d3), sc = va_switch(d3, d2), sm = va_switch(d2, d1);
        const double fpr = fp - (sp / 4.) * ((1. - kap * sp) * d4 + (1. + kap * sp) * d3);
        const double fpl = fc + (sc / 4.) * ((1. - kap * sc) * d2 + (1. + kap * sc) * d3);
        const double fmr = fc - (sc / 4.) * ((1. - kap * sc) * d3 + (1. + kap * sc) * d2);
        const double fml = fm + (sm / 4.) * ((1. - kap * sm) * d1 + (1. + kap * sm) * d2);
        *flux_p = 0.5 * (Jp * (fpr + fpl) - fabs(Jp) * (fpr - fpl));
        *flux_m = 0.5 * (Jm * (fmr + fml) - fabs(Jm) * (fmr - fml));
        return;
    }
    double s4 = sgn(d4), s3 = sgn(d3), s2 = sgn(d2), s1 = sgn(d1);
    double g6 = s4 * fmax(0., fmin(fabs(d4), s4 * bb * d3));
    double g5 = s3 * fmax(0., fmin(fabs(d3), s3 * bb * d4));
    double g4 = s3 * fmax(0., fmin(fabs(d3), s3 * bb * d2));
    double g3 = s2 * fmax(0., fmin(fabs(d2), s2 * bb * d3));
    double g2 = s2 * fmax(0., fmin(fabs(d2), s2 * bb * d1));
    double g1 = s1 * fmax(0., fmin(fabs(d1), s1 * bb * d2));
    double fpr = fp - (e / 4.) * ((1. - kap) * g6 + (1. + kap) * g5);
    double fpl = fc + (e / 4.) * ((1. - kap) * g3 + (1. + kap) * g4);
    double fmr = fc - (e / 4.) * ((1. - kap) * g4 + (1. + kap) * g3);
    double fml = fm + (e / 4.) * ((1. - kap) * g1 + (1. + kap) * g2);
    *flux_p = 0.5 * (Jp * (fpr + fpl) - fabs(Jp) * (fpr - fpl));
    *flux_m = 0.5 * (Jm * (fmr + fml) - fabs(Jm) * (fmr - fml));
}

/* calc_intermediate_U_at_cell, src/cfd.h:176-242 with calc_convection_muscl
 * (src/cfd.h:9-109) and calc_diffusion (src/cfd.h:145-173) */
static void predictor_cell(dalm_oracle *o, int64_t i, int64_t j, int64_t k) {
    int64_t c = ID(o, i, j, k);
    int64_t e = ID(o, i + 1, j, k), ee = ID(o, i + 2, j, k);
    int64_t w = ID(o, i - 1, j, k), ww = ID(o, i - 2, j, k);
    int64_t n = ID(o, i, j + 1, k), nn = ID(o, i, j + 2, k);
    int64_t s = ID(o, i, j - 1, k), ss = ID(o, i, j - 2, k);
    int64_t t = ID(o, i, j, k + 1), tt = ID(o, i, j, k + 2);
    int64_t b = ID(o, i, j, k - 1), bb = ID(o, i, j, k - 2);
    double dxc = o->dx[i], dyc = o->dy[j], dzc = o->dz[k];
    double J = dxc * dyc * dzc;
    double visc = 1 / o->re + o->nut[c];
    double JUE = o->JU[c * 3 + 0], JUW = o->JU[w * 3 + 0];
    double JVN = o->JU[c * 3 + 1], JVS = o->JU[s * 3 + 1];
    double JWT = o->JU[c * 3 + 2], JWB = o->JU[b * 3 + 2];
    const double *V = o->Uold;
    for (int m = 0; m < 3; m++) {
        double fc = V[c * 3 + m];
        double fE, fW, fN, fS, fT, fB;
        muscl_axis(V[ww * 3 + m], V[w * 3 + m], fc, V[e * 3 + m], V[ee * 3 + m], JUE, JUW, &fE, &fW,
                   o->limiter);
        muscl_axis(V[ss * 3 + m], V[s * 3 + m], fc, V[n * 3 + m], V[nn * 3 + m], JVN, JVS, &fN, &fS,
                   o->limiter);
        muscl_axis(V[bb * 3 + m], V[b * 3 + m], fc, V[t * 3 + m], V[tt * 3 + m], JWT, JWB, &fT, &fB,
                   o->limiter);
        double conv = (fE - fW + fN - fS + fT - fB) / J;
        double diff = visc * (((V[e * 3 + m] - fc) / (o->x[i + 1] - o->x[i]) -
                               (fc - V[w * 3 + m]) / (o->x[i] - o->x[i - 1])) / dxc +
                              ((V[n * 3 + m] - fc) / (o->y[j + 1] - o->y[j]) -
                               (fc - V[s * 3 + m]) / (o->y[j] - o->y[j - 1])) / dyc +
                              ((V[t * 3 + m] - fc) / (o->z[k + 1] - o->z[k]) -
                               (fc - V[b * 3 + m]) / (o->z[k] - o->z[k - 1])) / dzc);
        o->U[c * 3 + m] = fc + o->dt * (-conv + diff + o->f[c * 3 + m]);
    }
}

/* cpy_array(Uold, U) + calc_intermediate_U, src/solver.h:1042-1053, src/cfd.h:244-322 */
static void stage_predict(dalm_oracle *o) {
    memcpy(o->Uold, o->U, 3 * o->len * sizeof(double));
    int64_t gc = o->gc;
    for (int64_t i = gc; i < o->nx - gc; i++)
        for (int64_t j = gc; j < o->ny - gc; j++)
            for (int64_t k = gc; k < o->nz - gc; k++) predictor_cell(o, i, j, k);
}

/* -------------------------------------------------- face flux and its BCs */

/* interpolate_JU, src/cfd.h:395-493 (faces i,j,k in [gc-1, N-gc)) */
static void interp_flux(dalm_oracle *o) {
    int64_t gc = o->gc;
    for (int64_t i = gc - 1; i < o->nx - gc; i++)
        for (int64_t j = gc - 1; j < o->ny - gc; j++)
            for (int64_t k = gc - 1; k < o->nz - gc; k++) {
                int64_t c = ID(o, i, j, k);
                int64_t e = ID(o, i + 1, j, k), n = ID(o, i, j + 1, k), t = ID(o, i, j, k + 1);
                double yz = o->dy[j] * o->dz[k];
                o->JU[c * 3 + 0] = 0.5 * (o->U[c * 3 + 0] * yz + o->U[e * 3 + 0] * yz);
                double xz = o->dx[i] * o->dz[k];
                o->JU[c * 3 + 1] = 0.5 * (o->U[c * 3 + 1] * xz + o->U[n * 3 + 1] * xz);
                double xy = o->dx[i] * o->dy[j];
                o->JU[c * 3 + 2] = 0.5 * (o->U[c * 3 + 2] * xy + o->U[t * 3 + 2] * xy);
            }
}

/* apply_JUbc, src/bc.h:235-302, plus the inflow-profile extension */
static void flux_bc(dalm_oracle *o) {
    int64_t gc = o->gc;
    for (int64_t j = gc; j < o->ny - gc; j++)
        for (int64_t k = gc; k < o->nz - gc; k++) {
            double yz = o->dy[j] * o->dz[k];
            double u = o->has_profile ? o->profile[(j * o->nz + k) * 3] : o->uin[0];
            o->JU[ID(o, gc - 1, j, k) * 3 + 0] = yz * u;
        }
    for (int64_t i = gc; i < o->nx - gc; i++)
        for (int64_t k = gc; k < o->nz - gc; k++) {
            o->JU[ID(o, i, gc - 1, k) * 3 + 1] = 0;
            o->JU[ID(o, i, o->ny - gc - 1, k) * 3 + 1] = 0;
        }
    for (int64_t i = gc; i < o->nx - gc; i++)
        for (int64_t j = gc; j < o->ny - gc; j++) {
            o->JU[ID(o, i, j, gc - 1) * 3 + 2] = 0;
            o->JU[ID(o, i, j, o->nz - gc - 1) * 3 + 2] = 0;
        }
}

static double cell_divergence(const dalm_oracle *o, int64_t i, int64_t j, int64_t k) {
    int64_t c = ID(o, i, j, k);
    double JUE = o->JU[c * 3 + 0], JUW = o->JU[ID(o, i - 1, j, k) * 3 + 0];
    double JVN = o->JU[c * 3 + 1], JVS = o->JU[ID(o, i, j - 1, k) * 3 + 1];
    double JWT = o->JU[c * 3 + 2], JWB = o->JU[ID(o, i, j, k - 1) * 3 + 2];
    double J = o->dx[i] * o->dy[j] * o->dz[k];
    return (JUE - JUW + JVN - JVS + JWT - JWB) / J;
}

/* calc_poisson_rhs, src/cfd.h:569-598 */
static void poisson_rhs(dalm_oracle *o) {
    int64_t gc = o->gc;
    for (int64_t i = gc; i < o->nx - gc; i++)
        for (int64_t j = gc; j < o->ny - gc; j++)
            for (int64_t k = gc; k < o->nz - gc; k++)
                o->b[ID(o, i, j, k)] = cell_divergence(o, i, j, k) / (o->dt * o->max_diag);
}

/* ------------------------------------------------------------ Poisson */

static inline double stencil_sum(const dalm_oracle *o, const double *v, int64_t i, int64_t j,
                                 int64_t k, const double **acoef) {
    int64_t c = ID(o, i, j, k);
    const double *a = &o->A[c * 7];
    *acoef = a;
    return a[0] * v[c] + a[1] * v[ID(o, i + 1, j, k)] + a[2] * v[ID(o, i - 1, j, k)] +
           a[3] * v[ID(o, i, j + 1, k)] + a[4] * v[ID(o, i, j - 1, k)] +
           a[5] * v[ID(o, i, j, k + 1)] + a[6] * v[ID(o, i, j, k - 1)];
}

#define FOR_INTERIOR(o)                                   \
    for (int64_t i = (o)->gc; i < (o)->nx - (o)->gc; i++) \
        for (int64_t j = (o)->gc; j < (o)->ny - (o)->gc; j++) \
            for (int64_t k = (o)->gc; k < (o)->nz - (o)->gc; k++)

/* calc_residual, src/mv.h:58-182 */
static void residual(dalm_oracle *o, const double *x, const double *b, double *r) {
    const double *a;
    FOR_INTERIOR(o) { r[ID(o, i, j, k)] = b[ID(o, i, j, k)] - stencil_sum(o, x, i, j, k, &a); }
}
/* calc_Ax, src/mv.h:185-309 */
static void matvec(dalm_oracle *o, const double *x, double *y) {
    const double *a;
    FOR_INTERIOR(o) { y[ID(o, i, j, k)] = stencil_sum(o, x, i, j, k, &a); }
}
/* Pairwise (recursive halving) sum, used only by the summation-order
 * sensitivity mode below. */
static double pairwise_sum(const double *v, int64_t n) {
    if (n <= 8) {
        double s = 0;
        for (int64_t i = 0; i < n; i++) s += v[i];
        return s;
    }
    int64_t h = n / 2;
    return pairwise_sum(v, h) + pairwise_sum(v + h, n - h);
}

/* calc_inner_product, src/mv.h:8-31.  With sum_order == 1 (a test-only
 * perturbation, never the default) the same products are summed pairwise
 * instead of serially, to measure how sensitive the solver is to the
 * summation order alone. */
static double dot(const dalm_oracle *o, const double *a, const double *b) {
    if (o->sum_order != 0) {
        double *v = malloc(sizeof(double) * (size_t)o->len);
        int64_t n = 0;
        FOR_INTERIOR(o) { v[n++] = a[ID(o, i, j, k)] * b[ID(o, i, j, k)]; }
        double s = 0;
        if (o->sum_order == 1) {
            s = pairwise_sum(v, n);
        } else if (o->sum_order == 2) { /* reversed serial */
            for (int64_t m = n - 1; m >= 0; m--) s += v[m];
        } else { /* 3: 1184 strided partial sums, then serial (a GPU-like order) */
            for (int64_t p = 0; p < 1184; p++) {
                double part = 0;
                for (int64_t m = p; m < n; m += 1184) part += v[m];
                s += part;
            }
        }
        free(v);
        return s;
    }
    double tot = 0;
    FOR_INTERIOR(o) { tot += a[ID(o, i, j, k)] * b[ID(o, i, j, k)]; }
    return tot;
}
/* calc_l2_norm, src/mv.h:33-55 */
static double l2norm(const dalm_oracle *o, const double *v) {
    if (o->sum_order == 1) return sqrt(dot(o, v, v));
    double tot = 0;
    FOR_INTERIOR(o) { tot += sq(v[ID(o, i, j, k)]); }
    return sqrt(tot);
}
static double interior_count(const dalm_oracle *o) {
    return (double)((o->nx - 2 * o->gc) * (o->ny - 2 * o->gc) * (o->nz - 2 * o->gc));
}

/* sweep_sor, src/eq.h:145-289: cells with (i+j+k)%2 == color (offsets 0) */
static void sor_sweep(dalm_oracle *o, double *x, const double *b, double w, int color) {
    const double *a;
    FOR_INTERIOR(o) {
        if ((i + j + k) % 2 != color) continue;
        int64_t c = ID(o, i, j, k);
        double xc = x[c];
        double sum = stencil_sum(o, x, i, j, k, &a);
        double rel = (b[c] - sum) / a[0];
        x[c] = xc + w * rel;
    }
}

/* sweep_jacobi, src/eq.h:6-143 */
static void jacobi_sweep(dalm_oracle *o, double *x, const double *xold, const double *b) {
    const double *a;
    FOR_INTERIOR(o) {
        int64_t c = ID(o, i, j, k);
        double sum = stencil_sum(o, xold, i, j, k, &a);
        x[c] = xold[c] + (b[c] - sum) / a[0];
    }
}

/* run_jacobi_pc, src/eq.h:320-331 (x is zero on entry) */
static void jacobi_pc(dalm_oracle *o, double *x, const double *b) {
    for (int64_t it = 0; it < o->pc_max_it; it++) {
        memcpy(o->tmp, x, o->len * sizeof(double));
        jacobi_sweep(o, x, o->tmp, b);
    }
}

/* run_sor_pc, src/eq.h:308-318 */
static void sor_pc(dalm_oracle *o, double *x, const double *b) {
    for (int64_t it = 0; it < o->pc_max_it; it++) {
        sor_sweep(o, x, b, o->pc_relax, 0);
        sor_sweep(o, x, b, o->pc_relax, 1);
    }
}

/* run_sor, src/eq.h:291-306 */
static void run_sor(dalm_oracle *o) {
    double *x = o->p;
    o->it = 0;
    do {
        sor_sweep(o, x, o->b, o->relax, 0);
        sor_sweep(o, x, o->b, o->relax, 1);
        residual(o, x, o->b, o->r);
        o->err = l2norm(o, o->r) / sqrt(interior_count(o));
        o->it++;
    } while (o->it < o->max_it && o->err > o->tol);
}

/* Standalone Jacobi (extension): the reference's own sweep_jacobi
 * (src/eq.h:41-143) iterated with run_sor's stop rule (src/eq.h:297-305). */
static void run_jacobi(dalm_oracle *o) {
    double *x = o->p;
    o->it = 0;
    do {
        memcpy(o->tmp, x, o->len * sizeof(double));
        jacobi_sweep(o, x, o->tmp, o->b);
        residual(o, x, o->b, o->r);
        o->err = l2norm(o, o->r) / sqrt(interior_count(o));
        o->it++;
    } while (o->it < o->max_it && o->err > o->tol);
}

/* run_pbicgstab (Jacobi-PC src/eq.h:333-402, SOR-PC src/eq.h:404-473) */
static void run_bicgstab(dalm_oracle *o) {
    int64_t L = o->len;
    double *x = o->p, *b = o->b, *r = o->r, *r0 = o->r0, *p = o->pk, *pp = o->pp, *q = o->q,
           *s = o->s, *ss = o->ss, *t = o->t;
    residual(o, x, b, r);
    memcpy(r0, r, L * sizeof(double));
    double alpha = 1, beta, omega = 1, rho, rhoold = 1;
    memset(q, 0, L * sizeof(double));
    o->it = 0;
    do {
        rho = dot(o, r0, r);
        if (fabs(rho) < FLT_MIN) {
            o->err = rho;
            break;
        }
        if (o->it == 0) {
            memcpy(p, r, L * sizeof(double));
        } else {
            beta = (rho / rhoold) * (alpha / omega);
            for (int64_t n = 0; n < L; n++) p[n] = r[n] + beta * (p[n] - omega * q[n]);
        }
        memset(pp, 0, L * sizeof(double));
        if (o->pc == OR_PC_SOR) sor_pc(o, pp, p); else jacobi_pc(o, pp, p);
        matvec(o, pp, q);
        alpha = rho / dot(o, r0, q);
        for (int64_t n = 0; n < L; n++) s[n] = r[n] - alpha * q[n];
        memset(ss, 0, L * sizeof(double));
        if (o->pc == OR_PC_SOR) sor_pc(o, ss, s); else jacobi_pc(o, ss, s);
        matvec(o, ss, t);
        omega = dot(o, t, s) / dot(o, t, t);
        for (int64_t n = 0; n < L; n++) x[n] = x[n] + alpha * pp[n] + omega * ss[n];
        for (int64_t n = 0; n < L; n++) r[n] = s[n] - omega * t[n];
        rhoold = rho;
        o->err = l2norm(o, r) / sqrt(interior_count(o));
        o->it++;
    } while (o->it < o->max_it && o->err > o->tol);
}

/* ----------------------------------------------------- projection + BCs */

/* apply_pbc, src/bc.h:304-411 */
static void pressure_bc(dalm_oracle *o) {
    int64_t gc = o->gc, NX = o->nx, NY = o->ny, NZ = o->nz;
    for (int64_t j = gc; j < NY - gc; j++)
        for (int64_t k = gc; k < NZ - gc; k++) o->p[ID(o, gc - 1, j, k)] = o->p[ID(o, gc, j, k)];
    for (int64_t j = gc; j < NY - gc; j++)
        for (int64_t k = gc; k < NZ - gc; k++) {
            int64_t ii = NX - gc - 1, io = NX - gc;
            double hi = 0.5 * o->dx[ii], ho = 0.5 * o->dx[io], pbc = 0;
            o->p[ID(o, io, j, k)] = pbc - (o->p[ID(o, ii, j, k)] - pbc) * (ho / hi);
        }
    for (int64_t i = gc; i < NX - gc; i++)
        for (int64_t k = gc; k < NZ - gc; k++) {
            o->p[ID(o, i, gc - 1, k)] = o->p[ID(o, i, gc, k)];
            o->p[ID(o, i, NY - gc, k)] = o->p[ID(o, i, NY - gc - 1, k)];
        }
    for (int64_t i = gc; i < NX - gc; i++)
        for (int64_t j = gc; j < NY - gc; j++) {
            o->p[ID(o, i, j, gc - 1)] = o->p[ID(o, i, j, gc)];
            o->p[ID(o, i, j, NZ - gc)] = o->p[ID(o, i, j, NZ - gc - 1)];
        }
}

/* project_p, src/cfd.h:601-783 */
static void project(dalm_oracle *o) {
    int64_t gc = o->gc;
    const double *p = o->p;
    FOR_INTERIOR(o) {
        int64_t c = ID(o, i, j, k);
        o->U[c * 3 + 0] -= o->dt * (p[ID(o, i + 1, j, k)] - p[ID(o, i - 1, j, k)]) / (o->x[i + 1] - o->x[i - 1]);
        o->U[c * 3 + 1] -= o->dt * (p[ID(o, i, j + 1, k)] - p[ID(o, i, j - 1, k)]) / (o->y[j + 1] - o->y[j - 1]);
        o->U[c * 3 + 2] -= o->dt * (p[ID(o, i, j, k + 1)] - p[ID(o, i, j, k - 1)]) / (o->z[k + 1] - o->z[k - 1]);
    }
    for (int64_t i = gc - 1; i < o->nx - gc; i++)
        for (int64_t j = gc - 1; j < o->ny - gc; j++)
            for (int64_t k = gc - 1; k < o->nz - gc; k++) {
                int64_t c = ID(o, i, j, k);
                double yz = o->dy[j] * o->dz[k];
                double dpdx = (p[ID(o, i + 1, j, k)] - p[c]) / (o->x[i + 1] - o->x[i]);
                o->JU[c * 3 + 0] -= o->dt * yz * dpdx;
                double xz = o->dx[i] * o->dz[k];
                double dpdy = (p[ID(o, i, j + 1, k)] - p[c]) / (o->y[j + 1] - o->y[j]);
                o->JU[c * 3 + 1] -= o->dt * xz * dpdy;
                double xy = o->dx[i] * o->dy[j];
                double dpdz = (p[ID(o, i, j, k + 1)] - p[c]) / (o->z[k + 1] - o->z[k]);
                o->JU[c * 3 + 2] -= o->dt * xy * dpdz;
            }
}

/* apply_Ubc, src/bc.h:5-233 (no retracted floor), plus the inflow profile */
static void velocity_bc(dalm_oracle *o) {
    int64_t gc = o->gc, NX = o->nx, NY = o->ny, NZ = o->nz;
    double *U = o->U;
    const double *V = o->Uold;
    for (int64_t i = 0; i < gc; i++)
        for (int64_t j = gc; j < NY - gc; j++)
            for (int64_t k = gc; k < NZ - gc; k++)
                for (int m = 0; m < 3; m++)
                    U[ID(o, i, j, k) * 3 + m] =
                        o->has_profile ? o->profile[(j * NZ + k) * 3 + m] : o->uin[m];
    for (int64_t i = NX - gc; i < NX; i++)
        for (int64_t j = gc; j < NY - gc; j++)
            for (int64_t k = gc; k < NZ - gc; k++) {
                int64_t i0 = ID(o, i, j, k), i1 = ID(o, i - 1, j, k), i2 = ID(o, i - 2, j, k);
                double uout = U[i0 * 3 + 0];
                for (int m = 0; m < 3; m++) {
                    double f0 = V[i0 * 3 + m], f1 = V[i1 * 3 + m], f2 = V[i2 * 3 + m];
                    double grad = (3 * f0 - 4 * f1 + f2) / 2;
                    U[i0 * 3 + m] = f0 - uout * o->dt * grad / o->dx[i];
                }
            }
    /* y- and y+ slip: quadratic through (j0, j1, wall) */
    for (int side = 0; side < 2; side++)
        for (int64_t i = gc; i < NX - gc; i++)
            for (int64_t k = gc; k < NZ - gc; k++) {
                int64_t j0 = side ? NY - gc - 2 : gc + 1, j1 = side ? NY - gc - 1 : gc;
                int64_t j3 = side ? NY - gc : gc - 1, j4 = side ? NY - gc + 1 : gc - 2;
                int64_t a0 = ID(o, i, j0, k), a1 = ID(o, i, j1, k);
                int64_t a3 = ID(o, i, j3, k), a4 = ID(o, i, j4, k);
                double y0 = o->y[j0], y1 = o->y[j1];
                double y2 = side ? o->y[j1] + 0.5 * o->dy[j1] : o->y[j1] - 0.5 * o->dy[j1];
                double y3 = o->y[j3], y4 = o->y[j4];
                double ubc[3] = {U[a1 * 3 + 0], 0, U[a1 * 3 + 2]};
                for (int m = 0; m < 3; m++) {
                    double f0 = U[a0 * 3 + m], f1 = U[a1 * 3 + m], f2 = ubc[m];
                    U[a3 * 3 + m] = quad_poly(y0, y1, y2, f0, f1, f2, y3);
                    U[a4 * 3 + m] = quad_poly(y0, y1, y2, f0, f1, f2, y4);
                }
            }
    /* z- no-slip and z+ slip */
    for (int side = 0; side < 2; side++)
        for (int64_t i = gc; i < NX - gc; i++)
            for (int64_t j = gc; j < NY - gc; j++) {
                int64_t k0 = side ? NZ - gc - 2 : gc + 1, k1 = side ? NZ - gc - 1 : gc;
                int64_t k3 = side ? NZ - gc : gc - 1, k4 = side ? NZ - gc + 1 : gc - 2;
                int64_t a0 = ID(o, i, j, k0), a1 = ID(o, i, j, k1);
                int64_t a3 = ID(o, i, j, k3), a4 = ID(o, i, j, k4);
                double z0 = o->z[k0], z1 = o->z[k1];
                double z2 = side ? o->z[k1] + 0.5 * o->dz[k1] : o->z[k1] - 0.5 * o->dz[k1];
                double z3 = o->z[k3], z4 = o->z[k4];
                double ubc[3] = {0, 0, 0};
                /* z+ slip; z- no slip, or slip upstream of a retracted floor (src/bc.h:140-160) */
                if (side || (o->retracted && o->x[i] < o->floor_start)) {
                    ubc[0] = U[a1 * 3 + 0];
                    ubc[1] = U[a1 * 3 + 1];
                }
                for (int m = 0; m < 3; m++) {
                    double f0 = U[a0 * 3 + m], f1 = U[a1 * 3 + m], f2 = ubc[m];
                    U[a3 * 3 + m] = quad_poly(z0, z1, z2, f0, f1, f2, z3);
                    U[a4 * 3 + m] = quad_poly(z0, z1, z2, f0, f1, f2, z4);
                }
            }
}

/* calc_nut_at_cell, src/cfd.h:786-825 */
static void eddy_viscosity(dalm_oracle *o) {
    const double *U = o->U;
    FOR_INTERIOR(o) {
        int64_t e = ID(o, i + 1, j, k), w = ID(o, i - 1, j, k), n = ID(o, i, j + 1, k),
                s = ID(o, i, j - 1, k), t = ID(o, i, j, k + 1), b = ID(o, i, j, k - 1);
        double dxew = o->x[i + 1] - o->x[i - 1];
        double dyns = o->y[j + 1] - o->y[j - 1];
        double dztb = o->z[k + 1] - o->z[k - 1];
        double volume = o->dx[i] * o->dy[j] * o->dz[k];
        double dudx = (U[e * 3 + 0] - U[w * 3 + 0]) / dxew;
        double dudy = (U[n * 3 + 0] - U[s * 3 + 0]) / dyns;
        double dudz = (U[t * 3 + 0] - U[b * 3 + 0]) / dztb;
        double dvdx = (U[e * 3 + 1] - U[w * 3 + 1]) / dxew;
        double dvdy = (U[n * 3 + 1] - U[s * 3 + 1]) / dyns;
        double dvdz = (U[t * 3 + 1] - U[b * 3 + 1]) / dztb;
        double dwdx = (U[e * 3 + 2] - U[w * 3 + 2]) / dxew;
        double dwdy = (U[n * 3 + 2] - U[s * 3 + 2]) / dyns;
        double dwdz = (U[t * 3 + 2] - U[b * 3 + 2]) / dztb;
        double s1 = 2 * sq(dudx), s2 = 2 * sq(dvdy), s3 = 2 * sq(dwdz);
        double s4 = sq(dudy + dvdx), s5 = sq(dudz + dwdx), s6 = sq(dvdz + dwdy);
        double shear = sqrt(s1 + s2 + s3 + s4 + s5 + s6);
        double filter = cbrt(volume);
        o->nut[ID(o, i, j, k)] = sq(o->cs * filter) * shear;
    }
}

/* calc_divergence, src/cfd.h:1079-1107 */
static void divergence(dalm_oracle *o) {
    FOR_INTERIOR(o) { o->div[ID(o, i, j, k)] = cell_divergence(o, i, j, k); }
}

/* calc_max_cfl, src/cfd.h:1109-1141 */
static double max_cfl(const dalm_oracle *o) {
    double m = 0;
    FOR_INTERIOR(o) {
        int64_t c = ID(o, i, j, k);
        double local = fabs(o->U[c * 3 + 0]) * o->dt / o->dx[i] +
                       fabs(o->U[c * 3 + 1]) * o->dt / o->dy[j] +
                       fabs(o->U[c * 3 + 2]) * o->dt / o->dz[k];
        if (local > m) m = local;
    }
    return m;
}

/* ------------------------------------------------------------- actuator line */

/* frame_transform, src/euler_angle.h:34-62 */
static void frame_transform(const double in[3], double out[3], double angle, int type) {
    double c = cos(angle), s = sin(angle);
    double x = in[0], y = in[1], z = in[2];
    switch (type) {
    case OR_EULER_ROLL: out[0] = x; out[1] = c * y + s * z; out[2] = -s * y + c * z; break;
    case OR_EULER_PITCH: out[0] = c * x - s * z; out[1] = y; out[2] = -s * x + c * z; break;
    case OR_EULER_YAW: out[0] = c * x + s * y; out[1] = -s * x + c * y; out[2] = z; break;
    default: out[0] = x; out[1] = y; out[2] = z; break;
    }
}

/* frame_transform_U, src/euler_angle.h:64-127, including its two typos
 * (roll Rdtdx[2] = -s*v + v*w; yaw dRdtx[1] = ow*(-c*s - s*y)) */
static void frame_transform_U(const double p[3], const double U[3], double out[3],
                              double angle, double ow, int type) {
    double c = cos(angle), s = sin(angle);
    double x = p[0], y = p[1], z = p[2], u = U[0], v = U[1], w = U[2];
    switch (type) {
    case OR_EULER_ROLL:
        out[0] = 0. + u;
        out[1] = ow * (-s * y + c * z) + (c * v + s * w);
        out[2] = ow * (-c * y - s * z) + (-s * v + v * w);
        break;
    case OR_EULER_PITCH:
        out[0] = ow * (-s * x - c * z) + (c * u - s * w);
        out[1] = 0. + v;
        out[2] = ow * (c * x - s * z) + (s * u + c * w);
        break;
    case OR_EULER_YAW:
        out[0] = ow * (-s * x + c * y) + (c * u + s * v);
        out[1] = ow * (-c * s - s * y) + (-s * u + c * v);
        out[2] = 0. + w;
        break;
    default: out[0] = u; out[1] = v; out[2] = w; break;
    }
}

/* trilinear_interpolate, src/util.h:176-199 */
static double trilinear(const double v[8], double x0, double x1, double y0, double y1,
                        double z0, double z1, double xp, double yp, double zp) {
    double fx = (xp - x0) / (x1 - x0), fy = (yp - y0) / (y1 - y0), fz = (zp - z0) / (z1 - z0);
    double v01 = v[0] * (1 - fx) + v[1] * fx;
    double v23 = v[2] * (1 - fx) + v[3] * fx;
    double v45 = v[4] * (1 - fx) + v[5] * fx;
    double v67 = v[6] * (1 - fx) + v[7] * fx;
    double v0123 = v01 * (1 - fy) + v23 * fy;
    double v4567 = v45 * (1 - fy) + v67 * fy;
    return v0123 * (1 - fz) + v4567 * fz;
}

static double lin_interp(double v0, double v1, double x0, double x1, double xp) {
    double fx = (xp - x0) / (x1 - x0); /* src/util.h:166-174 */
    return v0 * (1 - fx) + v1 * fx;
}

/* run_alm, src/alm.h:450-479: update_ap_position (src/alm.h:233-267),
 * calc_ap_force (src/alm.h:269-414), distribute_ap_force (src/alm.h:416-448) */
static void actuator_line(dalm_oracle *o) {
    if (o->ap_count <= 0) return;
    double tm = o->dt * (double)o->step;
    int64_t ap_per_wt = o->ap_per_blade * o->blades;
    for (int64_t w = 0; w < o->wt_count; w++) {
        or_turbine *wt = &o->wt[w];
        double A = wt->formula[0], B = wt->formula[1], C = wt->formula[2], D = wt->formula[3];
        wt->angle = A * sin(B * tm + C) + D;
        wt->ow = A * B * cos(B * tm + C);
    }
    for (int64_t a = 0; a < o->ap_count; a++) {
        or_point *ap = &o->ap[a];
        or_turbine *wt = &o->wt[a / ap_per_wt];
        int64_t bid = (a % ap_per_wt) / o->ap_per_blade;
        double start_theta = bid * (2 * ORACLE_PI / o->blades);
        ap->theta = start_theta + tm * wt->rot_speed;
        double xyz[3] = {wt->rot_center[0], wt->rot_center[1] + ap->r * cos(ap->theta),
                         wt->rot_center[2] + ap->r * sin(ap->theta)};
        frame_transform(xyz, ap->xyz, -wt->angle, wt->angle_type);
        for (int m = 0; m < 3; m++) ap->xyz[m] += wt->base[m];
    }
    int64_t gc = o->gc;
    for (int64_t a = 0; a < o->ap_count; a++) {
        or_point *ap = &o->ap[a];
        or_turbine *wt = &o->wt[a / ap_per_wt];
        int64_t i = floor_index(o->x, ap->xyz[0], o->nx);
        int64_t j = floor_index(o->y, ap->xyz[1], o->ny);
        int64_t k = floor_index(o->z, ap->xyz[2], o->nz);
        if (i >= gc && i < o->nx - gc && j >= gc && j < o->ny - gc && k >= gc && k < o->nz - gc) {
            int64_t id[8] = {ID(o, i, j, k),         ID(o, i + 1, j, k),
                             ID(o, i, j + 1, k),     ID(o, i + 1, j + 1, k),
                             ID(o, i, j, k + 1),     ID(o, i + 1, j, k + 1),
                             ID(o, i, j + 1, k + 1), ID(o, i + 1, j + 1, k + 1)};
            double Uap[3];
            for (int m = 0; m < 3; m++) {
                double v[8];
                for (int q = 0; q < 8; q++) v[q] = o->U[id[q] * 3 + m];
                Uap[m] = trilinear(v, o->x[i], o->x[i + 1], o->y[j], o->y[j + 1], o->z[k],
                                   o->z[k + 1], ap->xyz[0], ap->xyz[1], ap->xyz[2]);
            }
            double rel[3] = {ap->xyz[0] - wt->base[0], ap->xyz[1] - wt->base[1],
                             ap->xyz[2] - wt->base[2]};
            double Ur[3];
            frame_transform_U(rel, Uap, Ur, wt->angle, wt->ow, wt->angle_type);
            double ux_ = Ur[0];
            double ut_ = ap->r * wt->rot_speed + Ur[1] * sin(ap->theta) - Ur[2] * cos(ap->theta);
            double urel2 = ux_ * ux_ + ut_ * ut_;
            double phi = atan(ux_ / ut_);
            double atk = phi * 180 / ORACLE_PI - ap->twist;
            double cd, cl;
            int64_t ti = floor_index(o->atk, atk, o->atk_count);
            const double *cdt = &o->cd[a * o->atk_count], *clt = &o->cl[a * o->atk_count];
            if (ti < 0) {
                cd = cdt[0]; cl = clt[0];
            } else if (ti >= o->atk_count - 1) {
                cd = cdt[o->atk_count - 1]; cl = clt[o->atk_count - 1];
            } else {
                cd = lin_interp(cdt[ti], cdt[ti + 1], o->atk[ti], o->atk[ti + 1], atk);
                cl = lin_interp(clt[ti], clt[ti + 1], o->atk[ti], o->atk[ti + 1], atk);
            }
            double fd = 0.5 * cd * urel2 * ap->chord * ap->dr;
            double fl = 0.5 * cl * urel2 * ap->chord * ap->dr;
            double fx_ = fl * cos(phi) + fd * sin(phi);
            double ft_ = fl * sin(phi) - fd * cos(phi);
            ft_ *= sgn(wt->rot_speed);
            double f_[3] = {-fx_, ft_ * sin(ap->theta), -ft_ * cos(ap->theta)};
            frame_transform(f_, ap->f, -wt->angle, wt->angle_type);
            ap->torque = fabs(ft_) * ap->r;
            ap->thrust = fx_;
        } else {
            ap->f[0] = ap->f[1] = ap->f[2] = 0;
            ap->torque = ap->thrust = 0;
        }
    }
    for (int64_t w = 0; w < o->wt_count; w++) {
        double torque = 0, thrust = 0;
        for (int64_t a = w * ap_per_wt; a < (w + 1) * ap_per_wt; a++) {
            torque += o->ap[a].torque;
            thrust += o->ap[a].thrust;
        }
        o->wt[w].torque = torque;
        o->wt[w].thrust = thrust;
    }
    double pw = o->projection_width;
    FOR_INTERIOR(o) {
        double fx = 0, fy = 0, fz = 0;
        double xc = o->x[i], yc = o->y[j], zc = o->z[k];
        double e = 1 / cube(pw * sqrt(ORACLE_PI));
        for (int64_t a = 0; a < o->ap_count; a++) {
            const or_point *ap = &o->ap[a];
            double r2 = sq(xc - ap->xyz[0]) + sq(yc - ap->xyz[1]) + sq(zc - ap->xyz[2]);
            double wght = e * exp(-r2 / sq(pw));
            fx += wght * ap->f[0];
            fy += wght * ap->f[1];
            fz += wght * ap->f[2];
        }
        int64_t c = ID(o, i, j, k);
        o->f[c * 3 + 0] = fx;
        o->f[c * 3 + 1] = fy;
        o->f[c * 3 + 2] = fz;
    }
}

static void diagnostics(dalm_oracle *o) {
    o->avg_div = l2norm(o, o->div) / sqrt(interior_count(o)); /* src/solver.h:1184 */
    o->max_cfl = max_cfl(o);                                   /* src/solver.h:1186 */
}

/* ---------------------------------------------------------------- driver */

void oracle_stage(dalm_oracle *o, int stage) {
    switch (stage) {
    case 0: stage_predict(o); break;
    case 1: interp_flux(o); flux_bc(o); poisson_rhs(o); break;
    case 2:
        if (o->solver == OR_SOLVER_BICG) run_bicgstab(o);
        else if (o->solver == OR_SOLVER_SOR) run_sor(o);
        else run_jacobi(o);
        break;
    case 3:
        pressure_bc(o);
        project(o);
        solid_velocity(o);
        velocity_bc(o);
        flux_bc(o);
        eddy_viscosity(o);
        divergence(o);
        break;
    case 4: actuator_line(o); break;
    case 5: diagnostics(o); break;
    case 6: {
        /* time average, src/solver.h:1194-1204 with calc_ax_plus_by (src/mv.h:322-335) */
        double tm = o->dt * (double)o->step;
        if (tm >= o->tavg_start_time) {
            o->tavg_count++;
            double wgt = 1. / o->tavg_count;
            for (int64_t n = 0; n < 3 * o->len; n++)
                o->Utavg[n] = (1. - wgt) * o->Utavg[n] + wgt * o->U[n];
        }
        break;
    }
    default: break;
    }
}

/* main_loop_once without output and probes, src/solver.h:1034-1306 */
void oracle_step(dalm_oracle *o, int n) {
    for (int s = 0; s < n; s++) {
        if (o->step != 0)
            for (int st = 0; st <= 5; st++) oracle_stage(o, st);
        oracle_stage(o, 6);
        o->step++;
    }
}

void oracle_advance_clock(dalm_oracle *o) { o->step++; }

void oracle_set_state(dalm_oracle *o, const double *U, const double *JU, const double *p,
                      int flags) {
    int64_t L = o->len;
    memcpy(o->U, U, 3 * L * sizeof(double));
    if (p) memcpy(o->p, p, L * sizeof(double));
    if (flags & 1) {
        memcpy(o->Uold, o->U, 3 * L * sizeof(double));
        velocity_bc(o);
    }
    if ((flags & 2) || !JU) {
        interp_flux(o);
        flux_bc(o);
    } else {
        memcpy(o->JU, JU, 3 * L * sizeof(double));
    }
    eddy_viscosity(o);
    divergence(o);
    actuator_line(o);
    diagnostics(o);
}

void oracle_set_inflow_profile(dalm_oracle *o, const double *prof) {
    free(o->profile);
    o->profile = NULL;
    o->has_profile = 0;
    if (!prof) return;
    size_t n = (size_t)(o->ny * o->nz * 3);
    o->profile = malloc(n * sizeof(double));
    memcpy(o->profile, prof, n * sizeof(double));
    o->has_profile = 1;
}

void oracle_set_turbine_params(dalm_oracle *o, const double *yaw_deg, const double *pitch_deg,
                               const double *omega) {
    int64_t ap_per_wt = o->ap_per_blade * o->blades;
    for (int64_t w = 0; w < o->wt_count; w++) {
        or_turbine *wt = &o->wt[w];
        if (yaw_deg) {
            wt->angle_type = OR_EULER_YAW;
            wt->formula[0] = wt->formula[1] = wt->formula[2] = 0;
            wt->formula[3] = yaw_deg[w] * ORACLE_PI / 180; /* deg_to_rad, src/util.h:214-216 */
        }
        if (omega) wt->rot_speed = omega[w];
        if (pitch_deg)
            for (int64_t a = w * ap_per_wt; a < (w + 1) * ap_per_wt; a++)
                o->ap[a].twist = o->base_twist[a] + pitch_deg[w];
    }
}

static double *field(const dalm_oracle *o, int which, int *nc) {
    *nc = 1;
    switch (which) {
    case 0: *nc = 3; return o->U;
    case 1: *nc = 3; return o->Uold;
    case 2: *nc = 3; return o->JU;
    case 3: return o->p;
    case 4: return o->nut;
    case 5: return o->div;
    case 6: *nc = 3; return o->f;
    case 7: return o->b;
    case 8: *nc = 3; return o->Utavg;
    default: return NULL;
    }
}

void oracle_get_field(const dalm_oracle *o, int which, double *out) {
    int nc;
    double *p = field(o, which, &nc);
    if (p) memcpy(out, p, o->len * nc * sizeof(double));
}

void oracle_set_field(dalm_oracle *o, int which, const double *in) {
    int nc;
    double *p = field(o, which, &nc);
    if (p) memcpy(p, in, o->len * nc * sizeof(double));
}

void oracle_size(const dalm_oracle *o, int64_t out[4]) {
    out[0] = o->nx; out[1] = o->ny; out[2] = o->nz; out[3] = o->gc;
}

void oracle_mesh(const dalm_oracle *o, double *x, double *y, double *z, double *dx,
                 double *dy, double *dz) {
    memcpy(x, o->x, o->nx * sizeof(double));
    memcpy(y, o->y, o->ny * sizeof(double));
    memcpy(z, o->z, o->nz * sizeof(double));
    memcpy(dx, o->dx, o->nx * sizeof(double));
    memcpy(dy, o->dy, o->ny * sizeof(double));
    memcpy(dz, o->dz, o->nz * sizeof(double));
}

double oracle_max_diag(const dalm_oracle *o) { return o->max_diag; }

void oracle_matrix(const dalm_oracle *o, double *A) {
    memcpy(A, o->A, 7 * o->len * sizeof(double));
}

void oracle_stats(const dalm_oracle *o, int64_t *ints, double *reals) {
    ints[0] = o->step;
    ints[1] = o->it;
    ints[2] = o->max_step;
    ints[3] = o->tavg_count;
    reals[0] = o->err;
    reals[1] = o->avg_div;
    reals[2] = o->max_cfl;
    reals[3] = o->dt;
}

void oracle_set_poisson(dalm_oracle *o, int64_t max_it, double tol) {
    o->max_it = max_it;
    o->tol = tol;
}

void oracle_set_sum_order(dalm_oracle *o, int mode) { o->sum_order = mode; }
void oracle_set_limiter(dalm_oracle *o, int limiter) { o->limiter = limiter; }

void oracle_turbines(const dalm_oracle *o, double *torque, double *thrust) {
    for (int64_t w = 0; w < o->wt_count; w++) {
        torque[w] = o->wt[w].torque;
        thrust[w] = o->wt[w].thrust;
    }
}

void oracle_points(const dalm_oracle *o, double *xyz, double *f, double *torque,
                   double *thrust) {
    for (int64_t a = 0; a < o->ap_count; a++) {
        for (int m = 0; m < 3; m++) {
            xyz[a * 3 + m] = o->ap[a].xyz[m];
            f[a * 3 + m] = o->ap[a].f[m];
        }
        torque[a] = o->ap[a].torque;
        thrust[a] = o->ap[a].thrust;
    }
}

void oracle_point_tables(const dalm_oracle *o, double *r, double *dr, double *chord,
                         double *twist, double *cd, double *cl, double *atk) {
    for (int64_t a = 0; a < o->ap_count; a++) {
        r[a] = o->ap[a].r;
        dr[a] = o->ap[a].dr;
        chord[a] = o->ap[a].chord;
        twist[a] = o->ap[a].twist;
    }
    memcpy(cd, o->cd, o->ap_count * o->atk_count * sizeof(double));
    memcpy(cl, o->cl, o->ap_count * o->atk_count * sizeof(double));
    memcpy(atk, o->atk, o->atk_count * sizeof(double));
}
