// Host-side driver of the multigrid preconditioner (test infrastructure).
//
// Compiled by tests/test_multigrid_math.py with nvcc as host code only: it
// builds the levels with the product's set-up code (multigrid_setup.hpp)
// and runs the V-cycle's schedule (mg_vcycle) with the product's per-cell
// functions (multigrid.cuh) in plain loops, so the CPU test suite can check
// the operator against the oracle's matrix and the V-cycle's symmetry and
// convergence.  Level 0 uses the solver's padded layout (2 guide cells).
#include <algorithm>
#include <vector>

#include "../3dalm_b200/csrc/multigrid.cuh"
#include "../3dalm_b200/csrc/multigrid_setup.hpp"

using namespace dalm;

namespace {

struct HostMg {
    std::vector<MgGeometry> geo;
    std::vector<std::vector<float>> cf[3], w[3];
    std::vector<std::vector<float>> x, f;
    std::vector<float> kinv;
    MgLevel L[MG_MAX_LEVELS];
    int levels = 0, ncoarse = 0;

    std::vector<std::vector<float>> cp;
    void smooth(int l, int color, bool zero) {
        const MgLevel &v = L[l];
        const long long half = (long long)v.n[0] * ((v.n[1] + 1) / 2);
        for (long long n = 0; n < half; n++) {
            int i, j;
            if (mg_color_column(v, n, color, i, j))
                mg_zline_column(v, x[l].data(), f[l].data(), cp[l].data(), i, j, zero);
        }
    }
    void restrict(int l) {
        const MgLevel &c = L[l + 1];
        for (int I = 0; I < c.n[0]; I++)
            for (int J = 0; J < c.n[1]; J++)
                for (int K = 0; K < c.n[2]; K++)
                    mg_restrict_cell(L[l], c, x[l].data(), f[l].data(), f[l + 1].data(), I, J, K);
    }
    void coarse() {
        const int l = levels - 1;
        for (int r = 0; r < ncoarse; r++) {
            float s = 0;
            for (int c = 0; c < ncoarse; c++)
                s += kinv[(size_t)r * ncoarse + c] * f[l][mg_cell_index(L[l], c)];
            x[l][mg_cell_index(L[l], r)] = s;
        }
    }
    void prolong(int l) {
        const MgLevel &v = L[l];
        for (int i = 0; i < v.n[0]; i++)
            for (int j = 0; j < v.n[1]; j++)
                for (int k = 0; k < v.n[2]; k++)
                    mg_prolong_cell(v, L[l + 1], x[l].data(), x[l + 1].data(), i, j, k);
    }
};

// The V-cycle as the CUDA executor (DeviceCycle in multigrid.cu) runs it:
// the restriction leaves out the children of the colour smoothed last, and
// each prolongation is not applied as a pass but by the next half-sweep,
// which reads its interior x/y neighbours as x + the parent's correction.
struct HostMgFolded {
    HostMg &m;
    int last_color[MG_MAX_LEVELS] = {};
    bool pending[MG_MAX_LEVELS] = {};
    void smooth(int l, int color, bool zero) {
        const MgLevel &v = m.L[l];
        std::vector<float> &x = m.x[l];
        const long long half = (long long)v.n[0] * ((v.n[1] + 1) / 2);
        for (long long n = 0; n < half; n++) {
            int i, j;
            if (!mg_color_column(v, n, color, i, j)) continue;
            const long long c0 = v.at(i, j, 0);
            for (int k = 0; k < v.n[2]; k++) {
                const long long c = c0 + k;
                float r = m.f[l][c];
                if (!zero) {
                    auto nb = [&](int ii, int jj, long long q) {
                        float val = x[q];
                        if (pending[l] && ii >= 0 && ii < v.n[0] && jj >= 0 && jj < v.n[1]) {
                            const MgLevel &C = m.L[l + 1];
                            val += m.x[l + 1][C.at(ii / C.fac[0], jj / C.fac[1], k / C.fac[2])];
                        }
                        return val;
                    };
                    const float wi = v.w[0][i], wj = v.w[1][j];
                    const float ax = wj * v.w[2][k], ay = wi * v.w[2][k];
                    r += ax * (v.cf[0][i + 1] * nb(i + 1, j, c + v.g.sx) + v.cf[0][i] * nb(i - 1, j, c - v.g.sx)) +
                         ay * (v.cf[1][j + 1] * nb(i, j + 1, c + v.g.sy) + v.cf[1][j] * nb(i, j - 1, c - v.g.sy));
                }
                x[c] = r;
            }
            mg_thomas(v, i, j, x.data() + c0, m.cp[l].data() + c0, 1);
        }
        pending[l] = false;
        last_color[l] = color;
    }
    void restrict(int l) {
        const MgLevel &c = m.L[l + 1];
        for (int I = 0; I < c.n[0]; I++)
            for (int J = 0; J < c.n[1]; J++)
                for (int K = 0; K < c.n[2]; K++)
                    m.f[l + 1][c.at(I, J, K)] = mg_restrict_sum(m.L[l], c, m.x[l].data(), m.f[l].data(),
                                                                I, J, K, last_color[l]);
    }
    void coarse() { m.coarse(); }
    void prolong(int l) { pending[l] = true; }
};

}  // namespace

extern "C" {

void *mgx_create(int n0, int n1, int n2, const double *cx, const double *cy, const double *cz,
                 const double *wx, const double *wy, const double *wz) {
    HostMg *m = new HostMg();
    std::vector<double> cen[3] = {{cx, cx + n0}, {cy, cy + n1}, {cz, cz + n2}};
    std::vector<double> w[3] = {{wx, wx + n0}, {wy, wy + n1}, {wz, wz + n2}};
    m->geo = mg_build_levels(cen, w, MG_MAX_LEVELS, MG_COARSE_TARGET);
    m->levels = (int)m->geo.size();
    for (int a = 0; a < 3; a++) {
        m->cf[a].resize(m->levels);
        m->w[a].resize(m->levels);
    }
    m->x.resize(m->levels);
    m->f.resize(m->levels);
    for (int l = 0; l < m->levels; l++) {
        const MgGeometry &G = m->geo[l];
        MgLevel &v = m->L[l];
        const int gc = l == 0 ? 2 : 1;
        v.g = Grid::make(G.n[0] + 2 * gc, G.n[1] + 2 * gc, G.n[2] + 2 * gc, gc);
        for (int a = 0; a < 3; a++) {
            v.n[a] = G.n[a];
            v.fac[a] = G.fac[a];
            m->cf[a][l].assign(G.cf[a].begin(), G.cf[a].end());
            m->w[a][l].assign(G.w[a].begin(), G.w[a].end());
            v.cf[a] = m->cf[a][l].data();
            v.w[a] = m->w[a][l].data();
        }
        m->x[l].assign((size_t)v.g.total, 0.f);
        m->f[l].assign((size_t)v.g.total, 0.f);
        m->cp.emplace_back((size_t)v.g.total, 0.f);
    }
    const MgGeometry &C = m->geo.back();
    m->ncoarse = (int)C.cells();
    if (m->ncoarse <= MG_MAX_COARSE) {
        std::vector<double> inv = mg_spd_inverse(mg_dense_operator(C), C.cells());
        m->kinv.assign(inv.begin(), inv.end());
    }
    return m;
}

void mgx_destroy(void *ctx) { delete (HostMg *)ctx; }

int mgx_levels(void *ctx, int *out) {
    HostMg *m = (HostMg *)ctx;
    for (int l = 0; l < m->levels; l++)
        for (int a = 0; a < 3; a++) out[3 * l + a] = m->L[l].n[a];
    return m->levels;
}

long long mgx_total(void *ctx) { return ((HostMg *)ctx)->L[0].g.total; }

void mgx_apply(void *ctx, const float *x, float *y) {
    HostMg *m = (HostMg *)ctx;
    const MgLevel &v = m->L[0];
    for (int i = 0; i < v.n[0]; i++)
        for (int j = 0; j < v.n[1]; j++)
            for (int k = 0; k < v.n[2]; k++) y[v.at(i, j, k)] = mg_apply(v, x, i, j, k);
}

// x = V-cycle(f), level-0 arrays in the padded layout
int mgx_vcycle(void *ctx, const float *f, float *x) {
    HostMg *m = (HostMg *)ctx;
    if (m->kinv.empty()) return -1;
    m->f[0].assign(f, f + m->L[0].g.total);
    std::fill(m->x[0].begin(), m->x[0].end(), 0.f);
    mg_vcycle_nu(*m, m->levels, mg_nu);
    std::copy(m->x[0].begin(), m->x[0].end(), x);
    return 0;
}

// Storage facts of level l: {at(0, 0, 0), sx, sy} (the smoother's vector
// path needs all three to be multiples of 8 elements).
void mgx_layout(void *ctx, int l, long long *out) {
    const MgLevel &v = ((HostMg *)ctx)->L[l];
    out[0] = v.at(0, 0, 0);
    out[1] = v.g.sx;
    out[2] = v.g.sy;
}

// The level's FP32 arrays as the device holds them (cf: n + 1, w: n).
void mgx_level_arrays(void *ctx, int l, int a, float *cf, float *w) {
    HostMg *m = (HostMg *)ctx;
    std::copy(m->cf[a][l].begin(), m->cf[a][l].end(), cf);
    std::copy(m->w[a][l].begin(), m->w[a][l].end(), w);
}

// The smoother's z-line factor table of level l (mg_line_table): info gets
// {built, ky, nclass, nf}; with non-null outputs also the classes and table.
void mgx_line_table(void *ctx, int l, int *info, int *cls_x, int *cls_y, float *tab) {
    HostMg *m = (HostMg *)ctx;
    std::vector<float> cf[3], w[3];
    for (int a = 0; a < 3; a++) {
        cf[a] = m->cf[a][l];
        w[a] = m->w[a][l];
    }
    MgLineTable T;
    const bool ok = mg_line_table(m->L[l].n, cf, w, T);
    info[0] = ok ? 1 : 0;
    info[1] = T.ky;
    info[2] = T.nclass;
    info[3] = T.nf;
    if (!ok) return;
    if (cls_x) std::copy(T.cls[0].begin(), T.cls[0].end(), cls_x);
    if (cls_y) std::copy(T.cls[1].begin(), T.cls[1].end(), cls_y);
    if (tab) std::copy(T.tab.begin(), T.tab.end(), tab);
}

// x = the V-cycle as the CUDA executor folds it (HostMgFolded)
int mgx_vcycle_folded(void *ctx, const float *f, float *x) {
    HostMg *m = (HostMg *)ctx;
    if (m->kinv.empty()) return -1;
    m->f[0].assign(f, f + m->L[0].g.total);
    std::fill(m->x[0].begin(), m->x[0].end(), 0.f);
    HostMgFolded e{*m};
    mg_vcycle_nu(e, m->levels, mg_nu);
    std::copy(m->x[0].begin(), m->x[0].end(), x);
    return 0;
}

}  // extern "C"
