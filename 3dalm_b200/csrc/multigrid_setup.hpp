// Host-side construction of the multigrid levels (multigrid.cuh): the
// merged-cell geometry per level, its face conductances, and the dense
// inverse of the coarsest operator.  FP64 here; the device stores FP32.
#pragma once

#include <array>
#include <cmath>
#include <stdexcept>
#include <vector>

#include "multigrid.cuh"

namespace dalm {

struct MgGeometry {
    int n[3] = {0, 0, 0}, fac[3] = {1, 1, 1};
    std::vector<double> cen[3], w[3], cf[3];  // centres, widths [n]; conductances [n + 1]

    long long cells() const { return (long long)n[0] * n[1] * n[2]; }

    // conductances of the finite-volume Laplacian: interior faces
    // 1 / (centre distance), the x+ outlet face 2 / width (p = 0 half a cell
    // away), inflow and wall faces 0
    void finish() {
        for (int a = 0; a < 3; a++) {
            n[a] = (int)cen[a].size();
            cf[a].assign(n[a] + 1, 0.0);
            for (int f = 0; f + 1 < n[a]; f++) cf[a][f + 1] = 1.0 / (cen[a][f + 1] - cen[a][f]);
            if (a == 0) cf[a][n[a]] = 2.0 / w[a][n[a] - 1];
        }
    }
};

// Levels from the interior cell centres and widths of the finest grid,
// down to the first level of at most `target` cells (solved directly).
inline std::vector<MgGeometry> mg_build_levels(const std::vector<double> (&cen)[3],
                                               const std::vector<double> (&w)[3],
                                               int max_levels, long long target) {
    std::vector<MgGeometry> L(1);
    for (int a = 0; a < 3; a++) {
        L[0].cen[a] = cen[a];
        L[0].w[a] = w[a];
    }
    L[0].finish();
    while ((int)L.size() < max_levels && L.back().cells() > target) {
        const MgGeometry &F = L.back();
        MgGeometry C;
        bool any = false;
        // x and y halve while they can (z-line relaxation handles z on every
        // level); z halves only once neither x nor y can
        auto can = [&](int a) { return F.n[a] % 2 == 0 && F.n[a] >= 4; };
        for (int a = 0; a < 2; a++) {
            C.fac[a] = can(a) ? 2 : 1;
            any = any || C.fac[a] == 2;
        }
        C.fac[2] = (!any && can(2)) ? 2 : 1;
        any = any || C.fac[2] == 2;
        if (!any) break;
        for (int a = 0; a < 3; a++) {
            for (int I = 0; I < F.n[a] / C.fac[a]; I++) {
                if (C.fac[a] == 2) {
                    C.cen[a].push_back(0.5 * (F.cen[a][2 * I] + F.cen[a][2 * I + 1]));
                    C.w[a].push_back(F.w[a][2 * I] + F.w[a][2 * I + 1]);
                } else {
                    C.cen[a].push_back(F.cen[a][I]);
                    C.w[a].push_back(F.w[a][I]);
                }
            }
        }
        C.finish();
        L.push_back(C);
    }
    return L;
}

// Dense K = -L of a level, row-major over (i n1 + j) n2 + k.
inline std::vector<double> mg_dense_operator(const MgGeometry &G) {
    const long long N = G.cells();
    std::vector<double> K((size_t)(N * N), 0.0);
    auto id = [&](int i, int j, int k) { return ((long long)i * G.n[1] + j) * G.n[2] + k; };
    for (int i = 0; i < G.n[0]; i++)
        for (int j = 0; j < G.n[1]; j++)
            for (int k = 0; k < G.n[2]; k++) {
                const long long r = id(i, j, k);
                const double area[3] = {G.w[1][j] * G.w[2][k], G.w[0][i] * G.w[2][k],
                                        G.w[0][i] * G.w[1][j]};
                const int idx[3] = {i, j, k};
                for (int a = 0; a < 3; a++) {
                    const double lo = G.cf[a][idx[a]], hi = G.cf[a][idx[a] + 1];
                    K[(size_t)(r * N + r)] += area[a] * (lo + hi);
                    int nb[3] = {i, j, k};
                    if (idx[a] > 0) {
                        nb[a] = idx[a] - 1;
                        K[(size_t)(r * N + id(nb[0], nb[1], nb[2]))] -= area[a] * lo;
                    }
                    nb[a] = idx[a] + 1;
                    if (idx[a] + 1 < G.n[a])
                        K[(size_t)(r * N + id(nb[0], nb[1], nb[2]))] -= area[a] * hi;
                }
            }
    return K;
}

// Inverse of a symmetric positive definite matrix by Cholesky.
inline std::vector<double> mg_spd_inverse(std::vector<double> A, long long N) {
    for (long long j = 0; j < N; j++) {  // A = L L^T in the lower triangle
        double d = A[(size_t)(j * N + j)];
        for (long long k = 0; k < j; k++) d -= A[(size_t)(j * N + k)] * A[(size_t)(j * N + k)];
        if (!(d > 0)) throw std::runtime_error("multigrid coarse operator is not positive definite");
        d = std::sqrt(d);
        A[(size_t)(j * N + j)] = d;
        for (long long i = j + 1; i < N; i++) {
            double s = A[(size_t)(i * N + j)];
            for (long long k = 0; k < j; k++) s -= A[(size_t)(i * N + k)] * A[(size_t)(j * N + k)];
            A[(size_t)(i * N + j)] = s / d;
        }
    }
    std::vector<double> X((size_t)(N * N), 0.0), y((size_t)N);
    for (long long c = 0; c < N; c++) {  // column c of the inverse
        for (long long i = 0; i < N; i++) {
            double s = (i == c) ? 1.0 : 0.0;
            for (long long k = 0; k < i; k++) s -= A[(size_t)(i * N + k)] * y[(size_t)k];
            y[(size_t)i] = s / A[(size_t)(i * N + i)];
        }
        for (long long i = N - 1; i >= 0; i--) {
            double s = y[(size_t)i];
            for (long long k = i + 1; k < N; k++) s -= A[(size_t)(k * N + i)] * X[(size_t)(k * N + c)];
            X[(size_t)(i * N + c)] = s / A[(size_t)(i * N + i)];
        }
    }
    return X;
}

// Z-line factor table of a level (MgLevel::ltab): the classes of columns
// with equal line matrices and, per class, the matrix-only quantities of the
// partition-method solve (mglf_* layout), computed in FP64 from the FP32
// level arrays the device holds and the same formulas as k_mg_smooth's
// generic path.  False (no table) when the columns are longer than 256
// cells or there are more than MG_MAX_LINE_CLASSES classes (a mesh that is
// not uniform in x or y); the smoother then forms and eliminates each
// column's matrix itself.
constexpr int MG_MAX_LINE_CLASSES = 64;

struct MgLineTable {
    std::vector<int> cls[2];
    int ky = 0, nclass = 0, nf = 0;
    std::vector<float> tab;
};

inline bool mg_line_table(const int (&n)[3], const std::vector<float> (&cf)[3],
                          const std::vector<float> (&w)[3], MgLineTable &T) {
    const int nk = n[2], R = (nk + 31) / 32;
    if (R < 1 || R > 8) return false;
    std::vector<std::array<float, 3>> keys[2];
    for (int a = 0; a < 2; a++) {
        T.cls[a].assign(n[a], 0);
        for (int q = 0; q < n[a]; q++) {
            const std::array<float, 3> key = {w[a][q], cf[a][q + 1], cf[a][q]};
            size_t c = 0;
            while (c < keys[a].size() && keys[a][c] != key) c++;
            if (c == keys[a].size()) {
                if ((int)keys[a].size() >= MG_MAX_LINE_CLASSES) return false;
                keys[a].push_back(key);
            }
            T.cls[a][q] = (int)c;
        }
    }
    T.ky = (int)keys[1].size();
    T.nclass = (int)keys[0].size() * T.ky;
    if (T.nclass > MG_MAX_LINE_CLASSES) return false;
    T.nf = mglf_count(R);
    T.tab.assign((size_t)T.nclass * T.nf * 32, 0.f);
    const int N = 32 * R;
    std::vector<double> A(N), B(N), C(N), q(N), fa(N), g(N), xa(N), xc(N);
    double ra[32], rb[32], rc[32];
    for (int cx = 0; cx < (int)keys[0].size(); cx++)
        for (int cy = 0; cy < T.ky; cy++) {
            float *tab = T.tab.data() + (size_t)(cx * T.ky + cy) * T.nf * 32;
            auto put = [&](int field, int lane, double v) { tab[field * 32 + lane] = (float)v; };
            const double wi = keys[0][cx][0], xe = keys[0][cx][1], xw = keys[0][cx][2];
            const double wj = keys[1][cy][0], yn = keys[1][cy][1], ys = keys[1][cy][2];
            const double az = wi * wj, sxy = wj * (xe + xw) + wi * (yn + ys);
            for (int k = 0; k < N; k++) {
                if (k < nk) {
                    const double lo = az * cf[2][k], hi = az * cf[2][k + 1];
                    A[k] = -lo;
                    B[k] = w[2][k] * sxy + lo + hi;
                    C[k] = -hi;
                } else {
                    A[k] = 0;
                    B[k] = 1;
                    C[k] = 0;
                }
            }
            // each lane's first R - 1 rows: forward, then back sweep
            for (int l = 0; l < 32; l++) {
                const int k0 = R * l;
                for (int s = 0; s + 1 < R; s++) {
                    const int k = k0 + s;
                    const double den = s == 0 ? B[k] : B[k] - A[k] * g[k - 1];
                    q[k] = 1.0 / den;
                    fa[k] = (s == 0 ? A[k] : -A[k] * fa[k - 1]) * q[k];
                    g[k] = C[k] * q[k];
                    put(mglf_q(s), l, q[k]);
                    put(mglf_a(s), l, A[k]);
                    put(mglf_g(s), l, g[k]);
                }
                for (int s = R - 2; s >= 0; s--) {
                    const int k = k0 + s;
                    if (s == R - 2) {
                        xa[k] = fa[k];
                        xc[k] = g[k];
                    } else {
                        xa[k] = fa[k] - g[k] * xa[k + 1];
                        xc[k] = -g[k] * xc[k + 1];
                    }
                    put(mglf_xa(s), l, xa[k]);
                    put(mglf_xc(s), l, xc[k]);
                }
            }
            // the lanes' last rows, in the segment ends y_l alone
            for (int l = 0; l < 32; l++) {
                const int kl = R * l + R - 1;
                if (R == 1) {
                    ra[l] = A[kl];
                    rb[l] = B[kl];
                    rc[l] = C[kl];
                    continue;
                }
                const double An = l < 31 ? xa[R * (l + 1)] : 0.0, Cn = l < 31 ? xc[R * (l + 1)] : 0.0;
                ra[l] = -A[kl] * xa[kl - 1];
                rb[l] = B[kl] - A[kl] * xc[kl - 1] - C[kl] * An;
                rc[l] = -C[kl] * Cn;
                put(mglf_al(R), l, A[kl]);
                put(mglf_cl(R), l, C[kl]);
            }
            // parallel cyclic reduction over the lanes (identity rows outside)
            for (int t = 0; t < 5; t++) {
                const int d = 1 << t;
                double na[32], nb[32], nc[32];
                for (int l = 0; l < 32; l++) {
                    const bool m = l >= d, p = l + d < 32;
                    const double am = m ? ra[l - d] : 0, bm = m ? rb[l - d] : 1, cm = m ? rc[l - d] : 0;
                    const double ap = p ? ra[l + d] : 0, bp = p ? rb[l + d] : 1, cp = p ? rc[l + d] : 0;
                    const double alpha = -ra[l] / bm, gamma = -rc[l] / bp;
                    put(mglf_alpha(R, t), l, alpha);
                    put(mglf_gamma(R, t), l, gamma);
                    nb[l] = rb[l] + alpha * cm + gamma * ap;
                    na[l] = alpha * am;
                    nc[l] = gamma * cp;
                }
                for (int l = 0; l < 32; l++) {
                    ra[l] = na[l];
                    rb[l] = nb[l];
                    rc[l] = nc[l];
                }
            }
            for (int l = 0; l < 32; l++) put(mglf_invrb(R), l, 1.0 / rb[l]);
        }
    return true;
}

}  // namespace dalm
