// Host-side construction of the multigrid levels (multigrid.cuh): the
// merged-cell geometry per level, its face conductances, and the dense
// inverse of the coarsest operator.  FP64 here; the device stores FP32.
#pragma once

#include <cmath>
#include <stdexcept>
#include <vector>

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

}  // namespace dalm
