// The predictor of the mixed-precision form (DALM_MIXED): the same stage as
// k_predict (cpy_array(Uold, U) + calc_intermediate_U, src/cfd.h:176-322)
// with the increment dt (-conv + diff + f) computed in FP32 from the FP64
// fields and added to the FP64 velocity:  U* = Uold + (double) increment.
// The increment is of order dt |U| / dx, so its FP32 rounding is ~1e-7 of it
// (~1e-10 of U per step).  Storage stays FP64; the FP64 divergence, Poisson
// residual and projection follow unchanged.  Compiled with contraction and
// fast quotients: this form has no parity to keep with the reference.
#include <algorithm>

#include "flow.cuh"

namespace dalm {

namespace {

__device__ __forceinline__ float qf(float a, float b) { return __fdividef(a, b); }

__device__ __forceinline__ float va_switch_f(float a, float b) {
    const float eps = 1e-12f;
    return qf(2.f * a * b + eps, a * a + b * b + eps);
}

// the b=4 limiter term s_a max(0, min(|a|, s_a bb b)) for (a, b) and
// (b, a): zero unless a and b have the same sign, else min(|a|, bb |b|)
// with a's sign
__device__ __forceinline__ void minmod_pair(float a, float b, float bb, float &gab,
                                            float &gba) {
    const bool same = a * b > 0.f;
    gab = same ? copysignf(fminf(fabsf(a), bb * fabsf(b)), a) : 0.f;
    gba = same ? copysignf(fminf(fabsf(b), bb * fabsf(a)), b) : 0.f;
}

// kappa = 1/3 MUSCL face values and upwind fluxes along one axis
// (src/cfd.h:37-60; van Albada: the extension of DALM_LIMITER_VAN_ALBADA)
__device__ __forceinline__ void muscl_axis_f(float fmm, float fm, float fc, float fp, float fpp,
                                             float Jp, float Jm, float &flux_p, float &flux_m,
                                             int limiter) {
    const float kap = 1.f / 3.f;
    const float bb = (3.f - kap) / (1.f - kap);
    const float d4 = fpp - fp, d3 = fp - fc, d2 = fc - fm, d1 = fm - fmm;
    float fpr, fpl, fmr, fml;
    if (limiter == 1) {
        const float sp = va_switch_f(d4, d3), sc = va_switch_f(d3, d2), sm = va_switch_f(d2, d1);
        fpr = fp - (sp * 0.25f) * ((1.f - kap * sp) * d4 + (1.f + kap * sp) * d3);
        fpl = fc + (sc * 0.25f) * ((1.f - kap * sc) * d2 + (1.f + kap * sc) * d3);
        fmr = fc - (sc * 0.25f) * ((1.f - kap * sc) * d3 + (1.f + kap * sc) * d2);
        fml = fm + (sm * 0.25f) * ((1.f - kap * sm) * d1 + (1.f + kap * sm) * d2);
    } else {
        float g6, g5, g4, g3, g2, g1;
        minmod_pair(d4, d3, bb, g6, g5);
        minmod_pair(d3, d2, bb, g4, g3);
        minmod_pair(d2, d1, bb, g2, g1);
        fpr = fp - 0.25f * ((1.f - kap) * g6 + (1.f + kap) * g5);
        fpl = fc + 0.25f * ((1.f - kap) * g3 + (1.f + kap) * g4);
        fmr = fc - 0.25f * ((1.f - kap) * g4 + (1.f + kap) * g3);
        fml = fm + 0.25f * ((1.f - kap) * g1 + (1.f + kap) * g2);
    }
    flux_p = 0.5f * (Jp * (fpr + fpl) - fabsf(Jp) * (fpr - fpl));
    flux_m = 0.5f * (Jm * (fmr + fml) - fabsf(Jm) * (fmr - fml));
}

// The interior cells in column segments (a block owns 32 k x 8 j columns
// and marches along a chunk of i planes; interior-aligned, so no warp is
// spent on the guide cells, which k_copy_guides copies).  The geometry
// comes from the per-axis FP32 table (MixedGeom) instead of per-cell FP64
// differences and quotients.  Three blocks per SM (80 registers, no
// spills) hide the FP64 loads better than two.
__global__ void __launch_bounds__(TILE_THREADS, 3)
k_predict_f32(StepParams P, Segments T, MixedGeom Gm, float inv_re, Vec3<const double> V,
              Vec3<double> Un, Vec3<const double> JU, Vec3<const double> F) {
    const Grid &g = P.g;
    const long long sx = g.sx, sy = g.sy;
    const float dt = (float)P.dt;
    for (int u = blockIdx.x; u < T.count; u += gridDim.x) {
        int i0, i1, j, k;
        if (!T.column(u, i0, i1, j, k)) continue;
        const float4 gy = Gm.ax[1][j], gz = Gm.ax[2][k];
        for (int i = i0; i < i1; i++) {
            const long long c = g.at(i, j, k);
            const float4 gx = Gm.ax[0][i];
            const float inv_vol = gx.x * gy.x * gz.x;
            // central differences over x[i+1] - x[i-1] (calc_nut_at_cell, src/cfd.h:786-825)
            float G[3][3];
#pragma unroll
            for (int m = 0; m < 3; m++) {
                const double *v = V.c[m];
                G[m][0] = (float)(v[c + sx] - v[c - sx]) * gx.w;
                G[m][1] = (float)(v[c + sy] - v[c - sy]) * gy.w;
                G[m][2] = (float)(v[c + 1] - v[c - 1]) * gz.w;
            }
            const float S = 2.f * (G[0][0] * G[0][0] + G[1][1] * G[1][1] + G[2][2] * G[2][2]) +
                            (G[0][1] + G[1][0]) * (G[0][1] + G[1][0]) +
                            (G[0][2] + G[2][0]) * (G[0][2] + G[2][0]) +
                            (G[1][2] + G[2][1]) * (G[1][2] + G[2][1]);
            const float visc = inv_re + (float)P.filter2[c] * sqrtf(S);
            const float JUE = (float)JU.c[0][c], JUW = (float)JU.c[0][c - sx];
            const float JVN = (float)JU.c[1][c], JVS = (float)JU.c[1][c - sy];
            const float JWT = (float)JU.c[2][c], JWB = (float)JU.c[2][c - 1];
            const float divJ = JUE - JUW + JVN - JVS + JWT - JWB;
            const bool has_f = P.fbox.contains(i, j, k);
#pragma unroll
            for (int m = 0; m < 3; m++) {
                const double *v = V.c[m];
                const double fc64 = v[c];
                // differences to the cell value in FP32: the stencil in the
                // velocity's own frame keeps full relative accuracy
                const float fc = 0.f;
                const float fe = (float)(v[c + sx] - fc64), fee = (float)(v[c + 2 * sx] - fc64);
                const float fw = (float)(v[c - sx] - fc64), fww = (float)(v[c - 2 * sx] - fc64);
                const float fn = (float)(v[c + sy] - fc64), fnn = (float)(v[c + 2 * sy] - fc64);
                const float fs = (float)(v[c - sy] - fc64), fss = (float)(v[c - 2 * sy] - fc64);
                const float ft = (float)(v[c + 1] - fc64), ftt = (float)(v[c + 2] - fc64);
                const float fb = (float)(v[c - 1] - fc64), fbb = (float)(v[c - 2] - fc64);
                float fE, fW, fN, fS, fT, fB;
                muscl_axis_f(fww, fw, fc, fe, fee, JUE, JUW, fE, fW, P.limiter);
                muscl_axis_f(fss, fs, fc, fn, fnn, JVN, JVS, fN, fS, P.limiter);
                muscl_axis_f(fbb, fb, fc, ft, ftt, JWT, JWB, fT, fB, P.limiter);
                // the flux differences of the shifted values plus the shift's own
                // (fc64 times the face-flux divergence)
                const float conv = (fE - fW + fN - fS + fT - fB + (float)fc64 * divJ) * inv_vol;
                const float diff = visc * ((fe * gx.y + fw * gx.z) * gx.x +
                                           (fn * gy.y + fs * gy.z) * gy.x +
                                           (ft * gz.y + fb * gz.z) * gz.x);
                const float fm = has_f ? (float)F.c[m][c] : 0.f;
                Un.c[m][c] = fc64 + (double)(dt * (-conv + diff + fm));
            }
            // the guide cells at the ends of this k row (U* = U^n there)
            if (k == g.gc || k == g.nz - g.gc - 1) {
                const long long d = k == g.gc ? -1 : 1;
                for (int t = 1; t <= g.gc; t++)
#pragma unroll
                    for (int m = 0; m < 3; m++) Un.c[m][c + t * d] = V.c[m][c + t * d];
            }
        }
    }
}

// U* = U^n on the guide cells of the rows (i, j) outside the interior (no
// boundary condition after the predictor; k_predict_f32 copies the k ends of
// the interior rows): one warp per row, 2 gc planes of ny rows, then 2 gc
// strips of nx - 2 gc rows.
__global__ void __launch_bounds__(256) k_copy_guides(Grid g, Vec3<const double> V, Vec3<double> Un) {
    const int gc = g.gc, ni = g.nx - 2 * gc;
    const int lane = threadIdx.x & 31;
    const unsigned a = 2u * gc * g.ny;
    const unsigned rows = a + 2u * gc * ni;
    const unsigned nw = gridDim.x * (blockDim.x >> 5);
    for (unsigned r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += nw) {
        int i, j;
        if (r < a) {
            const int p = (int)(r / g.ny);
            i = p < gc ? p : g.nx - 2 * gc + p;
            j = (int)(r - (unsigned)p * g.ny);
        } else {
            const unsigned q = r - a;
            const int p = (int)(q / ni);
            j = p < gc ? p : g.ny - 2 * gc + p;
            i = gc + (int)(q - (unsigned)p * ni);
        }
        const long long c0 = g.at(i, j, 0);
        for (int k = lane; k < g.nz; k += 32)
            for (int m = 0; m < 3; m++) Un.c[m][c0 + k] = V.c[m][c0 + k];
    }
}

}  // namespace

void launch_predict_f32(const LaunchCtx &L, const StepParams &P, const MixedGeom &geo,
                        Vec3<const double> uold, Vec3<double> unew, Vec3<const double> ju,
                        Vec3<const double> f) {
    const Grid &g = P.g;
    const Segments T =
        Segments::make(Box{{g.gc, g.gc, g.gc}, {g.nx - g.gc, g.ny - g.gc, g.nz - g.gc}}, L.blocks);
    L.pre(KK_PREDICT);
    k_predict_f32<<<L.blocks, TILE_THREADS, 0, L.s>>>(P, T, geo, (float)(1.0 / P.re), uold, unew,
                                                       ju, f);
    L.post(KK_PREDICT);
    const long long outer = 2LL * g.gc * g.ny + 2LL * g.gc * (g.nx - 2 * g.gc);
    L.pre(KK_PREDICT);
    k_copy_guides<<<(int)std::min<long long>((outer + 7) / 8, 2 * 148), 256, 0, L.s>>>(g, uold,
                                                                                    unew);
    L.post(KK_PREDICT);
}

}  // namespace dalm
