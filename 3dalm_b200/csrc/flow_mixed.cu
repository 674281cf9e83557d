// The predictor of the mixed-precision form (DALM_MIXED): the same stage as
// k_predict (cpy_array(Uold, U) + calc_intermediate_U, src/cfd.h:176-322)
// with the increment dt (-conv + diff + f) computed in FP32 from the FP64
// fields and added to the FP64 velocity:  U* = Uold + (double) increment.
// The increment is of order dt |U| / dx, so its FP32 rounding is ~1e-7 of it
// (~1e-10 of U per step).  Storage stays FP64; the FP64 divergence, Poisson
// residual and projection follow unchanged.  Compiled with contraction and
// fast quotients: this form has no parity to keep with the reference.
#include "flow.cuh"

namespace dalm {

namespace {

__device__ __forceinline__ float sgnf(float v) { return (float)((v > 0.f) - (v < 0.f)); }
__device__ __forceinline__ float qf(float a, float b) { return __fdividef(a, b); }

__device__ __forceinline__ float va_switch_f(float a, float b) {
    const float eps = 1e-12f;
    return qf(2.f * a * b + eps, a * a + b * b + eps);
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
        const float s4 = sgnf(d4), s3 = sgnf(d3), s2 = sgnf(d2), s1 = sgnf(d1);
        const float g6 = s4 * fmaxf(0.f, fminf(fabsf(d4), s4 * bb * d3));
        const float g5 = s3 * fmaxf(0.f, fminf(fabsf(d3), s3 * bb * d4));
        const float g4 = s3 * fmaxf(0.f, fminf(fabsf(d3), s3 * bb * d2));
        const float g3 = s2 * fmaxf(0.f, fminf(fabsf(d2), s2 * bb * d3));
        const float g2 = s2 * fmaxf(0.f, fminf(fabsf(d2), s2 * bb * d1));
        const float g1 = s1 * fmaxf(0.f, fminf(fabsf(d1), s1 * bb * d2));
        fpr = fp - 0.25f * ((1.f - kap) * g6 + (1.f + kap) * g5);
        fpl = fc + 0.25f * ((1.f - kap) * g3 + (1.f + kap) * g4);
        fmr = fc - 0.25f * ((1.f - kap) * g4 + (1.f + kap) * g3);
        fml = fm + 0.25f * ((1.f - kap) * g1 + (1.f + kap) * g2);
    }
    flux_p = 0.5f * (Jp * (fpr + fpl) - fabsf(Jp) * (fpr - fpl));
    flux_m = 0.5f * (Jm * (fmr + fml) - fabsf(Jm) * (fmr - fml));
}

// every cell of the stored grid (guide cells copied) in column segments:
// a block owns 32 k x 8 j columns and marches along a chunk of i planes
__global__ void __launch_bounds__(TILE_THREADS, 2)
k_predict_f32(StepParams P, Segments T, Vec3<const double> V, Vec3<double> Un,
              Vec3<const double> JU, Vec3<const double> F) {
    const Grid &g = P.g;
    for (int u = blockIdx.x; u < T.count; u += gridDim.x) {
        int i0, i1, j, k;
        if (!T.column(u, i0, i1, j, k)) continue;
        for (int i = i0; i < i1; i++) {
            const long long c = g.at(i, j, k);
            const bool inner = i >= g.gc && i < g.nx - g.gc && j >= g.gc && j < g.ny - g.gc &&
                               k >= g.gc && k < g.nz - g.gc;
            if (!inner) {
                for (int m = 0; m < 3; m++) Un.c[m][c] = V.c[m][c];
                continue;
            }
            const long long sx = g.sx, sy = g.sy;
            const float dxc = (float)P.m.dx[i], dyc = (float)P.m.dy[j], dzc = (float)P.m.dz[k];
            const float vol = dxc * dyc * dzc;
            // central differences over x[i+1] - x[i-1] (calc_nut_at_cell, src/cfd.h:786-825)
            const float dxew = (float)(P.m.x[i + 1] - P.m.x[i - 1]);
            const float dyns = (float)(P.m.y[j + 1] - P.m.y[j - 1]);
            const float dztb = (float)(P.m.z[k + 1] - P.m.z[k - 1]);
            float G[3][3];
            for (int m = 0; m < 3; m++) {
                const double *v = V.c[m];
                G[m][0] = qf((float)(v[c + sx] - v[c - sx]), dxew);
                G[m][1] = qf((float)(v[c + sy] - v[c - sy]), dyns);
                G[m][2] = qf((float)(v[c + 1] - v[c - 1]), dztb);
            }
            const float S = 2.f * (G[0][0] * G[0][0] + G[1][1] * G[1][1] + G[2][2] * G[2][2]) +
                            (G[0][1] + G[1][0]) * (G[0][1] + G[1][0]) +
                            (G[0][2] + G[2][0]) * (G[0][2] + G[2][0]) +
                            (G[1][2] + G[2][1]) * (G[1][2] + G[2][1]);
            const float visc = (float)(1.0 / P.re) + (float)P.filter2[c] * sqrtf(S);
            const float JUE = (float)JU.c[0][c], JUW = (float)JU.c[0][c - sx];
            const float JVN = (float)JU.c[1][c], JVS = (float)JU.c[1][c - sy];
            const float JWT = (float)JU.c[2][c], JWB = (float)JU.c[2][c - 1];
            const float rxe = 1.f / (float)(P.m.x[i + 1] - P.m.x[i]), rxw = 1.f / (float)(P.m.x[i] - P.m.x[i - 1]);
            const float ryn = 1.f / (float)(P.m.y[j + 1] - P.m.y[j]), rys = 1.f / (float)(P.m.y[j] - P.m.y[j - 1]);
            const float rzt = 1.f / (float)(P.m.z[k + 1] - P.m.z[k]), rzb = 1.f / (float)(P.m.z[k] - P.m.z[k - 1]);
            const bool has_f = P.fbox.contains(i, j, k);
            const float dt = (float)P.dt;
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
                const float conv = qf(fE - fW + fN - fS + fT - fB +
                                          (float)fc64 * (JUE - JUW + JVN - JVS + JWT - JWB),
                                      vol);
                const float diff = visc * (qf(fe * rxe + fw * rxw, dxc) + qf(fn * ryn + fs * rys, dyc) +
                                           qf(ft * rzt + fb * rzb, dzc));
                const float fm = has_f ? (float)F.c[m][c] : 0.f;
                Un.c[m][c] = fc64 + (double)(dt * (-conv + diff + fm));
            }
        }
    }
}

}  // namespace

void launch_predict_f32(const LaunchCtx &L, const StepParams &P, Vec3<const double> uold,
                        Vec3<double> unew, Vec3<const double> ju, Vec3<const double> f) {
    L.pre(KK_PREDICT);
    const Segments T = Segments::make(Box{{0, 0, 0}, {P.g.nx, P.g.ny, P.g.nz}}, L.blocks);
    k_predict_f32<<<L.blocks, TILE_THREADS, 0, L.s>>>(P, T, uold, unew, ju, f);
    L.post(KK_PREDICT);
}

}  // namespace dalm
