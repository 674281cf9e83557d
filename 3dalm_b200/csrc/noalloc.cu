// dalm_diagnostics_noalloc: the divergence norm and maximum CFL number of a
// velocity / face-flux state that the caller already holds in device memory,
// computed without allocating anything.
//
// Who needs it: code that owns the solver's arrays itself and cannot let a
// library call cudaMalloc -- an OpenACC program that keeps U and JU in its
// own `acc enter data` region and hands device pointers over with
// `host_data use_device`, a caller whose memory pool already holds the
// whole device budget, or code that must not trigger an allocation (and
// the implicit synchronisation it brings) in the middle of a time step.
//
// The per-segment partial sums of the reduction live in the file-scope
// array below (g_partials), so every GPU that loads this library holds
// NOALLOC_MAX_SEGMENTS * 2 doubles (256 KiB) plus one counter until the
// process exits.  The first call on a device looks up the array's device
// address with cudaGetSymbolAddress (with that device current) and caches
// it; make that first call before any CUDA stream capture.  All calls share
// the array and it keeps the last call's contents; the completion counter is
// cleared on the caller's stream at the start of every call.  Calls whose
// work overlaps on the GPU (different streams, or other devices' calls are
// fine) race on the array: serialise them.
#include <cmath>
#include <mutex>
#include <string>

#include "../../include/dalm.h"
#include "common.cuh"

namespace dalm {
namespace {

constexpr int NOALLOC_MAX_SEGMENTS = 16384;
constexpr int NOALLOC_CHUNK = 16;  // i-planes per segment
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) double g_partials[NOALLOC_MAX_SEGMENTS * 2];
static __device__ __align__(256) unsigned int g_ticket;

struct ScratchPtrs {
    double *partials;
    unsigned int *ticket;
};

std::mutex g_setup_mutex;
ScratchPtrs g_scratch[NOALLOC_MAX_DEVICES];
bool g_ready[NOALLOC_MAX_DEVICES];

// Reference layout: cell (i,j,k) at (i*NY + j)*NZ + k, vectors AoS [len][3].
__global__ void __launch_bounds__(TILE_THREADS)
k_diag_ref_layout(Segments S, int ny, int nz, const double *U, const double *JU,
                  const double *dx, const double *dy, const double *dz, double dt, double ncell,
                  Partials<2> part, double *out) {
    double div2 = 0, cfl = 0;
    for (int u = blockIdx.x; u < S.count; u += gridDim.x) {
        int i0, i1, j, k;
        if (!S.column(u, i0, i1, j, k)) continue;
        for (int i = i0; i < i1; i++) {
            long long c = ((long long)i * ny + j) * nz + k;
            long long w = c - (long long)ny * nz, s = c - nz, b = c - 1;
            // calc_divergence (src/cfd.h:1093-1105)
            double J = dx[i] * dy[j] * dz[k];
            double d = (JU[c * 3 + 0] - JU[w * 3 + 0] + JU[c * 3 + 1] - JU[s * 3 + 1] +
                        JU[c * 3 + 2] - JU[b * 3 + 2]) / J;
            div2 += d * d;
            // calc_max_cfl (src/cfd.h:1126-1130)
            double local = fabs(U[c * 3 + 0]) * dt / dx[i] + fabs(U[c * 3 + 1]) * dt / dy[j] +
                           fabs(U[c * 3 + 2]) * dt / dz[k];
            cfl = local > cfl ? local : cfl;
        }
    }
    double v[2] = {div2, cfl};
    if (grid_reduce<2>(v, 2u, part) && threadIdx.x == 0) {
        out[0] = sqrt(v[0]) / sqrt(ncell);
        out[1] = v[1];
    }
}

}  // namespace
}  // namespace dalm

using namespace dalm;

extern "C" int dalm_diagnostics_noalloc(const double *U, const double *JU, const double *dx,
                                        const double *dy, const double *dz,
                                        const int64_t size[3], int64_t gc, double dt,
                                        double *out, void *stream) {
    if (!U || !JU || !dx || !dy || !dz || !size || !out) {
        set_last_error("dalm_diagnostics_noalloc: null argument");
        return DALM_ERR_ARG;
    }
    if (gc < 1 || size[0] <= 2 * gc || size[1] <= 2 * gc || size[2] <= 2 * gc ||
        size[0] > (1 << 30) || size[1] > (1 << 30) || size[2] > (1 << 30)) {
        set_last_error("dalm_diagnostics_noalloc: bad grid size");
        return DALM_ERR_ARG;
    }
    Box box{{(int)gc, (int)gc, (int)gc},
            {(int)(size[0] - gc), (int)(size[1] - gc), (int)(size[2] - gc)}};
    Segments S;
    S.box = box;
    S.ntk = (box.hi[2] - box.lo[2] + TK - 1) / TK;
    S.ntj = (box.hi[1] - box.lo[1] + TJ - 1) / TJ;
    S.ncol = S.ntk * S.ntj;
    S.ich = NOALLOC_CHUNK;
    S.nchunk = (box.hi[0] - box.lo[0] + S.ich - 1) / S.ich;
    int64_t segments = (int64_t)S.ncol * S.nchunk;
    if (segments > NOALLOC_MAX_SEGMENTS) {
        // too large for the fixed scratch array: one partial per segment of
        // 32 (k) x 8 (j) x 16 (i) interior cells, at most 16384 segments
        set_last_error("dalm_diagnostics_noalloc: grid needs " + std::to_string(segments) +
                       " segments of 32x8x16 interior cells; the fixed scratch holds 16384");
        return DALM_ERR_UNSUPPORTED;
    }
    S.count = (int)segments;

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        set_last_error(std::string("dalm_diagnostics_noalloc: no usable current device: ") +
                       cudaGetErrorString(e));
        return DALM_ERR_CUDA;
    }
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_ready[dev]) {
            // once per device, with that device current: the array's device
            // address (the host-side name is only a stand-in)
            ScratchPtrs p{};
            e = cudaGetSymbolAddress((void **)&p.partials, g_partials);
            if (e == cudaSuccess) e = cudaGetSymbolAddress((void **)&p.ticket, g_ticket);
            if (e != cudaSuccess) {
                set_last_error(std::string("dalm_diagnostics_noalloc: cudaGetSymbolAddress: ") +
                               cudaGetErrorString(e));
                return DALM_ERR_CUDA;
            }
            g_scratch[dev] = p;
            g_ready[dev] = true;
        }
    }
    ScratchPtrs p = g_scratch[dev];
    cudaStream_t s = (cudaStream_t)stream;
    // the completion counter must start at zero; the partials are fully
    // overwritten by every call
    e = cudaMemsetAsync(p.ticket, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) {
        set_last_error(std::string("dalm_diagnostics_noalloc: ") + cudaGetErrorString(e));
        return DALM_ERR_CUDA;
    }
    double ncell = (double)(size[0] - 2 * gc) * (double)(size[1] - 2 * gc) * (double)(size[2] - 2 * gc);
    k_diag_ref_layout<<<S.count, TILE_THREADS, 0, s>>>(S, (int)size[1], (int)size[2], U, JU, dx, dy,
                                                       dz, dt, ncell, Partials<2>{p.partials, p.ticket},
                                                       out);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_error(std::string("dalm_diagnostics_noalloc: ") + cudaGetErrorString(e));
        return DALM_ERR_CUDA;
    }
    return DALM_OK;
}
