// Shared device-side definitions: field layout in HBM, launch geometry,
// deterministic grid reductions.
//
// Layout.  Every field is SoA (one array per component) over the stored grid
// (interior + gc guide cells per side).  k (z) is contiguous like the
// reference (src/util.h:11-13), but each k-row is padded to a pitch that is
// a multiple of 8 elements and shifted by `off` so that the first interior
// cell k = gc of every row starts on a 64-byte (FP64) / 32-byte (FP32)
// boundary: a warp reading 32 consecutive interior cells touches exactly
// 8 (FP64) or 4 (FP32) 32-byte sectors.
#pragma once

#include <utility>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#include <cuda_runtime.h>

namespace dalm {

#define DALM_CUDA(call)                                                              \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess)                                                       \
            throw ::dalm::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct CudaError : std::runtime_error {
    explicit CudaError(const std::string &m) : std::runtime_error(m) {}
};

// A bounded device-side wait ran out (reported as DALM_ERR_DEVICE_WAIT).
struct DeviceWaitError : std::runtime_error {
    explicit DeviceWaitError(const std::string &m) : std::runtime_error(m) {}
};

// An option combination this build does not implement (DALM_ERR_UNSUPPORTED).
struct Unsupported : std::runtime_error {
    explicit Unsupported(const std::string &m) : std::runtime_error(m) {}
};

// Sets the message returned by dalm_last_error(NULL).
void set_last_error(const std::string &msg);

struct Grid {
    int nx, ny, nz, gc;      // stored sizes (incl. guide cells) and guide cells
    long long sx, sy, off;   // element strides and row offset
    long long total;         // elements per field allocation

    __host__ __device__ long long at(int i, int j, int k) const {
        return (long long)i * sx + (long long)j * sy + k + off;
    }
    static Grid make(int nx, int ny, int nz, int gc) {
        Grid g;
        g.nx = nx; g.ny = ny; g.nz = nz; g.gc = gc;
        g.off = (8 - gc % 8) % 8;
        g.sy = ((g.off + nz + 7) / 8) * 8;
        g.sx = g.sy * ny;
        g.total = g.sx * nx;
        return g;
    }
    // interior extents
    __host__ __device__ int ni() const { return nx - 2 * gc; }
    __host__ __device__ int nj() const { return ny - 2 * gc; }
    __host__ __device__ int nk() const { return nz - 2 * gc; }
};

// A box of cells [lo, hi) per axis in stored indices.
struct Box {
    int lo[3], hi[3];
    __host__ __device__ bool empty() const {
        return hi[0] <= lo[0] || hi[1] <= lo[1] || hi[2] <= lo[2];
    }
    __host__ __device__ bool contains(int i, int j, int k) const {
        return i >= lo[0] && i < hi[0] && j >= lo[1] && j < hi[1] && k >= lo[2] && k < hi[2];
    }
};

// Tiling of a box into (32 k) x (8 j) x (1 i) tiles; blocks of 256 threads
// walk the tiles with a block-stride loop so the number of blocks (and thus
// the number of reduction partials) is fixed per launch.
constexpr int TK = 32, TJ = 8, TILE_THREADS = TK * TJ;

struct Tiling {
    Box box;
    int ntk, ntj, nti;
    long long ntiles;
    __host__ static Tiling make(const Box &b) {
        Tiling t;
        t.box = b;
        t.ntk = (b.hi[2] - b.lo[2] + TK - 1) / TK;
        t.ntj = (b.hi[1] - b.lo[1] + TJ - 1) / TJ;
        t.nti = b.hi[0] - b.lo[0];
        if (b.empty()) t.ntk = t.ntj = t.nti = 0;
        t.ntiles = (long long)t.ntk * t.ntj * t.nti;
        return t;
    }
    // cell handled by this thread in tile `tile`; false when outside the box
    __device__ bool cell(long long tile, int &i, int &j, int &k) const {
        int tk = (int)(tile % ntk);
        long long r = tile / ntk;
        int tj = (int)(r % ntj);
        int ti = (int)(r / ntj);
        k = box.lo[2] + tk * TK + (int)(threadIdx.x % TK);
        j = box.lo[1] + tj * TJ + (int)(threadIdx.x / TK);
        i = box.lo[0] + ti;
        return k < box.hi[2] && j < box.hi[1];
    }
};

// Column segments: the box is cut into (32 k) x (8 j) columns, and each
// column into i-chunks of `ich` planes.  One block of 256 threads owns one
// segment; each thread marches along i through its chunk, so neighbours in i
// rotate through registers and every index is 32-bit arithmetic done once
// per block.  Segment u: column = u % ncol, chunk = u / ncol.
struct Segments {
    Box box;
    int ntk, ntj, ncol, nchunk, ich;
    int count;
    // Enough segments to fill the GPU, chunks of at most 32 planes.  (Sizing
    // the chunk count to fill whole waves of resident blocks was measured
    // slower on the 512x256x128 case: shorter chunks cost more than the
    // last wave's idle slots.)
    __host__ static Segments make(const Box &b, int target_blocks) {
        Segments s;
        s.box = b;
        s.ntk = (b.hi[2] - b.lo[2] + TK - 1) / TK;
        s.ntj = (b.hi[1] - b.lo[1] + TJ - 1) / TJ;
        s.ncol = s.ntk * s.ntj;
        int ni = b.hi[0] - b.lo[0];
        if (b.empty()) {
            s.ncol = s.nchunk = s.count = 0;
            s.ich = 1;
            return s;
        }
        // enough segments to fill the GPU, at most 32 planes per chunk
        int want_chunks = (target_blocks + s.ncol - 1) / s.ncol;
        s.ich = (ni + want_chunks - 1) / want_chunks;
        if (s.ich < 1) s.ich = 1;
        if (s.ich > 32) s.ich = 32;
        s.nchunk = (ni + s.ich - 1) / s.ich;
        s.count = s.ncol * s.nchunk;
        return s;
    }
    // planes [i0, i1) of a chunk: balanced, at most ich planes
    __host__ __device__ void chunk_range(int chunk, int &i0, int &i1) const {
        const long long ni = box.hi[0] - box.lo[0];
        i0 = box.lo[0] + (int)(chunk * ni / nchunk);
        i1 = box.lo[0] + (int)((chunk + 1) * ni / nchunk);
    }
    // this thread's (k, j) and the segment's [i0, i1); false when (k, j) is
    // outside the box
    __device__ bool column(int u, int &i0, int &i1, int &j, int &k) const {
        int col = u % ncol, chunk = u / ncol;
        k = box.lo[2] + (col % ntk) * TK + (int)(threadIdx.x & 31);
        j = box.lo[1] + (col / ntk) * TJ + (int)(threadIdx.x >> 5);
        chunk_range(chunk, i0, i1);
        return k < box.hi[2] && j < box.hi[1];
    }
};

// ---- deterministic reductions ---------------------------------------------
//
// Each block reduces its values in a fixed order (warp shuffles, then warps
// in order) and writes one partial per block.  The last block to finish
// (atomic ticket) sums the partials in block order and runs the finisher.
// The result is independent of block scheduling; no block ever waits on
// another, so there is no spin-wait anywhere.

template <int N>
struct Partials {
    double *buf;            // [max_blocks][N]
    unsigned int *ticket;   // one counter, reset by the last block
};

// Slot m of a reduction is a max when bit m of `maxmask` is set, else a sum.
__device__ inline double red_op(double a, double b, bool is_max) {
    return is_max ? (a > b ? a : b) : a + b;
}

__device__ inline double warp_reduce(double v, bool is_max) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = red_op(v, __shfl_down_sync(0xffffffffu, v, o), is_max);
    return v;
}

// Block reduction of N values; result valid in thread 0.
template <int N>
__device__ inline void block_reduce(double (&v)[N], unsigned maxmask, double *smem /*[32*N]*/) {
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int m = 0; m < N; m++) v[m] = warp_reduce(v[m], (maxmask >> m) & 1u);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int m = 0; m < N; m++) smem[warp * N + m] = v[m];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int m = 0; m < N; m++) {
            double a = smem[m];
            for (int w = 1; w < nwarps; w++) a = red_op(a, smem[w * N + m], (maxmask >> m) & 1u);
            v[m] = a;
        }
    }
    __syncthreads();
}

// Writes this block's partials; returns true in every thread of the last
// block, whose thread 0 then holds the grid totals in v.  Max slots assume
// non-negative values (identity 0).
template <int N>
__device__ inline bool grid_reduce(double (&v)[N], unsigned maxmask, Partials<N> P) {
    __shared__ double smem[32 * N];
    __shared__ bool is_last;
    block_reduce<N>(v, maxmask, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int m = 0; m < N; m++) P.buf[blockIdx.x * N + m] = v[m];
        __threadfence();
        unsigned int t = atomicAdd(P.ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    // last block: fixed-order sum of the partials (each thread a fixed
    // strided subset in block order, then the block reduction in warp order)
    double acc[N];
#pragma unroll
    for (int m = 0; m < N; m++) acc[m] = 0.0;
    for (unsigned int b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
        for (int m = 0; m < N; m++) {
            double x = ((volatile double *)P.buf)[b * N + m];
            acc[m] = (b == threadIdx.x) ? x : red_op(acc[m], x, (maxmask >> m) & 1u);
        }
    }
    block_reduce<N>(acc, maxmask, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int m = 0; m < N; m++) v[m] = acc[m];
        *P.ticket = 0u;
    }
    return true;
}

// Kinds of kernels, for launch counting and per-kernel event timing.
enum KernelKind {
    KK_PREDICT = 0, KK_FLUX_RHS, KK_PBC, KK_PROJECT, KK_UBC, KK_DIAG, KK_TAVG,
    KK_ALM_POINTS, KK_ALM_SUMS, KK_ALM_PROJECT,
    KK_SOR_SWEEP, KK_RESIDUAL_NORM, KK_JACOBI_SWEEP,
    KK_BICG_INIT, KK_BICG_P, KK_BICG_Q, KK_BICG_S, KK_BICG_T, KK_BICG_XR,
    KK_POISSON_BEGIN, KK_LAYOUT, KK_SEQ_SUM, KK_BICG_PF, KK_BICG_SF, KK_REFINE_RESIDUAL, KK_REFINE_UPDATE,
    // FP32 inner solves of iterative refinement
    KK_SOR_SWEEP32, KK_JACOBI_SWEEP32, KK_BICG_P32, KK_BICG_Q32, KK_BICG_S32, KK_BICG_T32, KK_BICG_XR32,
    // discrete adjoint
    KK_ADJ_BC, KK_ADJ_PROJECT, KK_ADJ_FACES, KK_ADJ_NUT, KK_ADJ_PREDICT, KK_ADJ_ALM,
    // multigrid-preconditioned CG (inner solves of DALM_MIXED)
    KK_MG_SMOOTH, KK_MG_TRANSFER, KK_MG_COARSE, KK_MG_PCG,
    // two FP64 Jacobi sweeps in one pass (the preconditioner's last two)
    KK_JACOBI_SWEEP2,
    KK_COUNT
};

// Everything a launcher needs besides its operands: the stream, the number
// of blocks for tile loops, and an optional hook called around each launch
// (the host uses it to record CUDA events per kernel kind).
struct LaunchCtx {
    cudaStream_t s = 0;
    int blocks = 1;
    void (*hook)(void *self, int kind, int phase) = nullptr;  // phase 0 before, 1 after
    void *self = nullptr;
    long long *launches = nullptr;
    // per-kind algorithmic bytes of the launches, for kernels whose bytes
    // depend on the launch (multigrid levels); accumulated when profiling
    double *kind_bytes = nullptr;
    void bytes(int kind, double b) const {
        if (kind_bytes) kind_bytes[kind] += b;
    }
    void pre(int kind) const {
        if (hook) hook(self, kind, 0);
    }
    void post(int kind) const {
        if (launches) (*launches)++;
        if (hook) hook(self, kind, 1);
        DALM_CUDA(cudaGetLastError());
    }
};

// Programmatic dependent launch: a kernel launched by pdl_launch may be
// scheduled while the previous kernel in the stream is finishing, so its
// launch latency overlaps that kernel's tail.  pdl_wait(), the first
// statement of every such kernel, holds it until the previous kernel has
// completed and its memory operations are visible (griddepcontrol.wait; a
// no-op when the kernel was launched without the attribute); it then lets
// the next kernel be scheduled as soon as every block of this one has
// started (griddepcontrol.launch_dependents: the waiting blocks of the next
// kernel never hold back a block of this one, which are all resident by
// then).
__device__ __forceinline__ void pdl_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;");
}

template <typename... Exp, typename... Act>
inline void pdl_launch(void (*kernel)(Exp...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Act &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    DALM_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Act>(args)...));
}

inline int reduction_blocks(int sm_count) { return sm_count * 8; }

}  // namespace dalm
