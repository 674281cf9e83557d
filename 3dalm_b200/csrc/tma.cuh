// TMA (cp.async.bulk.tensor) plane staging for the stencil kernels.
//
// A field is described to the TMA unit as a 3-D tensor {x = k + off (the
// padded row), y = j, z = i}.  Three maps per field: `halo` boxes of
// (32 + 2h) x 10 x 1 elements (the 32 x 8 tile of a block plus one cell in
// j and h cells in k each side, h = 16 B / element size so that the box
// starts on a 16-byte boundary), `plain` boxes of 32 x 8 x 1 and `wide`
// boxes (below).  Loads complete on an mbarrier per ring stage.  Every wait
// is bounded: after WAIT_LIMIT polls the kernel raises an error flag and
// returns.
#pragma once

#include <cuda.h>

#include "common.cuh"

namespace dalm {

// `wide` boxes carry the three-cell halo of the fused BiCGStab kernels:
// (32 + 2*4) x (8 + 2*3) x 1, starting 4 cells below the tile in k (a
// 16-byte boundary for 4- and 8-byte elements) and 3 rows below it in j.
constexpr int WIDE_HK = 4, WIDE_HJ = 3;

struct FieldMaps {
    CUtensorMap halo;
    CUtensorMap plain;
    CUtensorMap wide;
};

// Builds both maps for one field (element size 4 or 8) over grid g; throws
// CudaError when the driver rejects them.
FieldMaps make_field_maps(const Grid &g, const void *base, int elem_bytes);

constexpr unsigned WAIT_LIMIT = 1u << 24;

__device__ __forceinline__ unsigned smem_addr(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

// true once the phase with the given parity has completed
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// bounded wait; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity) {
    for (unsigned n = 0; n < WAIT_LIMIT; n++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// 3-D tiled TMA load of one box into shared memory, completing on `bar`.
// x (the element index within the padded row) must be a multiple of
// 16 bytes / element size; callers guarantee it.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
        "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

}  // namespace dalm
