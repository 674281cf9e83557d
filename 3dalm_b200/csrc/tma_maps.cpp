// Host side of tma.cuh: tensor maps through the driver's
// cuTensorMapEncodeTiled, reached with cudaGetDriverEntryPoint so the library
// needs no link-time dependency on libcuda.
#include <cudaTypedefs.h>

#include <mutex>

#include "tma.cuh"

namespace dalm {

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    if (!fn) throw CudaError("cuTensorMapEncodeTiled is not available from the driver");
    return fn;
}

void encode(CUtensorMap *map, const Grid &g, const void *base, int eb, cuuint32_t bx, cuuint32_t by) {
    cuuint64_t dims[3] = {(cuuint64_t)g.sy, (cuuint64_t)g.ny, (cuuint64_t)g.nx};
    cuuint64_t strides[2] = {(cuuint64_t)g.sy * eb, (cuuint64_t)g.sx * eb};
    cuuint32_t box[3] = {bx, by, 1};
    cuuint32_t estride[3] = {1, 1, 1};
    CUresult r = encode_fn()(map, eb == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                             3, const_cast<void *>(base), dims, strides, box, estride,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        throw CudaError("cuTensorMapEncodeTiled failed with code " + std::to_string((int)r));
}

}  // namespace

FieldMaps make_field_maps(const Grid &g, const void *base, int elem_bytes) {
    if (elem_bytes != 4 && elem_bytes != 8) throw std::invalid_argument("element size");
    if (((uintptr_t)base) % 16 != 0) throw std::invalid_argument("TMA base not 16-byte aligned");
    if ((g.sy * elem_bytes) % 16 != 0) throw std::invalid_argument("row pitch not 16-byte multiple");
    FieldMaps m;
    int h = 16 / elem_bytes;
    encode(&m.halo, g, base, elem_bytes, (cuuint32_t)(TK + 2 * h), (cuuint32_t)(TJ + 2));
    encode(&m.plain, g, base, elem_bytes, (cuuint32_t)TK, (cuuint32_t)TJ);
    encode(&m.wide, g, base, elem_bytes, (cuuint32_t)(TK + 2 * WIDE_HK), (cuuint32_t)(TJ + 2 * WIDE_HJ));
    return m;
}

}  // namespace dalm
