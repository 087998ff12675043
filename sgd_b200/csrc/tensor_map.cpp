#include "tensor_map.h"

#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "common.h"

namespace sgd {

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    if (!fn) fail("cuTensorMapEncodeTiled is not available from the CUDA driver");
    return fn;
}

}  // namespace

CUtensorMap encode_tensor_3d_f32(const float* base, uint64_t n0, uint64_t n1, uint64_t n2, uint32_t b0, uint32_t b1,
                                 uint32_t b2) {
    if (reinterpret_cast<uintptr_t>(base) % 16) fail("tensor map: base address not 16-byte aligned");
    if ((n0 * 4) % 16 || (b0 * 4) % 16) fail("tensor map: rows of %llu floats, boxes of %u: not whole 16-byte words",
                                             (unsigned long long)n0, b0);
    if (b0 > 256 || b1 > 256 || b2 > 256) fail("tensor map: box extents above 256");
    CUtensorMap map;
    const cuuint64_t dims[3] = {n0, n1, n2};
    const cuuint64_t strides[2] = {n0 * 4, n0 * n1 * 4};  // bytes, dimensions 1 and 2
    const cuuint32_t box[3] = {b0, b1, b2};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box,
                                 estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail("cuTensorMapEncodeTiled failed (%d)", (int)r);
    return map;
}

}  // namespace sgd
