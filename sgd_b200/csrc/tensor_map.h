// Host encoding of TMA tensor maps (cuTensorMapEncodeTiled, reached through
// the runtime's driver entry point: no link against the driver library).
#pragma once

#include <cuda.h>

#include <cstdint>

namespace sgd {

// A 3D FP32 tensor of extents (n0, n1, n2), n0 contiguous, at `base`, read in
// boxes of (b0, b1, b2) elements; out-of-range elements read as zero.
// Requirements checked: base 16-byte aligned, n0 * 4 a multiple of 16,
// b0 * 4 a multiple of 16, every box extent <= 256.  Throws through fail().
CUtensorMap encode_tensor_3d_f32(const float* base, uint64_t n0, uint64_t n1, uint64_t n2, uint32_t b0, uint32_t b1,
                                 uint32_t b2);

}  // namespace sgd
