// Parameters of the generic 2D fan-beam kernels (fan2d.cuh); plain C++ so that
// host-only translation units can hold them.
#pragma once

#include <cuda_runtime.h>

namespace sgd {

struct Fan2DParams {
    int ni = 0, nj = 0;       // cell grid: cell (i, j) at index i * nj + j
    int np = 0, nu = 0;
    const float* view = nullptr;     // [np][B::kViewFloats]
    const float4* bins = nullptr;    // basis-specific per-(view, bin) table, or null
    const int2* wins = nullptr;      // [tiles][np] forward-tile bin windows
    int wcap = 0;                    // max window width (bins)
    int tiles_j = 0;                 // tiles along j
    int aux_i = 0;                   // basis-specific integer (e.g. hex row count)
};

constexpr int kF2TileI = 8, kF2TileJ = 32, kF2Threads = kF2TileI * kF2TileJ, kF2Views = 4;

}  // namespace sgd
