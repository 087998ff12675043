// Parameters of the generic 2D fan-beam kernels (fan2d.cuh); plain C++ so that
// host-only translation units can hold them.
#pragma once

#include <cuda_runtime.h>

namespace sgd {

struct Fan2DParams {
    int ni = 0, nj = 0;       // cell grid: cell (i, j) at index i * nj + j
    int np = 0, nu = 0;
    const float* view = nullptr;     // [np][B::kViewFloats], 16-byte rows
    const float4* bins = nullptr;    // basis-specific per-(view, bin) table [np][B::kBinF4][nu] (planes), or null
    float* imgT = nullptr;           // [nj][ni] transposed copy of the image for i-major strips (forward scratch)
    double* part = nullptr;          // [kF2FwdParts][np][nu] the forward's partial sums (scratch)
    const float4* strips = nullptr;  // [np][nblk][2] forward block strips (fan2d.cuh)
    int nblk = 0;                    // bin blocks of kF2Block bins per view
    const int2* twin = nullptr;      // [tiles][np] back-projection tile bin windows
    int tiles_j = 0;                 // back tiles along j
    int wcap = 0;                    // widest back window (bins)
    int aux_i = 0;                   // basis-specific integer
    int* err = nullptr;              // device status word (bounded waits), 0 = ok
    unsigned wait_limit = 1u << 22;  // polls of the back kernel's staging wait before it gives up
    double* out64 = nullptr;         // when set, the kernels write their FP64 sums here instead of the FP32 output
};

// forward: one single-warp CTA per (view, block of kF2Block bins, part of
// the block's lines), kF2FwdParts parts
constexpr int kF2Block = 32, kF2FwdParts = 4;
// back: one CTA per kF2TileI x kF2TileJ cells (one per thread), views staged
// kF2Views at a time in a ring of fan2d_back_stages<B>() slots
constexpr int kF2TileI = 8, kF2TileJ = 32, kF2BackThreads = kF2TileI * kF2TileJ, kF2Views = 4;

// Ring slots of the back projection: four with no per-bin table, three with
// one (so that a basis with a two-word table keeps its CTAs per SM)
template <class B>
constexpr int fan2d_back_stages() {
    return B::kBinF4 == 0 ? 4 : 3;
}

}  // namespace sgd
