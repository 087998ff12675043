// Bin ranges through a view's bin homography (fan_geometry.h: BinHomography),
// shared by the B1 kernels and the system-matrix builders.
#pragma once

#include <cuda_runtime.h>

namespace sgd {

__device__ __forceinline__ float hom_u(const float* h, float fi, float fj) {
    return __fdividef(fmaf(h[0], fi, fmaf(h[1], fj, h[2])), fmaf(h[3], fi, fmaf(h[4], fj, h[5])));
}

// Clamped bin range of the box [i0, i1] x [j0, j1] (pixel-index coordinates)
// under the view's homography: extremes of a linear-fractional map over a box
// are at its corners.
__device__ __forceinline__ void box_bins(const float* h, float i0, float i1, float j0, float j1, int nu, int& lo,
                                         int& hi) {
    const float u00 = hom_u(h, i0, j0), u01 = hom_u(h, i0, j1), u10 = hom_u(h, i1, j0), u11 = hom_u(h, i1, j1);
    lo = max(0, (int)floorf(fminf(fminf(u00, u01), fminf(u10, u11))));
    hi = min(nu - 1, (int)floorf(fmaxf(fmaxf(u00, u01), fmaxf(u10, u11))));
}

}  // namespace sgd
