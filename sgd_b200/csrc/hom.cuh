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

// Bin range of the box [fi-1, fi+1] x [fj-1, fj+1] from its centre: with
// u = N / D linear-fractional, |u - u_c| <= (|n0 - u_c d0| + |n1 - u_c d1|) /
// (|D_c| - |d0| - |d1|) over the box (h[6] = |d0| + |d1|); a range at least as
// wide as the corners', from one division instead of four.  A box reaching
// the source plane gets every bin.
__device__ __forceinline__ void box_bins_bound(const float* h, float fi, float fj, int nu, int& lo, int& hi) {
    const float N = fmaf(h[0], fi, fmaf(h[1], fj, h[2]));
    const float D = fmaf(h[3], fi, fmaf(h[4], fj, h[5]));
    const float uc = __fdividef(N, D);
    const float spread = fabsf(fmaf(-uc, h[3], h[0])) + fabsf(fmaf(-uc, h[4], h[1]));
    const float dmin = fabsf(D) - h[6];
    const float w = dmin > 0.f ? __fdividef(spread, dmin) : 1e30f;
    lo = max(0, (int)floorf(uc - w));
    hi = min(nu - 1, (int)floorf(uc + w));
}

}  // namespace sgd
