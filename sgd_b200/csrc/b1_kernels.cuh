// B1 (bilinear box-spline) fan-beam footprint, evaluated identically by the
// forward and the back kernels so that the pair is an exact transpose.
//
// All arithmetic is written with explicit round-to-nearest intrinsics: the
// compiler may not contract or reorder it differently in the two kernels, so
// conv(i, j, p, u) is bit-identical wherever it is computed.
#pragma once

#include <cuda_runtime.h>

namespace sgd {

// Footprint threshold of the reference (layers/A_B1.cu:203, :347).
constexpr float kConvEps = 1e-7f;

// G(x) = sign(x) S(|x|), S a quartic on each of five intervals of |x|.
// `T(k)` returns table field k of the bin record (see fan_geometry.h).
template <class Tab>
__device__ __forceinline__ float b1_G(float x, float k1, float k2, float k3, float k4, const Tab& T) {
    const float ax = fabsf(x);
    const int r = (ax >= k1) + (ax >= k2) + (ax >= k3) + (ax >= k4);
    const int o = 10 + 6 * r;
    const float h = __fsub_rn(ax, T(o));
    float s = __fmaf_rn(h, T(o + 5), T(o + 4));
    s = __fmaf_rn(h, s, T(o + 3));
    s = __fmaf_rn(h, s, T(o + 2));
    s = __fmaf_rn(h, s, T(o + 1));
    return copysignf(s, x);
}

// conv of layers/A_B1.cu:182-197 for pixel (fi, fj) given as float indices.
// c[0..9] are the bin's affine edge offsets and interval ends.
template <class Tab>
__device__ __forceinline__ float b1_conv(float fi, float fj, const float* c, const Tab& T) {
    const float xa = __fmaf_rn(fi, c[0], __fmaf_rn(fj, c[1], c[2]));
    const float xb = __fmaf_rn(fi, c[3], __fmaf_rn(fj, c[4], c[5]));
    const float ga = b1_G(xa, c[6], c[7], c[8], c[9], T);
    const float gb = b1_G(xb, c[6], c[7], c[8], c[9], T);
    return __fdividef(__fsub_rn(gb, ga), __fsub_rn(xb, xa));
}

}  // namespace sgd
