// The 3-direction box spline of the B0 and H0 footprints: the unit-area
// convolution of three boxes of widths |v1|, |v2|, |v3|, evaluated at y
// measured from the support's left end (layers/A_B0.cu:20-35 and
// layers/A_H0.cu:21-36 with layers/spline_conv.hh:239-293).  The reference
// sorts the widths, centres y and picks one of six quadratic pieces with a
// chain of branches and IEEE divisions by the widths' product; here the two
// reciprocals are fast (MUFU) reciprocals and the piece is chosen by selects
// (lanes of a warp sit on different pieces).  Each value is within a few units
// in the last place of the reference's; the bin ranges, which decide which
// pairs exist, are not computed here.
#pragma once

#include <cuda_runtime.h>

namespace sgd {

__device__ __forceinline__ void order_desc(float& a, float& b) {
    const float hi = fmaxf(a, b), lo = fminf(a, b);
    a = hi;
    b = lo;
}

__device__ __forceinline__ float box3(float y, float v1, float v2, float v3) {
    float x0 = fabsf(v1), x1 = fabsf(v2), x2 = fabsf(v3);
    const float yc = fabsf(y - (v1 + v2 + v3) * 0.5f);
    order_desc(x1, x2);
    order_desc(x0, x1);
    order_desc(x1, x2);
    if (!(x2 > 1e-7f)) {
        // two boxes (the third width vanished): a trapezoid
        const float h = __fdividef(1.0f, x0);
        const float r = __fdividef((x0 + x1) * 0.5f - yc, x0 * x1);
        return fmaxf(0.0f, fminf(h, r));
    }
    const float h = __fdividef(1.0f, x0);
    const float rp = __fdividef(1.0f, x0 * x1 * x2);
    const float K0 = (x0 - x1 - x2) * 0.5f, K1 = (x0 - x1 + x2) * 0.5f;
    const float K2 = (x0 + x1 - x2) * 0.5f, K3 = (x0 + x1 + x2) * 0.5f;
    const float a = K3 - yc, b = K0 - yc;
    const float p_top = 0.5f * a * a * rp;                      // K2 <= y < K3
    const float p_ramp = ((x0 + x1) * 0.5f - yc) * x2 * rp;     // K1 <= y < K2
    const float p_flat_in = h - __fmaf_rn(K0, K0, __fmul_rn(yc, yc)) * rp;  // y < -K0 (K0^2 + yc^2, one fixed contraction)
    const float p_shoulder = h - 0.5f * b * b * rp;             // K0 <= y < K1
    float v = yc < K0 ? h : p_shoulder;
    v = yc < -K0 ? p_flat_in : v;
    v = yc >= K1 ? p_ramp : v;
    v = yc >= K2 ? p_top : v;
    return yc >= K3 ? 0.0f : v;
}

}  // namespace sgd
