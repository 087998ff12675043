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

// One bin's 64-byte record (layout in fan_geometry.h).
struct B1Bin {
    float4 q0, q1, q2, q3;
};

// G(x) = sign(x) S(|x|); S in closed form (fan_geometry.h).
__device__ __forceinline__ float b1_G(float x, const B1Bin& r) {
    const float a = r.q1.z, b = r.q1.w, apb = r.q2.x, amb = r.q2.y;
    const float c1 = r.q2.z, c2 = r.q2.w, c3 = r.q3.x, c4 = r.q3.y, c5 = r.q3.z;
    const float ax = fabsf(x);
    const float w = fmaxf(__fsub_rn(b, ax), 0.f);
    const float w2 = __fmul_rn(w, w);
    const float w4 = __fmul_rn(w2, w2);
    // inner: x/a - x^2/(2a^2) - b^2/(12a^2) + w^4/(12a^2b^2)
    float sin_ = __fmaf_rn(ax, __fmaf_rn(-ax, c2, c1), -c3);
    sin_ = __fmaf_rn(c4, w4, sin_);
    // outer: 1/2 - (p^4 - 2q^4 - 2w^4)/(24a^2b^2)
    const float p = fmaxf(__fsub_rn(apb, ax), 0.f);
    const float q = fmaxf(__fsub_rn(a, ax), 0.f);
    const float p2 = __fmul_rn(p, p), q2 = __fmul_rn(q, q);
    float t = __fmaf_rn(p2, p2, -__fadd_rn(w4, w4));
    t = __fmaf_rn(__fmul_rn(-2.f, q2), q2, t);
    const float sout = __fmaf_rn(-c5, t, 0.5f);
    return copysignf(ax <= amb ? sin_ : sout, x);
}

// Edge offsets of pixel (fi, fj): xa = fi*c0 + (fj*c1 + c2), rounded in that
// order (the forward kernel hoists the bracket out of its row loop).
__device__ __forceinline__ float b1_xa_inner(float fj, const B1Bin& r) { return __fmaf_rn(fj, r.q0.y, r.q0.z); }
__device__ __forceinline__ float b1_xb_inner(float fj, const B1Bin& r) { return __fmaf_rn(fj, r.q1.x, r.q1.y); }
__device__ __forceinline__ float b1_xa(float fi, float inner, const B1Bin& r) { return __fmaf_rn(fi, r.q0.x, inner); }
__device__ __forceinline__ float b1_xb(float fi, float inner, const B1Bin& r) { return __fmaf_rn(fi, r.q0.w, inner); }

// One MUFU reciprocal (|x| >= 2^-126 here: xb - xa is a bin width at the
// pixel, ~0.1..10 mm).
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// conv from the two edge offsets.
__device__ __forceinline__ float b1_conv_x(float xa, float xb, const B1Bin& r) {
    const float ga = b1_G(xa, r);
    const float gb = b1_G(xb, r);
    return __fmul_rn(__fsub_rn(gb, ga), rcp_approx(__fsub_rn(xb, xa)));
}

// conv of layers/A_B1.cu:182-197 for pixel (fi, fj) given as float indices.
__device__ __forceinline__ float b1_conv(float fi, float fj, const B1Bin& r) {
    return b1_conv_x(b1_xa(fi, b1_xa_inner(fj, r), r), b1_xb(fi, b1_xb_inner(fj, r), r), r);
}

}  // namespace sgd
