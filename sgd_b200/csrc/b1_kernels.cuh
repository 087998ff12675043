// B1 (bilinear box-spline) fan-beam footprint, evaluated identically by the
// forward and the back kernels so that the pair is an exact transpose.
//
// All arithmetic is written with explicit round-to-nearest intrinsics: the
// compiler may not contract or reorder it differently in the two kernels, so
// conv(i, j, p, u) is bit-identical wherever it is computed.  Two forms:
//   scalar (b1_conv)       the two edges one after the other (the system-
//                          matrix builder);
//   packed (b1_conv_pair)  both edges at once on the sm_100 packed-FP32
//                          instructions (__ffma2_rn, __fadd2_rn, __fmul2_rn),
//                          on constant pairs built from the record (once per
//                          bin in the forward kernel, which reuses a bin for
//                          dozens of pixels; per evaluation in the back
//                          kernel, where the register moves still cost less
//                          than the scalar form).  Each half of a packed
//                          operation rounds exactly as the scalar operation
//                          does, so the two forms give the same bits.
#pragma once

#include <cuda_runtime.h>

namespace sgd {

// Footprint threshold of the reference (layers/A_B1.cu:203, :347).
constexpr float kConvEps = 1e-7f;

// One bin's 64-byte record (layout in fan_geometry.h).
struct B1Bin {
    float4 q0, q1, q2, q3;
};

// Derived constants, formed identically in both forms: a - b and
// -1/(24a^2b^2) = -0.5 * 1/(12a^2b^2) (exact).
__device__ __forceinline__ float b1_amb(const B1Bin& r) { return __fsub_rn(r.q2.x, r.q1.z); }

// G(x) = sign(x) S(|x|); S in closed form (fan_geometry.h).
__device__ __forceinline__ float b1_G(float x, const B1Bin& r) {
    const float b = r.q1.z, a = r.q2.x, apb = r.q2.z, amb = b1_amb(r);
    const float c1 = r.q3.x, c2 = r.q3.y, nc3 = r.q3.z, c4 = r.q3.w, nc5 = __fmul_rn(-0.5f, c4);
    const float ax = fabsf(x);
    const float w = fmaxf(__fsub_rn(b, ax), 0.f);
    const float w2 = __fmul_rn(w, w);
    const float w4 = __fmul_rn(w2, w2);
    // inner: x/a - x^2/(2a^2) - b^2/(12a^2) + w^4/(12a^2b^2)
    float sin_ = __fmaf_rn(ax, __fmaf_rn(-ax, c2, c1), nc3);
    sin_ = __fmaf_rn(c4, w4, sin_);
    // outer: 1/2 - (p^4 - 2q^4 - 2w^4)/(24a^2b^2)
    const float p = fmaxf(__fsub_rn(apb, ax), 0.f);
    const float q = fmaxf(__fsub_rn(a, ax), 0.f);
    const float p2 = __fmul_rn(p, p), q2 = __fmul_rn(q, q);
    float t = __fmaf_rn(p2, p2, __fmul_rn(w4, -2.f));  // -(w4 + w4) exactly
    t = __fmaf_rn(__fmul_rn(-2.f, q2), q2, t);
    const float sout = __fmaf_rn(nc5, t, 0.5f);
    return copysignf(ax <= amb ? sin_ : sout, x);
}

// Edge offsets of pixel (fi, fj): xa = fi*ci + (fj*cj + c0), rounded in that
// order (the forward kernel hoists the bracket out of its row loop).
__device__ __forceinline__ float b1_xa_inner(float fj, const B1Bin& r) { return __fmaf_rn(fj, r.q0.z, r.q1.x); }
__device__ __forceinline__ float b1_xb_inner(float fj, const B1Bin& r) { return __fmaf_rn(fj, r.q0.w, r.q1.y); }
__device__ __forceinline__ float b1_xa(float fi, float inner, const B1Bin& r) { return __fmaf_rn(fi, r.q0.x, inner); }
__device__ __forceinline__ float b1_xb(float fi, float inner, const B1Bin& r) { return __fmaf_rn(fi, r.q0.y, inner); }

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

__device__ __forceinline__ float2 pair(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 relu2(float2 v) { return make_float2(fmaxf(v.x, 0.f), fmaxf(v.y, 0.f)); }

// A bin's constants as operand pairs: (xa, xb) coefficients, and every
// profile constant duplicated.
struct B1Pair {
    float2 ci, cj, c0;                          // xa, xb = fi * ci + (fj * cj + c0)
    float2 b, apb, a, k2, k1, nk3, k4, nk5;     // b, a+b, a, 1/(2a^2), 1/a, -b^2/(12a^2), 1/(12a^2b^2), -1/(24a^2b^2)
    float amb;                                  // a - b
};

// The record's first three chunks are already operand pairs; the four
// single constants of the last are duplicated.
__device__ __forceinline__ B1Pair b1_pair(const B1Bin& r) {
    B1Pair k;
    k.ci = make_float2(r.q0.x, r.q0.y);
    k.cj = make_float2(r.q0.z, r.q0.w);
    k.c0 = make_float2(r.q1.x, r.q1.y);
    k.b = make_float2(r.q1.z, r.q1.w);
    k.a = make_float2(r.q2.x, r.q2.y);
    k.apb = make_float2(r.q2.z, r.q2.w);
    k.amb = b1_amb(r);
    k.k1 = pair(r.q3.x);
    k.k2 = pair(r.q3.y);
    k.nk3 = pair(r.q3.z);
    k.k4 = pair(r.q3.w);
    k.nk5 = __fmul2_rn(k.k4, pair(-0.5f));
    return k;
}

// b1_G at both halves of x.
__device__ __forceinline__ float2 b1_G2(float2 x, const B1Pair& k) {
    const float2 ax = make_float2(fabsf(x.x), fabsf(x.y));
    const float2 nax = make_float2(-ax.x, -ax.y);
    const float2 w = relu2(__fadd2_rn(k.b, nax));
    const float2 w2 = __fmul2_rn(w, w);
    const float2 w4 = __fmul2_rn(w2, w2);
    float2 sin_ = __ffma2_rn(ax, __ffma2_rn(nax, k.k2, k.k1), k.nk3);
    sin_ = __ffma2_rn(k.k4, w4, sin_);
    const float2 p = relu2(__fadd2_rn(k.apb, nax));
    const float2 q = relu2(__fadd2_rn(k.a, nax));
    const float2 p2 = __fmul2_rn(p, p), q2 = __fmul2_rn(q, q);
    float2 t = __ffma2_rn(p2, p2, __fmul2_rn(w4, pair(-2.f)));  // -(w4 + w4) exactly
    t = __ffma2_rn(__fmul2_rn(pair(-2.f), q2), q2, t);
    const float2 sout = __ffma2_rn(k.nk5, t, pair(0.5f));
    return make_float2(copysignf(ax.x <= k.amb ? sin_.x : sout.x, x.x),
                       copysignf(ax.y <= k.amb ? sin_.y : sout.y, x.y));
}

// (xa, xb) = fi * ci + inner, inner = fj * cj + c0: the scalar rounding order.
__device__ __forceinline__ float2 b1_inner2(float2 fj, const B1Pair& k) { return __ffma2_rn(fj, k.cj, k.c0); }
__device__ __forceinline__ float2 b1_edges2(float2 fi, float2 inner, const B1Pair& k) {
    return __ffma2_rn(fi, k.ci, inner);
}

// b1_conv_x on the edge pair e = (xa, xb).
__device__ __forceinline__ float b1_conv_pair(float2 e, const B1Pair& k) {
    const float2 g = b1_G2(e, k);
    return __fmul_rn(__fsub_rn(g.y, g.x), rcp_approx(__fsub_rn(e.y, e.x)));
}

}  // namespace sgd
