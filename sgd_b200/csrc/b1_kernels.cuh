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
//                          on the record's constant pairs, which it stores
//                          duplicated so that no kernel builds a pair.  Each
//                          half of a packed operation rounds exactly as the
//                          scalar operation does, so the two forms give the
//                          same bits.
#pragma once

#include <cuda_runtime.h>

namespace sgd {

// Footprint threshold of the reference (layers/A_B1.cu:203, :347).
constexpr float kConvEps = 1e-7f;

// One bin's 64-byte record (layout in fan_geometry.h).
struct B1Bin {
    float4 q0, q1, q2, q3;
};

// G(y) = sign(y) S(|y|), y in units of the profile's half-width a (records in
// fan_geometry.h): S in closed form, the inner piece where 1 - |y| >= beta.
// The packed form (b1_G2) performs the same operations in the same order.
__device__ __forceinline__ float b1_G(float y, const B1Bin& r) {
    const float beta = r.q1.z, opb = r.q2.x, nk3 = r.q2.z, k4 = r.q3.x;
    const float ay = fabsf(y), nay = -ay;
    const float qr = __fadd_rn(1.f, nay);
    const float w = fmaxf(__fadd_rn(beta, nay), 0.f);
    const float w2 = __fmul_rn(w, w);
    const float w4 = __fmul_rn(w2, w2);
    // inner: y - y^2/2 - beta^2/12 + w^4/(12 beta^2)
    float sin_ = __fmaf_rn(ay, __fmaf_rn(nay, 0.5f, 1.f), nk3);
    sin_ = __fmaf_rn(k4, w4, sin_);
    // outer: 1/2 + (q^4 + w^4 - p^4/2)/(12 beta^2)
    const float p = fmaxf(__fadd_rn(opb, nay), 0.f);
    const float q = fmaxf(qr, 0.f);
    const float p2 = __fmul_rn(p, p), q2 = __fmul_rn(q, q);
    float t = __fmaf_rn(q2, q2, w4);
    t = __fmaf_rn(p2, __fmul_rn(p2, -0.5f), t);
    const float sout = __fmaf_rn(k4, t, 0.5f);
    return copysignf(qr >= beta ? sin_ : sout, y);
}

// Edge offsets of pixel (fi, fj): ya = fi*ci + (fj*cj + c0), rounded in that
// order (the forward kernel hoists the bracket out of its row loop).
__device__ __forceinline__ float b1_xa_inner(float fj, const B1Bin& r) { return __fmaf_rn(fj, r.q0.z, r.q1.x); }
__device__ __forceinline__ float b1_xb_inner(float fj, const B1Bin& r) { return __fmaf_rn(fj, r.q0.w, r.q1.y); }
__device__ __forceinline__ float b1_xa(float fi, float inner, const B1Bin& r) { return __fmaf_rn(fi, r.q0.x, inner); }
__device__ __forceinline__ float b1_xb(float fi, float inner, const B1Bin& r) { return __fmaf_rn(fi, r.q0.y, inner); }

// One MUFU reciprocal (|x| >= 2^-126 here: yb - ya is a bin width at the
// pixel over a, ~0.1..100).
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// conv from the two edge offsets (units of a): the difference quotient of G,
// scaled back to mm by 1/a.
__device__ __forceinline__ float b1_conv_x(float ya, float yb, const B1Bin& r) {
    const float ga = b1_G(ya, r);
    const float gb = b1_G(yb, r);
    return __fmul_rn(__fmul_rn(__fsub_rn(gb, ga), rcp_approx(__fsub_rn(yb, ya))), r.q3.z);
}

// conv of layers/A_B1.cu:182-197 for pixel (fi, fj) given as float indices.
__device__ __forceinline__ float b1_conv(float fi, float fj, const B1Bin& r) {
    return b1_conv_x(b1_xa(fi, b1_xa_inner(fj, r), r), b1_xb(fi, b1_xb_inner(fj, r), r), r);
}

__device__ __forceinline__ float2 pair(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 relu2(float2 v) { return make_float2(fmaxf(v.x, 0.f), fmaxf(v.y, 0.f)); }

// A bin's constants as operand pairs, taken from the record as they lie in it
// (no moves: each pair is the low or high half of a 16-byte chunk).
struct B1Pair {
    float2 ci, cj, c0;        // ya, yb = fi * ci + (fj * cj + c0)
    float2 beta, opb, nk3, k4;  // beta, 1 + beta, -beta^2/12, 1/(12 beta^2)
    float inv_a;              // 1/a
};

__device__ __forceinline__ B1Pair b1_pair(const B1Bin& r) {
    B1Pair k;
    k.ci = make_float2(r.q0.x, r.q0.y);
    k.cj = make_float2(r.q0.z, r.q0.w);
    k.c0 = make_float2(r.q1.x, r.q1.y);
    k.beta = make_float2(r.q1.z, r.q1.w);
    k.opb = make_float2(r.q2.x, r.q2.y);
    k.nk3 = make_float2(r.q2.z, r.q2.w);
    k.k4 = make_float2(r.q3.x, r.q3.y);
    k.inv_a = r.q3.z;
    return k;
}

// b1_G at both halves of y.
__device__ __forceinline__ float2 b1_G2(float2 y, const B1Pair& k) {
    const float2 ay = make_float2(fabsf(y.x), fabsf(y.y));
    const float2 nay = make_float2(-ay.x, -ay.y);
    const float2 qr = __fadd2_rn(pair(1.f), nay);
    const float2 w = relu2(__fadd2_rn(k.beta, nay));
    const float2 w2 = __fmul2_rn(w, w);
    const float2 w4 = __fmul2_rn(w2, w2);
    float2 sin_ = __ffma2_rn(ay, __ffma2_rn(nay, pair(0.5f), pair(1.f)), k.nk3);
    sin_ = __ffma2_rn(k.k4, w4, sin_);
    const float2 p = relu2(__fadd2_rn(k.opb, nay));
    const float2 q = relu2(qr);
    const float2 p2 = __fmul2_rn(p, p), q2 = __fmul2_rn(q, q);
    float2 t = __ffma2_rn(q2, q2, w4);
    t = __ffma2_rn(p2, __fmul2_rn(p2, pair(-0.5f)), t);
    const float2 sout = __ffma2_rn(k.k4, t, pair(0.5f));
    return make_float2(copysignf(qr.x >= k.beta.x ? sin_.x : sout.x, y.x),
                       copysignf(qr.y >= k.beta.y ? sin_.y : sout.y, y.y));
}

// (ya, yb) = fi * ci + inner, inner = fj * cj + c0: the scalar rounding order.
__device__ __forceinline__ float2 b1_inner2(float2 fj, const B1Pair& k) { return __ffma2_rn(fj, k.cj, k.c0); }
__device__ __forceinline__ float2 b1_edges2(float2 fi, float2 inner, const B1Pair& k) {
    return __ffma2_rn(fi, k.ci, inner);
}

// b1_conv_x on the edge pair e = (ya, yb).
__device__ __forceinline__ float b1_conv_pair(float2 e, const B1Pair& k) {
    const float2 g = b1_G2(e, k);
    return __fmul_rn(__fmul_rn(__fsub_rn(g.y, g.x), rcp_approx(__fsub_rn(e.y, e.x))), k.inv_a);
}

}  // namespace sgd
