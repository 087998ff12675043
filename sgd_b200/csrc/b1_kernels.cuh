// B1 (bilinear box-spline) fan-beam footprint, evaluated identically by the
// forward, back and matrix kernels so that the pair is an exact transpose.
//
// All arithmetic is written with explicit round-to-nearest operations: the
// compiler may not contract or reorder it differently in different kernels,
// so conv(i, j, p, u) is bit-identical wherever it is computed.  The two edge
// offsets of a bin and the profile G at both run as pairs on the sm_100
// packed-FP32 instructions (__ffma2_rn, __fadd2_rn, __fmul2_rn): one
// instruction evaluates both edges, each half rounded exactly as the scalar
// operation would be.
#pragma once

#include <cuda_runtime.h>

namespace sgd {

// Footprint threshold of the reference (layers/A_B1.cu:203, :347).
constexpr float kConvEps = 1e-7f;

// One bin's 96-byte record (layout and constants in fan_geometry.h): six
// float4 whose halves are the operand pairs of the packed instructions.
struct B1Bin {
    float4 q0, q1, q2, q3, q4, q5;
    __device__ __forceinline__ float2 ci() const { return make_float2(q0.x, q0.y); }    // i coefficient (a, b)
    __device__ __forceinline__ float2 cj() const { return make_float2(q0.z, q0.w); }    // j coefficient (a, b)
    __device__ __forceinline__ float2 c0() const { return make_float2(q1.x, q1.y); }    // constant term (a, b)
    __device__ __forceinline__ float2 b() const { return make_float2(q1.z, q1.w); }
    __device__ __forceinline__ float2 apb() const { return make_float2(q2.x, q2.y); }
    __device__ __forceinline__ float2 a() const { return make_float2(q2.z, q2.w); }
    __device__ __forceinline__ float2 k2() const { return make_float2(q3.x, q3.y); }    // 1/(2a^2)
    __device__ __forceinline__ float2 k1() const { return make_float2(q3.z, q3.w); }    // 1/a
    __device__ __forceinline__ float2 nk3() const { return make_float2(q4.x, q4.y); }   // -b^2/(12a^2)
    __device__ __forceinline__ float2 k4() const { return make_float2(q4.z, q4.w); }    // 1/(12a^2b^2)
    __device__ __forceinline__ float2 nk5() const { return make_float2(q5.x, q5.y); }   // -1/(24a^2b^2)
    __device__ __forceinline__ float amb() const { return q5.z; }                        // a - b
};

__device__ __forceinline__ float2 pair(float v) { return make_float2(v, v); }

__device__ __forceinline__ float2 relu2(float2 v) { return make_float2(fmaxf(v.x, 0.f), fmaxf(v.y, 0.f)); }

// G(x) = sign(x) S(|x|) at both halves of x; S in closed form (fan_geometry.h):
//   S = |x| (1/a - |x|/(2a^2)) - b^2/(12a^2) + w^4/(12a^2b^2)   for |x| <= a - b
//   S = 1/2 - (p^4 - 2q^4 - 2w^4)/(24a^2b^2)                    otherwise
// with w = (b - |x|)+, p = (a + b - |x|)+, q = (a - |x|)+.
__device__ __forceinline__ float2 b1_G2(float2 x, const B1Bin& r) {
    const float2 ax = make_float2(fabsf(x.x), fabsf(x.y));
    const float2 nax = make_float2(-ax.x, -ax.y);
    const float2 w = relu2(__fadd2_rn(r.b(), nax));
    const float2 w2 = __fmul2_rn(w, w);
    const float2 w4 = __fmul2_rn(w2, w2);
    float2 sin_ = __ffma2_rn(ax, __ffma2_rn(nax, r.k2(), r.k1()), r.nk3());
    sin_ = __ffma2_rn(r.k4(), w4, sin_);
    const float2 p = relu2(__fadd2_rn(r.apb(), nax));
    const float2 q = relu2(__fadd2_rn(r.a(), nax));
    const float2 p2 = __fmul2_rn(p, p), q2 = __fmul2_rn(q, q);
    float2 t = __ffma2_rn(p2, p2, __fmul2_rn(w4, pair(-2.f)));  // p^4 - 2 w^4 (w4 * -2 is exact)
    t = __ffma2_rn(__fmul2_rn(pair(-2.f), q2), q2, t);
    const float2 sout = __ffma2_rn(r.nk5(), t, pair(0.5f));
    const float amb = r.amb();
    return make_float2(copysignf(ax.x <= amb ? sin_.x : sout.x, x.x), copysignf(ax.y <= amb ? sin_.y : sout.y, x.y));
}

// Edge offsets (xa, xb) of pixel (fi, fj): fi * ci + (fj * cj + c0), rounded
// in that order (the forward kernel hoists the bracket out of its loop).
__device__ __forceinline__ float2 b1_inner(float2 fj, const B1Bin& r) { return __ffma2_rn(fj, r.cj(), r.c0()); }
__device__ __forceinline__ float2 b1_edges(float2 fi, float2 inner, const B1Bin& r) {
    return __ffma2_rn(fi, r.ci(), inner);
}

// One MUFU reciprocal (|x| >= 2^-126 here: xb - xa is a bin width at the
// pixel, ~0.1..10 mm).
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// conv from the two edge offsets e = (xa, xb).
__device__ __forceinline__ float b1_conv_x(float2 e, const B1Bin& r) {
    const float2 g = b1_G2(e, r);
    return __fmul_rn(__fsub_rn(g.y, g.x), rcp_approx(__fsub_rn(e.y, e.x)));
}

// conv of layers/A_B1.cu:182-197 for pixel (fi, fj) given as float indices.
__device__ __forceinline__ float b1_conv(float fi, float fj, const B1Bin& r) {
    return b1_conv_x(b1_edges(pair(fi), b1_inner(pair(fj), r), r), r);
}

}  // namespace sgd
