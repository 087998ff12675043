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

namespace sgd {

// The 4-direction box spline of widths (-w, va, vb, vc) at y for lattice
// directions with va + vb + vc = 0 (the hexagonal lattice's, dt sin(theta +
// {0, 2pi/3, 4pi/3})), as the difference over the blur width w > 0 of the
// 3-direction spline's CDF: (F(y + w) - F(y)) / w (the truncated-power sign
// convention: support's left end at the sum of the negative widths).  The
// 3-direction spline's largest magnitude is the sum of the other two, x0 =
// x1 + x2, and its centre is 0, so F(y) = 1/2 + sgn(y) G(|y|) with the
// cumulative from the centre G(t) = h t - rp6 t^3 up to x2, GK2 - 3 rp6 x2
// (x1 - t)(x1 + x2 - t) up to x1, 1/2 - rp6 (x1 + x2 - t)^3 up to x1 + x2,
// 1/2 beyond (each piece written with distances to a nearby knot, so FP32
// keeps its accuracy).  Per bin: x1 >= x2 > 0, h = 1/(x1 + x2), rp6 = 1/(6
// (x1 + x2) x1 x2) and GK2 = 1/2 - rp6 x2^3.
__device__ __forceinline__ float box4_hex_by_cum(float y, float w, float x1, float x2, float h, float rp6,
                                                 float GK2) {
    const float K3 = x1 + x2, r3 = 3.0f * rp6 * x2;
    auto G = [&](float e) {
        const float t = fabsf(e);
        const float d3 = K3 - t, d2 = x1 - t;
        const float top = __fmaf_rn(-rp6 * d3 * d3, d3, 0.5f);
        const float ramp = __fmaf_rn(-r3 * d2, d3, GK2);
        const float inner = __fmaf_rn(h, t, -rp6 * t * t * t);
        float g = t > x2 ? ramp : inner;
        g = t >= x1 ? top : g;
        return copysignf(t >= K3 ? 0.5f : g, e);
    };
    return __fdividef(G(y + w) - G(y), w);
}

// The 2-direction box spline of signed widths p, q (a trapezoid of unit area
// on [sum of the negative widths, sum of the positive ones]): its CDF F2 at
// e0 and e1, both measured from the support's centre, as F2(e1) - F2(e0).
// G2(t) = t / x0 on the plateau t <= (x0 - x1)/2, 1/2 - (k1 - t)^2 / (2 x0
// x1) on the ramp up to k1 = (x0 + x1)/2, 1/2 beyond (x0 >= x1 the widths'
// magnitudes; a zero x1 leaves the box, whose ramp is empty).
__device__ __forceinline__ float box2_cum_diff(float e1, float e0, float p, float q) {
    const float x0 = fmaxf(fabsf(p), fabsf(q)), x1 = fminf(fabsf(p), fabsf(q));
    const float k0 = (x0 - x1) * 0.5f, k1 = (x0 + x1) * 0.5f;
    const float ih = __fdividef(1.0f, x0), ir = __fdividef(0.5f, x0 * x1);
    auto G = [&](float t) {
        const float d = k1 - t;
        const float g = t <= k0 ? t * ih : __fmaf_rn(-ir * d, d, 0.5f);
        return t >= k1 ? 0.5f : g;
    };
    return copysignf(G(fabsf(e1)), e1) - copysignf(G(fabsf(e0)), e0);
}

// x0 F2 - x0 / 2 at e (measured from the trapezoid's centre) for the
// trapezoid of magnitudes x0 >= x1: sgn(e) (min(|e|, k0) + x1 tau (1 - tau /
// 2)), tau = sat((|e| - k0) / x1) the covered fraction of the ramp, k0 = (x0 -
// x1) / 2, o = -k0 / x1.  On the plateau this is |e|; on the ramp it is k0 +
// x1 tau - x1 tau^2 / 2 = x0 / 2 - x1 (1 - tau)^2 / 2; beyond it x0 / 2.  All
// of it on the FMA pipe (saturated products, a minimum, a sign copy).  For x1
// = 0 (a box: 1/x1 infinite) tau is 0 or 1 (0 for the NaN at the knot) and
// the ramp term is 0.
__device__ __forceinline__ float trap_cum_scaled(float e, float k0, float x1, float rx1, float o) {
    const float t = fabsf(e);
    const float tau = __saturatef(__fmaf_rn(t, rx1, o));
    return copysignf(__fmaf_rn(x1 * tau, __fmaf_rn(-0.5f, tau, 1.0f), fminf(t, k0)), e);
}

// The 3-direction box spline of signed widths p, q, v at y (box3's
// convention) as the difference of the (p, q) trapezoid's CDF over v:
// (F2(y) - F2(y - v)) / v, with the trapezoid's 1/x0 and 1/x1 given (per-bin
// constants of a table; x0 >= x1 the widths' magnitudes).
__device__ __forceinline__ float box3_by_cum(float y, float p, float q, float v, float ih, float rx1) {
    const float x0 = fmaxf(fabsf(p), fabsf(q)), x1 = fminf(fabsf(p), fabsf(q));
    const float k0 = (x0 - x1) * 0.5f, c = (p + q) * 0.5f, o = -k0 * rx1;
    const float e1 = y - c, e0 = (y - v) - c;
    const float d = trap_cum_scaled(e1, k0, x1, rx1, o) - trap_cum_scaled(e0, k0, x1, rx1, o);
    return __fdividef(d * ih, v);
}

// The sum of the three 3-direction box splines (-w, va, vb), (-w, vb, vc),
// (-w, vc, va) at y (the H0 footprint, layers/A_H0.cu:21-36 with
// spline_conv.hh:244-293): each is the difference over the blur width w > 0
// of its pair's trapezoid CDF, (F2(y + w) - F2(y)) / w, so the three share one
// division.
__device__ __forceinline__ float box3_sum3_by_cum(float y, float w, float va, float vb, float vc) {
    const float cab = (va + vb) * 0.5f, cbc = (vb + vc) * 0.5f, cca = (vc + va) * 0.5f;
    const float d = box2_cum_diff((y + w) - cab, y - cab, va, vb) + box2_cum_diff((y + w) - cbc, y - cbc, vb, vc) +
                    box2_cum_diff((y + w) - cca, y - cca, vc, va);
    return __fdividef(d, w);
}

}  // namespace sgd
