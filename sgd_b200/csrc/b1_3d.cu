// A_B1_3D: bilinear (in-plane) x separable-footprint (axial) cone-beam
// projector.  Reference: layers/A_B1_3D.cu:22-66 (gamma), :68-80 (footprint),
// :82-312 (forward), :314-531 (backward), :686-773 (C entry points).
//
// Per voxel (ix, iy, iz) and view: the in-plane B1 footprint conv(u) of the
// column (ix, iy) over the bins u of its +-1 voxel support (the reference's
// FP32 formula, its FP32 bin stepping included), times the integral g(v)
// of the axial trapezoid (corners ix +- 1 at iy, iz +- 1/2 through pmi) over
// bin row v, times vol * dx dy dz * sqrt(r3^2 / r2^2).  The reference's
// forward also multiplies by 2 / (trapezoid width) (:210), its backward does
// not (:436), and the backward skips single-bin u or v ranges (:404, :433):
//   mode 0 "reference": both kernels as the reference (parity);
//   mode 1 "adjoint":   the forward as the reference and the back projector its
//                       exact transpose (dot-product test, autograd).
//
// conv(u) does not depend on z and g(v) does not depend on u, so per view and
// column the projection factors through the column's axial profile:
//   forward   proj(u, v) += conv(u) A(v),  A(v) = sum_z C(z) w(z) g(z, v)
//   back      vol(z) += w(z) sum_v g(z, v) B(v),  B(v) = sum_u conv(u) proj(u, v)
// (w the reference's amplitude), evaluated by
//   b1_3d_fwd_kernel   a CTA per (view, block of 16 u bins).  Its columns are
//                      the block's in-plane strip (the 2D kernels' plan, B1
//                      support); a warp takes one column at a time, its lanes
//                      the column's voxels (z contiguous in a transposed copy
//                      of the volume, one reference z chunk of 32 per pass),
//                      and builds A in shared memory; after each batch of one
//                      column per warp the threads, each owning detector
//                      rows, add conv(u) A(v) into the block's FP64
//                      accumulators.  Every bin is written once: no atomics
//                      in global memory.
//   b1_3d_back_kernel  a CTA per 4 x 2 columns (a warp each) and 256 voxels
//                      of z (a lane each owns 8, FP64 accumulators in
//                      registers).  Per view the CTA's window of 16 u bins
//                      x all v rows is staged by a TMA tensor load (double
//                      buffered on mbarriers with bounded waits); each warp
//                      forms B of its column from it and each lane its
//                      voxels' sums.  Every voxel is written once.
// The reference's z chunks of 32 are kept: the FP32 stepping oz += dz from a
// chunk's start, and its `return` at the first voxel whose trapezoid starts
// beyond the detector top, which ends the rest of that chunk (a warp ballot
// here).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.h"
#include "cone_columns.cuh"
#include "fan_geometry.h"
#include "proj2d.h"
#include "tensor_map.h"
#include "tma.cuh"

namespace sgd {

namespace {

constexpr int kZChunk = 32;      // the reference's Z_SIZE (layers/A_B1_3D.cu:25)
constexpr float kEps = 1e-7f;
constexpr int kUB = 16;          // forward: u bins per block
constexpr int kFW = 8;           // forward: warps, columns per batch
constexpr int kMaxLines = 2048;  // forward: strip lines held in shared memory
constexpr int kTX = 4, kTY = 2;  // back: columns per CTA (a warp each)
constexpr int kWin = 20;         // back: staged u window (bins); rows of 80 bytes keep float4 row reads free of bank conflicts
constexpr int kRowBox = 192;     // back: rows per TMA box
constexpr int kZPer = 8;         // back: voxels per lane (z = l + 32 k)
constexpr uint32_t kDrainLimit = 1u << 22;  // back: polls of the drain after a failed wait

struct View3 {
    float pm[12];
    float puvx, puvy, srcx, srcy, srcz, dtvx, dtvy, singular;
};

__device__ __forceinline__ void load_view3(const float* g, View3& V) {
    const float4* q = reinterpret_cast<const float4*>(g);
    float t[20];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const float4 a = __ldg(q + k);
        t[4 * k] = a.x; t[4 * k + 1] = a.y; t[4 * k + 2] = a.z; t[4 * k + 3] = a.w;
    }
#pragma unroll
    for (int k = 0; k < 12; ++k) V.pm[k] = t[k];
    V.puvx = t[12]; V.puvy = t[13]; V.srcx = t[14]; V.srcy = t[15]; V.srcz = t[16];
    V.dtvx = t[17]; V.dtvy = t[18]; V.singular = t[19];
}

__device__ __forceinline__ void sort4(float* a) {
    auto s2 = [](float& x, float& y) {
        if (x > y) {
            const float t = y;
            y = x;
            x = t;
        }
    };
    s2(a[0], a[1]);
    s2(a[2], a[3]);
    s2(a[0], a[2]);
    s2(a[1], a[3]);
    s2(a[1], a[2]);
}

// layers/spline_conv.hh:295-405 (T = float), the reference's FP32 forms
__device__ float conv_ag2b(float a, float b, float x) {
    float a3 = a * a * a, ab2 = a * b * b, b3 = b * b * b;
    float k1 = (6 * a * a * b * b);
    float sum = 0.0f;
    if (x <= b) return (x * (12 * ab2 - 4 * b3 - 4 * b * x * x + x * x * x)) / (2 * k1);
    sum += ((12 * a - 7 * b) * b) / (12 * a * a);
    if (x <= a - b) return sum + (-2 * a * b + b * b + 2 * a * x - x * x) / (2 * a * a);
    sum += 0.5f - b / a;
    if (x <= a)
        return sum + ((a - b - x) * (a3 - 13 * b3 + 9 * b * b * x - 3 * b * x * x - x * x * x - 3 * a * a * (b + x) -
                                     3 * a * (b - x) * (3 * b + x))) / (4 * k1);
    sum += (13 * b * b) / (24 * a * a);
    if (x < a + b)
        return sum + ((x - a) * (a + 2 * b - x) * (a * a + 2 * a * b + 2 * b * b - 2 * (a + b) * x + x * x)) / (4 * k1);
    return sum + b * b / (24 * a * a);
}
__device__ float conv_al2b(float a, float b, float x) {
    float a3 = a * a * a, a2b = a * a * b, ab2 = a * b * b, b3 = b * b * b;
    float k1 = (6 * a * a * b * b), k2 = a - b;
    float sum = 0.0f;
    if (x <= a - b) return (x * (12 * ab2 - 4 * b3 - 4 * b * x * x + x * x * x)) / (2 * k1);
    sum += ((a - b) * (a3 - 7 * a2b + 23 * ab2 - 9 * b3)) / (2 * k1);
    if (x <= b)
        return sum + (((x - a + b) * (a3 - 11 * a2b + 43 * ab2 - 17 * b3 + (5 * a - 13 * b) * k2 * x - (a + 7 * b) * x * x +
                                      3 * x * x * x)) / (4 * k1));
    sum += (((2 * b - a) * (a3 - 6 * a2b + 24 * ab2 - 8 * b3)) / (4 * k1));
    if (x <= a)
        return sum + (((b - x) * (4 * a3 - 3 * b3 + b * b * x - 5 * b * x * x - x * x * x - 6 * a * a * (3 * b + x) +
                                  4 * a * (b * b + 4 * b * x + x * x))) / (4 * k1));
    sum += (((b - a) * (a3 - 7 * a2b + 5 * ab2 - 3 * b3)) / (4 * k1));
    if (x < a + b)
        return sum + ((x - a) * (a + 2 * b - x) * (a * a + 2 * a * b + 2 * b * b - 2 * (a + b) * x + x * x)) / (4 * k1);
    return sum + b * b / (24 * a * a);
}
__device__ float lc1d(float x1, float x2, float a, float b) {  // layers/A_B1_3D.cu:68-80
    const bool side = (x1 * x2) > 0;
    const float y1 = fabsf(x1), y2 = fabsf(x2);
    float s1, s2;
    if (b > 1e-7f) {
        if (b <= a - b) {
            s1 = conv_ag2b(a, b, y1);
            s2 = conv_ag2b(a, b, y2);
        } else {
            s1 = conv_al2b(a, b, y1);
            s2 = conv_al2b(a, b, y2);
        }
    } else {
        s1 = (y1 >= a) ? 0.5f : (y1 / a - (y1 * y1) / (2 * a * a));
        s2 = (y2 >= a) ? 0.5f : (y2 / a - (y2 * y2) / (2 * a * a));
    }
    return (side ? fabsf(s1 - s2) : (s1 + s2)) / fabsf(x2 - x1);
}

struct Column {
    float ox, oy, v1, v2, v3, v4;
    int minu, maxu;
};

// layers/A_B1_3D.cu:120-176 (the column part, independent of z)
__device__ __forceinline__ void column_setup(const View3& V, int ix, int iy, int nx, int ny, int nu, float dx,
                                             float dy, Column& c) {
    const float* pm = V.pm;
    c.ox = (ix - 0.5f * (nx - 1)) * dx;
    c.oy = (iy - 0.5f * (ny - 1)) * dy;
    const float signy1 = iy - 1.0f, signy2 = iy + 1.0f, signx1 = ix - 1.0f, signx2 = ix + 1.0f;
    const float u1 = pm[0] * signx1 + pm[1] * signy1 + pm[3];
    const float u2 = pm[8] * signx1 + pm[9] * signy1 + pm[11];
    const float u3 = pm[0] * signx2 + pm[1] * signy1 + pm[3];
    const float u4 = pm[8] * signx2 + pm[9] * signy1 + pm[11];
    const float u5 = pm[0] * signx1 + pm[1] * signy2 + pm[3];
    const float u6 = pm[8] * signx1 + pm[9] * signy2 + pm[11];
    const float u7 = pm[0] * signx2 + pm[1] * signy2 + pm[3];
    const float u8 = pm[8] * signx2 + pm[9] * signy2 + pm[11];
    c.v1 = pm[4] * signx1 + pm[5] * iy + pm[7];
    c.v2 = pm[4] * signx2 + pm[5] * iy + pm[7];
    c.v3 = pm[8] * signx1 + pm[9] * iy + pm[11];
    c.v4 = pm[8] * signx2 + pm[9] * iy + pm[11];
    float us[4];
    if (V.singular == 0.f) {
        us[0] = (u1) / (u2);
        us[1] = (u3) / (u4);
        us[2] = (u5) / (u6);
        us[3] = (u7) / (u8);
    } else {
        us[0] = ((u1) / (u2) * 1.5f - 1.0f) / V.puvx;
        us[1] = ((u3) / (u4) * 1.5f - 1.0f) / V.puvx;
        us[2] = ((u5) / (u6) * 1.5f - 1.0f) / V.puvx;
        us[3] = ((u7) / (u8) * 1.5f - 1.0f) / V.puvx;
    }
    sort4(us);
    c.minu = min(max(0, (int)floorf(us[0])), nu - 1);
    c.maxu = min(max(0, (int)floorf(us[3])), nu - 1);
}

// in-plane footprint of bin minu + ti of the column (layers/A_B1_3D.cu:252-278):
// the FP32 bin centre is stepped from minu as the reference steps it
__device__ __forceinline__ float column_conv_at(const View3& V, const Column& c, const float2* __restrict__ vecs,
                                                int nu, int ti) {
    const float px = V.srcx, py = V.srcy, ox = c.ox, oy = c.oy;
    float sx = V.dtvx + V.puvx * (c.minu - 0.5f * nu + 0.5f);
    float sy = V.dtvy + V.puvy * (c.minu - 0.5f * nu + 0.5f);
    for (int k = 0; k < ti; ++k) {
        sx += V.puvx;
        sy += V.puvy;
    }
    const float2 v = __ldg(vecs + c.minu + ti);
    const float ax = sx - V.puvx * 0.5f, ay = sy - V.puvy * 0.5f;
    const float bx = sx + V.puvx * 0.5f, by = sy + V.puvy * 0.5f;
    const float ra = ((ox - px) * (sx - px) + (oy - py) * (sy - py)) / ((ax - px) * (sx - px) + (ay - py) * (sy - py));
    const float rb = ((ox - px) * (sx - px) + (oy - py) * (sy - py)) / ((bx - px) * (sx - px) + (by - py) * (sy - py));
    const float ax1 = px + (ax - px) * ra, ay1 = py + (ay - py) * ra;
    const float bx1 = px + (bx - px) * rb, by1 = py + (by - py) * rb;
    const float x1 = sqrtf((ax1 - ox) * (ax1 - ox) + (ay1 - oy) * (ay1 - oy));
    const float x2 = sqrtf((bx1 - ox) * (bx1 - ox) + (by1 - oy) * (by1 - oy));
    const float sgn = ((ax1 - ox) * (bx1 - ox) + (ay1 - oy) * (by1 - oy) > 0) ? 1.0f : -1.0f;
    return lc1d(x1 * sgn, x2, fmaxf(v.x, v.y), fminf(v.x, v.y));
}

// axial trapezoid of voxel iz (layers/A_B1_3D.cu:188-205); false: beyond the
// detector top (the reference returns for the rest of its chunk)
__device__ __forceinline__ bool voxel_v(const View3& V, const Column& c, int iz, int nv, float* vs, int& minv,
                                        int& maxv) {
    const float* pm = V.pm;
    const float signz1 = (iz - 0.5f), signz2 = (iz + 0.5f);
    if (V.singular == 0.f) {
        vs[0] = (c.v1 + pm[6] * signz1) / (c.v3 + pm[10] * signz1);
        vs[1] = (c.v1 + pm[6] * signz2) / (c.v3 + pm[10] * signz2);
        vs[2] = (c.v2 + pm[6] * signz1) / (c.v4 + pm[10] * signz1);
        vs[3] = (c.v2 + pm[6] * signz2) / (c.v4 + pm[10] * signz2);
    } else {
        vs[0] = ((c.v1 + pm[6] * signz1) / (c.v3 + pm[10] * signz1) * 1.5f - 1.0f) / V.puvy;
        vs[1] = ((c.v1 + pm[6] * signz2) / (c.v3 + pm[10] * signz2) * 1.5f - 1.0f) / V.puvy;
        vs[2] = ((c.v2 + pm[6] * signz1) / (c.v4 + pm[10] * signz1) * 1.5f - 1.0f) / V.puvy;
        vs[3] = ((c.v2 + pm[6] * signz2) / (c.v4 + pm[10] * signz2) * 1.5f - 1.0f) / V.puvy;
    }
    sort4(vs);
    if (vs[0] >= nv) return false;
    minv = min(max(0, (int)floorf(vs[0])), nv - 1);
    maxv = min(max(0, (int)floorf(vs[3])), nv - 1);
    return true;
}


struct Geo3 {
    int nx, ny, nz, np, nu, nv;
    float dx, dy, dz;
    const float* view;    // [np][20]
    const float2* vecs;   // [np][nu]
};

// Launch tables of the new kernels.
struct Plan3 {
    const float4* strips;  // [np][nblk][2]: forward block strips (fan2d.cuh record)
    int nblk;
    const int* twin;       // [tiles][np]: back window's first bin (a multiple of 4), -1: read global memory
    int tiles_x, tiles_y;
    int* err;              // bounded-wait status, 0 = ok
    unsigned wait_limit;   // polls of one staged view before the back projection gives up
};

// Axial footprint of voxel iz of column c (layers/A_B1_3D.cu:188-210): the
// trapezoid vs[0..3] in v, its first and last rows, the reference's axial
// normalisation 2 / width and the ramp factors of its row integrals (fast
// reciprocals: within an ulp or two of the reference's divisions).  Returns
// false when the trapezoid starts beyond the detector top.
struct Axial {
    float vs[4];
    float k01, k23, width2;
    int minv, maxv;
};

__device__ __forceinline__ bool axial(const View3& V, const Column& c, int iz, int nv, Axial& a) {
    const float* pm = V.pm;
    const float signz1 = (iz - 0.5f), signz2 = (iz + 0.5f);
    float* vs = a.vs;
    vs[0] = __fdividef(c.v1 + pm[6] * signz1, c.v3 + pm[10] * signz1);
    vs[1] = __fdividef(c.v1 + pm[6] * signz2, c.v3 + pm[10] * signz2);
    vs[2] = __fdividef(c.v2 + pm[6] * signz1, c.v4 + pm[10] * signz1);
    vs[3] = __fdividef(c.v2 + pm[6] * signz2, c.v4 + pm[10] * signz2);
    if (V.singular != 0.f) {
        const float r = __fdividef(1.0f, V.puvy);
#pragma unroll
        for (int k = 0; k < 4; ++k) vs[k] = (vs[k] * 1.5f - 1.0f) * r;
    }
    sort4(vs);
    if (!(vs[0] < (float)nv)) return false;
    a.minv = min(max(0, (int)floorf(vs[0])), nv - 1);
    a.maxv = min(max(0, (int)floorf(vs[3])), nv - 1);
    // a zero-width ramp contributes nothing (the reference drops its NaN)
    a.k01 = vs[1] > vs[0] ? __fdividef(0.5f, vs[1] - vs[0]) : 0.f;
    a.k23 = vs[3] > vs[2] ? __fdividef(0.5f, vs[3] - vs[2]) : 0.f;
    a.width2 = __fdividef(2.0f, (vs[3] - vs[0]) + (vs[2] - vs[1]));
    return true;
}

// Cumulative of the axial trapezoid up to s: each of its three pieces'
// integral over a row [j, j + 1] (layers/A_B1_3D.cu:30-66) is the difference
// of the piece's terms at the row's ends clamped into the piece, so a row's
// share is axial_cdf(j + 1) - axial_cdf(j), one evaluation per row boundary.
// The clamped distances are exact (Sterbenz); written with round-to-nearest
// intrinsics so that the forward and back kernels form the same bits.
__device__ __forceinline__ float axial_cdf(const Axial& a, float s) {
    const float* u = a.vs;
    const float c01 = __fsub_rn(fminf(fmaxf(s, u[0]), u[1]), u[0]);
    const float c12 = __fsub_rn(fminf(fmaxf(s, u[1]), u[2]), u[1]);
    const float d23 = __fsub_rn(u[3], fminf(fmaxf(s, u[2]), u[3]));
    const float g = __fmaf_rn(__fmul_rn(a.k01, c01), c01, c12);
    return __fmaf_rn(-__fmul_rn(a.k23, d23), d23, g);
}

// The reference's amplitude sqrt(r3^2 / r2^2) of a voxel at height oz.
__device__ __forceinline__ float amplitude(float ir2, float dzz) { return sqrtf(fmaf(dzz * dzz, ir2, 1.0f)); }

// Lane l's voxel of a 32-voxel pass is live unless it or an earlier voxel of
// its reference chunk started beyond the detector top (the reference's
// `return`, layers/A_B1_3D.cu:202): `beyond` is the pass's ballot.
__device__ __forceinline__ bool chunk_live(unsigned beyond, int l) { return (beyond & ((2u << l) - 1u)) == 0u; }

// oz of voxel iz: the reference steps it by dz from its 32-voxel chunk's start.
__device__ __forceinline__ float chunk_oz(int iz, int nz, float dz) {
    const int z0 = iz & ~(kZChunk - 1);
    float oz = (z0 - 0.5f * (nz - 1)) * dz;
    for (int q = z0; q < iz; ++q) oz += dz;
    return oz;
}

__host__ __device__ constexpr size_t fwd3_smem(int nv, int nz) {
    return (size_t)kUB * nv * 8 + (size_t)kFW * nv * 4 + kFW * kUB * 4 + (kMaxLines + 1) * 4 + (size_t)nz * 4;
}

__global__ void __launch_bounds__(kFW * 32, 3) b1_3d_fwd_kernel(Geo3 G, Plan3 K, const float* __restrict__ volT,
                                                             float* __restrict__ proj, float scale) {
    extern __shared__ __align__(16) unsigned char f3_smem[];
    const int nv = G.nv, nz = G.nz;
    double* acc = reinterpret_cast<double*>(f3_smem);   // [kUB][nv]
    float* A = reinterpret_cast<float*>(acc + kUB * nv);  // [kFW][nv]: each warp's column profile
    float* cs = A + kFW * nv;                             // [kFW][kUB]: its conv per block bin
    int* pref = reinterpret_cast<int*>(cs + kFW * kUB);   // [kMaxLines + 1]: candidates before each line
    float* soz = reinterpret_cast<float*>(pref + kMaxLines + 1);  // [nz]
    __shared__ int s_act[kFW][2];
    const int k = blockIdx.x, p = blockIdx.y, tid = threadIdx.x, w = tid >> 5, l = tid & 31;
    const int u0 = k * kUB, nb = min(kUB, G.nu - u0);

    for (int e = tid; e < kUB * nv; e += blockDim.x) acc[e] = 0.0;
    for (int z = tid; z < nz; z += blockDim.x) soz[z] = chunk_oz(z, nz, G.dz);
    const float4* st = K.strips + ((size_t)p * K.nblk + k) * 2;
    const float4 s0 = __ldg(st), s1 = __ldg(st + 1);
    const bool jmaj = s0.x > 0.5f;
    const int nmin = jmaj ? G.nx : G.ny;
    const int mlo = (int)s1.z, nlines = (int)s1.w - mlo + 1;
    auto span = [&](int m, int& nlo, int& nhi) {
        const float fm = (float)m;
        const float na = fmaf(s0.z, fm, s0.y), nbb = fmaf(s1.x, fm, s0.w);
        nlo = max(0, (int)ceilf(fminf(na, nbb) - s1.y));
        nhi = min(nmin - 1, (int)floorf(fmaxf(na, nbb) + s1.y));
    };
    // candidates per line, then their running sum (warp 0)
    for (int t = tid; t < nlines; t += blockDim.x) {
        int a, b;
        span(mlo + t, a, b);
        pref[t + 1] = max(0, b - a + 1);
    }
    __syncthreads();
    if (w == 0) {
        int carry = 0;
        if (l == 0) pref[0] = 0;
        for (int t0 = 0; t0 < nlines; t0 += 32) {
            int v = t0 + l < nlines ? pref[t0 + l + 1] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int n = __shfl_up_sync(0xffffffffu, v, o);
                if (l >= o) v += n;
            }
            if (t0 + l < nlines) pref[t0 + l + 1] = v + carry;
            carry += __shfl_sync(0xffffffffu, v, 31);
        }
    }
    __syncthreads();
    const int total = nlines > 0 ? pref[nlines] : 0;

    View3 V;
    load_view3(G.view + (size_t)p * 20, V);
    const float2* vecs = G.vecs + (size_t)p * G.nu;
    float* Aw = A + w * nv;
    for (int base = 0; base < total; base += kFW) {
        const int idx = base + w;
        int blo = 1, bhi = 0;
        if (idx < total) {
            int lo = 0, hi = nlines;  // pref[lo] <= idx < pref[hi]
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (pref[mid] <= idx) lo = mid;
                else hi = mid;
            }
            int nlo, nhi;
            span(mlo + lo, nlo, nhi);
            const int n = nlo + (idx - pref[lo]), m = mlo + lo;
            const int ix = jmaj ? n : m, iy = jmaj ? m : n;
            Column c;
            column_setup(V, ix, iy, G.nx, G.ny, G.nu, G.dx, G.dy, c);
            const int tlo = max(c.minu, u0), thi = min(c.maxu, u0 + nb - 1);
            if (tlo <= thi) {
                blo = tlo - u0;
                bhi = thi - u0;
                // the column's footprint in each of its block bins, a lane each
                if (l < kUB) {
                    float cv = 0.f;
                    if (l >= blo && l <= bhi) {
                        cv = column_conv_at(V, c, vecs, G.nu, u0 + l - c.minu);
                        if (!(cv == cv)) cv = 0.f;  // the reference skips a NaN product (:283)
                    }
                    cs[w * kUB + l] = cv;
                }
                for (int v = l; v < nv; v += 32) Aw[v] = 0.f;
                __syncwarp();
                const float px = V.srcx, py = V.srcy, pz = V.srcz;
                const float ir2 = __fdividef(1.0f, (c.ox - px) * (c.ox - px) + (c.oy - py) * (c.oy - py));
                const float* colv = volT + ((size_t)iy * G.nx + ix) * nz;
                for (int z0 = 0; z0 < nz; z0 += 32) {
                    const int iz = z0 + l;
                    Axial a;
                    const bool in = iz < nz;
                    const bool ok = in && axial(V, c, iz, nv, a);
                    const unsigned beyond = __ballot_sync(0xffffffffu, in && !ok);
                    if (!ok || !chunk_live(beyond, l)) continue;
                    const float C0 = __ldg(colv + iz);
                    if (C0 == 0.f) continue;
                    const float C = C0 * amplitude(ir2, soz[iz] - pz) * a.width2;
                    if (!(C == C)) continue;
                    float gp = axial_cdf(a, (float)a.minv);
                    for (int j = a.minv; j <= a.maxv; ++j) {
                        const float gn = axial_cdf(a, (float)(j + 1));
                        const float g = __fsub_rn(gn, gp);
                        gp = gn;
                        if (g > kEps) atomicAdd(Aw + j, C * g);
                    }
                }
            }
        }
        if (l == 0) {
            s_act[w][0] = blo;
            s_act[w][1] = bhi;
        }
        __syncthreads();  // every warp's A and conv of this batch
        for (int v = tid; v < nv; v += blockDim.x) {
#pragma unroll 1
            for (int q = 0; q < kFW; ++q) {
                const int b0 = s_act[q][0], b1 = s_act[q][1];
                if (b1 < b0) continue;
                const float av = A[q * nv + v];
                if (av == 0.f) continue;
                for (int b = b0; b <= b1; ++b) {
                    const float cv = cs[q * kUB + b];
                    if (cv != 0.f) acc[b * nv + v] = fma((double)cv, (double)av, acc[b * nv + v]);
                }
            }
        }
        __syncthreads();  // before the warps overwrite A
    }
    for (int e = tid; e < nb * nv; e += blockDim.x) {
        const int v = e / nb, b = e - v * nb;
        proj[((size_t)p * nv + v) * G.nu + u0 + b] = (float)acc[b * nv + v] * scale;
    }
}

__host__ __device__ constexpr int rows_padded(int nv) { return (nv + kRowBox - 1) / kRowBox * kRowBox; }

// 128 bytes of slack: the staging buffer is placed on a 128-byte boundary
__host__ __device__ constexpr size_t back3_smem(int nv) {
    return 128 + (size_t)2 * rows_padded(nv) * kWin * 4 + (size_t)kTX * kTY * nv * 4 + 16;
}

// mode 0: the reference's backward (no 2/width factor, conv > 1e-7 kept,
// single-bin u or v ranges skipped); mode 1: the exact transpose of the
// forward.  use_tma: the projection is staged through `map` (a tensor map of
// proj, extents (nu, nv, np)); otherwise read from global memory.
__global__ void __launch_bounds__(kTX * kTY * 32, 3) b1_3d_back_kernel(const __grid_constant__ CUtensorMap map,
                                                                    Geo3 G, Plan3 K, const float* __restrict__ proj,
                                                                    float* __restrict__ vol, int mode, int use_tma) {
    extern __shared__ __align__(128) unsigned char b3_smem[];
    const int nv = G.nv, nvp = rows_padded(nv), nboxes = nvp / kRowBox;
    // [2][nvp][kWin], every TMA box (kRowBox rows of kWin floats, 12 KB) on a
    // 128-byte boundary
    float* stage = reinterpret_cast<float*>(b3_smem + ((128 - (smem_addr(b3_smem) & 127u)) & 127u));
    float* Bs = stage + (size_t)2 * nvp * kWin;                 // [warps][nv]
    uint64_t* bars = reinterpret_cast<uint64_t*>(Bs + kTX * kTY * nv);
    __shared__ int s_abort;
    const int tid = threadIdx.x, w = tid >> 5, l = tid & 31;
    const int tile = blockIdx.y * K.tiles_x + blockIdx.x;
    const int ix = blockIdx.x * kTX + (w % kTX), iy = blockIdx.y * kTY + (w / kTX);
    const bool col_ok = ix < G.nx && iy < G.ny;
    const int zbase = blockIdx.z * 32 * kZPer;
    const int* twin = K.twin + (size_t)tile * G.np;
    float* Bw = Bs + w * nv;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
        s_abort = 0;
    }
    __syncthreads();
    // view p's window into buffer p & 1 (a plain arrival when it is read from
    // global memory, so that every view completes one phase)
    auto issue = [&](int p) {
        const int ulo = use_tma ? __ldg(twin + p) : -1;
        uint64_t* bar = &bars[p & 1];
        if (ulo < 0) {
            mbar_arrive_expect_tx(bar, 0);
            return;
        }
        mbar_arrive_expect_tx(bar, (uint32_t)(nboxes * kRowBox * kWin * 4));
        fence_proxy_async_smem();
        for (int r = 0; r < nboxes; ++r)
            tma_load_3d(stage + ((size_t)(p & 1) * nvp + (size_t)r * kRowBox) * kWin, &map, ulo, r * kRowBox, p, bar);
    };
    // view f's copies never arrived: wait (bounded, full limit) for them and
    // for view f + 1's, issued before f's wait, so that no bulk copy is still
    // landing in this CTA's shared memory when it exits
    auto drain = [&](int f) {
        if (tid == 0) {
            mbar_wait_bounded(&bars[f & 1], (uint32_t)(f >> 1) & 1u, kDrainLimit);
            if (f + 1 < G.np) mbar_wait_bounded(&bars[(f + 1) & 1], (uint32_t)((f + 1) >> 1) & 1u, kDrainLimit);
        }
    };
    if (tid == 0) {
        issue(0);
        if (G.np > 1) issue(1);
    }
    double acc[kZPer];
    float oz[kZPer];
#pragma unroll
    for (int q = 0; q < kZPer; ++q) {
        acc[q] = 0.0;
        oz[q] = chunk_oz(min(zbase + 32 * q + l, G.nz - 1), G.nz, G.dz);
    }
    for (int p = 0; p < G.np; ++p) {
        if (!mbar_wait_bounded(&bars[p & 1], (uint32_t)(p >> 1) & 1u, K.wait_limit)) {
            s_abort = 1;
            if (K.err) atomicExch(K.err, 1);
        }
        __syncthreads();
        if (s_abort) {
            drain(p);
            return;
        }
        const int ulo = use_tma ? __ldg(twin + p) : -1;
        const float* sp = stage + (size_t)(p & 1) * nvp * kWin;
        const float* gp = proj + (size_t)p * nv * G.nu;
        View3 V;
        load_view3(G.view + (size_t)p * 20, V);
        Column c;
        bool active = col_ok;
        if (active) {
            column_setup(V, ix, iy, G.nx, G.ny, G.nu, G.dx, G.dy, c);
            if (mode == 0 && c.minu >= c.maxu) active = false;  // layers/A_B1_3D.cu:404
        }
        if (active) {
            const int ncv = c.maxu - c.minu + 1;
            // conv of bin minu + l (lane l), then B(v) = sum over kept bins
            // of conv(u) proj(u, v), a lane per row
            float cv = 0.f;
            if (l < ncv) {
                cv = column_conv_at(V, c, G.vecs + (size_t)p * G.nu, G.nu, l);
                const bool keep = mode == 0 ? (cv == cv && cv > kEps) : (cv == cv);
                if (!keep) cv = 0.f;
            }
            const int du0 = c.minu - ulo, q0 = du0 >> 2, sh = du0 & 3;
            if (ulo >= 0 && du0 >= 0 && ncv + sh <= 8 && 4 * q0 + 8 <= kWin) {
                // the column's bins lie in two 16-byte words of each staged
                // row: B(v) = sum_k coef[k] row[4 q0 + k], coef the column's
                // footprint shifted by sh (the same for every lane)
                float coef[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const float ck = __shfl_sync(0xffffffffu, cv, max(0, min(31, k - sh)));
                    coef[k] = (k >= sh && k - sh < ncv) ? ck : 0.f;
                }
                for (int v = l; v < nv; v += 32) {
                    const float4* row = reinterpret_cast<const float4*>(sp + (size_t)v * kWin) + q0;
                    const float4 a = row[0], b4 = row[1];
                    float b = coef[0] * a.x;
                    b = fmaf(coef[1], a.y, b);
                    b = fmaf(coef[2], a.z, b);
                    b = fmaf(coef[3], a.w, b);
                    b = fmaf(coef[4], b4.x, b);
                    b = fmaf(coef[5], b4.y, b);
                    b = fmaf(coef[6], b4.z, b);
                    b = fmaf(coef[7], b4.w, b);
                    Bw[v] = b;
                }
            } else {
                // not in the staged window (or a snapped view's wide range):
                // global memory, a lane per row
                for (int v0 = 0; v0 < nv; v0 += 32) {  // uniform trip count: the shuffles need every lane
                    const int v = v0 + l;
                    float b = 0.f;
                    for (int t = 0; t < min(ncv, 32); ++t) {
                        const float ct = __shfl_sync(0xffffffffu, cv, t);
                        if (ct != 0.f && v < nv) b = fmaf(ct, __ldg(gp + (size_t)v * G.nu + c.minu + t), b);
                    }
                    if (v < nv) Bw[v] = b;
                }
                if (ncv > 32) {  // the reference's degenerate ranges on snapped views: the rest
                    for (int v = l; v < nv; v += 32) {
                        float b = Bw[v];
                        for (int t = 32; t < ncv; ++t) {
                            const float ct = column_conv_at(V, c, G.vecs + (size_t)p * G.nu, G.nu, t);
                            if (!(mode == 0 ? (ct == ct && ct > kEps) : (ct == ct))) continue;
                            b = fmaf(ct, __ldg(gp + (size_t)v * G.nu + c.minu + t), b);
                        }
                        Bw[v] = b;
                    }
                }
            }
            __syncwarp();
            const float px = V.srcx, py = V.srcy, pz = V.srcz;
            const float ir2 = __fdividef(1.0f, (c.ox - px) * (c.ox - px) + (c.oy - py) * (c.oy - py));
#pragma unroll
            for (int q = 0; q < kZPer; ++q) {
                const int iz = zbase + 32 * q + l;
                Axial a;
                const bool in = iz < G.nz;
                const bool ok = in && axial(V, c, iz, nv, a);
                const unsigned beyond = __ballot_sync(0xffffffffu, in && !ok);
                if (!ok || !chunk_live(beyond, l)) continue;
                if (mode == 0 && a.minv >= a.maxv) continue;  // :433
                float val = 0.f;
                float gp = axial_cdf(a, (float)a.minv);
                for (int j = a.minv; j <= a.maxv; ++j) {
                    const float gn = axial_cdf(a, (float)(j + 1));
                    const float g = __fsub_rn(gn, gp);
                    gp = gn;
                    if (g > kEps) val = fmaf(g, Bw[j], val);
                }
                const float C = mode == 0 ? amplitude(ir2, oz[q] - pz) : amplitude(ir2, oz[q] - pz) * a.width2;
                acc[q] += (double)(val * C);
            }
        }
        __syncthreads();  // buffer p & 1 fully read
        if (tid == 0 && p + 2 < G.np) issue(p + 2);
    }
    if (!col_ok) return;
    const float dxyz = G.dx * G.dy * G.dz;
    const size_t plane = (size_t)G.nx * G.ny;
#pragma unroll
    for (int q = 0; q < kZPer; ++q) {
        const int iz = zbase + 32 * q + l;
        if (iz < G.nz) vol[(size_t)iz * plane + (size_t)iy * G.nx + ix] = (float)(acc[q] * (double)dxyz);
    }
}

// footprint evaluations the reference counts (:50): one per u bin of each
// voxel with a v range, in its forward
__global__ void b1_3d_count_kernel(Geo3 G, unsigned long long* out) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long ncol = (long long)G.nx * G.ny;
    unsigned long long n = 0;
    if (t < ncol) {
        const int ix = (int)(t % G.nx), iy = (int)(t / G.nx);
        for (int p = 0; p < G.np; ++p) {
            View3 V;
            load_view3(G.view + (size_t)p * 20, V);
            Column c;
            column_setup(V, ix, iy, G.nx, G.ny, G.nu, G.dx, G.dy, c);
            for (int z0 = 0; z0 < G.nz; z0 += kZChunk)
                for (int iz = z0; iz < min(G.nz, z0 + kZChunk); ++iz) {
                    float vs[4];
                    int a, b;
                    if (!voxel_v(V, c, iz, G.nv, vs, a, b)) break;
                    n += (unsigned long long)(c.maxu - c.minu + 1);
                }
        }
    }
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(out, n);
}

}  // namespace

class B1Cone {
public:
    int mode;
    int nx, ny, nz, np, nu, nv;
    double dx, dy, dz, du, dv;
    int device = 0;
    cudaStream_t stream = nullptr;
    unsigned long long count = 0;
    Geo3 G{};

    B1Cone(int mode_, int nx_, int ny_, int nz_, int np_, int nu_, int nv_, double dx_, double dy_, double dz_,
           double du_, double dv_, double lsd, double lso, const double* angles)
        : mode(mode_), nx(nx_), ny(ny_), nz(nz_), np(np_), nu(nu_), nv(nv_), dx(dx_), dy(dy_), dz(dz_), du(du_), dv(dv_) {
        if (nx <= 0 || ny <= 0 || nz <= 0 || np <= 0 || nu <= 0 || nv <= 0) fail("invalid sizes");
        check_pitches({dx, dy, dz, du, dv});
        check_distances(lsd, lso);
        check_views(np, angles, nullptr, nullptr);
        SGD_CUDA(cudaGetDevice(&device));
        SGD_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        // GeoData(nx, ny, nz, nu, nv, np, dx, dy, dz, du, dv) + geo_init_angles (layers/A_B1_3D.cu:686-694)
        const std::vector<ViewFrame> fr = view_frames(np, lsd, lso, du, dv, angles, nullptr, nullptr);
        std::vector<float> view((size_t)np * 20, 0.f);
        std::vector<float2> vecs((size_t)np * nu);
        for (int p = 0; p < np; ++p) {
            double pm[12];
            float* v = &view[(size_t)p * 20];
            reference_pmi(fr[p], nu / 2.0, nv / 2.0, nx, ny, nz, dx, dy, dz, pm, v);
            v[12] = (float)fr[p].puv[0]; v[13] = (float)fr[p].puv[1];
            v[14] = (float)fr[p].src[0]; v[15] = (float)fr[p].src[1]; v[16] = (float)fr[p].src[2];
            v[17] = (float)fr[p].dtv[0]; v[18] = (float)fr[p].dtv[1];
            v[19] = (std::fabs((float)fr[p].puv[0] - (float)fr[p].puv[1]) < 1e-7f) ? 1.f : 0.f;
            // layers/A_B1_3D.cu:533-561
            const double cx = fr[p].dtv[0], cy = fr[p].dtv[1], ux = fr[p].puv[0], uy = fr[p].puv[1];
            const double px = fr[p].src[0], py = fr[p].src[1];
            for (int u = 0; u < nu; ++u) {
                const double sx = cx + ux * (u - 0.5 * nu + 0.5), sy = cy + uy * (u - 0.5 * nu + 0.5);
                const double th = std::atan2(std::fabs(px - sx), std::fabs(py - sy));
                vecs[(size_t)p * nu + u] = make_float2((float)std::fabs(dx * std::cos(th)), (float)std::fabs(dy * std::sin(th)));
            }
        }
        SGD_CUDA(cudaMalloc(&d_view_, view.size() * sizeof(float)));
        SGD_CUDA(cudaMemcpy(d_view_, view.data(), view.size() * sizeof(float), cudaMemcpyHostToDevice));
        SGD_CUDA(cudaMalloc(&d_vecs_, vecs.size() * sizeof(float2)));
        SGD_CUDA(cudaMemcpy(d_vecs_, vecs.data(), vecs.size() * sizeof(float2), cudaMemcpyHostToDevice));
        G = Geo3{nx, ny, nz, np, nu, nv, (float)dx, (float)dy, (float)dz, d_view_, d_vecs_};
        plan(lsd, lso, angles);
        const size_t nvol = (size_t)nx * ny * nz, nproj = (size_t)np * nu * nv;
        SGD_CUDA(cudaMalloc(&d_volT_, nvol * sizeof(float)));
        SGD_CUDA(cudaMalloc(&d_vol_, nvol * sizeof(float)));
        SGD_CUDA(cudaMalloc(&d_proj_, nproj * sizeof(float)));
        SGD_CUDA(cudaMallocHost(&h_vol_, nvol * sizeof(float)));
        SGD_CUDA(cudaMallocHost(&h_proj_, nproj * sizeof(float)));
        unsigned long long* dc = nullptr;
        SGD_CUDA(cudaMalloc(&dc, sizeof(unsigned long long)));
        SGD_CUDA(cudaMemset(dc, 0, sizeof(unsigned long long)));
        const long long ncol = (long long)nx * ny;
        b1_3d_count_kernel<<<(unsigned)((ncol + 255) / 256), 256, 0, stream>>>(G, dc);
        SGD_LAUNCH_CHECK();
        SGD_CUDA(cudaMemcpyAsync(&count, dc, sizeof(count), cudaMemcpyDeviceToHost, stream));
        SGD_CUDA(cudaStreamSynchronize(stream));
        cudaFree(dc);
    }
    ~B1Cone() {
        if (stream) cudaStreamSynchronize(stream);
        cudaFree(d_view_); cudaFree(d_vecs_); cudaFree(d_volT_); cudaFree(d_vol_); cudaFree(d_proj_);
        cudaFree(d_strips_); cudaFree(d_twin_); cudaFree(d_err_);
        cudaFreeHost(h_vol_); cudaFreeHost(h_proj_);
        if (stream) cudaStreamDestroy(stream);
    }
    // vol [z][y][x], proj [p][v][u], FP32 device
    void forward_dev(const float* vol, float* proj, cudaStream_t s) {
        launch_to_columns(vol, d_volT_, nx, ny, nz, s);
        SGD_LAUNCH_CHECK();
        b1_3d_fwd_kernel<<<dim3(K.nblk, np), kFW * 32, fwd3_smem(nv, nz), s>>>(G, K, d_volT_, proj,
                                                                             (float)dx * (float)dy * (float)dz);
        SGD_LAUNCH_CHECK();
    }
    void backward_dev(const float* proj, float* vol, cudaStream_t s) {
        // the projection through TMA tensor loads when its rows are whole
        // 16-byte words and it is 16-byte aligned; from global memory otherwise
        const bool tma = (nu % 4) == 0 && (reinterpret_cast<uintptr_t>(proj) % 16) == 0;
        CUtensorMap map;
        std::memset(&map, 0, sizeof(map));
        if (tma) map = encode_tensor_3d_f32(proj, (uint64_t)nu, (uint64_t)nv, (uint64_t)np, kWin, kRowBox, 1);
        const dim3 grid(K.tiles_x, K.tiles_y, (nz + 32 * kZPer - 1) / (32 * kZPer));
        b1_3d_back_kernel<<<grid, kTX * kTY * 32, back3_smem(nv), s>>>(map, G, K, proj, vol, mode, tma ? 1 : 0);
        SGD_LAUNCH_CHECK();
    }
    // 0, or -1 when a back projection's staging wait gave up (those voxels
    // were left unwritten); synchronises the device and clears the flag
    void set_wait_limit(unsigned limit) {
        SGD_CUDA(cudaStreamSynchronize(stream));
        K.wait_limit = limit;
    }
    int status() {
        int h = 0;
        SGD_CUDA(cudaDeviceSynchronize());
        SGD_CUDA(cudaMemcpy(&h, d_err_, sizeof(int), cudaMemcpyDeviceToHost));
        SGD_CUDA(cudaMemset(d_err_, 0, sizeof(int)));
        return h ? -1 : 0;
    }
    void forward_host(double* b, const double* x) {
        const long long nvol = (long long)nx * ny * nz, nproj = (long long)np * nu * nv;
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < nvol; ++e) h_vol_[e] = (float)x[e];
        SGD_CUDA(cudaMemcpyAsync(d_vol_, h_vol_, nvol * sizeof(float), cudaMemcpyHostToDevice, stream));
        forward_dev(d_vol_, d_proj_, stream);
        SGD_CUDA(cudaMemcpyAsync(h_proj_, d_proj_, nproj * sizeof(float), cudaMemcpyDeviceToHost, stream));
        SGD_CUDA(cudaStreamSynchronize(stream));
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < nproj; ++e) b[e] = (double)h_proj_[e];
    }
    void backward_host(const double* b, double* x) {
        const long long nvol = (long long)nx * ny * nz, nproj = (long long)np * nu * nv;
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < nproj; ++e) h_proj_[e] = (float)b[e];
        SGD_CUDA(cudaMemcpyAsync(d_proj_, h_proj_, nproj * sizeof(float), cudaMemcpyHostToDevice, stream));
        backward_dev(d_proj_, d_vol_, stream);
        SGD_CUDA(cudaMemcpyAsync(h_vol_, d_vol_, nvol * sizeof(float), cudaMemcpyDeviceToHost, stream));
        int e = 0;
        SGD_CUDA(cudaMemcpyAsync(&e, d_err_, sizeof(int), cudaMemcpyDeviceToHost, stream));
        SGD_CUDA(cudaStreamSynchronize(stream));
        if (e) {
            SGD_CUDA(cudaMemset(d_err_, 0, sizeof(int)));
            fail("A_B1_3D back projection: a staged view did not arrive within the bounded wait; output incomplete");
        }
#pragma omp parallel for schedule(static)
        for (long long e2 = 0; e2 < nvol; ++e2) x[e2] = (double)h_vol_[e2];
    }

private:
    // The launch tables: the forward's block strips from the in-plane fan
    // geometry (B1 support +-1 voxel, blocks of kUB bins), and per back tile
    // of kTX x kTY columns and view the first bin of its staged window (a
    // multiple of 4 for the TMA box), -1 when its bins span more than kWin.
    void plan(double lsd, double lso, const double* angles) {
        if (nx > kMaxLines || ny > kMaxLines) fail("A_B1_3D: %d x %d columns exceed %d per line", nx, ny, kMaxLines);
        if (fwd3_smem(nv, nz) > 227 * 1024 || back3_smem(nv) > 227 * 1024)
            fail("A_B1_3D: %d detector rows do not fit the kernels' shared memory", nv);
        FanGeometry g;
        g.init(nx, ny, np, nu, dx, dy, du, lsd, lso, angles, nullptr, nullptr);
        auto map = [&](int p) {
            double hw[6];
            fan_world_hom(g, p, hw);
            return grid_range_map(hw, g.x0(), g.dx, g.y0(), g.dy, 1.0, 1.0);
        };
        std::vector<float4> strips;
        std::vector<int2> unused;
        plan_fan2d(nx, ny, np, nu, map, strips, unused, kUB);
        K.nblk = (nu + kUB - 1) / kUB;
        K.tiles_x = (nx + kTX - 1) / kTX;
        K.tiles_y = (ny + kTY - 1) / kTY;
        std::vector<int> twin((size_t)K.tiles_x * K.tiles_y * np, -1);
        for (int p = 0; p < np; ++p) {
            const RangeMap m = map(p);
            for (int ty = 0; ty < K.tiles_y; ++ty)
                for (int tx = 0; tx < K.tiles_x; ++tx) {
                    const double i0 = tx * kTX - 1.0, i1 = std::min(nx, (tx + 1) * kTX) - 1 + 1.0;
                    const double j0 = ty * kTY - 1.0, j1 = std::min(ny, (ty + 1) * kTY) - 1 + 1.0;
                    double umin = 1e300, umax = -1e300;
                    int pos = 0, neg = 0;
                    for (double i : {i0, i1})
                        for (double j : {j0, j1}) {
                            const double D = m.h[3] * i + m.h[4] * j + m.h[5];
                            (D > 0 ? pos : neg)++;
                            const double u = (m.h[0] * i + m.h[1] * j + m.h[2]) / D;
                            umin = std::min(umin, u);
                            umax = std::max(umax, u);
                        }
                    if (pos && neg) continue;
                    const int lo = std::max(0, (int)std::floor(umin) - 1);
                    const int hi = std::min(nu - 1, (int)std::floor(umax) + 1);
                    const int ulo = lo & ~3;
                    if (hi - ulo + 1 <= kWin) twin[((size_t)ty * K.tiles_x + tx) * np + p] = ulo;
                }
        }
        SGD_CUDA(cudaMalloc(&d_strips_, strips.size() * sizeof(float4)));
        SGD_CUDA(cudaMemcpy(d_strips_, strips.data(), strips.size() * sizeof(float4), cudaMemcpyHostToDevice));
        SGD_CUDA(cudaMalloc(&d_twin_, twin.size() * sizeof(int)));
        SGD_CUDA(cudaMemcpy(d_twin_, twin.data(), twin.size() * sizeof(int), cudaMemcpyHostToDevice));
        SGD_CUDA(cudaMalloc(&d_err_, sizeof(int)));
        SGD_CUDA(cudaMemset(d_err_, 0, sizeof(int)));
        K.strips = d_strips_;
        K.twin = d_twin_;
        K.err = d_err_;
        K.wait_limit = 1u << 22;
        SGD_CUDA(cudaFuncSetAttribute(b1_3d_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)fwd3_smem(nv, nz)));
        SGD_CUDA(cudaFuncSetAttribute(b1_3d_back_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)back3_smem(nv)));
    }

    Plan3 K{};
    float4* d_strips_ = nullptr;
    int* d_twin_ = nullptr;
    int* d_err_ = nullptr;
    float* d_volT_ = nullptr;
    float* d_view_ = nullptr;
    float2* d_vecs_ = nullptr;
    float* d_vol_ = nullptr;
    float* d_proj_ = nullptr;
    float* h_vol_ = nullptr;
    float* h_proj_ = nullptr;
};

}  // namespace sgd

using sgd::B1Cone;

extern "C" {

void* sgd_b1_3d_init(int mode, int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy, double dz,
                     double du, double dv, double lsd, double lso, double* angles) {
    return sgd::guarded<void*>(nullptr, [&]() -> void* {
        if (mode != 0 && mode != 1) sgd::fail("sgd_b1_3d_init: mode must be 0 or 1");
        return new B1Cone(mode, nx, ny, nz, np, nu, nv, dx, dy, dz, du, dv, lsd, lso, angles);
    });
}
void* b1_3d_init(int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy, double dz, double du,
                 double dv, double lsd, double lso, double* angles) {
    return sgd_b1_3d_init(0, nx, ny, nz, np, nu, nv, dx, dy, dz, du, dv, lsd, lso, angles);
}
unsigned long long b1_3d_forward_projection(double* b, double* x, void* layer) {
    return sgd::guarded<unsigned long long>(~0ull, [&]() -> unsigned long long {
        if (!layer || !b || !x) sgd::fail("b1_3d_forward_projection: null argument");
        B1Cone* L = static_cast<B1Cone*>(layer);
        L->forward_host(b, x);
        return L->count;
    });
}
void b1_3d_backward_projection(double* b, double* x, void* layer) {
    sgd::guarded_status([&] {
        if (!layer || !b || !x) sgd::fail("b1_3d_backward_projection: null argument");
        static_cast<B1Cone*>(layer)->backward_host(b, x);
    });
}
int sgd_b1_3d_backward_projection(double* b, double* x, void* layer) {
    return sgd::guarded_status([&] {
        if (!layer || !b || !x) sgd::fail("b1_3d_backward_projection: null argument");
        static_cast<B1Cone*>(layer)->backward_host(b, x);
    });
}
void b1_3d_destroy(void* layer) { delete static_cast<B1Cone*>(layer); }
int sgd_b1_3d_forward_dev(void* layer, const float* d_vol, float* d_proj, void* stream) {
    return sgd::guarded_status([&] {
        if (!layer || !d_vol || !d_proj) sgd::fail("sgd_b1_3d_forward_dev: null argument");
        static_cast<B1Cone*>(layer)->forward_dev(d_vol, d_proj, static_cast<cudaStream_t>(stream));
    });
}
int sgd_b1_3d_backward_dev(void* layer, const float* d_proj, float* d_vol, void* stream) {
    return sgd::guarded_status([&] {
        if (!layer || !d_vol || !d_proj) sgd::fail("sgd_b1_3d_backward_dev: null argument");
        static_cast<B1Cone*>(layer)->backward_dev(d_proj, d_vol, static_cast<cudaStream_t>(stream));
    });
}
unsigned long long sgd_b1_3d_count(void* layer) { return layer ? static_cast<B1Cone*>(layer)->count : 0ull; }
int sgd_b1_3d_set_wait_limit(void* layer, unsigned limit) {
    return sgd::guarded_status([&] {
        if (!layer) sgd::fail("sgd_b1_3d_set_wait_limit: null layer");
        static_cast<B1Cone*>(layer)->set_wait_limit(limit);
    });
}
int sgd_b1_3d_status(void* layer) {
    return sgd::guarded_status([&] {
        if (!layer) sgd::fail("sgd_b1_3d_status: null layer");
        if (static_cast<B1Cone*>(layer)->status() != 0)
            sgd::fail("A_B1_3D back projection: a staged view did not arrive within the bounded wait; "
                      "the affected voxels were left unwritten");
    });
}

}  // extern "C"
