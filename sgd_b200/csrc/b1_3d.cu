// A_B1_3D: bilinear (in-plane) x separable-footprint (axial) cone-beam
// projector.  Reference: layers/A_B1_3D.cu:22-66 (gamma), :68-80 (footprint),
// :82-312 (forward), :314-531 (backward), :686-773 (C entry points).
//
// Per voxel (ix, iy, iz) and view: the in-plane B1 footprint conv(u) of the
// column (ix, iy) over the bins u of its +-1 voxel support (the reference's
// FP32 formula, its FP32 bin stepping included), times the integral gamma(v)
// of the axial trapezoid (corners ix +- 1 at iy, iz +- 1/2 through pmi) over
// bin row v, times vol * dx dy dz * sqrt(r3^2 / r2^2).  The reference's
// forward also multiplies by 2 / (trapezoid width) (:210), its backward does
// not (:436), and the backward skips single-bin u or v ranges (:404, :433):
//   mode 0 "reference": both kernels as the reference (parity);
//   mode 1 "adjoint":   the forward as the reference and the back projector its
//                       exact transpose (dot-product test, autograd).
// conv(u) does not depend on z; both kernels compute it once per column and
// view and reuse it for the column's voxels (the reference recomputes it per
// voxel).  Voxels are processed in the reference's z chunks of 32 so that the
// FP32 stepping oz += dz is identical.
//
//   b1_3d_forward_kernel  a CTA per 16 x 16 columns x one z chunk; per view the
//                         CTA's (u, v) window (block min/max of its voxels'
//                         ranges) is accumulated in shared memory and flushed
//                         to an FP64 sinogram, or added directly when a window
//                         is larger than the shared buffer.
//   b1_3d_back_kernel     gather: a thread per column and 16 voxels of a chunk,
//                         FP64 accumulators, each voxel written once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.h"
#include "fan_geometry.h"

namespace sgd {

namespace {

constexpr int kZChunk = 32;      // the reference's Z_SIZE (layers/A_B1_3D.cu:25)
constexpr int kTile = 16;        // forward: 16 x 16 columns per CTA
constexpr int kWinCap = 6144;    // forward: shared (u, v) window, floats
constexpr int kBackZ = 16;       // back: voxels of a chunk per thread
constexpr int kMaxConv = 8;      // cached in-plane footprints per column
constexpr int kMaxRows = 4;      // cached axial integrals per voxel (v rows)
constexpr float kEps = 1e-7f;

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

// layers/A_B1_3D.cu:30-66
__device__ __forceinline__ float gamma_trap(float s1, float s2, const float* us) {
    float g = 0.0f, tmp, b1, b2;
    b1 = fmaxf(s1, us[0]);
    b2 = fminf(s2, us[1]);
    tmp = (b2 > b1) ? (1 / (2 * (us[1] - us[0]))) * ((b2 - us[0]) * (b2 - us[0]) - (b1 - us[0]) * (b1 - us[0])) : 0.0f;
    if (tmp == tmp) g += tmp;
    b1 = fmaxf(s1, us[1]);
    b2 = fminf(s2, us[2]);
    tmp = (b2 > b1) ? b2 - b1 : 0.0f;
    if (tmp == tmp) g += tmp;
    b1 = fmaxf(s1, us[2]);
    b2 = fminf(s2, us[3]);
    tmp = (b2 > b1) ? (1 / (2 * (us[3] - us[2]))) * ((b1 - us[3]) * (b1 - us[3]) - (b2 - us[3]) * (b2 - us[3])) : 0.0f;
    if (tmp == tmp) g += tmp;
    return g;
}

// gamma_trap of rows minv .. minv + kMaxRows - 1 (those up to maxv), once per
// voxel: the (u, v) loops below reuse them for every u.  Unrolled so that
// they stay in registers.
__device__ __forceinline__ void voxel_rows(const float* vs, int minv, int maxv, float* g) {
#pragma unroll
    for (int r = 0; r < kMaxRows; ++r) g[r] = (minv + r <= maxv) ? gamma_trap((float)(minv + r), minv + r + 1.0f, vs) : 0.f;
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

// the first kMaxConv footprints of the column, cached; bins beyond (only the
// reference's degenerate ranges of odd-45-degree views reach them) are
// recomputed by column_conv_at
__device__ __forceinline__ void column_conv(const View3& V, const Column& c, const float2* __restrict__ vecs, int nu,
                                            float* conv) {
    const int n = min(c.maxu - c.minu + 1, kMaxConv);
    for (int ti = 0; ti < n; ++ti) conv[ti] = column_conv_at(V, c, vecs, nu, ti);
}

__device__ __forceinline__ float conv_of(const View3& V, const Column& c, const float2* __restrict__ vecs, int nu,
                                         const float* conv, int ti) {
    return ti < kMaxConv ? conv[ti] : column_conv_at(V, c, vecs, nu, ti);
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

__global__ void __launch_bounds__(kTile * kTile, 6) b1_3d_forward_kernel(Geo3 G, const float* __restrict__ vol,
                                                                     double* __restrict__ proj64) {
    __shared__ float s_acc[kWinCap];
    __shared__ int s_win[4];
    const int ix = blockIdx.x * kTile + threadIdx.x, iy = blockIdx.y * kTile + threadIdx.y;
    const int z_start = blockIdx.z * kZChunk, z_end = min(G.nz, z_start + kZChunk);
    const int tid = threadIdx.y * kTile + threadIdx.x;
    const bool mine = ix < G.nx && iy < G.ny;
    const size_t plane = (size_t)G.nx * G.ny;
    for (int p = 0; p < G.np; ++p) {
        View3 V;
        load_view3(G.view + (size_t)p * 20, V);
        Column c;
        float conv[kMaxConv];
        int ncv = 0;
        int ulo = 1 << 30, uhi = -1, vlo = 1 << 30, vhi = -1;
        const float2* vecs = G.vecs + (size_t)p * G.nu;
        if (mine) {
            column_setup(V, ix, iy, G.nx, G.ny, G.nu, G.dx, G.dy, c);
            column_conv(V, c, vecs, G.nu, conv);
            ncv = c.maxu - c.minu + 1;
            // v extent of the chunk: trapezoids at its first and last voxels
            float vs[4];
            int a, b;
            if (voxel_v(V, c, z_start, G.nv, vs, a, b)) {
                vlo = min(vlo, a); vhi = max(vhi, b);
            }
            if (voxel_v(V, c, z_end - 1, G.nv, vs, a, b)) {
                vlo = min(vlo, a); vhi = max(vhi, b);
            } else {
                vhi = G.nv - 1;
            }
            ulo = c.minu;
            uhi = c.minu + ncv - 1;
        }
        if (tid == 0) {
            s_win[0] = 1 << 30; s_win[1] = -1; s_win[2] = 1 << 30; s_win[3] = -1;
        }
        __syncthreads();
        if (mine && vhi >= vlo) {
            atomicMin(&s_win[0], ulo); atomicMax(&s_win[1], uhi);
            atomicMin(&s_win[2], vlo); atomicMax(&s_win[3], vhi);
        }
        __syncthreads();
        const int wul = s_win[0], wuh = s_win[1], wvl = s_win[2], wvh = s_win[3];
        const int wu = wuh - wul + 1, wv = wvh - wvl + 1;
        const bool in_smem = wu > 0 && wv > 0 && wu * wv <= kWinCap;
        if (in_smem)
            for (int e = tid; e < wu * wv; e += kTile * kTile) s_acc[e] = 0.f;
        __syncthreads();
        if (mine && wu > 0 && wv > 0) {
            float* dp = nullptr;
            double* gp = proj64 + (size_t)p * G.nu * G.nv;
            float oz = (z_start - 0.5f * (G.nz - 1)) * G.dz;
            for (int iz = z_start; iz < z_end; ++iz, oz += G.dz) {
                const float C0 = vol[(size_t)iz * plane + (size_t)iy * G.nx + ix];
                float vs[4];
                int minv, maxv;
                if (!voxel_v(V, c, iz, G.nv, vs, minv, maxv)) break;
                if (C0 == 0.f) continue;
                const float px = V.srcx, py = V.srcy, pz = V.srcz;
                const float weight = sqrtf(((c.ox - px) * (c.ox - px) + (c.oy - py) * (c.oy - py) + (oz - pz) * (oz - pz)) /
                                           ((c.ox - px) * (c.ox - px) + (c.oy - py) * (c.oy - py)));
                const float C = C0 * weight * (2 / (((vs[3] - vs[0]) + (vs[2] - vs[1]))));
                auto add = [&](int u, int j, float val, float g) {
                    if (!(g > kEps)) return;
                    if (in_smem) {
                        dp = s_acc + (j - wvl) * wu + (u - wul);
                        atomicAdd(dp, val * g);
                    } else {
                        atomicAdd(gp + (size_t)j * G.nu + u, (double)(val * g));
                    }
                };
                if (maxv - minv < kMaxRows) {
                    float gr[kMaxRows];
                    voxel_rows(vs, minv, maxv, gr);
                    for (int ti = 0; ti < ncv; ++ti) {
                        const float val = conv_of(V, c, vecs, G.nu, conv, ti) * C;
                        if (!(val == val)) continue;
#pragma unroll
                        for (int r = 0; r < kMaxRows; ++r)
                            if (minv + r <= maxv) add(c.minu + ti, minv + r, val, gr[r]);
                    }
                } else {
                    for (int ti = 0; ti < ncv; ++ti) {
                        const float val = conv_of(V, c, vecs, G.nu, conv, ti) * C;
                        if (!(val == val)) continue;
                        for (int j = minv; j <= maxv; ++j)
                            add(c.minu + ti, j, val, gamma_trap((float)j, j + 1.0f, vs));
                    }
                }
            }
        }
        __syncthreads();
        if (in_smem) {
            double* gp = proj64 + (size_t)p * G.nu * G.nv;
            for (int e = tid; e < wu * wv; e += kTile * kTile) {
                const float a = s_acc[e];
                if (a != 0.f) {
                    const int j = wvl + e / wu, u = wul + e % wu;
                    atomicAdd(gp + (size_t)j * G.nu + u, (double)a);
                }
            }
        }
        __syncthreads();
    }
}

// mode 0: the reference's backward (no 2/width factor, conv > 1e-7 kept,
// single-bin u or v ranges skipped); mode 1: the exact transpose of the forward
__global__ void __launch_bounds__(256, 4) b1_3d_back_kernel(Geo3 G, const float* __restrict__ proj,
                                                         float* __restrict__ vol, int mode) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int per_col = (G.nz + kBackZ - 1) / kBackZ;
    const long long ncol = (long long)G.nx * G.ny;
    if (t >= ncol * per_col) return;
    const int col = (int)(t % ncol), part = (int)(t / ncol);
    const int ix = col % G.nx, iy = col / G.nx;
    const int z0 = part * kBackZ, z1 = min(G.nz, z0 + kBackZ);
    const int z_start = (z0 / kZChunk) * kZChunk;  // the reference's chunk: oz is stepped from its start
    double acc[kBackZ];
#pragma unroll
    for (int k = 0; k < kBackZ; ++k) acc[k] = 0.0;
    const float dxyz = G.dx * G.dy * G.dz;
    for (int p = 0; p < G.np; ++p) {
        View3 V;
        load_view3(G.view + (size_t)p * 20, V);
        Column c;
        column_setup(V, ix, iy, G.nx, G.ny, G.nu, G.dx, G.dy, c);
        if (mode == 0 && c.minu >= c.maxu) continue;  // layers/A_B1_3D.cu:404
        float conv[kMaxConv];
        const float2* vecs = G.vecs + (size_t)p * G.nu;
        column_conv(V, c, vecs, G.nu, conv);
        const int ncv = c.maxu - c.minu + 1;
        const float* pp = proj + (size_t)p * G.nu * G.nv;
        float oz = (z_start - 0.5f * (G.nz - 1)) * G.dz;
        for (int iz = z_start; iz < z0; ++iz) oz += G.dz;
        for (int iz = z0; iz < z1; ++iz, oz += G.dz) {
            float vs[4];
            int minv, maxv;
            if (!voxel_v(V, c, iz, G.nv, vs, minv, maxv)) break;
            if (mode == 0 && minv >= maxv) continue;  // :433
            const float px = V.srcx, py = V.srcy, pz = V.srcz;
            const float weight = sqrtf(((c.ox - px) * (c.ox - px) + (c.oy - py) * (c.oy - py) + (oz - pz) * (oz - pz)) /
                                       ((c.ox - px) * (c.ox - px) + (c.oy - py) * (c.oy - py)));
            float C = weight;
            if (mode == 1) C = weight * (2 / (((vs[3] - vs[0]) + (vs[2] - vs[1]))));
            float val = 0.f;
            if (maxv - minv < kMaxRows) {
                float gr[kMaxRows];
                voxel_rows(vs, minv, maxv, gr);
                for (int ti = 0; ti < ncv; ++ti) {
                    const float cv = conv_of(V, c, vecs, G.nu, conv, ti);
                    if (mode == 0 ? !(cv == cv && cv > kEps) : !(cv * C == cv * C)) continue;
                    const float* pu = pp + (size_t)minv * G.nu + c.minu + ti;
#pragma unroll
                    for (int r = 0; r < kMaxRows; ++r)
                        if (minv + r <= maxv && gr[r] > kEps) val = fmaf(__ldg(pu + (size_t)r * G.nu), gr[r] * cv, val);
                }
            } else {
                for (int ti = 0; ti < ncv; ++ti) {
                    const float cv = conv_of(V, c, vecs, G.nu, conv, ti);
                    if (mode == 0 ? !(cv == cv && cv > kEps) : !(cv * C == cv * C)) continue;
                    const int u = c.minu + ti;
                    for (int j = minv; j <= maxv; ++j) {
                        const float g = gamma_trap((float)j, j + 1.0f, vs);
                        if (g > kEps) val = fmaf(__ldg(pp + (size_t)j * G.nu + u), g * cv, val);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < kBackZ; ++k)
                if (k == iz - z0) acc[k] += (double)(val * C);
        }
    }
    const size_t plane = (size_t)G.nx * G.ny;
#pragma unroll
    for (int k = 0; k < kBackZ; ++k)
        if (z0 + k < z1) vol[(size_t)(z0 + k) * plane + col] = (float)(acc[k] * (double)dxyz);
}

__global__ void b1_3d_finish_kernel(const double* __restrict__ s64, float* __restrict__ s32, long long n, float scale) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) s32[e] = (float)(s64[e] * (double)scale);
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
        const size_t nvol = (size_t)nx * ny * nz, nproj = (size_t)np * nu * nv;
        SGD_CUDA(cudaMalloc(&d_proj64_, nproj * sizeof(double)));
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
        cudaFree(d_view_); cudaFree(d_vecs_); cudaFree(d_proj64_); cudaFree(d_vol_); cudaFree(d_proj_);
        cudaFreeHost(h_vol_); cudaFreeHost(h_proj_);
        if (stream) cudaStreamDestroy(stream);
    }
    // vol [z][y][x], proj [p][v][u], FP32 device
    void forward_dev(const float* vol, float* proj, cudaStream_t s) {
        const long long nproj = (long long)np * nu * nv;
        SGD_CUDA(cudaMemsetAsync(d_proj64_, 0, nproj * sizeof(double), s));
        dim3 grid((nx + kTile - 1) / kTile, (ny + kTile - 1) / kTile, (nz + kZChunk - 1) / kZChunk);
        b1_3d_forward_kernel<<<grid, dim3(kTile, kTile), 0, s>>>(G, vol, d_proj64_);
        SGD_LAUNCH_CHECK();
        b1_3d_finish_kernel<<<(unsigned)((nproj + 255) / 256), 256, 0, s>>>(d_proj64_, proj, nproj,
                                                                          (float)dx * (float)dy * (float)dz);
        SGD_LAUNCH_CHECK();
    }
    void backward_dev(const float* proj, float* vol, cudaStream_t s) {
        const long long n = (long long)nx * ny * ((nz + kBackZ - 1) / kBackZ);
        b1_3d_back_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(G, proj, vol, mode);
        SGD_LAUNCH_CHECK();
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
        SGD_CUDA(cudaStreamSynchronize(stream));
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < nvol; ++e) x[e] = (double)h_vol_[e];
    }

private:
    float* d_view_ = nullptr;
    float2* d_vecs_ = nullptr;
    double* d_proj64_ = nullptr;
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

}  // extern "C"
