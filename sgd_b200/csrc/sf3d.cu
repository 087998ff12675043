// SF_projector: 3D separable-footprint (SF-TR, optionally SF-TT) cone-beam
// projector.  Reference: layers/SF_projector.cu:42-78 (gamma), :81-234
// (SF_project), :237-356 (SF_backproject), :359-400 (SF::project /
// back_project); it has no C entry points there.
//
// Per voxel (ix, iy, iz) and view, through the view's index-space matrix pmi:
// the four in-plane corners (ix +- 1/2, iy +- 1/2) at iz give a trapezoid
// us[0..3] in u; the voxel's z extent gives a rectangle vs[0..1] in v (SF-TR),
// or the corners (ix +- 1/2, iy) at iz +- 1/2 a trapezoid (SF-TT, forward
// only in the reference).  This projector takes bins as [i - 1/2, i + 1/2]
// (ranges ceil(us - 1/2), :165-166), unlike the 2D projectors.  Amplitudes:
//   forward   lsd^2 dy dz / (du dv) * (1/r^2) * 2/(trapezoid width) * 1/(v width)
//   backward  lsd dx / np          * (1/r)   * 2/(trapezoid width) * 1/(v width)
// with r the distance from the source to (dx (ix - nx/2), dy (iy - ny/2),
// dz (iz - nz/2)) (integer halves, :104-105).
//
// Reference behaviour (mode 0), reproduced for parity:
//   * the forward adds the footprint alone, without the voxel value or the
//     amplitude (C is computed and never used, :190-221): it projects the
//     indicator of the non-zero voxels;
//   * bin indices are not clamped, j * nu + i is only bounds-checked, so bins
//     beyond the u edges wrap into neighbouring rows (:216, :336).
//   * on the snapped 3pi/4 and -pi/4 views its index-space matrices degenerate
//     (utils/geo.cu:36-41) and voxels project onto spans of hundreds of bins;
//     here a voxel whose span exceeds twice the detector is skipped (the one
//     deviation: the reference visits those spans).
// Mode 1 ("fixed"): exact projection matrices on every view, the forward
// scales by the voxel value and amplitude and drops out-of-detector bins; the
// back projection is its exact transpose.
//
// Mode 0 runs the reference's scatter and gather as written (a thread per
// voxel column chunk and view, FP64 atomics; a thread per voxel): its bins
// wrap into neighbouring rows and its snapped views visit hundreds of bins,
// neither of which fits a detector-block decomposition.  Mode 1 runs the
// factored kernels.  With a circular orbit the detector's u row of every
// exact matrix has no z term (pm[2] = pm[10] = 0, checked at init), so the
// in-plane trapezoid g(u) of a column does not depend on z and the axial
// footprint f_z(v) does not depend on u; per view and column
//   forward   proj(u, v) += g(u) A(v),   A(v) = sum_z C(z) vol(z) f_z(v)
//   back      vol(z) += C(z) sum_v f_z(v) B(v),   B(v) = sum_u g(u) proj(u, v)
// with C the amplitude.  sf3d_fwd_kernel takes a CTA per (view, block of 16
// u bins): its columns are the block's in-plane strip, a warp builds one
// column's A in shared memory (lanes over z, a transposed copy of the volume),
// and threads that own detector rows add g(u) A(v) into FP64 block
// accumulators: every bin is written once, no atomics in global memory.
// sf3d_back1_kernel takes a CTA per 4 x 2 columns and 256 voxels of z; per
// view a TMA tensor load stages the tile's window of 20 u bins x all rows
// (double buffered on mbarriers with bounded waits), each warp forms B of its
// column and each lane its voxels' sums.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include <cuda.h>

#include "common.h"
#include "cone_columns.cuh"
#include "fan_geometry.h"
#include "proj2d.h"
#include "tensor_map.h"
#include "tma.cuh"

namespace sgd {

namespace {

constexpr int kSFZ = 64;  // the reference's Z_SIZE (layers/SF_projector.hh:3)

struct SFGeo {
    int nx, ny, nz, np, nu, nv, trap, mode;
    double dx, dy, dz;
    const float* pmi;    // [np][12]
    const double* src;   // [np][3]
    const double* fwdf;  // [np] forward factor lsd^2 dy dz / (du dv) (times dx in mode 1)
    double backf;        // lsd dx / np
};

__device__ __forceinline__ void sort4f(float* a) {
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

// layers/SF_projector.cu:42-78
__device__ __forceinline__ float sf_gamma(float s1, float s2, const float* us) {
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

struct SFVoxel {
    float us[4], vs[4];
    int min_u, max_u, min_v, max_v;
    float C;  // amplitude (forward or backward normalisation)
};

// Returns 0: voxel contributes, 1: skip this voxel, 2: skip the rest of the
// thread's z chunk (the reference's `return`, :150, :286).
__device__ int sf_voxel(const SFGeo& G, const float* pm, const double* src, double factor, bool fwd, int ix, int iy,
                        int iz, SFVoxel& o) {
    const int nxh = G.nx / 2, nyh = G.ny / 2, nzh = G.nz / 2;
    const float pmv2 = pm[4] * ix + pm[5] * iy + pm[7];
    const float pmv3 = pm[8] * ix + pm[9] * iy + pm[11];
    const float signy1 = iy - 0.5f, signy2 = iy + 0.5f, signx1 = ix - 0.5f, signx2 = ix + 0.5f;
    const float u1 = pm[0] * signx1 + pm[1] * signy1 + pm[3], u2 = pm[8] * signx1 + pm[9] * signy1 + pm[11];
    const float u3 = pm[0] * signx2 + pm[1] * signy1 + pm[3], u4 = pm[8] * signx2 + pm[9] * signy1 + pm[11];
    const float u5 = pm[0] * signx1 + pm[1] * signy2 + pm[3], u6 = pm[8] * signx1 + pm[9] * signy2 + pm[11];
    const float u7 = pm[0] * signx2 + pm[1] * signy2 + pm[3], u8 = pm[8] * signx2 + pm[9] * signy2 + pm[11];
    const float signz1 = (iz - 0.5f), signz2 = (iz + 0.5f);
    float min_v, max_v;
    const bool trap = fwd && G.trap;
    if (!trap) {
        o.vs[0] = (pmv2 + pm[6] * signz1) / (pmv3 + pm[10] * signz1);
        min_v = ceilf(o.vs[0] - 0.5f);
        if (min_v >= G.nv) return 2;
        o.vs[1] = (pmv2 + pm[6] * signz2) / (pmv3 + pm[10] * signz2);
        max_v = ceilf(o.vs[1] - 0.5f);
        if (max_v < 0) return 1;
    } else {
        const float v1 = pm[4] * signx1 + pm[5] * iy + pm[7], v2 = pm[4] * signx2 + pm[5] * iy + pm[7];
        const float v3 = pm[8] * signx1 + pm[9] * iy + pm[11], v4 = pm[8] * signx2 + pm[9] * iy + pm[11];
        o.vs[0] = (v1 + pm[6] * signz1) / (v3 + pm[10] * signz1);
        o.vs[1] = (v1 + pm[6] * signz2) / (v3 + pm[10] * signz2);
        o.vs[2] = (v2 + pm[6] * signz1) / (v4 + pm[10] * signz1);
        o.vs[3] = (v2 + pm[6] * signz2) / (v4 + pm[10] * signz2);
        sort4f(o.vs);
        min_v = ceilf(o.vs[0] - 0.5f);
        max_v = ceilf(o.vs[3] - 0.5f);
        if ((max_v < 0) || (min_v >= G.nv)) return 1;
    }
    const double ddx = G.dx * (ix - nxh) - src[0], ddy = G.dy * (iy - nyh) - src[1], ddz = G.dz * (iz - nzh) - src[2];
    float weight = rsqrtf((float)(ddx * ddx + ddy * ddy + ddz * ddz));
    if (fwd) weight *= weight;
    o.us[0] = (u1 + pm[2] * iz) / (u2 + pm[10] * iz);
    o.us[1] = (u3 + pm[2] * iz) / (u4 + pm[10] * iz);
    o.us[2] = (u5 + pm[2] * iz) / (u6 + pm[10] * iz);
    o.us[3] = (u7 + pm[2] * iz) / (u8 + pm[10] * iz);
    sort4f(o.us);
    const float min_u = ceilf(o.us[0] - 0.5f), max_u = ceilf(o.us[3] - 0.5f);
    if ((max_u < 0) || (min_u >= G.nu)) return 1;
    const float tw = (2 / (((o.us[3] - o.us[0]) + (o.us[2] - o.us[1]))));
    // SF-TT amplitude: 2 / (sum of the trapezoid's parallel sides).  The
    // reference's expression (:194) groups it differently, but its forward
    // never applies the amplitude, so only the fixed mode reads this.
    if (trap)
        o.C = (float)(weight * factor * tw * (2 / ((o.vs[3] - o.vs[0]) + (o.vs[2] - o.vs[1]))));
    else
        o.C = (float)(weight * factor * tw * (1 / (o.vs[1] - o.vs[0])));
    // a voxel whose projection spans more bins than twice the detector (near
    // the source plane, or through a degenerate matrix) is skipped: its
    // footprint is meaningless and the loops below would run unbounded
    if (!(max_u - min_u <= 2.f * G.nu + 4.f) || !(max_v - min_v <= 2.f * G.nv + 4.f)) return 1;
    o.min_u = (int)min_u; o.max_u = (int)max_u; o.min_v = (int)min_v; o.max_v = (int)max_v;
    return 0;
}

__device__ __forceinline__ float sf_fv(const SFGeo& G, bool trap, const SFVoxel& o, int j) {
    if (trap) return sf_gamma(j - 0.5f, j + 0.5f, o.vs);
    return fmaxf(fminf(j + 0.5f, o.vs[1]) - fmaxf(j - 0.5f, o.vs[0]), 0);
}

// a thread per (ix, iy, z chunk of 64) and view (grid z = views); the volume
// is FP32 (device entry points) or FP64 (mode 1 host entry points)
template <typename TVol>
__global__ void __launch_bounds__(128) sf3d_forward_kernel(SFGeo G, const TVol* __restrict__ vol,
                                                           double* __restrict__ proj64) {
    const int ix = blockIdx.x * 16 + threadIdx.x, iy = blockIdx.y * 8 + threadIdx.y;
    const int chunks = (G.nz + kSFZ - 1) / kSFZ;
    const int p = blockIdx.z / chunks, zc = blockIdx.z % chunks;
    if (ix >= G.nx || iy >= G.ny || p >= G.np) return;
    const float* pm = G.pmi + 12 * (size_t)p;
    const double* src = G.src + 3 * (size_t)p;
    const int nuv = G.nu * G.nv;
    double* pp = proj64 + (size_t)p * nuv;
    const bool trap = G.trap != 0;
    for (int iz = zc * kSFZ; iz < min(G.nz, (zc + 1) * kSFZ); ++iz) {
        const TVol C0 = vol[((size_t)iz * G.ny + iy) * G.nx + ix];
        SFVoxel o;
        const int r = sf_voxel(G, pm, src, G.fwdf[p], true, ix, iy, iz, o);
        if (r == 2 && G.mode == 0) break;  // the reference leaves its z chunk (:150)
        if (r != 0 || C0 == TVol(0)) continue;  // o is only filled when r == 0
        // mode 1 multiplies in FP64 so that the back kernel's terms are the
        // same real numbers (an adjoint pair to FP64 accumulation)
        const double amp = (G.mode == 0) ? 1.0 : (double)o.C * (double)C0;
        for (int i = o.min_u; i <= o.max_u; ++i) {
            const float g = sf_gamma(i - 0.5f, i + 0.5f, o.us);
            if (G.mode == 1 && (i < 0 || i >= G.nu)) continue;
            for (int j = o.min_v; j <= o.max_v; ++j) {
                const float f2 = g * sf_fv(G, trap, o, j);
                const int idxv = j * G.nu + i;
                if (G.mode == 1 && (j < 0 || j >= G.nv)) continue;
                if (idxv < nuv && idxv >= 0 && f2 == f2 && f2 != 0.f) atomicAdd(pp + idxv, (double)f2 * amp);
            }
        }
    }
}

// mode 0: SF_backproject (rect in v); mode 1: exact transpose of the fixed
// forward.  FP32 in and out (device entry points) or FP64 (mode 1 host entry
// points, so that the pair stays an adjoint pair to FP64 rounding end to end)
template <typename TProj, typename TVol>
__global__ void __launch_bounds__(128) sf3d_back_kernel(SFGeo G, const TProj* __restrict__ proj,
                                                        TVol* __restrict__ vol) {
    const int ix = blockIdx.x * 16 + threadIdx.x, iy = blockIdx.y * 8 + threadIdx.y;
    const int iz = blockIdx.z;
    if (ix >= G.nx || iy >= G.ny) return;
    const int nuv = G.nu * G.nv;
    const bool trap = G.mode == 1 && G.trap != 0;
    const int z0 = iz - iz % kSFZ;
    double acc = 0.0;
    for (int p = 0; p < G.np; ++p) {
        const float* pm = G.pmi + 12 * (size_t)p;
        const double* src = G.src + 3 * (size_t)p;
        SFVoxel o;
        // The reference walks z in chunks of 64 and leaves the chunk at the
        // first voxel whose v range starts beyond the detector.  v is monotone
        // in z along a column, so that voxel is either the chunk's first or
        // this one: test both.
        if (G.mode == 0 && iz != z0) {
            const float pmv2 = pm[4] * ix + pm[5] * iy + pm[7], pmv3 = pm[8] * ix + pm[9] * iy + pm[11];
            const float v0 = (pmv2 + pm[6] * (z0 - 0.5f)) / (pmv3 + pm[10] * (z0 - 0.5f));
            if (ceilf(v0 - 0.5f) >= G.nv) continue;
        }
        const int r = sf_voxel(G, pm, src, G.mode == 0 ? G.backf : G.fwdf[p], G.mode == 1, ix, iy, iz, o);
        if (r != 0) continue;
        const TProj* pp = proj + (size_t)p * nuv;
        double sumV = 0.0;
        for (int i = o.min_u; i <= o.max_u; ++i) {
            if (G.mode == 1 && (i < 0 || i >= G.nu)) continue;
            const float g = sf_gamma(i - 0.5f, i + 0.5f, o.us);
            for (int j = o.min_v; j <= o.max_v; ++j) {
                if (G.mode == 1 && (j < 0 || j >= G.nv)) continue;
                const float f = g * sf_fv(G, trap, o, j);
                const int idxv = j * G.nu + i;
                if (idxv < nuv && idxv >= 0 && (G.mode == 0 || (f == f && f != 0.f)))
                    sumV += (double)pp[idxv] * (double)f;
            }
        }
        sumV *= (double)o.C;
        if (sumV == sumV) acc += sumV;
    }
    vol[((size_t)iz * G.ny + iy) * G.nx + ix] = (TVol)acc;
}

__global__ void sf3d_finish_kernel(const double* __restrict__ s64, float* __restrict__ s32, long long n) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) s32[e] = (float)s64[e];
}

// ---------------------------------------------------------------------------
// Mode 1: the factored kernels.

constexpr int kUB = 16;          // forward: u bins per block
constexpr int kFW = 8;           // forward: warps, columns per batch
constexpr int kMaxLines = 2048;  // forward: strip lines held in shared memory
constexpr int kTX = 4, kTY = 2;  // back: columns per CTA (a warp each)
constexpr int kWin = 20;         // back: staged u window (bins); 80-byte rows keep float4 row reads free of bank conflicts
constexpr int kRowBox = 192;     // back: rows per TMA box
constexpr int kZPer = 8;         // back: voxels per lane (z = l + 32 k)
constexpr int kZC = 256;         // forward: voxels of a column staged at a time (rectangle footprints)
constexpr uint32_t kDrainLimit = 1u << 22;  // back: polls of the drain after a failed wait

struct SFPlan {
    const float4* strips;  // [np][nblk][2]: forward block strips (the 2D projectors' record)
    int nblk;
    const int* twin;       // [tiles][np]: back window's first bin (a multiple of 4), -1: read global memory
    int tiles_x, tiles_y;
    int* err;              // bounded-wait status, 0 = ok
    unsigned wait_limit;
};

// The z-independent part of a column's footprint in one view (the same
// expressions as sf_voxel): the sorted in-plane trapezoid us[0..3] and its
// bins [min_u, max_u] (bins are [i - 1/2, i + 1/2]), the amplitude's 2 /
// (trapezoid width), and the per-column terms of the axial corners and the
// source distance.  False when the column projects off the detector in u or
// over more than twice its width (sf_voxel's skip).
struct SFCol {
    float us[4];
    float tw, pmv2, inv3, tv1, tv2, invt3, invt4;
    float rho2;  // squared in-plane distance of the column from the source
    int min_u, max_u;
};

// a * b + c * d + e with fixed contractions, so that every kernel inlining
// these functions forms the same bits
__device__ __forceinline__ float lin3(float a, float b, float c, float d, float e) {
    return __fadd_rn(__fmaf_rn(a, b, __fmul_rn(c, d)), e);
}

__device__ __forceinline__ bool sf_column(const SFGeo& G, const float* pm, const double* src, int ix, int iy,
                                          SFCol& c) {
    const float signy1 = iy - 0.5f, signy2 = iy + 0.5f, signx1 = ix - 0.5f, signx2 = ix + 0.5f;
    const float u1 = lin3(pm[0], signx1, pm[1], signy1, pm[3]), u2 = lin3(pm[8], signx1, pm[9], signy1, pm[11]);
    const float u3 = lin3(pm[0], signx2, pm[1], signy1, pm[3]), u4 = lin3(pm[8], signx2, pm[9], signy1, pm[11]);
    const float u5 = lin3(pm[0], signx1, pm[1], signy2, pm[3]), u6 = lin3(pm[8], signx1, pm[9], signy2, pm[11]);
    const float u7 = lin3(pm[0], signx2, pm[1], signy2, pm[3]), u8 = lin3(pm[8], signx2, pm[9], signy2, pm[11]);
    c.us[0] = u1 / u2;
    c.us[1] = u3 / u4;
    c.us[2] = u5 / u6;
    c.us[3] = u7 / u8;
    sort4f(c.us);
    const float min_u = ceilf(c.us[0] - 0.5f), max_u = ceilf(c.us[3] - 0.5f);
    if ((max_u < 0) || (min_u >= G.nu) || !(max_u - min_u <= 2.f * G.nu + 4.f)) return false;
    c.min_u = (int)min_u;
    c.max_u = (int)max_u;
    c.tw = (2 / (((c.us[3] - c.us[0]) + (c.us[2] - c.us[1]))));
    // the axial rectangle's ends and trapezoid's corners are (n + pm[6] s) /
    // d with d free of z (pm[10] = 0): one reciprocal per column
    const float fix = (float)ix, fiy = (float)iy;
    c.pmv2 = lin3(pm[4], fix, pm[5], fiy, pm[7]);
    c.inv3 = __frcp_rn(lin3(pm[8], fix, pm[9], fiy, pm[11]));
    c.tv1 = lin3(pm[4], signx1, pm[5], fiy, pm[7]);
    c.tv2 = lin3(pm[4], signx2, pm[5], fiy, pm[7]);
    c.invt3 = __frcp_rn(lin3(pm[8], signx1, pm[9], fiy, pm[11]));
    c.invt4 = __frcp_rn(lin3(pm[8], signx2, pm[9], fiy, pm[11]));
    const double ddx = G.dx * (ix - G.nx / 2) - src[0], ddy = G.dy * (iy - G.ny / 2) - src[1];
    c.rho2 = (float)(ddx * ddx + ddy * ddy);
    return true;
}

// Voxel iz of the column: its axial rectangle (SF-TR) or trapezoid (SF-TT)
// vs, its rows [min_v, max_v] clamped to the detector and the forward
// amplitude C (squared inverse distance, as sf_voxel with fwd).  False when
// sf_voxel skips the voxel.
struct SFAx {
    float vs[4];
    float C;
    int min_v, max_v;
};

// sf_gamma with its differences of squares contracted one fixed way
// (a*a - b*b as fma(a, a, -(b*b))), for the corrected pair, whose forward and
// back kernels must form the same bits.
__device__ __forceinline__ float sf_gamma1(float s1, float s2, const float* us) {
    auto sq_diff = [](float a, float b) { return __fmaf_rn(a, a, -__fmul_rn(b, b)); };
    float g = 0.0f, tmp, b1, b2;
    b1 = fmaxf(s1, us[0]);
    b2 = fminf(s2, us[1]);
    tmp = (b2 > b1) ? (1 / (2 * (us[1] - us[0]))) * sq_diff(b2 - us[0], b1 - us[0]) : 0.0f;
    if (tmp == tmp) g += tmp;
    b1 = fmaxf(s1, us[1]);
    b2 = fminf(s2, us[2]);
    tmp = (b2 > b1) ? b2 - b1 : 0.0f;
    if (tmp == tmp) g += tmp;
    b1 = fmaxf(s1, us[2]);
    b2 = fminf(s2, us[3]);
    tmp = (b2 > b1) ? (1 / (2 * (us[3] - us[2]))) * sq_diff(b1 - us[3], b2 - us[3]) : 0.0f;
    if (tmp == tmp) g += tmp;
    return g;
}

// End k of a column's axial rectangles: the image of z = k - 1/2 (consecutive
// voxels share their ends bit for bit).
__device__ __forceinline__ float sf_end(const SFCol& c, float pm6, int k) {
    return __fmul_rn(__fmaf_rn(pm6, k - 0.5f, c.pmv2), c.inv3);
}

// The forward amplitude of voxel iz without its axial width: the view factor
// times 2 / (trapezoid width) over the squared distance from the source
// (FP32, fast reciprocal: the FP64 distance of sf_voxel agrees to ~1e-7).
__device__ __forceinline__ float sf_amp(const SFGeo& G, const SFCol& c, float dzf, float srcz, float factor, int iz) {
    const float ddz = __fmaf_rn(dzf, (float)(iz - G.nz / 2), -srcz);
    return __fdividef(__fmul_rn(factor, c.tw), __fmaf_rn(ddz, ddz, c.rho2));
}

__device__ __forceinline__ bool sf_axial(const SFGeo& G, const float* pm, const SFCol& c, float dzf, float srcz,
                                         float factor, bool trap, int iz, SFAx& a) {
    float min_v, max_v;
    if (!trap) {
        a.vs[0] = sf_end(c, pm[6], iz);
        min_v = ceilf(a.vs[0] - 0.5f);
        if (min_v >= G.nv) return false;
        a.vs[1] = sf_end(c, pm[6], iz + 1);
        max_v = ceilf(a.vs[1] - 0.5f);
        if (max_v < 0) return false;
    } else {
        const float signz1 = (iz - 0.5f), signz2 = (iz + 0.5f);
        a.vs[0] = __fmul_rn(__fmaf_rn(pm[6], signz1, c.tv1), c.invt3);
        a.vs[1] = __fmul_rn(__fmaf_rn(pm[6], signz2, c.tv1), c.invt3);
        a.vs[2] = __fmul_rn(__fmaf_rn(pm[6], signz1, c.tv2), c.invt4);
        a.vs[3] = __fmul_rn(__fmaf_rn(pm[6], signz2, c.tv2), c.invt4);
        sort4f(a.vs);
        min_v = ceilf(a.vs[0] - 0.5f);
        max_v = ceilf(a.vs[3] - 0.5f);
        if ((max_v < 0) || (min_v >= G.nv)) return false;
    }
    if (!(max_v - min_v <= 2.f * G.nv + 4.f)) return false;
    const float amp = sf_amp(G, c, dzf, srcz, factor, iz);
    if (trap)
        a.C = amp * __fdividef(2.f, (a.vs[3] - a.vs[0]) + (a.vs[2] - a.vs[1]));
    else
        a.C = amp * __fdividef(1.f, a.vs[1] - a.vs[0]);
    a.min_v = max(0, (int)min_v);
    a.max_v = min(G.nv - 1, (int)max_v);
    return true;
}

// axial footprint of row j (sf_fv)
__device__ __forceinline__ float sf_row(const SFAx& a, bool trap, int j) {
    if (trap) return sf_gamma1(j - 0.5f, j + 0.5f, a.vs);
    return fmaxf(fminf(j + 0.5f, a.vs[1]) - fmaxf(j - 0.5f, a.vs[0]), 0.f);
}

__host__ __device__ constexpr size_t sf_fwd_smem(int nv) {
    return (size_t)kUB * nv * 8 + (size_t)kFW * nv * 8 + (size_t)kFW * kZC * 8 + (size_t)kFW * (kZC + 2) * 4 +
           kFW * kUB * 4 + (kMaxLines + 1) * 4;
}

// The voxel weight C(z) vol(z) of sf_axial for a rectangle whose ends vs0,
// vs1 were formed already (the same expressions): 0 where sf_axial skips.
__device__ __forceinline__ double sf_rect_weight(const SFGeo& G, const SFCol& c, float dzf, float srcz, float factor,
                                                 int iz, float vs0, float vs1, float C0) {
    const float min_v = ceilf(vs0 - 0.5f), max_v = ceilf(vs1 - 0.5f);
    if (min_v >= G.nv || max_v < 0 || !(max_v - min_v <= 2.f * G.nv + 4.f)) return 0.0;
    const float C = sf_amp(G, c, dzf, srcz, factor, iz) * __fdividef(1.f, vs1 - vs0);
    return C == C ? (double)C * (double)C0 : 0.0;
}

// A(v) += sum_z C(z) vol(z) f_z(v) of one column, rectangle footprints, by
// the warp: the rectangles of consecutive voxels share their ends (t_z, t_z+1
// with t_k the image of k - 1/2), so per chunk of kZC voxels the lanes stage
// the ends T and the weights W, then each lane takes detector rows and sums
// the few voxels that overlap its row in FP64 (rows at the chunk's edges add
// to what the previous chunk left).  No atomics; every term as the back
// projection forms it.
__device__ __forceinline__ void sf_rect_profile(const SFGeo& G, const float* pm, const SFCol& c, float dzf,
                                                float srcz, float factor, const float* __restrict__ colv, int l,
                                                float* T, double* W, double* Aw) {
    const int nz = G.nz, nv = G.nv;
    for (int z0 = 0; z0 < nz; z0 += kZC) {
        const int zn = min(kZC, nz - z0);
        for (int k = l; k <= zn; k += 32) T[k] = sf_end(c, pm[6], z0 + k);
        __syncwarp();
        for (int k = l; k < zn; k += 32) {
            const float C0 = __ldg(colv + z0 + k);
            W[k] = C0 == 0.f ? 0.0 : sf_rect_weight(G, c, dzf, srcz, factor, z0 + k, T[k], T[k + 1], C0);
        }
        __syncwarp();
        const float tlo = T[0], thi = T[zn];
        // ends that decrease along z give empty rectangles (f = 0 on every row)
        if (thi > tlo) {
            const int rlo = max(0, (int)ceilf(tlo - 0.5f)), rhi = min(nv - 1, (int)ceilf(thi - 0.5f));
            const float invh = (float)zn / (thi - tlo);
            for (int j = rlo + l; j <= rhi; j += 32) {
                const float bl = j - 0.5f, br = j + 0.5f;
                // the rectangle holding the row's lower edge: estimate, then step
                int k = min(max((int)floorf((bl - tlo) * invh), 0), zn - 1);
                while (k > 0 && T[k] > bl) --k;
                while (k < zn - 1 && T[k + 1] <= bl) ++k;
                double a = 0.0;
                for (; k < zn && T[k] < br; ++k) {
                    const float f = fmaxf(fminf(br, T[k + 1]) - fmaxf(bl, T[k]), 0.f);
                    if (f != 0.f) a = fma((double)f, W[k], a);
                }
                Aw[j] += a;
            }
        }
        __syncwarp();
    }
}

// TOut: float (device entry points) or double (the FP64 host entry points
// return the FP64 accumulators as they are)
template <typename TOut>
__global__ void __launch_bounds__(kFW * 32, 3) sf3d_fwd_kernel(SFGeo G, SFPlan K, const float* __restrict__ volT,
                                                            TOut* __restrict__ proj) {
    extern __shared__ __align__(16) unsigned char sf_fsmem[];
    const int nv = G.nv, nz = G.nz;
    double* acc = reinterpret_cast<double*>(sf_fsmem);  // [kUB][nv]
    double* A = acc + kUB * nv;                         // [kFW][nv]: each warp's column profile
    double* Wz = A + kFW * nv;                          // [kFW][kZC]: its staged voxel weights
    float* Tz = reinterpret_cast<float*>(Wz + kFW * kZC);  // [kFW][kZC + 2]: their rectangles' ends
    float* cs = Tz + kFW * (kZC + 2);                   // [kFW][kUB]: its g per block bin
    int* pref = reinterpret_cast<int*>(cs + kFW * kUB);   // [kMaxLines + 1]: candidates before each line
    __shared__ int s_act[kFW][2];
    const int k = blockIdx.x, p = blockIdx.y, tid = threadIdx.x, w = tid >> 5, l = tid & 31;
    const int u0 = k * kUB, nb = min(kUB, G.nu - u0);

    for (int e = tid; e < kUB * nv; e += blockDim.x) acc[e] = 0.0;
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

    const float* pm = G.pmi + 12 * (size_t)p;
    const double* src = G.src + 3 * (size_t)p;
    const float factor = (float)G.fwdf[p], srcz = (float)src[2], dzf = (float)G.dz;
    const bool trap = G.trap != 0;
    double* Aw = A + w * nv;
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
            SFCol c;
            if (sf_column(G, pm, src, ix, iy, c)) {
                const int tlo = max(c.min_u, u0), thi = min(c.max_u, u0 + nb - 1);
                if (tlo <= thi) {
                    blo = tlo - u0;
                    bhi = thi - u0;
                    if (l < kUB) {
                        float gv = 0.f;
                        if (l >= blo && l <= bhi) {
                            const int i = u0 + l;
                            gv = sf_gamma1(i - 0.5f, i + 0.5f, c.us);
                            if (!(gv == gv)) gv = 0.f;
                        }
                        cs[w * kUB + l] = gv;
                    }
                    for (int v = l; v < nv; v += 32) Aw[v] = 0.0;
                    __syncwarp();
                    const float* colv = volT + ((size_t)iy * G.nx + ix) * nz;
                    if (!trap) {
                        sf_rect_profile(G, pm, c, dzf, srcz, factor, colv, l, Tz + w * (kZC + 2), Wz + w * kZC, Aw);
                    } else {
                        // trapezoids of neighbouring voxels overlap: FP64
                        // shared-memory atomics over each voxel's rows
                        for (int iz = l; iz < nz; iz += 32) {
                            const float C0 = __ldg(colv + iz);
                            if (C0 == 0.f) continue;
                            SFAx a;
                            if (!sf_axial(G, pm, c, dzf, srcz, factor, trap, iz, a)) continue;
                            const double wv = (double)a.C * (double)C0;
                            for (int j = a.min_v; j <= a.max_v; ++j) {
                                const float f = sf_row(a, trap, j);
                                if (f != 0.f) atomicAdd(Aw + j, wv * (double)f);
                            }
                        }
                    }
                }
            }
        }
        if (l == 0) {
            s_act[w][0] = blo;
            s_act[w][1] = bhi;
        }
        __syncthreads();  // every warp's A and g of this batch
        for (int v = tid; v < nv; v += blockDim.x) {
#pragma unroll 1
            for (int q = 0; q < kFW; ++q) {
                const int b0 = s_act[q][0], b1 = s_act[q][1];
                if (b1 < b0) continue;
                const double av = A[q * nv + v];
                if (av == 0.0) continue;
                for (int b = b0; b <= b1; ++b) {
                    const float gv = cs[q * kUB + b];
                    if (gv != 0.f) acc[b * nv + v] = fma((double)gv, av, acc[b * nv + v]);
                }
            }
        }
        __syncthreads();  // before the warps overwrite A
    }
    for (int e = tid; e < nb * nv; e += blockDim.x) {
        const int v = e / nb, b = e - v * nb;
        proj[((size_t)p * nv + v) * G.nu + u0 + b] = (TOut)acc[b * nv + v];
    }
}

__host__ __device__ constexpr int sf_rows_padded(int nv) { return (nv + kRowBox - 1) / kRowBox * kRowBox; }

// 128 bytes of slack: the staging buffer is placed on a 128-byte boundary
__host__ __device__ constexpr size_t sf_back_smem(int nv) {
    return 128 + (size_t)2 * sf_rows_padded(nv) * kWin * 4 + (size_t)kTX * kTY * nv * 8 + 16;
}

// The exact transpose of sf3d_fwd_kernel.  use_tma: the projection is staged
// through `map` (a tensor map of proj, extents (nu, nv, np)); otherwise read
// from global memory.
template <typename TOut>
__global__ void __launch_bounds__(kTX * kTY * 32, 2) sf3d_back1_kernel(const __grid_constant__ CUtensorMap map,
                                                                    SFGeo G, SFPlan K, const float* __restrict__ proj,
                                                                    TOut* __restrict__ vol, int use_tma) {
    extern __shared__ __align__(128) unsigned char sf_bsmem[];
    const int nv = G.nv, nu = G.nu, nvp = sf_rows_padded(nv), nboxes = nvp / kRowBox;
    // [2][nvp][kWin], every TMA box (kRowBox rows of kWin floats) on a
    // 128-byte boundary
    float* stage = reinterpret_cast<float*>(sf_bsmem + ((128 - (smem_addr(sf_bsmem) & 127u)) & 127u));
    double* Bs = reinterpret_cast<double*>(stage + (size_t)2 * nvp * kWin);  // [warps][nv]
    uint64_t* bars = reinterpret_cast<uint64_t*>(Bs + kTX * kTY * nv);
    __shared__ int s_abort;
    const int tid = threadIdx.x, w = tid >> 5, l = tid & 31;
    const int tile = blockIdx.y * K.tiles_x + blockIdx.x;
    const int ix = blockIdx.x * kTX + (w % kTX), iy = blockIdx.y * kTY + (w / kTX);
    const bool col_ok = ix < G.nx && iy < G.ny;
    const int zbase = blockIdx.z * 32 * kZPer;
    const int* twin = K.twin + (size_t)tile * G.np;
    double* Bw = Bs + w * nv;
    const bool trap = G.trap != 0;
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
#pragma unroll
    for (int q = 0; q < kZPer; ++q) acc[q] = 0.0;
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
        const float* gp = proj + (size_t)p * nv * nu;
        const float* pm = G.pmi + 12 * (size_t)p;
        const double* src = G.src + 3 * (size_t)p;
        const float srczf = (float)src[2], factorf = (float)G.fwdf[p], dzf = (float)G.dz;
        SFCol c;
        if (col_ok && sf_column(G, pm, src, ix, iy, c)) {
            const int lo = max(c.min_u, 0), ncv = min(c.max_u, nu - 1) - lo + 1;
            // g of bin lo + l (lane l), then B(v) = sum_u g(u) proj(u, v), a
            // lane per row
            float gv = 0.f;
            if (l < ncv) {
                const int i = lo + l;
                gv = sf_gamma1(i - 0.5f, i + 0.5f, c.us);
                if (!(gv == gv)) gv = 0.f;
            }
            const int du0 = lo - ulo, q0 = du0 >> 2, sh = du0 & 3;
            if (ulo >= 0 && du0 >= 0 && ncv + sh <= 8 && 4 * q0 + 8 <= kWin) {
                // the column's bins lie in two 16-byte words of each staged
                // row, from word element sh on: B(v) = sum_t g_t row[4 q0 +
                // sh + t] over its ncv bins, FP64 sums of the FP32 products
                // (each exact in FP64; only the ncv elements are converted)
                double gd[8];
#pragma unroll
                for (int t = 0; t < 8; ++t) gd[t] = (double)__shfl_sync(0xffffffffu, gv, t);
                auto form = [&](auto shc) {
                    constexpr int SH = decltype(shc)::value;
                    for (int v = l; v < nv; v += 32) {
                        const float4* row = reinterpret_cast<const float4*>(sp + (size_t)v * kWin) + q0;
                        const float4 a = row[0], b4 = row[1];
                        const float e[8] = {a.x, a.y, a.z, a.w, b4.x, b4.y, b4.z, b4.w};
                        double b = 0.0;
#pragma unroll
                        for (int t = 0; t < 8 - SH; ++t)
                            if (t < ncv) b = fma(gd[t], (double)e[SH + t], b);
                        Bw[v] = b;
                    }
                };
                switch (sh) {
                    case 0: form(std::integral_constant<int, 0>{}); break;
                    case 1: form(std::integral_constant<int, 1>{}); break;
                    case 2: form(std::integral_constant<int, 2>{}); break;
                    default: form(std::integral_constant<int, 3>{}); break;
                }
            } else {
                // not in the staged window: global memory, a lane per row
                for (int v0 = 0; v0 < nv; v0 += 32) {  // uniform trip count: the shuffles need every lane
                    const int v = v0 + l;
                    double b = 0.0;
                    for (int t = 0; t < min(ncv, 32); ++t) {
                        const float ct = __shfl_sync(0xffffffffu, gv, t);
                        if (ct != 0.f && v < nv) b = fma((double)ct, (double)__ldg(gp + (size_t)v * nu + lo + t), b);
                    }
                    if (v < nv) Bw[v] = b;
                }
                if (ncv > 32) {  // columns wider than a warp (near the source): the rest
                    for (int v = l; v < nv; v += 32) {
                        double b = Bw[v];
                        for (int t = 32; t < ncv; ++t) {
                            const int i = lo + t;
                            const float ct = sf_gamma1(i - 0.5f, i + 0.5f, c.us);
                            if (ct == ct && ct != 0.f) b = fma((double)ct, (double)__ldg(gp + (size_t)v * nu + i), b);
                        }
                        Bw[v] = b;
                    }
                }
            }
            __syncwarp();
#pragma unroll
            for (int q = 0; q < kZPer; ++q) {
                const int iz = zbase + 32 * q + l;
                SFAx a;
                if (iz >= G.nz || !sf_axial(G, pm, c, dzf, srczf, factorf, trap, iz, a)) continue;
                double val = 0.0;
                for (int j = a.min_v; j <= a.max_v; ++j) val = fma((double)sf_row(a, trap, j), Bw[j], val);
                const double s = val * (double)a.C;
                if (s == s) acc[q] += s;
            }
        }
        __syncthreads();  // buffer p & 1 fully read
        if (tid == 0 && p + 2 < G.np) issue(p + 2);
    }
    if (!col_ok) return;
    const size_t plane = (size_t)G.nx * G.ny;
#pragma unroll
    for (int q = 0; q < kZPer; ++q) {
        const int iz = zbase + 32 * q + l;
        if (iz < G.nz) vol[(size_t)iz * plane + (size_t)iy * G.nx + ix] = (TOut)acc[q];
    }
}

}  // namespace

class SF3D {
public:
    SFGeo G{};
    SFPlan K{};
    int device = 0;
    cudaStream_t stream = nullptr;

    SF3D(int mode, int trap, int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy, double dz, double du,
         double dv, double lsd, double lso, const double* angles) {
        if (nx <= 0 || ny <= 0 || nz <= 0 || np <= 0 || nu <= 0 || nv <= 0) fail("invalid sizes");
        check_pitches({dx, dy, dz, du, dv});
        check_distances(lsd, lso);
        check_views(np, angles, nullptr, nullptr);
        SGD_CUDA(cudaGetDevice(&device));
        SGD_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        const std::vector<ViewFrame> fr = view_frames(np, lsd, lso, du, dv, angles, nullptr, nullptr);
        std::vector<float> pmi((size_t)np * 12);
        std::vector<double> src((size_t)np * 3), fwdf(np);
        for (int p = 0; p < np; ++p) {
            double pm[12];
            // mode 0 keeps the reference's matrices, degenerate views included;
            // the corrected pair projects through the exact ones
            if (mode == 0) reference_pmi(fr[p], nu / 2.0, nv / 2.0, nx, ny, nz, dx, dy, dz, pm, &pmi[12 * (size_t)p]);
            else exact_pmi(fr[p], nu / 2.0, nv / 2.0, nx, ny, nz, dx, dy, dz, &pmi[12 * (size_t)p]);
            for (int k = 0; k < 3; ++k) src[3 * p + k] = fr[p].src[k];
            const float flsd = (float)lsd;  // SF::project: float lsd (:362)
            // the reference's factor lsd^2 dy dz / (du dv) (:364) lacks the
            // voxel's third side: the corrected pair multiplies it in, so
            // that its forward carries the voxel's line integrals for any dx
            fwdf[p] = flsd * flsd * dy * dz / (du * dv) * (mode == 1 ? dx : 1.0);
        }
        SGD_CUDA(cudaMalloc(&d_pmi_, pmi.size() * sizeof(float)));
        SGD_CUDA(cudaMemcpy(d_pmi_, pmi.data(), pmi.size() * sizeof(float), cudaMemcpyHostToDevice));
        SGD_CUDA(cudaMalloc(&d_src_, src.size() * sizeof(double)));
        SGD_CUDA(cudaMemcpy(d_src_, src.data(), src.size() * sizeof(double), cudaMemcpyHostToDevice));
        SGD_CUDA(cudaMalloc(&d_fwdf_, fwdf.size() * sizeof(double)));
        SGD_CUDA(cudaMemcpy(d_fwdf_, fwdf.data(), fwdf.size() * sizeof(double), cudaMemcpyHostToDevice));
        G = SFGeo{nx, ny, nz, np, nu, nv, trap, mode, dx, dy, dz, d_pmi_, d_src_, d_fwdf_,
                  (double)(float)lsd * dx / np};
        const size_t nvol = (size_t)nx * ny * nz, nproj = (size_t)np * nu * nv;
        if (mode == 1) {
            plan(pmi);
            SGD_CUDA(cudaMalloc(&d_volT_, nvol * sizeof(float)));
        } else {
            SGD_CUDA(cudaMalloc(&d_proj64_, nproj * sizeof(double)));
        }
        SGD_CUDA(cudaMalloc(&d_err_, sizeof(int)));
        SGD_CUDA(cudaMemset(d_err_, 0, sizeof(int)));
        K.err = d_err_;
        K.wait_limit = 1u << 22;
        SGD_CUDA(cudaMalloc(&d_vol_, nvol * sizeof(float)));
        SGD_CUDA(cudaMalloc(&d_proj_, nproj * sizeof(float)));
        SGD_CUDA(cudaMallocHost(&h_vol_, nvol * sizeof(float)));
        SGD_CUDA(cudaMallocHost(&h_proj_, nproj * sizeof(float)));
    }
    ~SF3D() {
        if (stream) cudaStreamSynchronize(stream);
        cudaFree(d_pmi_); cudaFree(d_src_); cudaFree(d_fwdf_); cudaFree(d_proj64_); cudaFree(d_vol64_);
        cudaFree(d_volT_);
        cudaFree(d_strips_); cudaFree(d_twin_); cudaFree(d_err_);
        cudaFree(d_vol_); cudaFree(d_proj_); cudaFreeHost(h_vol_); cudaFreeHost(h_proj_);
        if (stream) cudaStreamDestroy(stream);
    }
    // FP64 host arrays x[(iz*ny + iy)*nx + ix], b[(p*nv + v)*nu + u]: the
    // inputs are rounded to FP32 as the reference's SF class does; mode 1
    // returns its FP64 accumulators, mode 0 rounds its output to FP32 as the
    // reference does
    void forward_host(double* b, const double* x) {
        const long long nvol = (long long)G.nx * G.ny * G.nz, nproj = (long long)G.np * G.nu * G.nv;
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < nvol; ++e) h_vol_[e] = (float)x[e];
        SGD_CUDA(cudaMemcpyAsync(d_vol_, h_vol_, nvol * sizeof(float), cudaMemcpyHostToDevice, stream));
        if (G.mode == 1) {
            ensure_fp64();
            forward1(d_vol_, d_proj64_, stream);
            SGD_CUDA(cudaMemcpyAsync(b, d_proj64_, nproj * sizeof(double), cudaMemcpyDeviceToHost, stream));
            SGD_CUDA(cudaStreamSynchronize(stream));
            return;
        }
        forward_dev(d_vol_, d_proj_, stream);
        SGD_CUDA(cudaMemcpyAsync(h_proj_, d_proj_, nproj * sizeof(float), cudaMemcpyDeviceToHost, stream));
        SGD_CUDA(cudaStreamSynchronize(stream));
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < nproj; ++e) b[e] = (double)h_proj_[e];
    }
    void backward_host(const double* b, double* x) {
        const long long nvol = (long long)G.nx * G.ny * G.nz, nproj = (long long)G.np * G.nu * G.nv;
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < nproj; ++e) h_proj_[e] = (float)b[e];
        SGD_CUDA(cudaMemcpyAsync(d_proj_, h_proj_, nproj * sizeof(float), cudaMemcpyHostToDevice, stream));
        if (G.mode == 1) {
            ensure_fp64();
            back1(d_proj_, d_vol64_, stream);
            SGD_CUDA(cudaMemcpyAsync(x, d_vol64_, nvol * sizeof(double), cudaMemcpyDeviceToHost, stream));
        } else {
            backward_dev(d_proj_, d_vol_, stream);
            SGD_CUDA(cudaMemcpyAsync(h_vol_, d_vol_, nvol * sizeof(float), cudaMemcpyDeviceToHost, stream));
        }
        int e = 0;
        SGD_CUDA(cudaMemcpyAsync(&e, d_err_, sizeof(int), cudaMemcpyDeviceToHost, stream));
        SGD_CUDA(cudaStreamSynchronize(stream));
        if (e) {
            SGD_CUDA(cudaMemset(d_err_, 0, sizeof(int)));
            fail("SF_projector back projection: a staged view did not arrive within the bounded wait; output incomplete");
        }
        if (G.mode == 1) return;
#pragma omp parallel for schedule(static)
        for (long long e2 = 0; e2 < nvol; ++e2) x[e2] = (double)h_vol_[e2];
    }
    // vol [z][y][x], proj [p][v][u], FP32 device
    void forward_dev(const float* vol, float* proj, cudaStream_t s) {
        if (G.mode == 1) {
            forward1(vol, proj, s);
            return;
        }
        const long long n = (long long)G.np * G.nu * G.nv;
        SGD_CUDA(cudaMemsetAsync(d_proj64_, 0, n * sizeof(double), s));
        const int chunks = (G.nz + kSFZ - 1) / kSFZ;
        dim3 grid((G.nx + 15) / 16, (G.ny + 7) / 8, G.np * chunks);
        sf3d_forward_kernel<float><<<grid, dim3(16, 8), 0, s>>>(G, vol, d_proj64_);
        SGD_LAUNCH_CHECK();
        sf3d_finish_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d_proj64_, proj, n);
        SGD_LAUNCH_CHECK();
    }
    void backward_dev(const float* proj, float* vol, cudaStream_t s) {
        if (G.mode == 1) {
            back1(proj, vol, s);
            return;
        }
        dim3 grid((G.nx + 15) / 16, (G.ny + 7) / 8, G.nz);
        sf3d_back_kernel<float, float><<<grid, dim3(16, 8), 0, s>>>(G, proj, vol);
        SGD_LAUNCH_CHECK();
    }
    // 0, or -1 when a back projection's staging wait gave up (those voxels
    // were left unwritten); synchronises the device and clears the flag
    int status() {
        int h = 0;
        SGD_CUDA(cudaDeviceSynchronize());
        SGD_CUDA(cudaMemcpy(&h, d_err_, sizeof(int), cudaMemcpyDeviceToHost));
        SGD_CUDA(cudaMemset(d_err_, 0, sizeof(int)));
        return h ? -1 : 0;
    }
    void set_wait_limit(unsigned limit) {
        SGD_CUDA(cudaStreamSynchronize(stream));
        K.wait_limit = limit;
    }

private:
    // mode 1: the column copy and the factored forward
    template <typename TOut>
    void forward1(const float* vol, TOut* proj, cudaStream_t s) {
        launch_to_columns(vol, d_volT_, G.nx, G.ny, G.nz, s);
        SGD_LAUNCH_CHECK();
        sf3d_fwd_kernel<TOut><<<dim3(K.nblk, G.np), kFW * 32, sf_fwd_smem(G.nv), s>>>(G, K, d_volT_, proj);
        SGD_LAUNCH_CHECK();
    }
    // mode 1: the projection through TMA tensor loads when its rows are whole
    // 16-byte words and it is 16-byte aligned; from global memory otherwise
    template <typename TOut>
    void back1(const float* proj, TOut* vol, cudaStream_t s) {
        const bool tma = (G.nu % 4) == 0 && (reinterpret_cast<uintptr_t>(proj) % 16) == 0;
        CUtensorMap map;
        std::memset(&map, 0, sizeof(map));
        if (tma) map = encode_tensor_3d_f32(proj, (uint64_t)G.nu, (uint64_t)G.nv, (uint64_t)G.np, kWin, kRowBox, 1);
        const dim3 grid(K.tiles_x, K.tiles_y, (G.nz + 32 * kZPer - 1) / (32 * kZPer));
        sf3d_back1_kernel<TOut><<<grid, kTX * kTY * 32, sf_back_smem(G.nv), s>>>(map, G, K, proj, vol, tma ? 1 : 0);
        SGD_LAUNCH_CHECK();
    }
    void ensure_fp64() {
        const size_t nvol = (size_t)G.nx * G.ny * G.nz, nproj = (size_t)G.np * G.nu * G.nv;
        if (!d_proj64_) SGD_CUDA(cudaMalloc(&d_proj64_, nproj * sizeof(double)));
        if (!d_vol64_) SGD_CUDA(cudaMalloc(&d_vol64_, nvol * sizeof(double)));
    }
    // Mode 1's launch tables.  The in-plane footprint of column (i, j) in
    // view p spans u' in the image of its corners (i +- 1/2, j +- 1/2) under
    // u' = (pm0 i + pm1 j + pm3) / (pm8 i + pm9 j + pm11), bins are
    // [b - 1/2, b + 1/2]: as a range map with floor(u) = bin that is u' + 1/2
    // with radii 1/2.  The forward's block strips come from it (blocks of kUB
    // bins), and per back tile of kTX x kTY columns and view the first bin of
    // its staged window (a multiple of 4 for the TMA box), -1 when its bins
    // span more than kWin.
    void plan(const std::vector<float>& pmi) {
        const int nx = G.nx, ny = G.ny, np = G.np, nu = G.nu, nv = G.nv;
        if (nx > kMaxLines || ny > kMaxLines) fail("SF_projector: %d x %d columns exceed %d per line", nx, ny, kMaxLines);
        if (sf_fwd_smem(nv) > 227 * 1024 || sf_back_smem(nv) > 227 * 1024)
            fail("SF_projector: %d detector rows do not fit the kernels' shared memory", nv);
        for (int p = 0; p < np; ++p)
            if (pmi[12 * (size_t)p + 2] != 0.f || pmi[12 * (size_t)p + 10] != 0.f)
                fail("SF_projector: view %d's u row depends on z (not a circular orbit)", p);
        auto map = [&](int p) {
            const float* q = &pmi[12 * (size_t)p];
            RangeMap m;
            m.h[0] = (double)q[0] + 0.5 * q[8];
            m.h[1] = (double)q[1] + 0.5 * q[9];
            m.h[2] = (double)q[3] + 0.5 * q[11];
            m.h[3] = q[8];
            m.h[4] = q[9];
            m.h[5] = q[11];
            m.ri = 0.5;
            m.rj = 0.5;
            return m;
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
                    const double i0 = tx * kTX - m.ri, i1 = std::min(nx, (tx + 1) * kTX) - 1 + m.ri;
                    const double j0 = ty * kTY - m.rj, j1 = std::min(ny, (ty + 1) * kTY) - 1 + m.rj;
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
                    if (hi < lo) continue;
                    const int ulo = lo & ~3;
                    if (hi - ulo + 1 <= kWin) twin[((size_t)ty * K.tiles_x + tx) * np + p] = ulo;
                }
        }
        SGD_CUDA(cudaMalloc(&d_strips_, strips.size() * sizeof(float4)));
        SGD_CUDA(cudaMemcpy(d_strips_, strips.data(), strips.size() * sizeof(float4), cudaMemcpyHostToDevice));
        SGD_CUDA(cudaMalloc(&d_twin_, twin.size() * sizeof(int)));
        SGD_CUDA(cudaMemcpy(d_twin_, twin.data(), twin.size() * sizeof(int), cudaMemcpyHostToDevice));
        K.strips = d_strips_;
        K.twin = d_twin_;
        SGD_CUDA(cudaFuncSetAttribute(sf3d_fwd_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sf_fwd_smem(nv)));
        SGD_CUDA(cudaFuncSetAttribute(sf3d_fwd_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sf_fwd_smem(nv)));
        SGD_CUDA(cudaFuncSetAttribute(sf3d_back1_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sf_back_smem(nv)));
        SGD_CUDA(cudaFuncSetAttribute(sf3d_back1_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sf_back_smem(nv)));
    }
    float* d_pmi_ = nullptr;
    double* d_src_ = nullptr;
    double* d_fwdf_ = nullptr;
    double* d_proj64_ = nullptr;
    double* d_vol64_ = nullptr;
    float* d_volT_ = nullptr;
    float4* d_strips_ = nullptr;
    int* d_twin_ = nullptr;
    int* d_err_ = nullptr;
    float* d_vol_ = nullptr;
    float* d_proj_ = nullptr;
    float* h_vol_ = nullptr;
    float* h_proj_ = nullptr;
};

}  // namespace sgd

extern "C" {

void* sgd_sf3d_init(int mode, int trap_v, int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy,
                    double dz, double du, double dv, double lsd, double lso, double* angles) {
    return sgd::guarded<void*>(nullptr, [&]() -> void* {
        if (mode != 0 && mode != 1) sgd::fail("sgd_sf3d_init: mode must be 0 or 1");
        return new sgd::SF3D(mode, trap_v, nx, ny, nz, np, nu, nv, dx, dy, dz, du, dv, lsd, lso, angles);
    });
}
void sgd_sf3d_destroy(void* layer) { delete static_cast<sgd::SF3D*>(layer); }
int sgd_sf3d_forward_dev(void* layer, const float* d_vol, float* d_proj, void* stream) {
    return sgd::guarded_status([&] {
        if (!layer || !d_vol || !d_proj) sgd::fail("sgd_sf3d_forward_dev: null argument");
        static_cast<sgd::SF3D*>(layer)->forward_dev(d_vol, d_proj, static_cast<cudaStream_t>(stream));
    });
}
int sgd_sf3d_forward_projection(double* b, double* x, void* layer) {
    return sgd::guarded_status([&] {
        if (!layer || !b || !x) sgd::fail("sgd_sf3d_forward_projection: null argument");
        static_cast<sgd::SF3D*>(layer)->forward_host(b, x);
    });
}
int sgd_sf3d_backward_projection(double* b, double* x, void* layer) {
    return sgd::guarded_status([&] {
        if (!layer || !b || !x) sgd::fail("sgd_sf3d_backward_projection: null argument");
        static_cast<sgd::SF3D*>(layer)->backward_host(b, x);
    });
}
int sgd_sf3d_backward_dev(void* layer, const float* d_proj, float* d_vol, void* stream) {
    return sgd::guarded_status([&] {
        if (!layer || !d_vol || !d_proj) sgd::fail("sgd_sf3d_backward_dev: null argument");
        static_cast<sgd::SF3D*>(layer)->backward_dev(d_proj, d_vol, static_cast<cudaStream_t>(stream));
    });
}
int sgd_sf3d_status(void* layer) {
    return sgd::guarded_status([&] {
        if (!layer) sgd::fail("sgd_sf3d_status: null layer");
        if (static_cast<sgd::SF3D*>(layer)->status() != 0)
            sgd::fail("SF_projector back projection: a staged view did not arrive within the bounded wait; "
                      "the affected voxels were left unwritten");
    });
}
int sgd_sf3d_set_wait_limit(void* layer, unsigned limit) {
    return sgd::guarded_status([&] {
        if (!layer) sgd::fail("sgd_sf3d_set_wait_limit: null layer");
        static_cast<sgd::SF3D*>(layer)->set_wait_limit(limit);
    });
}

}  // extern "C"
