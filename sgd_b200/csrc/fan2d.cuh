// Generic 2D fan-beam projector kernels, parameterised by a footprint basis.
//
// A basis B supplies, for cell (i, j) of the grid and view p:
//   B::kViewFloats          per-view constants (a multiple of 4 floats)
//   B::kBinF4               float4 words per (view, bin) in the basis table
//                           P.bins (0: no table), stored as kBinF4 planes of
//                           nu words per view ([view][word][bin]) so that
//                           lanes on neighbouring bins read neighbouring
//                           16-byte words of shared memory
//   B::View, B::Cell        per-view constants; per-(cell, view) state with the
//                           bin range [lo, hi] (the reference's rule, clamped
//                           to the detector as the reference clamps it)
//   B::load_view(v, V)      from shared or global memory
//   B::valid(i, j, P)       whether (i, j) is a cell of the grid
//   B::setup(V, i, j, P, c)
//   B::value(V, c, u, t, P) footprint in bin u (0 where the reference drops
//                           it), t = the bin's table entry (t[k]: word k, a
//                           BinRef over the planes); bins are walked in
//                           order from c.lo, each by value() or skip(), which
//                           lets a basis step its bin position as the
//                           reference does
//   B::skip(V, c)           steps past a bin without evaluating it
//   B::start(V, c, u)       before the first bin u a walk evaluates
// The forward's strips and the back's windows come from each cell's true
// footprint (plan_fan2d, proj2d.h); a bin outside it has footprint exactly 0.
// So both kernels evaluate every (cell, bin) pair with a non-zero value and
// u in [lo, hi] (the pairs the reference keeps) through the same functions;
// sums run in FP32 over the few terms of a lane's lines in one bin (fused
// multiply-adds) and, in the back projection, compensated over a cell's bins
// in a chunk of views (exact products), then in FP64, so the pair is an
// adjoint pair well below 1e-6 even on heavily cancelling Gaussian inputs.
//
//   fan2d_forward_kernel  detector-block driven: a single-warp CTA per (view,
//                         block of 32 bins, part of the block's lines).  The
//                         block's ray strip is crossed by the lines of the
//                         grid's major axis; each lane owns lines and walks
//                         the few cells of its line inside the strip
//                         (host-computed strip records), adding each value to
//                         its own FP32 shared-memory column of the block's
//                         bins.  Neighbouring lanes own neighbouring lines and
//                         read the image (j-major strips) or its transposed
//                         copy (i-major) at neighbouring addresses.  The
//                         columns are summed across lanes in FP64 and each
//                         part's sums written once; fan2d_forward_sum_kernel
//                         adds the parts in order: no atomics, and no warp
//                         waits for another at a barrier.
//   fan2d_back_kernel     voxel driven: a CTA per tile of cells, a thread per
//                         cell.  Per chunk of kF2Views views warp 0 stages the
//                         view constants and the tile's window of the basis
//                         table by bulk asynchronous copies (TMA) into a ring
//                         of kF2Stages slots, with full/empty mbarriers per
//                         slot instead of CTA barriers; the sinogram is read
//                         through the read-only cache.  Each thread
//                         accumulates over all views in registers and writes
//                         its cell once.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "fan2d_params.h"
#include "tma.cuh"

namespace sgd {

constexpr uint32_t kF2WaitLimit = 1u << 22;

// a * b + c * d with the first product fused: the contraction the compiler
// picks for that source form, written out so that every kernel (and the
// system-matrix visitor) that inlines a basis forms the same bits.  The
// forward and back projections are transposes of each other only if they
// evaluate identical values.
__device__ __forceinline__ float dot2f(float a, float b, float c, float d) { return __fmaf_rn(a, b, __fmul_rn(c, d)); }

// x within |x| 2^-21 (4 ulp) plus 2^-22 of an integer: a fast quotient x
// (within 2 ulp of the IEEE one) and the IEEE quotient may then have
// different floors.  Bases whose bin ranges are the reference's floors of
// IEEE quotients take fast quotients and fall back to IEEE division where
// this holds (about one extreme in 2000 at bin indices of a few hundred).
__device__ __forceinline__ bool near_integer(float x) {
    const float f = x - floorf(x), tol = __fmaf_rn(fabsf(x), 0x1p-21f, 0x1p-22f);
    return f < tol || f > 1.0f - tol;
}

// One bin's entry of a basis table held as planes: word k at p[k * stride].
struct BinRef {
    const float4* p;
    int stride;
    __device__ __forceinline__ float4 operator[](int k) const { return p[k * stride]; }
};

// Compensated (Kahan) FP32 accumulation: s holds the sum, c the part of it
// that is rounding error (true sum = s - c), four FP32 operations per term
// and no conversions.  Written with round-to-nearest intrinsics so that the
// compiler can neither fuse nor reassociate them.
__device__ __forceinline__ void kahan_add(float& s, float& c, float x) {
    const float y = __fsub_rn(x, c);
    const float t = __fadd_rn(s, y);
    c = __fsub_rn(__fsub_rn(t, s), y);
    s = t;
}

// s - c += a * b with the product exact: its rounding error (one fused
// multiply-add) joins the compensation.  Forward and back then round no
// product differently, and the pair stays an adjoint pair to FP64 level.
__device__ __forceinline__ void kahan_fma(float& s, float& c, float a, float b) {
    const float p = __fmul_rn(a, b);
    const float e = __fmaf_rn(a, b, -p);
    kahan_add(s, c, p);
    c = __fsub_rn(c, e);
}

// Forward block strips (host: plan_fan2d, proj2d.h).  For block k of view p,
// along the major axis m the block's two bounding rays cross the minor axis
// at alpha_a + beta_a m and alpha_b + beta_b m; candidate cells lie within
// `margin` of the span between them.  s0 = (j_major, alpha_a, beta_a,
// alpha_b), s1 = (beta_b, margin, first line, last line).
//
// One warp per (block, view, part): part q takes the block's lines first +
// 32 q + lane + 32 kF2FwdParts t.  A warp that runs out of lines retires
// and frees its slot; nothing waits for the other parts, whose FP64 sums
// fan2d_forward_sum_kernel adds in part order.
template <class B>
__global__ void __launch_bounds__(32, 32) fan2d_forward_kernel(Fan2DParams P, const float* __restrict__ img) {
    constexpr int kBF4 = B::kBinF4 > 0 ? B::kBinF4 : 1;
    // each lane's FP32 column of the block's bins over its lines (a few terms
    // per bin), summed across lanes in FP64
    __shared__ float s_acc[kF2Block][33];
    __shared__ float4 s_bin[kBF4 * kF2Block];  // [word][bin of the block]
    __shared__ __align__(16) float s_view[B::kViewFloats];
    const int k = blockIdx.x, p = blockIdx.y, q = blockIdx.z;
    const int u0 = k * kF2Block, nb = min(kF2Block, P.nu - u0);
    const int l = threadIdx.x;
    for (int e = l; e < B::kViewFloats; e += 32) s_view[e] = __ldg(P.view + (size_t)p * B::kViewFloats + e);
    if (B::kBinF4 > 0)
        for (int e = l; e < nb * B::kBinF4; e += 32) {
            const int k = e / nb, b = e - k * nb;
            s_bin[k * kF2Block + b] = __ldg(P.bins + ((size_t)p * B::kBinF4 + k) * P.nu + u0 + b);
        }
    for (int e = l; e < kF2Block * 33; e += 32) (&s_acc[0][0])[e] = 0.f;
    __syncwarp();

    typename B::View V;
    B::load_view(s_view, V);
    const float4* st = P.strips + ((size_t)p * P.nblk + k) * 2;
    const float4 s0 = __ldg(st), s1 = __ldg(st + 1);
    const bool jmaj = s0.x > 0.5f;
    const int nmin = jmaj ? P.ni : P.nj;
    const int mlo = (int)s1.z, mhi = (int)s1.w;
    // cell (m, n) of line m: lanes own consecutive lines, so that j-major
    // strips read the image and i-major ones its transposed copy coalesced
    const int nmaj = jmaj ? P.nj : P.ni;
    const float* src = jmaj ? img : P.imgT;
    float* acc = &s_acc[0][l];  // bin b at acc[33 b]: this lane's column
    for (int m = mlo + 32 * q + l; m <= mhi; m += 32 * kF2FwdParts) {
        const float fm = (float)m;
        const float na = fmaf(s0.z, fm, s0.y), nbb = fmaf(s1.x, fm, s0.w);
        const int nlo = max(0, (int)ceilf(fminf(na, nbb) - s1.y));
        const int nhi = min(nmin - 1, (int)floorf(fmaxf(na, nbb) + s1.y));
        for (int n = nlo; n <= nhi; ++n) {
            const int i = jmaj ? n : m, j = jmaj ? m : n;
            if (!B::valid(i, j, P)) continue;
            const float C = __ldg(src + (size_t)n * nmaj + m);
            if (C == 0.f) continue;
            typename B::Cell c;
            B::setup(V, i, j, P, c);
            if (c.hi < u0 || c.lo >= u0 + nb) continue;
            const int ue = min(c.hi, u0 + nb - 1);
            int u = c.lo;
            for (; u < u0; ++u) B::skip(V, c);
            B::start(V, c, u);
            for (; u <= ue; ++u) {
                // a dropped bin's value is 0: adding 0 * C leaves the column as
                // it is (for a finite image value)
                const float v = B::value(V, c, u, BinRef{s_bin + (u - u0), kF2Block}, P);
                acc[33 * (u - u0)] = fmaf(v, C, acc[33 * (u - u0)]);
            }
        }
    }
    __syncwarp();
    if (l < nb) {
        double t = 0.0;
        for (int r = 0; r < 32; ++r) t += (double)s_acc[l][r];
        P.part[((size_t)q * P.np + p) * P.nu + u0 + l] = t;
    }
}

// sino (or out64) = scale * the sum of the forward's parts, in part order
static __global__ void fan2d_forward_sum_kernel(Fan2DParams P, float* __restrict__ sino, float scale) {
    const size_t n = (size_t)P.np * P.nu;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        double t = 0.0;
#pragma unroll
        for (int q = 0; q < kF2FwdParts; ++q) t += P.part[q * n + e];
        if (P.out64) P.out64[e] = t * (double)scale;
        else sino[e] = (float)t * scale;
    }
}

// in [rows][cols] -> out [cols][rows] (the forward's line-major image copy)
static __global__ void fan2d_transpose_kernel(const float* __restrict__ in, float* __restrict__ out, int rows,
                                              int cols) {
    __shared__ float t[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        if (r < rows && c < cols) t[k][threadIdx.x] = in[(size_t)r * cols + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (r < rows && c < cols) out[(size_t)c * rows + r] = t[threadIdx.x][k];
    }
}

// Shared memory of the back kernel: mbarriers full[S], empty[S] | view
// constants [S][VC][kViewFloats] | tables [S][VC][kBinF4][wcap] float4.
template <class B, int VC, int S>
__host__ __device__ constexpr size_t fan2d_back_header() {
    return (size_t)2 * S * 8 + (size_t)S * VC * B::kViewFloats * 4;
}
template <class B, int VC, int S>
__host__ __device__ constexpr size_t fan2d_back_smem(int wcap) {
    return fan2d_back_header<B, VC, S>() + (size_t)S * VC * wcap * (B::kBinF4 * 16);
}

// The back projection's staging ring: chunk c (views c VC .. c VC + VC - 1)
// lives in slot c % S.  Warp 0 stages chunk c + S - 2 when it starts chunk c
// (after every warp has released that slot's previous chunk, c - 2); each warp
// waits for its chunk's copies on full[slot] and releases the slot on
// empty[slot] when done.  No warp waits for the others at a CTA barrier: the
// warps of a tile drift apart by up to S - 1 chunks, so that a chunk's uneven
// work (cells' bin counts differ per view) evens out over several chunks.
template <class B, int VC, int S>
__global__ void __launch_bounds__(kF2BackThreads) fan2d_back_kernel(Fan2DParams P, const float* __restrict__ sino,
                                                                    float* __restrict__ img, float scale) {
    static_assert(B::kViewFloats % 4 == 0, "view rows must be whole 16-byte words");
    static_assert(fan2d_back_header<B, VC, S>() % 16 == 0, "staged tables must start 16-byte aligned");
    static_assert(S >= 3 && VC <= 32, "the ring needs three slots; a lane per view of a chunk");
    extern __shared__ __align__(16) unsigned char f2_smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(f2_smem);                          // [S]
    uint64_t* empty = full + S;                                                       // [S]
    float* sview = reinterpret_cast<float*>(f2_smem + 2 * S * 8);                     // [S][VC][kViewFloats]
    float4* sbin = reinterpret_cast<float4*>(f2_smem + fan2d_back_header<B, VC, S>());  // [S][VC][kBinF4][wcap]
    __shared__ int s_abort;

    const int tid = threadIdx.x, w = tid >> 5, l = tid & 31;
    const int tile = blockIdx.y * P.tiles_j + blockIdx.x;
    const int i = blockIdx.y * kF2TileI + w, j = blockIdx.x * kF2TileJ + l;
    const bool mine = i < P.ni && j < P.nj && B::valid(i, j, P);
    const int2* twin = P.twin + (size_t)tile * P.np;
    const int nchunks = (P.np + VC - 1) / VC;

    if (tid == 0) {
        for (int k = 0; k < S; ++k) {
            mbar_init(&full[k], 1);
            mbar_init(&empty[k], kF2TileI);  // one arrival per warp
        }
        fence_mbar_init();
        s_abort = 0;
    }
    __syncthreads();

    // warp 0: stage chunk n into slot n % S, lane v taking view v (view
    // constants and table window by bulk copies, completed on full[slot]).
    // For n >= S the slot's previous chunk n - S must have been released by
    // every warp first.  Returns false when that wait gives up.
    auto stage = [&](int n) -> bool {
        const int slot = n % S;
        if (n >= S) {
            // every lane acquires the release itself before its copies overwrite the slot
            const bool ok = mbar_wait_bounded(&empty[slot], (uint32_t)(n / S - 1) & 1u, P.wait_limit);
            if (!__all_sync(0xffffffffu, ok)) return false;
        }
        const int p = n * VC + l;
        int2 lh = make_int2(0, -1);
        uint32_t bytes = 0;
        if (l < VC && p < P.np) {
            lh = __ldg(twin + p);
            bytes = B::kViewFloats * 4;
            if (B::kBinF4 > 0 && lh.y >= lh.x) bytes += (uint32_t)(lh.y - lh.x + 1) * B::kBinF4 * 16;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
        if (l == 0) mbar_arrive_expect_tx(&full[slot], bytes);
        __syncwarp();
        if (l < VC && p < P.np) {
            fence_proxy_async_smem();
            bulk_copy_g2s(sview + (slot * VC + l) * B::kViewFloats, P.view + (size_t)p * B::kViewFloats,
                          B::kViewFloats * 4, &full[slot]);
            if (B::kBinF4 > 0 && lh.y >= lh.x)
                for (int k = 0; k < B::kBinF4; ++k)
                    bulk_copy_g2s(sbin + ((size_t)(slot * VC + l) * B::kBinF4 + k) * P.wcap,
                                  P.bins + ((size_t)p * B::kBinF4 + k) * P.nu + lh.x,
                                  (uint32_t)(lh.y - lh.x + 1) * 16, &full[slot]);
        }
        return true;
    };

    int staged = 0;  // warp 0: chunks staged so far
    if (w == 0)
        for (; staged < min(S - 2, nchunks); ++staged) stage(staged);
    double acc = 0.0;
    for (int c = 0; c < nchunks; ++c) {
        if (*(volatile int*)&s_abort) break;
        if (w == 0 && c + S - 2 < nchunks) {
            if (!stage(c + S - 2)) {
                if (l == 0) {
                    s_abort = 1;
                    if (P.err) atomicExch(P.err, 1);
                }
                break;
            }
            staged = c + S - 1;
        }
        const int slot = c % S;
        if (!mbar_wait_bounded(&full[slot], (uint32_t)(c / S) & 1u, P.wait_limit)) {
            s_abort = 1;
            if (P.err) atomicExch(P.err, 1);
            break;
        }
        if (mine) {
            // a compensated FP32 sum within a chunk of views, FP64 across chunks
            float csum = 0.f, ccmp = 0.f;
#pragma unroll 1
            for (int v = 0; v < VC; ++v) {
                const int p = c * VC + v;
                if (p >= P.np) break;
                const int2 lh = __ldg(twin + p);
                if (lh.y < lh.x) continue;
                typename B::View V;
                B::load_view(sview + (slot * VC + v) * B::kViewFloats, V);
                typename B::Cell cl;
                B::setup(V, i, j, P, cl);
                if (cl.hi < lh.x || cl.lo > lh.y) continue;
                const float4* tb = sbin + (size_t)(slot * VC + v) * P.wcap * B::kBinF4 - lh.x;
                const float* sb = sino + (size_t)p * P.nu;
                const int ue = min(cl.hi, lh.y);
                int u = cl.lo;
                for (; u < lh.x; ++u) B::skip(V, cl);
                B::start(V, cl, u);
                for (; u <= ue; ++u) {
                    // (a dropped bin's 0 adds nothing: s - c stays as it is)
                    kahan_fma(csum, ccmp, B::value(V, cl, u, BinRef{tb + u, P.wcap}, P), __ldg(sb + u));
                }
            }
            acc += (double)csum - (double)ccmp;
        }
        __syncwarp();
        if (l == 0) mbar_arrive(&empty[slot]);
    }
    __syncthreads();
    if (s_abort) {
        // copies that may still be landing: the last chunk staged into each
        // slot (a chunk whose phase already completed passes at once).  The
        // tile is left unwritten.
        if (w == 0 && l < S) {
            const int n = staged - 1 - ((staged - 1 - l) % S + S) % S;  // the last staged chunk in slot l
            if (staged > 0 && n >= 0 && n % S == l) mbar_wait_bounded(&full[l], (uint32_t)(n / S) & 1u, kF2WaitLimit);
        }
        return;
    }
    if (i < P.ni && j < P.nj) {
        if (P.out64) P.out64[(size_t)i * P.nj + j] = mine ? acc * (double)scale : 0.0;
        else img[(size_t)i * P.nj + j] = mine ? (float)acc * scale : 0.f;
    }
}

// The reference's footprint-evaluation count: sum over cells and views of the
// width of the (clamped) bin range.  One atomic per warp.
template <class B>
__global__ void fan2d_count_kernel(Fan2DParams P, unsigned long long* out) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long n = 0;
    if (idx < (long long)P.ni * P.nj) {
        const int i = (int)(idx / P.nj), j = (int)(idx - (long long)i * P.nj);
        if (B::valid(i, j, P))
            for (int p = 0; p < P.np; ++p) {
                typename B::View V;
                B::load_view(P.view + (size_t)p * B::kViewFloats, V);
                typename B::Cell c;
                B::setup(V, i, j, P, c);
                if (c.hi >= c.lo) n += (unsigned long long)(c.hi - c.lo + 1);
            }
    }
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(out, n);
}

}  // namespace sgd
