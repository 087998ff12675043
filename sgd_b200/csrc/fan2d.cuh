// Generic 2D fan-beam projector kernels, parameterised by a footprint basis.
//
// A basis B supplies, for cell (i, j) of the image grid and view p:
//   B::View                 per-view constants (B::kViewFloats floats in global memory)
//   B::Cell                 per-(cell, view) state: bin range [lo, hi] and whatever
//                           the footprint needs (projected corners, weights ...)
//   B::valid(i, j, P)       whether (i, j) is a cell of the grid
//   B::setup(V, i, j, P, c) fills c (c.lo > c.hi: no bins)
//   B::value(V, c, u, P)    footprint of the cell in bin u, 0 where the reference
//                           drops it (its thresholds), area factors included
// Both kernels call the same functions, so the pair is an exact transpose up
// to summation order.
//
//   fan2d_back_kernel     gather: one thread per cell, all views, FP32 within a
//                         view and FP64 across views, each cell written once.
//   fan2d_forward_kernel  scatter within a tile: a CTA per tile of cells; per
//                         chunk of views the tile's bins are accumulated in a
//                         shared-memory window (FP32 atomics), then each window
//                         is added to an FP64 sinogram (one atomic per bin per
//                         tile and view); fan2d_finish converts to FP32.
#pragma once

#include <cuda_runtime.h>

#include "fan2d_params.h"

namespace sgd {

template <class B>
__global__ void __launch_bounds__(256) fan2d_back_kernel(Fan2DParams P, const float* __restrict__ sino,
                                                         float* __restrict__ img) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)P.ni * P.nj) return;
    const int i = (int)(idx / P.nj), j = (int)(idx - (long long)i * P.nj);
    if (!B::valid(i, j, P)) {
        img[idx] = 0.f;
        return;
    }
    // FP64 products and sums, as the forward kernel: the pair is an adjoint
    // pair to FP64 rounding, whatever the cancellation in the inputs
    double acc = 0.0;
    for (int p = 0; p < P.np; ++p) {
        typename B::View V;
        B::load_view(P.view + (size_t)p * B::kViewFloats, V);
        typename B::Cell c;
        B::setup(V, i, j, P, c);
        const float* sp = sino + (size_t)p * P.nu;
        for (int u = c.lo; u <= c.hi; ++u) {
            const float val = B::value(V, c, u, p, P);
            if (val != 0.f) acc = fma((double)val, (double)__ldg(sp + u), acc);
        }
    }
    img[idx] = (float)acc;
}

template <class B>
__global__ void __launch_bounds__(kF2Threads) fan2d_forward_kernel(Fan2DParams P, const float* __restrict__ img,
                                                                  double* __restrict__ sino64) {
    extern __shared__ __align__(8) unsigned char f2_smem[];
    double* s_acc = reinterpret_cast<double*>(f2_smem);  // [kF2Views][wcap], FP64: see the back kernel
    const int tid = threadIdx.x;
    const int i = blockIdx.y * kF2TileI + (tid >> 5), j = blockIdx.x * kF2TileJ + (tid & 31);
    const int2* twin = P.wins + (size_t)(blockIdx.y * P.tiles_j + blockIdx.x) * P.np;
    const bool mine = i < P.ni && j < P.nj && B::valid(i, j, P);
    const float C = mine ? __ldg(img + (size_t)i * P.nj + j) : 0.f;
    for (int p0 = 0; p0 < P.np; p0 += kF2Views) {
        __syncthreads();  // previous chunk's windows flushed
        for (int e = tid; e < kF2Views * P.wcap; e += kF2Threads) s_acc[e] = 0.0;
        __syncthreads();
        if (C != 0.f) {
            for (int v = 0; v < kF2Views && p0 + v < P.np; ++v) {
                const int p = p0 + v;
                const int2 w = __ldg(twin + p);
                typename B::View V;
                B::load_view(P.view + (size_t)p * B::kViewFloats, V);
                typename B::Cell c;
                B::setup(V, i, j, P, c);
                const int lo = max(c.lo, w.x), hi = min(c.hi, w.y);
                double* acc = s_acc + v * P.wcap - w.x;
                for (int u = lo; u <= hi; ++u) {
                    const float val = B::value(V, c, u, p, P);
                    if (val != 0.f) atomicAdd(acc + u, (double)val * (double)C);
                }
            }
        }
        __syncthreads();
        for (int v = 0; v < kF2Views && p0 + v < P.np; ++v) {
            const int2 w = __ldg(twin + p0 + v);
            for (int k = tid; k <= w.y - w.x; k += kF2Threads) {
                const double a = s_acc[v * P.wcap + k];
                if (a != 0.0) atomicAdd(sino64 + (size_t)(p0 + v) * P.nu + w.x + k, a);
            }
        }
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

__global__ void fan2d_finish_kernel(const double* __restrict__ s64, float* __restrict__ s32, long long n, float scale);

}  // namespace sgd
