// Template parts of Proj2D, included by each basis translation unit:
// launches of the generic kernels and the system-matrix visitor.
#pragma once

#include <algorithm>

#include "common.h"
#include "csr_build.cuh"
#include "fan2d.cuh"
#include "proj2d.h"

namespace sgd {

template <class B>
void fan2d_forward(const Fan2DParams& P, const float* img, float* sino, float scale, cudaStream_t s) {
    fan2d_transpose_kernel<<<dim3((P.nj + 31) / 32, (P.ni + 31) / 32), dim3(32, 8), 0, s>>>(img, P.imgT, P.ni, P.nj);
    SGD_LAUNCH_CHECK();
    dim3 grid(P.nblk, P.np, kF2FwdParts);
    fan2d_forward_kernel<B><<<grid, 32, 0, s>>>(P, img);
    SGD_LAUNCH_CHECK();
    const size_t n = (size_t)P.np * P.nu;
    fan2d_forward_sum_kernel<<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 16), 256, 0, s>>>(P, sino, scale);
    SGD_LAUNCH_CHECK();
}

template <class B>
void fan2d_back(const Fan2DParams& P, const float* sino, float* img, float scale, cudaStream_t s) {
    const size_t smem = fan2d_back_smem<B, kF2Views, fan2d_back_stages<B>()>(P.wcap);
    if (smem > 227 * 1024) fail("back projection: tile window of %d bins does not fit in shared memory", P.wcap);
    if (smem > 48 * 1024)
        SGD_CUDA(cudaFuncSetAttribute(fan2d_back_kernel<B, kF2Views, fan2d_back_stages<B>()>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    dim3 grid(P.tiles_j, (P.ni + kF2TileI - 1) / kF2TileI);
    fan2d_back_kernel<B, kF2Views, fan2d_back_stages<B>()><<<grid, kF2BackThreads, smem, s>>>(P, sino, img, scale);
    SGD_LAUNCH_CHECK();
}

template <class B>
unsigned long long fan2d_count(const Fan2DParams& P, cudaStream_t s) {
    unsigned long long* d = nullptr;
    SGD_CUDA(cudaMallocAsync(&d, sizeof(unsigned long long), s));
    SGD_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), s));
    const long long n = (long long)P.ni * P.nj;
    fan2d_count_kernel<B><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P, d);
    SGD_LAUNCH_CHECK();
    unsigned long long h = 0;
    SGD_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s));
    SGD_CUDA(cudaFreeAsync(d, s));
    SGD_CUDA(cudaStreamSynchronize(s));
    return h;
}

// System-matrix visitor of basis B: the pairs and values the kernels use.
template <class B>
struct Fan2DVisit {
    Fan2DParams P;
    float scale;
    __device__ bool valid(int i, int j) const { return B::valid(i, j, P); }
    template <class F>
    __device__ void visit(int p, int i, int j, F&& f) const {
        typename B::View V;
        B::load_view(P.view + (size_t)p * B::kViewFloats, V);
        typename B::Cell c;
        B::setup(V, i, j, P, c);
        B::start(V, c, c.lo);
        for (int u = c.lo; u <= c.hi; ++u) {
            const float v = B::value(V, c, u, BinRef{P.bins + (size_t)p * B::kBinF4 * P.nu + u, P.nu}, P);
            if (v != 0.f) f(u, v * scale);
        }
    }
};

template <class B>
long long fan2d_csr(const Fan2DParams& P, float scale, const CsrOut& out, cudaStream_t s) {
    return build_csr(Fan2DVisit<B>{P, scale}, P.np, P.nu, P.ni, P.nj, out, s);
}

}  // namespace sgd
