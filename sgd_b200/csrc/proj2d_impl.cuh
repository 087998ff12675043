// Template parts of Proj2D, included by each basis translation unit.
#pragma once

#include <algorithm>

#include "common.h"
#include "csr_build.cuh"
#include "fan2d.cuh"
#include "proj2d.h"

namespace sgd {

template <class BoxFn>
void Proj2D::finish_init(const std::vector<float>& view, int view_floats, const std::vector<float4>& bins,
                         BoxFn box) {
    SGD_CUDA(cudaGetDevice(&device));
    SGD_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    P.np = geo.np;
    P.nu = geo.nu;
    SGD_CUDA(cudaMalloc(&d_view_, view.size() * sizeof(float)));
    SGD_CUDA(cudaMemcpy(d_view_, view.data(), view.size() * sizeof(float), cudaMemcpyHostToDevice));
    P.view = d_view_;
    if (!bins.empty()) {
        SGD_CUDA(cudaMalloc(&d_bins_, bins.size() * sizeof(float4)));
        SGD_CUDA(cudaMemcpy(d_bins_, bins.data(), bins.size() * sizeof(float4), cudaMemcpyHostToDevice));
        P.bins = d_bins_;
    }
    (void)view_floats;
    // forward tiles of kF2TileI x kF2TileJ cells and their bin windows per view
    const int ti = (P.ni + kF2TileI - 1) / kF2TileI, tj = (P.nj + kF2TileJ - 1) / kF2TileJ;
    std::vector<int2> wins((size_t)ti * tj * geo.np);
    int wmax = 1;
    for (int a = 0; a < ti; ++a)
        for (int b = 0; b < tj; ++b) {
            const Box2 bx = box(a * kF2TileI, std::min(P.ni, (a + 1) * kF2TileI) - 1, b * kF2TileJ,
                                std::min(P.nj, (b + 1) * kF2TileJ) - 1);
            for (int p = 0; p < geo.np; ++p) {
                int lo, hi;
                window(p, bx, lo, hi);
                wins[((size_t)a * tj + b) * geo.np + p] = make_int2(lo, hi);
                wmax = std::max(wmax, hi - lo + 1);
            }
        }
    P.tiles_j = tj;
    P.wcap = wmax;
    smem_fwd_ = (size_t)kF2Views * wmax * sizeof(double);
    if (smem_fwd_ > 48 * 1024) fail("forward tile window of %d bins does not fit in shared memory", wmax);
    SGD_CUDA(cudaMalloc(&d_wins_, wins.size() * sizeof(int2)));
    SGD_CUDA(cudaMemcpy(d_wins_, wins.data(), wins.size() * sizeof(int2), cudaMemcpyHostToDevice));
    P.wins = d_wins_;
    const size_t nimg = (size_t)P.ni * P.nj, nsino = (size_t)geo.np * geo.nu;
    SGD_CUDA(cudaMalloc(&d_sino64_, nsino * sizeof(double)));
    SGD_CUDA(cudaMalloc(&d_img_, nimg * sizeof(float)));
    SGD_CUDA(cudaMalloc(&d_sino_, nsino * sizeof(float)));
    SGD_CUDA(cudaMallocHost(&h_img_, nimg * sizeof(float)));
    SGD_CUDA(cudaMallocHost(&h_sino_, nsino * sizeof(float)));
}

// Launches of the generic kernels for basis B.
template <class B>
void fan2d_forward(const Fan2DParams& P, const float* img, double* s64, float* sino, float scale, size_t smem,
                   cudaStream_t s) {
    const long long ns = (long long)P.np * P.nu;
    SGD_CUDA(cudaMemsetAsync(s64, 0, ns * sizeof(double), s));
    dim3 grid(P.tiles_j, (P.ni + kF2TileI - 1) / kF2TileI);
    fan2d_forward_kernel<B><<<grid, kF2Threads, smem, s>>>(P, img, s64);
    SGD_LAUNCH_CHECK();
    fan2d_finish_kernel<<<(unsigned)((ns + 255) / 256), 256, 0, s>>>(s64, sino, ns, scale);
    SGD_LAUNCH_CHECK();
}

__global__ void scale_kernel(float* a, long long n, float scale);

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

template <class B>
void fan2d_back(const Fan2DParams& P, const float* sino, float* img, float scale, cudaStream_t s) {
    const long long n = (long long)P.ni * P.nj;
    fan2d_back_kernel<B><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P, sino, img);
    SGD_LAUNCH_CHECK();
    if (scale != 1.f) {
        scale_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(img, n, scale);
        SGD_LAUNCH_CHECK();
    }
}

// System-matrix visitor of basis B: the bins and values the kernels use.
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
        for (int u = c.lo; u <= c.hi; ++u) {
            const float v = B::value(V, c, u, p, P);
            if (v != 0.f) f(u, v * scale);
        }
    }
};

template <class B>
long long fan2d_csr(const Fan2DParams& P, float scale, const CsrOut& out, cudaStream_t s) {
    return build_csr(Fan2DVisit<B>{P, scale}, P.np, P.nu, P.ni, P.nj, out, s);
}

}  // namespace sgd
