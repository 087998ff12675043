#include <cmath>

#include "common.h"
#include "fan2d.cuh"
#include "proj2d.h"

namespace sgd {

__global__ void fan2d_finish_kernel(const double* __restrict__ s64, float* __restrict__ s32, long long n,
                                    float scale) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) s32[e] = (float)s64[e] * scale;
}

__global__ void scale_kernel(float* a, long long n, float scale) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) a[e] *= scale;
}

void box_window(const FanGeometry& g, int p, const Box2& b, int& lo, int& hi) {
    const double px = g.src[2 * p], py = g.src[2 * p + 1];
    const double Dx = g.dtv[2 * p], Dy = g.dtv[2 * p + 1];
    const double ex = g.puv[2 * p], ey = g.puv[2 * p + 1];
    double umin = 1e300, umax = -1e300;
    const double xs[2] = {b.x0, b.x1}, ys[2] = {b.y0, b.y1};
    for (double x : xs)
        for (double y : ys) {
            // detector coordinate of the ray P -> (x, y): s = cross(P - D, X - P) / cross(e, X - P)
            const double wx = x - px, wy = y - py;
            const double s = ((px - Dx) * wy - (py - Dy) * wx) / (ex * wy - ey * wx);
            const double u = s + 0.5 * g.nu;
            umin = std::min(umin, u);
            umax = std::max(umax, u);
        }
    lo = std::max(0, (int)std::floor(umin) - 1);
    hi = std::min(g.nu - 1, (int)std::floor(umax) + 1);
    if (umax < -1.0 || umin > g.nu + 1.0) {
        lo = 0;
        hi = -1;
    }
}

void Proj2D::window(int p, const Box2& b, int& lo, int& hi) const { box_window(geo, p, b, lo, hi); }

Proj2D::~Proj2D() {
    if (stream) cudaStreamSynchronize(stream);
    cudaFree(d_view_);
    cudaFree(d_bins_);
    cudaFree(d_wins_);
    cudaFree(d_sino64_);
    cudaFree(d_img_);
    cudaFree(d_sino_);
    cudaFreeHost(h_img_);
    cudaFreeHost(h_sino_);
    if (stream) cudaStreamDestroy(stream);
}

void Proj2D::forward_host(double* b, const double* x) {
    const long long nimg = (long long)P.ni * P.nj, nsino = (long long)P.np * P.nu;
#pragma omp parallel for schedule(static) if (nimg > (1 << 16))
    for (long long e = 0; e < nimg; ++e) h_img_[e] = (float)x[e];
    SGD_CUDA(cudaMemcpyAsync(d_img_, h_img_, nimg * sizeof(float), cudaMemcpyHostToDevice, stream));
    forward_dev(d_img_, d_sino_, stream);
    SGD_CUDA(cudaMemcpyAsync(h_sino_, d_sino_, nsino * sizeof(float), cudaMemcpyDeviceToHost, stream));
    SGD_CUDA(cudaStreamSynchronize(stream));
#pragma omp parallel for schedule(static) if (nsino > (1 << 16))
    for (long long e = 0; e < nsino; ++e) b[e] = (double)h_sino_[e];
}

void Proj2D::backward_host(const double* b, double* x) {
    const long long nimg = (long long)P.ni * P.nj, nsino = (long long)P.np * P.nu;
#pragma omp parallel for schedule(static) if (nsino > (1 << 16))
    for (long long e = 0; e < nsino; ++e) h_sino_[e] = (float)b[e];
    SGD_CUDA(cudaMemcpyAsync(d_sino_, h_sino_, nsino * sizeof(float), cudaMemcpyHostToDevice, stream));
    backward_dev(d_sino_, d_img_, stream);
    SGD_CUDA(cudaMemcpyAsync(h_img_, d_img_, nimg * sizeof(float), cudaMemcpyDeviceToHost, stream));
    SGD_CUDA(cudaStreamSynchronize(stream));
#pragma omp parallel for schedule(static) if (nimg > (1 << 16))
    for (long long e = 0; e < nimg; ++e) x[e] = (double)h_img_[e];
}

}  // namespace sgd
