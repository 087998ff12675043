// B1 fan-beam projector: single-geometry kernels (bodies in b1_body.cuh),
// their launchers, the back kernel's tile windows and the footprint count.
//
// Reference: layers/A_B1.cu:62-208 (forward, one launch per view, FP64
// atomics) and :211-353 (backward).
#include "b1.h"

#include <algorithm>
#include <cmath>

#include "b1_body.cuh"
#include "b1_kernels.cuh"
#include "common.h"

namespace sgd {

namespace {

constexpr int kFwdWarps = 8;

__global__ void __launch_bounds__(kFwdWarps * 32)
b1_forward_kernel(const float4* __restrict__ rec, const float* __restrict__ strip, const float* __restrict__ img,
                  const float* __restrict__ imgT, float* __restrict__ sino, int nx, int ny, int np, int nu,
                  float dxdy) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long gw = (long long)blockIdx.x * kFwdWarps + warp;
    if (gw >= (long long)np * nu) return;
    b1_forward_row(rec, strip, img, imgT, sino, nx, ny, nu, dxdy, gw, lane);
}

// One CTA per 32x8 tile; wins[tile * np + p] = (lo, hi), the tile's bins in
// view p.  Staged planes of WCAP bins (b1_back_tile), four views per chunk up
// to 320 bins and two beyond.  Seven CTAs of 128 threads per SM (72
// registers): a 512^2 image's 1024 tiles run in one wave on 148 SMs.
template <int WCAP>
__global__ void __launch_bounds__(kBackThreads, 7)
b1_back_kernel(const float4* __restrict__ rec, const BinHomography* __restrict__ hom, const int2* __restrict__ wins,
               const float* __restrict__ sino, float* __restrict__ img, int nx, int ny, int np, int nu, float dxdy,
               int* __restrict__ err, uint32_t wait_limit) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (threadIdx.x == 0) {
        uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    uint32_t use0 = 0, use1 = 0;
    const int2* twin = wins + (size_t)(blockIdx.y * gridDim.x + blockIdx.x) * np;
    b1_back_tile<b1_back_vc(WCAP), WCAP>(rec, hom, twin, sino, img, nx, ny, np, nu, dxdy, err, wait_limit,
                                         blockIdx.y * kBackTI, blockIdx.x * kBackTJ, smem, use0, use1);
}

__global__ void transpose_kernel(const float* __restrict__ in, float* __restrict__ out, int rows, int cols) {
    // in[r * cols + c] -> out[c * rows + r]
    __shared__ float t[32][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int r = blockIdx.y * 32 + k;
        if (r < rows && c < cols) t[k][threadIdx.x] = in[(size_t)r * cols + c];
    }
    __syncthreads();
    const int r = blockIdx.y * 32 + threadIdx.x;
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int cc = blockIdx.x * 32 + k;
        if (r < rows && cc < cols) out[(size_t)cc * rows + r] = t[threadIdx.x][k];
    }
}

// Footprint evaluations the reference performs (its conv_count): per pixel and
// view, the width of the clamped bin range of the +-1 pixel support
// (layers/A_B1.cu:148-160).  One atomic per warp.
__global__ void b1_count_kernel(const BinHomography* __restrict__ hom, int nx, int ny, int np, int nu,
                                unsigned long long* out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    unsigned long long n = 0;
    if (j < ny) {
        const float fi = (float)i, fj = (float)j;
        for (int p = 0; p < np; ++p) {
            const BinHomography H = hom[p];
            const float h[6] = {H.n0, H.n1, H.n2, H.d0, H.d1, H.d2};
            const float a = hom_u(h, fi - 1.f, fj - 1.f), b = hom_u(h, fi - 1.f, fj + 1.f);
            const float c = hom_u(h, fi + 1.f, fj - 1.f), d = hom_u(h, fi + 1.f, fj + 1.f);
            const int lo = min(max(0, (int)floorf(fminf(fminf(a, b), fminf(c, d)))), nu - 1);
            const int hi = min(max(0, (int)floorf(fmaxf(fmaxf(a, b), fmaxf(c, d)))), nu - 1);
            n += (unsigned long long)(hi - lo + 1);
        }
    }
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, n);
}

}  // namespace

int b1_back_windows(const FanGeometry& g, const std::vector<BinHomography>& hom, std::vector<int>& wins) {
    // Per 32x8 tile and view, the bins its pixels' +-1 supports can reach: the
    // kernel's corner rule in double, one extra bin each side so the kernel's
    // FP32 per-pixel ranges always fall inside.  Returns the widest window.
    const int gx = (g.ny + kBackTJ - 1) / kBackTJ, gy = (g.nx + kBackTI - 1) / kBackTI;
    wins.assign((size_t)gx * gy * g.np * 2, 0);
    int wmax = 1;
    for (int by = 0; by < gy; ++by)
        for (int bx = 0; bx < gx; ++bx) {
            const int i0 = by * kBackTI, j0 = bx * kBackTJ;
            const double is[2] = {i0 - 1.0, (double)(i0 + kBackTI)}, js[2] = {j0 - 1.0, (double)(j0 + kBackTJ)};
            int* out = &wins[((size_t)by * gx + bx) * g.np * 2];
            for (int p = 0; p < g.np; ++p) {
                const BinHomography& H = hom[p];
                double umin = 1e300, umax = -1e300;
                for (double a : is)
                    for (double b : js) {
                        const double u = ((double)H.n0 * a + (double)H.n1 * b + H.n2) /
                                         ((double)H.d0 * a + (double)H.d1 * b + H.d2);
                        umin = std::min(umin, u);
                        umax = std::max(umax, u);
                    }
                const int lo = std::max(0, (int)std::floor(umin) - 1);
                const int hi = std::min(g.nu - 1, (int)std::floor(umax) + 1);
                out[2 * p] = lo;
                out[2 * p + 1] = hi;
                wmax = std::max(wmax, hi - lo + 1);
            }
        }
    return wmax;
}

int b1_back_plane(int widest) {
    for (int c : kBackCaps)
        if (widest + 1 <= c) return c;
    fail("B1 back projector: a tile's bin window of %d bins does not fit in shared memory (at most %d)", widest,
         kBackCaps[sizeof(kBackCaps) / sizeof(kBackCaps[0]) - 1] - 1);
}

namespace {

// Calls f(kernel, dynamic shared memory bytes) for the back kernel of plane stride wcap.
template <class F>
void with_back_kernel(int wcap, F&& f) {
    switch (wcap) {
#define SGD_B1_BACK_CASE(W) \
    case W: f(b1_back_kernel<W>, b1_back_smem<b1_back_vc(W), W>()); break;
        SGD_B1_BACK_CASE(16) SGD_B1_BACK_CASE(32) SGD_B1_BACK_CASE(48) SGD_B1_BACK_CASE(64)
        SGD_B1_BACK_CASE(96) SGD_B1_BACK_CASE(128) SGD_B1_BACK_CASE(192) SGD_B1_BACK_CASE(256)
        SGD_B1_BACK_CASE(320) SGD_B1_BACK_CASE(448) SGD_B1_BACK_CASE(640)
#undef SGD_B1_BACK_CASE
        default: fail("B1 back projector: no kernel for a window plane of %d bins", wcap);
    }
}

}  // namespace

size_t b1_back_smem_bytes(int wcap) {
    size_t bytes = 0;
    with_back_kernel(wcap, [&](auto, size_t smem) { bytes = smem; });
    return bytes;
}

void b1_prepare_device(int wcap) {
    with_back_kernel(wcap, [](auto kern, size_t smem) {
        SGD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        // the whole unified L1 as shared memory: seven CTAs of staged windows per SM
        SGD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      cudaSharedmemCarveoutMaxShared));
    });
}

void b1_forward_launch(const B1Device& d, const float* img, float* imgT, float* sino, cudaStream_t s) {
    dim3 tb(32, 8), tg((d.ny + 31) / 32, (d.nx + 31) / 32);
    transpose_kernel<<<tg, tb, 0, s>>>(img, imgT, d.nx, d.ny);
    SGD_LAUNCH_CHECK();
    const long long warps = (long long)d.np * d.nu;
    const unsigned blocks = (unsigned)((warps + kFwdWarps - 1) / kFwdWarps);
    b1_forward_kernel<<<blocks, kFwdWarps * 32, 0, s>>>(reinterpret_cast<const float4*>(d.rec), d.strip, img,
                                                        imgT, sino, d.nx, d.ny, d.np, d.nu, d.dxdy);
    SGD_LAUNCH_CHECK();
}

void b1_back_launch(const B1Device& d, const float* sino, float* img, cudaStream_t s) {
    dim3 tg((d.ny + kBackTJ - 1) / kBackTJ, (d.nx + kBackTI - 1) / kBackTI);
    with_back_kernel(d.wcap, [&](auto kern, size_t smem) {
        kern<<<tg, kBackThreads, smem, s>>>(reinterpret_cast<const float4*>(d.rec), d.hom,
                                            reinterpret_cast<const int2*>(d.wins), sino, img, d.nx, d.ny, d.np, d.nu,
                                            d.dxdy, d.err, d.wait_limit);
    });
    SGD_LAUNCH_CHECK();
}

unsigned long long b1_count(const B1Device& d, cudaStream_t s) {
    unsigned long long* dc = nullptr;
    SGD_CUDA(cudaMallocAsync(&dc, sizeof(unsigned long long), s));
    SGD_CUDA(cudaMemsetAsync(dc, 0, sizeof(unsigned long long), s));
    dim3 tb(128), tg((d.ny + 127) / 128, d.nx);
    b1_count_kernel<<<tg, tb, 0, s>>>(d.hom, d.nx, d.ny, d.np, d.nu, dc);
    SGD_LAUNCH_CHECK();
    unsigned long long h = 0;
    SGD_CUDA(cudaMemcpyAsync(&h, dc, sizeof(h), cudaMemcpyDeviceToHost, s));
    SGD_CUDA(cudaFreeAsync(dc, s));
    SGD_CUDA(cudaStreamSynchronize(s));
    return h;
}

}  // namespace sgd
