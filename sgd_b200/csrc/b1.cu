// B1 fan-beam projector kernels (sm_100a).
//
//   b1_forward_kernel   detector-driven: one warp per (view, bin).  Lanes split
//                       the rows (major axis) the bin's ray strip crosses, each
//                       lane evaluates the footprint of the few pixels of its
//                       row inside the strip, and the warp reduces with
//                       shuffles.  The sinogram is written once, no atomics.
//   b1_back_kernel      voxel-driven: one thread per pixel, a CTA per 32x8
//                       tile.  Per chunk of views the CTA stages the bin
//                       window its tile projects onto (footprint tables and
//                       sinogram values) in shared memory; each thread
//                       accumulates over all views in registers and writes
//                       its pixel once, no atomics.
//
// Reference: layers/A_B1.cu:62-208 (forward, one launch per view, FP64
// atomics) and :211-353 (backward).
#include "b1.h"

#include <algorithm>
#include <cmath>

#include "b1_kernels.cuh"
#include "common.h"

namespace sgd {

namespace {

constexpr int kFwdWarps = 8;
constexpr int kBackTI = 8;    // tile extent along i (x), threadIdx.y
constexpr int kBackTJ = 32;   // tile extent along j (y), threadIdx.x: contiguous in memory
constexpr int kBackThreads = kBackTI * kBackTJ;

struct RegTab {
    const float* p;
    __device__ __forceinline__ float operator()(int k) const { return p[k]; }
};

struct SoATab {
    const float* p;  // field k of this bin at p[k * stride]
    int stride;
    __device__ __forceinline__ float operator()(int k) const { return p[k * stride]; }
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// img (i, j) at img[i * ny + j]; imgT (i, j) at imgT[j * nx + i].
__global__ void __launch_bounds__(kFwdWarps * 32)
b1_forward_kernel(const float* __restrict__ rec, const float* __restrict__ strip, const float* __restrict__ img,
                  const float* __restrict__ imgT, float* __restrict__ sino, int nx, int ny, int np, int nu,
                  float dxdy) {
    __shared__ float s_tab[kFwdWarps][kB1Rec];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long gw = (long long)blockIdx.x * kFwdWarps + warp;
    if (gw >= (long long)np * nu) return;
    const float* r = rec + gw * kB1Rec;
    s_tab[warp][lane] = __ldg(r + lane);
    if (lane < kB1Rec - 32) s_tab[warp][32 + lane] = __ldg(r + 32 + lane);
    __syncwarp();
    float c[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) c[k] = s_tab[warp][k];
    const RegTab T{s_tab[warp]};

    const float4 st = __ldg(reinterpret_cast<const float4*>(strip + gw * kStripRec));
    const bool ydom = __ldg(strip + gw * kStripRec + 4) > 0.5f;
    const int nmaj = ydom ? ny : nx, nmin = ydom ? nx : ny;
    const float* src = ydom ? img : imgT;   // minor index n, major m: src[n * nmaj + m]
    const float aa = fabsf(st.y), ab = fabsf(st.w);

    // FP32 sums within a row (a few terms), FP64 across rows and lanes: the
    // forward and back kernels then round the same products to within FP64
    // accumulation error, which the dot-product adjoint test needs.
    double acc = 0.0;
    for (int m = lane; m < nmaj; m += 32) {
        const float fa = fmaf(st.y, (float)m, st.x);
        const float fb = fmaf(st.w, (float)m, st.z);
        // strip extent over the rows m-1..m+1 covered by a pixel's support,
        // widened by the +-1 pixel support along the minor axis
        const float lo = fminf(fa - aa, fb - ab) - 1.0f;
        const float hi = fmaxf(fa + aa, fb + ab) + 1.0f;
        const int nlo = max(0, (int)ceilf(lo));
        const int nhi = min(nmin - 1, (int)floorf(hi));
        float row = 0.f;
        for (int n = nlo; n <= nhi; ++n) {
            const float fi = ydom ? (float)n : (float)m;
            const float fj = ydom ? (float)m : (float)n;
            const float conv = b1_conv(fi, fj, c, T);
            if (conv > kConvEps) row = fmaf(conv, __ldg(src + (size_t)n * nmaj + m), row);
        }
        acc += (double)row;
    }
    acc = warp_sum(acc);
    if (lane == 0) sino[gw] = (float)acc * dxdy;
}

// Bin window [lo, hi] covered by pixels i in [i0, i1], j in [j0, j1] (with the
// +-1 pixel B1 support already applied by the caller), clamped to the detector.
__device__ __forceinline__ void bin_window(const BinHomography& H, float i0, float i1, float j0, float j1, int nu,
                                           int& lo, int& hi) {
    const float u00 = __fdividef(fmaf(H.n0, i0, fmaf(H.n1, j0, H.n2)), fmaf(H.d0, i0, fmaf(H.d1, j0, H.d2)));
    const float u01 = __fdividef(fmaf(H.n0, i0, fmaf(H.n1, j1, H.n2)), fmaf(H.d0, i0, fmaf(H.d1, j1, H.d2)));
    const float u10 = __fdividef(fmaf(H.n0, i1, fmaf(H.n1, j0, H.n2)), fmaf(H.d0, i1, fmaf(H.d1, j0, H.d2)));
    const float u11 = __fdividef(fmaf(H.n0, i1, fmaf(H.n1, j1, H.n2)), fmaf(H.d0, i1, fmaf(H.d1, j1, H.d2)));
    const float umin = fminf(fminf(u00, u01), fminf(u10, u11));
    const float umax = fmaxf(fmaxf(u00, u01), fmaxf(u10, u11));
    lo = max(0, (int)floorf(umin));
    hi = min(nu - 1, (int)floorf(umax));
}

// Shared memory per view: header (8 floats: homography) | window start |
// footprint fields [kB1Rec][wpad] | sinogram [wpad].
__host__ __device__ __forceinline__ int back_view_floats(int wpad) { return 16 + (kB1Rec + 1) * wpad; }

__global__ void __launch_bounds__(kBackThreads)
b1_back_kernel(const float* __restrict__ rec, const BinHomography* __restrict__ hom, const float* __restrict__ sino,
               float* __restrict__ img, int nx, int ny, int np, int nu, int wpad, int vchunk, float dxdy) {
    extern __shared__ float smem[];
    const int tj = threadIdx.x, ti = threadIdx.y, tid = ti * kBackTJ + tj;
    const int i0 = blockIdx.y * kBackTI, j0 = blockIdx.x * kBackTJ;
    const int i = i0 + ti, j = j0 + tj;
    const float fi = (float)i, fj = (float)j;
    const int vfl = back_view_floats(wpad);
    int* s_lo = reinterpret_cast<int*>(smem);            // [vchunk]
    int* s_hi = s_lo + vchunk;                            // [vchunk]
    float* s_view = smem + 2 * ((vchunk + 3) & ~3);       // [vchunk][vfl]

    double acc = 0.0;  // FP32 within a view (a few bins), FP64 across views
    for (int p0 = 0; p0 < np; p0 += vchunk) {
        const int nv = min(vchunk, np - p0);
        __syncthreads();
        if (tid < nv) {
            const BinHomography H = hom[p0 + tid];
            int lo, hi;
            bin_window(H, (float)i0 - 1.f, (float)(i0 + kBackTI), (float)j0 - 1.f, (float)(j0 + kBackTJ), nu, lo, hi);
            if (hi - lo + 1 > wpad) hi = lo + wpad - 1;  // cannot happen: wpad is sized on the host
            s_lo[tid] = lo;
            s_hi[tid] = hi;
            float* v = s_view + tid * vfl;
            v[0] = H.n0; v[1] = H.n1; v[2] = H.n2; v[3] = H.d0; v[4] = H.d1; v[5] = H.d2;
        }
        __syncthreads();
        // stage footprint records and sinogram values of each view's window
        for (int v = 0; v < nv; ++v) {
            const int lo = s_lo[v], W = s_hi[v] - lo + 1;
            if (W <= 0) continue;
            const float* g = rec + ((size_t)(p0 + v) * nu + lo) * kB1Rec;
            float* f = s_view + v * vfl + 16;
            for (int e = tid; e < W * kB1Rec; e += kBackThreads) {
                const int w = e / kB1Rec, k = e - w * kB1Rec;
                f[k * wpad + w] = __ldg(g + e);
            }
            const float* sp = sino + (size_t)(p0 + v) * nu + lo;
            for (int w = tid; w < W; w += kBackThreads) f[kB1Rec * wpad + w] = __ldg(sp + w);
        }
        __syncthreads();
        if (i < nx && j < ny) {
            for (int v = 0; v < nv; ++v) {
                const float* vw = s_view + v * vfl;
                const BinHomography H = {vw[0], vw[1], vw[2], vw[3], vw[4], vw[5], 0.f, 0.f};
                int ulo, uhi;
                bin_window(H, fi - 1.f, fi + 1.f, fj - 1.f, fj + 1.f, nu, ulo, uhi);
                const int lo = s_lo[v];
                ulo = max(ulo, lo);
                uhi = min(uhi, s_hi[v]);
                float vsum = 0.f;
                for (int u = ulo; u <= uhi; ++u) {
                    const float* fb = vw + 16 + (u - lo);
                    const SoATab T{fb, wpad};
                    float c[10];
#pragma unroll
                    for (int k = 0; k < 10; ++k) c[k] = fb[k * wpad];
                    const float conv = b1_conv(fi, fj, c, T);
                    if (conv > kConvEps) vsum = fmaf(conv, fb[kB1Rec * wpad], vsum);
                }
                acc += (double)vsum;
            }
        }
    }
    if (i < nx && j < ny) img[(size_t)i * ny + j] = (float)acc * dxdy;
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
// (layers/A_B1.cu:148-160).  Accumulated per block, one atomic per block.
__global__ void b1_count_kernel(const BinHomography* __restrict__ hom, int nx, int ny, int np, int nu,
                                unsigned long long* out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    unsigned long long n = 0;
    if (j < ny) {
        for (int p = 0; p < np; ++p) {
            const BinHomography H = hom[p];
            const float fi = (float)i, fj = (float)j;
            const float a = (fmaf(H.n0, fi - 1.f, fmaf(H.n1, fj - 1.f, H.n2))) / fmaf(H.d0, fi - 1.f, fmaf(H.d1, fj - 1.f, H.d2));
            const float b = (fmaf(H.n0, fi - 1.f, fmaf(H.n1, fj + 1.f, H.n2))) / fmaf(H.d0, fi - 1.f, fmaf(H.d1, fj + 1.f, H.d2));
            const float c = (fmaf(H.n0, fi + 1.f, fmaf(H.n1, fj - 1.f, H.n2))) / fmaf(H.d0, fi + 1.f, fmaf(H.d1, fj - 1.f, H.d2));
            const float d = (fmaf(H.n0, fi + 1.f, fmaf(H.n1, fj + 1.f, H.n2))) / fmaf(H.d0, fi + 1.f, fmaf(H.d1, fj + 1.f, H.d2));
            const int lo = min(max(0, (int)floorf(fminf(fminf(a, b), fminf(c, d)))), nu - 1);
            const int hi = min(max(0, (int)floorf(fmaxf(fmaxf(a, b), fmaxf(c, d)))), nu - 1);
            n += (unsigned long long)(hi - lo + 1);
        }
    }
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, n);
}

}  // namespace

int b1_back_wpad(const FanGeometry& g, const std::vector<BinHomography>& hom) {
    // Largest bin window of any 32x8 tile over all views (host replay of the
    // kernel's window rule, in double with a one-bin margin), rounded up to odd
    // so that per-bin fields fall into distinct shared-memory banks.
    int wmax = 1;
    for (int p = 0; p < g.np; ++p) {
        const BinHomography& H = hom[p];
        for (int i0 = 0; i0 < g.nx; i0 += kBackTI)
            for (int j0 = 0; j0 < g.ny; j0 += kBackTJ) {
                double is[2] = {i0 - 1.0, (double)(i0 + kBackTI)}, js[2] = {j0 - 1.0, (double)(j0 + kBackTJ)};
                double umin = 1e300, umax = -1e300;
                for (double a : is)
                    for (double b : js) {
                        double u = (H.n0 * a + H.n1 * b + H.n2) / (H.d0 * a + H.d1 * b + H.d2);
                        umin = std::min(umin, u);
                        umax = std::max(umax, u);
                    }
                int lo = std::max(0, (int)std::floor(umin) - 1), hi = std::min(g.nu - 1, (int)std::floor(umax) + 1);
                wmax = std::max(wmax, hi - lo + 1);
            }
    }
    return wmax | 1;
}

size_t b1_back_smem_bytes(int wpad, int vchunk) {
    return sizeof(float) * (2 * ((vchunk + 3) & ~3) + (size_t)vchunk * back_view_floats(wpad));
}

void b1_prepare_device() {
    SGD_CUDA(cudaFuncSetAttribute(b1_back_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
}

void b1_forward_launch(const B1Device& d, const float* img, float* imgT, float* sino, cudaStream_t s) {
    dim3 tb(32, 8), tg((d.ny + 31) / 32, (d.nx + 31) / 32);
    transpose_kernel<<<tg, tb, 0, s>>>(img, imgT, d.nx, d.ny);
    SGD_LAUNCH_CHECK();
    const long long warps = (long long)d.np * d.nu;
    const unsigned blocks = (unsigned)((warps + kFwdWarps - 1) / kFwdWarps);
    b1_forward_kernel<<<blocks, kFwdWarps * 32, 0, s>>>(d.rec, d.strip, img, imgT, sino, d.nx, d.ny, d.np, d.nu,
                                                        d.dxdy);
    SGD_LAUNCH_CHECK();
}

void b1_back_launch(const B1Device& d, const float* sino, float* img, cudaStream_t s) {
    const size_t smem = b1_back_smem_bytes(d.wpad, d.vchunk);
    dim3 tb(kBackTJ, kBackTI), tg((d.ny + kBackTJ - 1) / kBackTJ, (d.nx + kBackTI - 1) / kBackTI);
    b1_back_kernel<<<tg, tb, smem, s>>>(d.rec, d.hom, sino, img, d.nx, d.ny, d.np, d.nu, d.wpad, d.vchunk, d.dxdy);
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
