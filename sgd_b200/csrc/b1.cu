// B1 fan-beam projector kernels (sm_100a).
//
//   b1_forward_kernel   detector-driven: one warp per (view, bin).  Lanes split
//                       the rows (major axis) the bin's ray strip crosses; each
//                       lane evaluates the footprint of the few pixels of its
//                       row inside the strip, and the warp reduces with
//                       shuffles.  The sinogram is written once, no atomics.
//   b1_back_kernel      voxel-driven: one thread per pixel, a CTA per 32x8
//                       tile.  Per chunk of views the CTA stages the bin window
//                       its tile projects onto in shared memory: the 64-byte
//                       footprint records by TMA bulk copies completed on an
//                       mbarrier (double-buffered, the next chunk in flight
//                       while this one is evaluated), the sinogram values by
//                       plain loads.  Each thread accumulates over all views in
//                       registers and writes its pixel once, no atomics.
//
// Reference: layers/A_B1.cu:62-208 (forward, one launch per view, FP64
// atomics) and :211-353 (backward).
#include "b1.h"

#include <algorithm>
#include <cmath>

#include "b1_kernels.cuh"
#include "common.h"
#include "hom.cuh"
#include "tma.cuh"

namespace sgd {

namespace {

constexpr int kFwdWarps = 8;
constexpr int kBackTI = 8;    // tile extent along i (x), threadIdx.y
constexpr int kBackTJ = 32;   // tile extent along j (y), threadIdx.x: contiguous in memory
constexpr int kBackThreads = kBackTI * kBackTJ;
constexpr int kVC = 4;        // views per staged chunk
constexpr uint32_t kWaitLimit = 1u << 22;
constexpr int kHeaderBytes = 16 + 3 * kVC * 8 + 3 * kVC * 32;  // 2 mbarriers | 3 x kVC windows | 3 x kVC homographies
static_assert(kHeaderBytes % 16 == 0, "staged records must start 16-byte aligned");

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Records are float4 chunks laid out [view][chunk][bin] (fan_geometry.h).
__device__ __forceinline__ B1Bin load_bin(const float4* rec, int p, int u, int nu) {
    const float4* q = rec + (size_t)p * 4 * nu + u;
    return B1Bin{__ldg(q), __ldg(q + nu), __ldg(q + 2 * nu), __ldg(q + 3 * nu)};
}

// Candidate minor indices of major line m: the strip between the edge rays over
// the lines m-1..m+1 a pixel's support covers, widened by the +-1 pixel support
// along the minor axis.
__device__ __forceinline__ void strip_span(const float4& st, float aa, float ab, float fm, int nmin, int& nlo,
                                           int& nhi) {
    const float fa = fmaf(st.y, fm, st.x);
    const float fb = fmaf(st.w, fm, st.z);
    const float lo = fminf(fa - aa, fb - ab) - 1.0f;
    const float hi = fmaxf(fa + aa, fb + ab) + 1.0f;
    nlo = max(0, (int)ceilf(lo));
    nhi = min(nmin - 1, (int)floorf(hi));
}

// img (i, j) at img[i * ny + j]; imgT (i, j) at imgT[j * nx + i].
__global__ void __launch_bounds__(kFwdWarps * 32)
b1_forward_kernel(const float4* __restrict__ rec, const float* __restrict__ strip, const float* __restrict__ img,
                  const float* __restrict__ imgT, float* __restrict__ sino, int nx, int ny, int np, int nu,
                  float dxdy) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long gw = (long long)blockIdx.x * kFwdWarps + warp;
    if (gw >= (long long)np * nu) return;
    const int p = (int)(gw / nu), u = (int)(gw - (long long)p * nu);
    const B1Bin r = load_bin(rec, p, u, nu);
    const float4 st = __ldg(reinterpret_cast<const float4*>(strip + gw * kStripRec));
    const bool ydom = __ldg(strip + gw * kStripRec + 4) > 0.5f;
    const float aa = fabsf(st.y), ab = fabsf(st.w);

    // FP32 sums within a line (a few terms), FP64 across lines and lanes: the
    // forward and back kernels then round the same products to within FP64
    // accumulation error, which the dot-product adjoint test needs.
    double acc = 0.0;
    if (ydom) {
        // rows j = m, candidate columns i = n; the j terms are hoisted
        for (int m = lane; m < ny; m += 32) {
            const float fm = (float)m;
            int nlo, nhi;
            strip_span(st, aa, ab, fm, nx, nlo, nhi);
            const float ia = b1_xa_inner(fm, r), ib = b1_xb_inner(fm, r);
            float row = 0.f, fn = (float)nlo;
            const float* sp = img + (size_t)nlo * ny + m;
            for (int n = nlo; n <= nhi; ++n, fn += 1.0f, sp += ny) {
                const float conv = b1_conv_x(b1_xa(fn, ia, r), b1_xb(fn, ib, r), r);
                if (conv > kConvEps) row = fmaf(conv, __ldg(sp), row);
            }
            acc += (double)row;
        }
    } else {
        // columns i = m, candidate rows j = n
        for (int m = lane; m < nx; m += 32) {
            const float fm = (float)m;
            int nlo, nhi;
            strip_span(st, aa, ab, fm, ny, nlo, nhi);
            float row = 0.f, fn = (float)nlo;
            const float* sp = imgT + (size_t)nlo * nx + m;
            for (int n = nlo; n <= nhi; ++n, fn += 1.0f, sp += nx) {
                const float conv = b1_conv(fm, fn, r);
                if (conv > kConvEps) row = fmaf(conv, __ldg(sp), row);
            }
            acc += (double)row;
        }
    }
    acc = warp_sum(acc);
    if (lane == 0) sino[gw] = (float)acc * dxdy;
}

template <int N>
__device__ __forceinline__ int pick(const int (&a)[N], int v) {
    int r = a[0];
#pragma unroll
    for (int k = 1; k < N; ++k) r = (v == k) ? a[k] : r;
    return r;
}

// wins[tile * np + p] = (lo, hi): bins of view p that tile's pixels can touch
// (host-computed, conservative; fits in wcap).
__global__ void __launch_bounds__(kBackThreads, 5)
b1_back_kernel(const float4* __restrict__ rec, const BinHomography* __restrict__ hom, const int2* __restrict__ wins,
               const float* __restrict__ sino, float* __restrict__ img, int nx, int ny, int np, int nu, int wcap,
               float dxdy, int* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem);           // [2]
    int* win = reinterpret_cast<int*>(smem + 16);                   // [3][kVC][2]
    float* hs = reinterpret_cast<float*>(smem + 16 + 3 * kVC * 8);  // [3][kVC][8]
    float4* srec = reinterpret_cast<float4*>(smem + kHeaderBytes);  // [2][kVC][4 chunks][wcap]
    float* ssino = reinterpret_cast<float*>(srec + 2 * kVC * 4 * wcap);  // [2][kVC][wcap]
    __shared__ int s_abort;

    // each warp covers an 8 (j) x 4 (i) block of the 32 x 8 tile, so that its
    // lanes read few distinct bins of a view
    const int tid = threadIdx.x, w = tid >> 5, l = tid & 31;
    const int i0 = blockIdx.y * kBackTI, j0 = blockIdx.x * kBackTJ;
    const int i = i0 + 4 * (w >> 2) + (l >> 3), j = j0 + 8 * (w & 3) + (l & 7);
    const float fi = (float)i, fj = (float)j;
    const int nchunks = (np + kVC - 1) / kVC;
    const int2* twin = wins + (size_t)(blockIdx.y * gridDim.x + blockIdx.x) * np;

    // stage chunk c: windows and homographies (thread 0, read after the next
    // barrier), footprint records by TMA (thread 0), sinogram values (all)
    auto stage = [&](int c) {
        const int st = c & 1, slot = c % 3;
        if (tid == 0) {
            uint32_t bytes = 0;
            for (int v = 0; v < kVC; ++v) {
                const int p = c * kVC + v;
                int2 lh = make_int2(0, -1);
                if (p < np) {
                    lh = __ldg(twin + p);
                    const BinHomography H = hom[p];
                    float* h = hs + (slot * kVC + v) * 8;
                    h[0] = H.n0; h[1] = H.n1; h[2] = H.n2; h[3] = H.d0; h[4] = H.d1; h[5] = H.d2;
                }
                win[(slot * kVC + v) * 2] = lh.x;
                win[(slot * kVC + v) * 2 + 1] = lh.y;
                if (lh.y >= lh.x) bytes += (uint32_t)(lh.y - lh.x + 1) * sizeof(B1Bin);
            }
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&bars[st], bytes);
            for (int v = 0; v < kVC; ++v) {
                const int lo = win[(slot * kVC + v) * 2], W = win[(slot * kVC + v) * 2 + 1] - lo + 1;
                if (W > 0)
                    for (int q = 0; q < 4; ++q)
                        bulk_copy_g2s(srec + ((st * kVC + v) * 4 + q) * wcap,
                                      rec + ((size_t)(c * kVC + v) * 4 + q) * nu + lo, (uint32_t)W * 16u, &bars[st]);
            }
        }
        for (int v = 0; v < kVC; ++v) {
            const int p = c * kVC + v;
            if (p >= np) break;
            const int2 lh = __ldg(twin + p);
            const float* sp = sino + (size_t)p * nu + lh.x;
            float* dp = ssino + (st * kVC + v) * wcap;
            for (int k = tid; k <= lh.y - lh.x; k += kBackThreads) dp[k] = __ldg(sp + k);
        }
    };

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
        s_abort = 0;
    }
    __syncthreads();
    stage(0);

    double acc = 0.0;  // FP32 within a chunk (a few tens of terms), FP64 across chunks
    int c = 0;
    for (; c < nchunks; ++c) {
        __syncthreads();  // chunk c's windows and sinogram visible; chunk c-1 fully consumed
        if (s_abort) break;
        if (c + 1 < nchunks) stage(c + 1);
        const int st = c & 1, slot = c % 3;
        if (!mbar_wait_bounded(&bars[st], (uint32_t)((c >> 1) & 1), kWaitLimit)) {
            s_abort = 1;
            atomicExch(err, 1);
            continue;
        }
        if (i >= nx || j >= ny) continue;
        // this pixel's bins in each view of the chunk, then one flat loop over
        // all of them: lanes run nearly equal trip counts
        int ulo[kVC], uhi[kVC], roff[kVC], soff[kVC];
        int total = 0;
#pragma unroll
        for (int v = 0; v < kVC; ++v) {
            const int lo = win[(slot * kVC + v) * 2], hi = win[(slot * kVC + v) * 2 + 1];
            int a = 0, b = -1;
            if (hi >= lo) {
                box_bins(hs + (slot * kVC + v) * 8, fi - 1.f, fi + 1.f, fj - 1.f, fj + 1.f, nu, a, b);
                a = max(a, lo);
                b = min(b, hi);
            }
            ulo[v] = a;
            uhi[v] = b;
            roff[v] = (st * kVC + v) * 4 * wcap - lo;
            soff[v] = (st * kVC + v) * wcap - lo;
            total += max(0, b - a + 1);
        }
        float csum = 0.f;
        int v = 0, u = ulo[0], ue = uhi[0], ro = roff[0], so = soff[0];
        for (int k = 0; k < total; ++k) {
            while (u > ue) {
                ++v;
                u = pick(ulo, v);
                ue = pick(uhi, v);
                ro = pick(roff, v);
                so = pick(soff, v);
            }
            const float4* rb = srec + ro + u;
            const B1Bin r{rb[0], rb[wcap], rb[2 * wcap], rb[3 * wcap]};
            const float conv = b1_conv(fi, fj, r);
            if (conv > kConvEps) csum = fmaf(conv, ssino[so + u], csum);
            ++u;
        }
        acc += (double)csum;
    }
    if (c < nchunks) {
        // a staged chunk never arrived: wait (bounded) for the copies still in
        // flight into this CTA's shared memory, then leave the tile unwritten
        if (tid == 0) {
            mbar_wait_bounded(&bars[c & 1], (uint32_t)((c >> 1) & 1), kWaitLimit);
            if (c + 1 < nchunks) mbar_wait_bounded(&bars[(c + 1) & 1], (uint32_t)(((c + 1) >> 1) & 1), kWaitLimit);
        }
        return;
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
    // FP32 per-pixel ranges always fall inside.  Returns the largest window,
    // rounded up to a multiple of 4 (the shared-memory capacity per view).
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
    return (wmax + 3) & ~3;
}

size_t b1_back_smem_bytes(int wcap) {
    return kHeaderBytes + (size_t)2 * kVC * wcap * (sizeof(B1Bin) + sizeof(float));
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
    b1_forward_kernel<<<blocks, kFwdWarps * 32, 0, s>>>(reinterpret_cast<const float4*>(d.rec), d.strip, img,
                                                        imgT, sino, d.nx, d.ny, d.np, d.nu, d.dxdy);
    SGD_LAUNCH_CHECK();
}

void b1_back_launch(const B1Device& d, const float* sino, float* img, cudaStream_t s) {
    dim3 tg((d.ny + kBackTJ - 1) / kBackTJ, (d.nx + kBackTI - 1) / kBackTI);
    b1_back_kernel<<<tg, kBackThreads, b1_back_smem_bytes(d.wcap), s>>>(
        reinterpret_cast<const float4*>(d.rec), d.hom, reinterpret_cast<const int2*>(d.wins), sino, img, d.nx, d.ny,
        d.np, d.nu, d.wcap, d.dxdy, d.err);
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
