// 3x3 convolution of the warm-start CNN's 32-channel layers on the sm_100
// tensor cores: an implicit GEMM per tile of 128 output pixels (one row
// segment) with M = 128 pixels, N = 32 output channels and K = 9 taps x 32
// input channels, issued as tcgen05.mma (kind::f16, BF16 operands from shared
// memory, FP32 accumulator in tensor memory) and read back with tcgen05.ld.
//
// Precision: the weights are BF16 already (the network keeps FP32 masters and
// convolves with their BF16 copy); each FP32 activation is split into three
// BF16 terms hi + mid + lo (the value to within 2^-23 of itself), so that
// every product of the three MMA passes is exact and the sum is an FP32
// accumulation of the products the FP32 kernels form.
//
// Shared memory (no swizzle, the canonical K-major layout of 8 x 16-byte core
// matrices): per BF16 term, four 8-channel columns, each three staged input
// rows of 130 pixels (the tile and its halo) of 16 bytes; a tap (dy, dx) is
// the A operand starting dy rows and dx pixels into the column, so the nine
// taps read the same staged rows.  The weights as [tap][8-channel column]
// [output channel][8 channels].  One CTA of 256 threads per tile, persistent
// over tiles; thread 0 issues the 54 MMAs of a tile and commits them to an
// mbarrier; every thread then reads 16 of a pixel's 32 accumulators (TMEM
// lane = pixel) and writes them with the bias and ReLU fused.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "common.h"
#include "tma.cuh"

namespace sgd {

namespace {

constexpr int kTcM = 128;                 // output pixels per tile
constexpr int kTcC = 32;                  // input and output channels
constexpr int kTcX = kTcM + 2;            // staged input pixels per row (halo included)
constexpr int kTcCC = kTcC / 8;           // 8-channel core-matrix columns
constexpr int kTcSplit = 3;               // BF16 terms per FP32 activation
constexpr uint32_t kTcRowBytes = kTcX * 16;                  // one staged row of one column
constexpr uint32_t kTcColBytes = 3 * kTcRowBytes;            // a column: three rows
constexpr uint32_t kTcTermBytes = kTcCC * kTcColBytes;       // one BF16 term of the tile
constexpr uint32_t kTcABytes = kTcSplit * kTcTermBytes;      // 74880
constexpr uint32_t kTcBBytes = 9 * kTcCC * kTcC * 16;        // 18432
constexpr uint32_t kTcSmem = kTcABytes + kTcBBytes + kTcC * 4 + 16;
constexpr uint32_t kTcTmemCols = 32;      // FP32 accumulator columns (N)
constexpr uint32_t kTcWaitLimit = 1u << 22;
constexpr int kTcThreads = 2 * kTcM;      // two threads per pixel: each stages half the (row, column) pairs
constexpr int kTcBatch = 3;               // (row, column) pairs per thread whose loads are in flight together

// Instruction descriptor of kind::f16: FP32 D (bits 4-5 = 1), BF16 A and B
// (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bit 17,
// M >> 4 at bit 24.
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTcC >> 3) << 17) |
                              ((uint32_t)(kTcM >> 4) << 24);

// Shared-memory matrix descriptor, no swizzle: start address, leading byte
// offset (between the two 8-element K halves of an MMA's K = 16) and stride
// byte offset (between 8-row groups), each in 16-byte units; version 1 at
// bits 46-47.
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
        "}" ::"r"(tmem),
        "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// x = hi + mid + lo with each term the leading 8 significant bits of what is
// left (truncation: the high half of an FP32 is a BF16), every difference
// exact in FP32; the residual after three terms is below 2^-23 |x|.  Eight
// values per call, packed two BF16 per 32-bit word as the MMA reads them.
__device__ __forceinline__ void split3x8(const float* x, uint4& hi, uint4& mid, uint4& lo) {
    uint32_t h[8], m[8], l[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const uint32_t xb = __float_as_uint(x[k]);
        h[k] = xb & 0xFFFF0000u;
        const float r1 = __fsub_rn(x[k], __uint_as_float(h[k]));
        const uint32_t rb = __float_as_uint(r1);
        m[k] = rb & 0xFFFF0000u;
        const float r2 = __fsub_rn(r1, __uint_as_float(m[k]));
        l[k] = __float_as_uint(r2) & 0xFFFF0000u;
    }
    // the high halves of words 2k (low BF16) and 2k + 1 (high BF16)
    auto pack = [](uint32_t a, uint32_t b) { return __byte_perm(a, b, 0x7632); };
    hi = make_uint4(pack(h[0], h[1]), pack(h[2], h[3]), pack(h[4], h[5]), pack(h[6], h[7]));
    mid = make_uint4(pack(m[0], m[1]), pack(m[2], m[3]), pack(m[4], m[5]), pack(m[6], m[7]));
    lo = make_uint4(pack(l[0], l[1]), pack(l[2], l[3]), pack(l[4], l[5]), pack(l[6], l[7]));
}

__device__ int g_tc_err;  // set when a tile's MMAs never completed (bounded wait)

__global__ void __launch_bounds__(kTcThreads, 2)
conv3x3_c32_tc_kernel(const float* __restrict__ in, const __nv_bfloat16* __restrict__ w,
                      const float* __restrict__ bias, float* __restrict__ out, int N, int H, int W, int relu,
                      uint32_t wait_limit) {
    extern __shared__ __align__(128) unsigned char tsm[];
    unsigned char* sA = tsm;
    unsigned char* sB = tsm + kTcABytes;
    float* sbias = reinterpret_cast<float*>(sB + kTcBBytes);
    uint64_t* bar = reinterpret_cast<uint64_t*>(sbias + kTcC);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // weights w[n][ci][ky][kx] -> B[tap][ci / 8][n][ci % 8]
    for (int e = tid; e < kTcC * kTcC * 9; e += kTcThreads) {
        const int n = e / (kTcC * 9), r = e - n * kTcC * 9, ci = r / 9, t = r - ci * 9;
        *reinterpret_cast<__nv_bfloat16*>(sB + ((t * kTcCC + ci / 8) * kTcC + n) * 16 + (ci % 8) * 2) = w[e];
    }
    if (tid < kTcC) sbias[tid] = bias ? bias[tid] : 0.f;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                     "r"(kTcTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    fence_proxy_async_smem();  // the weights, written here, are read by the MMAs
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    const int tiles_x = (W + kTcM - 1) / kTcM;
    const long long ntiles = (long long)N * H * tiles_x;
    const size_t plane = (size_t)H * W;
    uint32_t phase = 0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int tx = (int)(tile % tiles_x);
        const long long ry = tile / tiles_x;
        const int y = (int)(ry % H), img = (int)(ry / H);
        const int x0 = tx * kTcM;

        // stage the three input rows (halo included) as three BF16 terms:
        // threads t and t + 128 take pixel x0 - 1 + t, each six of the twelve
        // (row, 8-channel column) pairs, three pairs' 24 loads in flight
        // together; threads 0, 1, 128 and 129 also take the last two halo
        // pixels
        const int half = tid / kTcM, qbeg = half * (3 * kTcCC / 2), qend = qbeg + 3 * kTcCC / 2;
        for (int xi = tid % kTcM; xi < kTcX; xi += kTcM) {
            const int gx = x0 - 1 + xi;
            const uint32_t xoff = xi * 16;
#pragma unroll 1
            for (int q0 = qbeg; q0 < qend; q0 += kTcBatch) {
                float v[kTcBatch][8];
#pragma unroll
                for (int b = 0; b < kTcBatch; ++b) {
                    const int q = q0 + b, cc = q % kTcCC, row = q / kTcCC, gy = y - 1 + row;
                    const bool in_img = gx >= 0 && gx < W && gy >= 0 && gy < H;
                    const float* src = in + ((size_t)img * kTcC + cc * 8) * plane + (size_t)gy * W + gx;
#pragma unroll
                    for (int k = 0; k < 8; ++k) v[b][k] = in_img ? __ldg(src + k * plane) : 0.f;
                }
#pragma unroll
                for (int b = 0; b < kTcBatch; ++b) {
                    const int q = q0 + b, cc = q % kTcCC, row = q / kTcCC;
                    uint4 h, m, l;
                    split3x8(v[b], h, m, l);
                    const uint32_t off = cc * kTcColBytes + row * kTcRowBytes + xoff;
                    *reinterpret_cast<uint4*>(sA + off) = h;
                    *reinterpret_cast<uint4*>(sA + kTcTermBytes + off) = m;
                    *reinterpret_cast<uint4*>(sA + 2 * kTcTermBytes + off) = l;
                }
            }
        }
        fence_proxy_async_smem();
        tc_fence_before();  // the previous tile's accumulator reads are done
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            const uint32_t a0 = smem_addr(sA), b0 = smem_addr(sB);
            uint32_t acc = 0;
#pragma unroll 1
            for (int s = 0; s < kTcSplit; ++s)
#pragma unroll 1
                for (int t = 0; t < 9; ++t)
#pragma unroll
                    for (int hk = 0; hk < 2; ++hk) {
                        const uint32_t aoff =
                            s * kTcTermBytes + 2 * hk * kTcColBytes + (t / 3) * kTcRowBytes + (t % 3) * 16;
                        const uint32_t boff = (t * kTcCC + 2 * hk) * kTcC * 16;
                        tc_mma(tmem, tc_desc(a0 + aoff, kTcColBytes, 128), tc_desc(b0 + boff, kTcC * 16, 128), acc);
                        acc = 1;
                    }
            tc_commit(bar);
        }
        const bool done = mbar_wait_bounded(bar, phase, wait_limit);
        if (!__syncthreads_and(done)) {
            if (tid == 0) atomicExch(&g_tc_err, 1);
            break;
        }
        phase ^= 1u;
        tc_fence_after();
        // warp w reads TMEM lanes 32 (w % 4) .. + 31 (its pixels), columns
        // 16 (w / 4) .. + 15 (its half of the output channels)
        const int quarter = warp & 3, n0 = (warp >> 2) * 16;
        float v[16];
        tc_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)n0, v);
        tc_wait_ld();
        const int x = x0 + quarter * 32 + lane;
        if (x < W) {
            float* dst = out + ((size_t)img * kTcC + n0) * plane + (size_t)y * W + x;
#pragma unroll
            for (int n = 0; n < 16; ++n) {
                const float r = v[n] + sbias[n0 + n];
                dst[n * plane] = relu ? fmaxf(r, 0.f) : r;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols)
                     : "memory");
}

}  // namespace

void conv3x3_c32_tc(const float* in, const __nv_bfloat16* w, const float* bias, float* out, int N, int H, int W,
                    int relu, cudaStream_t s) {
    if (N < 1 || H < 1 || W < 1) fail("conv3x3 (tensor cores): invalid sizes");
    int dev = 0, sms = 0;
    SGD_CUDA(cudaGetDevice(&dev));
    SGD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    SGD_CUDA(cudaFuncSetAttribute(conv3x3_c32_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
    const long long ntiles = (long long)N * H * ((W + kTcM - 1) / kTcM);
    const int grid = (int)std::min<long long>(ntiles, 2LL * sms);
    conv3x3_c32_tc_kernel<<<grid, kTcThreads, kTcSmem, s>>>(in, w, bias, out, N, H, W, relu, kTcWaitLimit);
    SGD_LAUNCH_CHECK();
}

}  // namespace sgd

extern "C" {

int sgd_conv3x3_forward_tc(const float* in, const void* w_bf16, const float* bias, float* out, int N, int Cin,
                           int Cout, int H, int W, int relu, void* stream) {
    return sgd::guarded_status([&] {
        if (!in || !w_bf16 || !out) sgd::fail("sgd_conv3x3_forward_tc: null argument");
        if (Cin != 32 || Cout != 32)
            sgd::fail("sgd_conv3x3_forward_tc: 32 input and 32 output channels only (got %d, %d)", Cin, Cout);
        sgd::conv3x3_c32_tc(in, static_cast<const __nv_bfloat16*>(w_bf16), bias, out, N, H, W, relu,
                            static_cast<cudaStream_t>(stream));
    });
}

int sgd_conv3x3_tc_status(void) {
    return sgd::guarded_status([&] {
        int e = 0;
        SGD_CUDA(cudaDeviceSynchronize());
        SGD_CUDA(cudaMemcpyFromSymbol(&e, sgd::g_tc_err, sizeof(int)));
        if (e) {
            const int zero = 0;
            SGD_CUDA(cudaMemcpyToSymbol(sgd::g_tc_err, &zero, sizeof(int)));
            sgd::fail("conv3x3 (tensor cores): a tile's MMAs did not complete (bounded wait); output incomplete");
        }
    });
}

}  // extern "C"
