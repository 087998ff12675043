// 3x3 convolution forward/backward, ReLU, MSE and Adam kernels for the small
// warm-start CNN of the ASD-POCS solver (5 layers, 32 channels).
//
// Layouts: activations NCHW FP32; weights [Cout][Cin][3][3] in BF16 (FP32
// master copies live with the optimiser); bias FP32 [Cout].  Zero padding,
// stride 1.  Every product is accumulated in FP32.
//
//   conv3x3_fwd_kernel    a CTA per 16x16 output tile, image and block of
//                         COB output channels; per input channel the 18x18
//                         input tile and the COB x 9 weights are staged in
//                         shared memory, each thread accumulates COB outputs
//                         in registers; bias and ReLU fused.
//   conv3x3_c32_kernel    32 output channels, input channels in groups of 8
//                         (the network's middle layers): a CTA per 32x8
//                         output tile and image, each thread 4 consecutive
//                         pixels x 8 output channels in registers, the 8
//                         input tiles and their 32x8x9 weights staged in
//                         shared memory per group.  Same summation order per
//                         output as conv3x3_fwd_kernel: bit-identical.
//   backward data         the same kernels on weights flipped in space and
//                         transposed in channels (flip_weights_kernel).
//   conv3x3_wgrad_kernel  a CTA per (output channel, input channel, image
//                         chunk): 9 + 1 sums per thread in registers over its
//                         pixels, block reduction, one FP32 atomic per tap.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "common.h"

namespace sgd {

namespace {

constexpr int kT = 16;  // output tile side

template <int COB>
__global__ void __launch_bounds__(kT * kT) conv3x3_fwd_kernel(const float* __restrict__ in,
                                                              const __nv_bfloat16* __restrict__ w,
                                                              const float* __restrict__ bias, float* __restrict__ out,
                                                              int Cin, int Cout, int H, int W, int relu) {
    __shared__ float tile[kT + 2][kT + 2];
    __shared__ float ws[COB][9];
    const int tx = threadIdx.x % kT, ty = threadIdx.x / kT;
    const int x = blockIdx.x * kT + tx, y = blockIdx.y * kT + ty;
    const int nblk = (Cout + COB - 1) / COB;
    const int n = blockIdx.z / nblk, co0 = (blockIdx.z % nblk) * COB;
    float acc[COB];
#pragma unroll
    for (int c = 0; c < COB; ++c) acc[c] = 0.f;
    const size_t plane = (size_t)H * W;
    for (int ci = 0; ci < Cin; ++ci) {
        const float* src = in + ((size_t)n * Cin + ci) * plane;
        for (int e = threadIdx.x; e < (kT + 2) * (kT + 2); e += kT * kT) {
            const int yy = blockIdx.y * kT + e / (kT + 2) - 1, xx = blockIdx.x * kT + e % (kT + 2) - 1;
            tile[e / (kT + 2)][e % (kT + 2)] =
                (yy >= 0 && yy < H && xx >= 0 && xx < W) ? __ldg(src + (size_t)yy * W + xx) : 0.f;
        }
        for (int e = threadIdx.x; e < COB * 9; e += kT * kT) {
            const int c = e / 9, k = e % 9;
            ws[c][k] = (co0 + c < Cout) ? __bfloat162float(w[((size_t)(co0 + c) * Cin + ci) * 9 + k]) : 0.f;
        }
        __syncthreads();
        float v[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) v[k] = tile[ty + k / 3][tx + k % 3];
#pragma unroll
        for (int c = 0; c < COB; ++c)
#pragma unroll
            for (int k = 0; k < 9; ++k) acc[c] = fmaf(ws[c][k], v[k], acc[c]);
        __syncthreads();
    }
    if (x >= W || y >= H) return;
#pragma unroll
    for (int c = 0; c < COB; ++c) {
        const int co = co0 + c;
        if (co >= Cout) break;
        float o = acc[c] + (bias ? bias[co] : 0.f);
        if (relu) o = fmaxf(o, 0.f);
        out[((size_t)n * Cout + co) * plane + (size_t)y * W + x] = o;
    }
}

constexpr int kCW = 32, kCH = 8;  // output tile of conv3x3_c32_kernel
constexpr int kCS = 35;            // staged row stride: lanes (row r, 4-pixel group g) read banks 3r + 4g + q
constexpr int kCG = 8;             // input channels per staged group

__global__ void __launch_bounds__(256, 2) conv3x3_c32_kernel(const float* __restrict__ in,
                                                             const __nv_bfloat16* __restrict__ w,
                                                             const float* __restrict__ bias, float* __restrict__ out,
                                                             int Cin, int H, int W, int relu) {
    __shared__ float tile[kCG][kCH + 2][kCS];
    __shared__ __align__(16) float ws[kCG][9][32];
    const int t = threadIdx.x;
    const int cg = t >> 6;                     // output channels 8 cg .. 8 cg + 7 (warp-uniform)
    const int ty = (t >> 3) & 7, tx4 = t & 7;  // output row, 4-pixel group
    const int n = blockIdx.z;
    const int x0 = blockIdx.x * kCW, y0 = blockIdx.y * kCH;
    const size_t plane = (size_t)H * W;
    float acc[4][8];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[p][c] = 0.f;
    for (int c0 = 0; c0 < Cin; c0 += kCG) {
        constexpr int kRow = kCW + 2, kPlane = (kCH + 2) * kRow;
        for (int e = t; e < kCG * kPlane; e += 256) {
            const int c = e / kPlane, r = (e - c * kPlane) / kRow, q = e - c * kPlane - r * kRow;
            const int yy = y0 + r - 1, xx = x0 + q - 1;
            tile[c][r][q] = (yy >= 0 && yy < H && xx >= 0 && xx < W)
                                ? __ldg(in + ((size_t)n * Cin + c0 + c) * plane + (size_t)yy * W + xx)
                                : 0.f;
        }
        for (int e = t; e < 32 * kCG * 9; e += 256) {
            const int co = e / (kCG * 9), c = (e / 9) % kCG, k = e % 9;
            ws[c][k][co] = __bfloat162float(w[((size_t)co * Cin + c0 + c) * 9 + k]);
        }
        __syncthreads();
#pragma unroll 1
        for (int c = 0; c < kCG; ++c) {
            float v[3][6];
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int q = 0; q < 6; ++q) v[r][q] = tile[c][ty + r][4 * tx4 + q];
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                const float4 wa = *reinterpret_cast<const float4*>(&ws[c][k][8 * cg]);
                const float4 wb = *reinterpret_cast<const float4*>(&ws[c][k][8 * cg + 4]);
                const float wk[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
#pragma unroll
                for (int p = 0; p < 4; ++p) {
                    const float a = v[k / 3][p + k % 3];
#pragma unroll
                    for (int co = 0; co < 8; ++co) acc[p][co] = fmaf(wk[co], a, acc[p][co]);
                }
            }
        }
        __syncthreads();
    }
    const int y = y0 + ty;
    if (y >= H) return;
#pragma unroll
    for (int co = 0; co < 8; ++co) {
        const int oc = 8 * cg + co;
        const float bv = bias ? bias[oc] : 0.f;
        float* dst = out + ((size_t)n * 32 + oc) * plane + (size_t)y * W;
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const int x = x0 + 4 * tx4 + p;
            float o = acc[p][co] + bv;
            if (relu) o = fmaxf(o, 0.f);
            if (x < W) dst[x] = o;
        }
    }
}

// wt[ci][co][8 - k] = w[co][ci][k]: the weights of the input-gradient convolution
__global__ void flip_weights_kernel(const __nv_bfloat16* __restrict__ w, __nv_bfloat16* __restrict__ wt, int Cin,
                                    int Cout) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Cin * Cout * 9) return;
    const int k = e % 9, ci = (e / 9) % Cin, co = e / (9 * Cin);
    wt[((size_t)ci * Cout + co) * 9 + (8 - k)] = w[e];
}

// block of 256 threads; result valid in thread 0
__device__ __forceinline__ float block_sum_f(float v, float* s) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
    __syncthreads();
    float t = 0.f;
    if (threadIdx.x < 32) {
        t = threadIdx.x < (blockDim.x >> 5) ? s[threadIdx.x] : 0.f;
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    }
    return t;
}

// gw[co][ci][k] += sum gout[n][co][y][x] in[n][ci][y+ky-1][x+kx-1]; gb[co] += sum gout
// grid (Cout, Cin, chunks of images), 256 threads.
__global__ void __launch_bounds__(256) conv3x3_wgrad_kernel(const float* __restrict__ in,
                                                            const float* __restrict__ gout, float* __restrict__ gw,
                                                            float* __restrict__ gb, int N, int Cin, int Cout, int H,
                                                            int W, int nper) {
    __shared__ float s[8];
    const int co = blockIdx.x, ci = blockIdx.y;
    const int n0 = blockIdx.z * nper, n1 = min(N, n0 + nper);
    const size_t plane = (size_t)H * W;
    float acc[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float accb = 0.f;
    for (int n = n0; n < n1; ++n) {
        const float* g = gout + ((size_t)n * Cout + co) * plane;
        const float* a = in + ((size_t)n * Cin + ci) * plane;
        for (size_t p = threadIdx.x; p < plane; p += blockDim.x) {
            const int y = (int)(p / W), x = (int)(p % W);
            const float gv = __ldg(g + p);
            accb += gv;
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                const int yy = y + k / 3 - 1, xx = x + k % 3 - 1;
                const float av = (yy >= 0 && yy < H && xx >= 0 && xx < W) ? __ldg(a + (size_t)yy * W + xx) : 0.f;
                acc[k] = fmaf(gv, av, acc[k]);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const float t = block_sum_f(acc[k], s);
        if (threadIdx.x == 0) atomicAdd(gw + ((size_t)co * Cin + ci) * 9 + k, t);
    }
    const float tb = block_sum_f(accb, s);
    if (threadIdx.x == 0 && ci == 0 && gb) atomicAdd(gb + co, tb);
}

__global__ void relu_bwd_kernel(float* __restrict__ g, const float* __restrict__ out, long long n) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n && !(out[e] > 0.f)) g[e] = 0.f;
}

// g = 2 (y - t) / n, loss += sum (y - t)^2
__global__ void mse_grad_kernel(const float* __restrict__ y, const float* __restrict__ t, float* __restrict__ g,
                                long long n, double* __restrict__ loss) {
    __shared__ float s[8];
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float d = 0.f;
    if (e < n) {
        d = y[e] - t[e];
        g[e] = 2.f * d / (float)n;
    }
    const float b = block_sum_f(d * d, s);
    if (threadIdx.x == 0) atomicAdd(loss, (double)b);
}

// Adam (Kingma and Ba 2015) on FP32 master weights, BF16 copy refreshed.
__global__ void adam_kernel(float* __restrict__ w, __nv_bfloat16* __restrict__ w16, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, long long n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const float gi = g[e];
    const float mi = b1 * m[e] + (1.f - b1) * gi, vi = b2 * v[e] + (1.f - b2) * gi * gi;
    m[e] = mi;
    v[e] = vi;
    const float wi = w[e] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[e] = wi;
    if (w16) w16[e] = __float2bfloat16(wi);
}

void conv_fwd(const float* in, const __nv_bfloat16* w, const float* bias, float* out, int N, int Cin, int Cout, int H,
              int W, int relu, cudaStream_t s) {
    if (N < 1 || Cin < 1 || Cout < 1 || H < 1 || W < 1) fail("conv3x3: invalid sizes");
    if (Cout == 32 && Cin % kCG == 0) {
        dim3 g((W + kCW - 1) / kCW, (H + kCH - 1) / kCH, N);
        conv3x3_c32_kernel<<<g, 256, 0, s>>>(in, w, bias, out, Cin, H, W, relu);
    } else if (Cout >= 8) {
        dim3 g((W + kT - 1) / kT, (H + kT - 1) / kT, N * ((Cout + 7) / 8));
        conv3x3_fwd_kernel<8><<<g, kT * kT, 0, s>>>(in, w, bias, out, Cin, Cout, H, W, relu);
    } else {
        dim3 g((W + kT - 1) / kT, (H + kT - 1) / kT, N * Cout);
        conv3x3_fwd_kernel<1><<<g, kT * kT, 0, s>>>(in, w, bias, out, Cin, Cout, H, W, relu);
    }
    SGD_LAUNCH_CHECK();
}

}  // namespace

}  // namespace sgd

extern "C" {

int sgd_conv3x3_forward(const float* in, const void* w_bf16, const float* bias, float* out, int N, int Cin, int Cout,
                        int H, int W, int relu, void* stream) {
    return sgd::guarded_status([&] {
        if (!in || !w_bf16 || !out) sgd::fail("sgd_conv3x3_forward: null argument");
        sgd::conv_fwd(in, static_cast<const __nv_bfloat16*>(w_bf16), bias, out, N, Cin, Cout, H, W, relu,
                      static_cast<cudaStream_t>(stream));
    });
}

// gin = conv^T(gout): gradient of the input.  scratch: Cin*Cout*9 BF16.
int sgd_conv3x3_backward_data(const float* gout, const void* w_bf16, void* scratch_bf16, float* gin, int N, int Cin,
                              int Cout, int H, int W, void* stream) {
    return sgd::guarded_status([&] {
        if (!gout || !w_bf16 || !scratch_bf16 || !gin) sgd::fail("sgd_conv3x3_backward_data: null argument");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        auto* wt = static_cast<__nv_bfloat16*>(scratch_bf16);
        const int n = Cin * Cout * 9;
        sgd::flip_weights_kernel<<<(n + 255) / 256, 256, 0, s>>>(static_cast<const __nv_bfloat16*>(w_bf16), wt, Cin,
                                                                 Cout);
        SGD_LAUNCH_CHECK();
        sgd::conv_fwd(gout, wt, nullptr, gin, N, Cout, Cin, H, W, 0, s);
    });
}

// gw (FP32 [Cout][Cin][9]) and gbias (FP32 [Cout], may be null) are accumulated into.
int sgd_conv3x3_backward_weight(const float* in, const float* gout, float* gw, float* gbias, int N, int Cin, int Cout,
                                int H, int W, void* stream) {
    return sgd::guarded_status([&] {
        if (!in || !gout || !gw) sgd::fail("sgd_conv3x3_backward_weight: null argument");
        if (N < 1 || Cin < 1 || Cout < 1 || H < 1 || W < 1) sgd::fail("sgd_conv3x3_backward_weight: invalid sizes");
        const int nper = 2;
        dim3 g(Cout, Cin, (N + nper - 1) / nper);
        sgd::conv3x3_wgrad_kernel<<<g, 256, 0, static_cast<cudaStream_t>(stream)>>>(in, gout, gw, gbias, N, Cin, Cout,
                                                                                   H, W, nper);
        SGD_LAUNCH_CHECK();
    });
}

int sgd_relu_backward(float* g, const float* out, long long n, void* stream) {
    return sgd::guarded_status([&] {
        if (!g || !out) sgd::fail("sgd_relu_backward: null argument");
        sgd::relu_bwd_kernel<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(g, out, n);
        SGD_LAUNCH_CHECK();
    });
}

int sgd_mse_grad(const float* y, const float* t, float* g, long long n, double* d_loss, void* stream) {
    return sgd::guarded_status([&] {
        if (!y || !t || !g || !d_loss) sgd::fail("sgd_mse_grad: null argument");
        sgd::mse_grad_kernel<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(y, t, g, n,
                                                                                                       d_loss);
        SGD_LAUNCH_CHECK();
    });
}

int sgd_adam_step(float* w, void* w_bf16, const float* g, float* m, float* v, long long n, float lr, float b1,
                  float b2, float eps, int step, void* stream) {
    return sgd::guarded_status([&] {
        if (!w || !g || !m || !v || step < 1) sgd::fail("sgd_adam_step: invalid argument");
        const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
        sgd::adam_kernel<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
            w, static_cast<__nv_bfloat16*>(w_bf16), g, m, v, n, lr, b1, b2, eps, c1, c2);
        SGD_LAUNCH_CHECK();
    });
}

}  // extern "C"
