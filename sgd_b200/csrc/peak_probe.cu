// FP32 issue-rate probe: measures the FMA throughput of this GPU at its
// current clocks, the denominator of the projectors' roofline (their bound is
// FP32 issue, not HBM or tensor cores).  Each thread runs 8 independent FMA
// chains so the pipe, not the dependency latency, limits the rate.
#include <cuda_runtime.h>

#include "common.h"

namespace {
__global__ void __launch_bounds__(256) fma_probe_kernel(float* out, int iters, float a, float b) {
    float x0 = threadIdx.x * 1e-3f, x1 = x0 + 1.f, x2 = x0 + 2.f, x3 = x0 + 3.f;
    float x4 = x0 + 4.f, x5 = x0 + 5.f, x6 = x0 + 6.f, x7 = x0 + 7.f;
    for (int k = 0; k < iters; ++k) {
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
            x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
        }
    }
    const float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == 1234.5f) out[blockIdx.x] = s;  // keeps the chains live
}
}  // namespace

extern "C" {
// Launches `blocks` x 256 threads, each doing iters*128 FMAs; returns the
// achieved FP32 rate in FLOP/s (FMA = 2 FLOPs) timed with CUDA events on
// `stream`, or -1 on failure.  `scratch` is any device buffer of >= blocks floats.
double sgd_fp32_fma_rate(float* scratch, int blocks, int iters, void* stream) {
    return sgd::guarded<double>(-1.0, [&]() -> double {
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        cudaEvent_t e0, e1;
        SGD_CUDA(cudaEventCreate(&e0));
        SGD_CUDA(cudaEventCreate(&e1));
        fma_probe_kernel<<<blocks, 256, 0, s>>>(scratch, iters, 0.999999f, 1e-6f);  // warm-up
        SGD_LAUNCH_CHECK();
        SGD_CUDA(cudaEventRecord(e0, s));
        fma_probe_kernel<<<blocks, 256, 0, s>>>(scratch, iters, 0.999999f, 1e-6f);
        SGD_LAUNCH_CHECK();
        SGD_CUDA(cudaEventRecord(e1, s));
        SGD_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        SGD_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        const double flops = 2.0 * 128.0 * (double)iters * 256.0 * (double)blocks;
        return flops / (ms * 1e-3);
    });
}
}
