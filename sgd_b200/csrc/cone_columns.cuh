// Column-major copy of a cone-beam volume for the factored forward
// projectors: vol [z][y][x] -> volT [y][x][z], so that the voxels of one
// (x, y) column are contiguous and a warp reads 32 of them in one request.
#pragma once

#include <cuda_runtime.h>

namespace sgd {
namespace {

__global__ void to_columns_kernel(const float* __restrict__ vol, float* __restrict__ volT, int nx, int ny, int nz) {
    __shared__ float t[32][33];
    const int col0 = blockIdx.x * 32, z0 = blockIdx.y * 32;
    const int ncol = nx * ny;
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int z = z0 + k, col = col0 + threadIdx.x;
        if (z < nz && col < ncol) t[k][threadIdx.x] = vol[(size_t)z * ncol + col];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int col = col0 + k, z = z0 + threadIdx.x;
        if (z < nz && col < ncol) volT[(size_t)col * nz + z] = t[threadIdx.x][k];
    }
}

inline void launch_to_columns(const float* vol, float* volT, int nx, int ny, int nz, cudaStream_t s) {
    const int ncol = nx * ny;
    to_columns_kernel<<<dim3((ncol + 31) / 32, (nz + 31) / 32), dim3(32, 8), 0, s>>>(vol, volT, nx, ny, nz);
}

}  // namespace
}  // namespace sgd
