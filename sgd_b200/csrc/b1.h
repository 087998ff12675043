// B1 fan-beam projector: device tables and kernel launchers.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "fan_geometry.h"

namespace sgd {

// Device-resident tables of one B1 geometry.
struct B1Device {
    int nx = 0, ny = 0, np = 0, nu = 0;
    float dxdy = 1.f;
    const float* rec = nullptr;          // [np][nu][kB1Rec]
    const float* strip = nullptr;        // [np][nu][kStripRec]
    const BinHomography* hom = nullptr;  // [np]
    const int* wins = nullptr;           // [tiles][np][2] bin windows of the back kernel's tiles
    int wcap = 4;                        // bins of a staged view window in the back kernel
    int* err = nullptr;                  // device flag: a bounded wait in a kernel gave up
    unsigned wait_limit = 1u << 22;      // polls of a back-projection staging wait before it gives up
};

int b1_back_windows(const FanGeometry& g, const std::vector<BinHomography>& hom, std::vector<int>& wins);
size_t b1_back_smem_bytes(int wcap);
void b1_prepare_device();

// sino[p * nu + u] = sum_{i,j} A[(p,u),(i,j)] img[i * ny + j]; imgT is scratch of nx*ny floats.
void b1_forward_launch(const B1Device& d, const float* img, float* imgT, float* sino, cudaStream_t s);
// img[i * ny + j] = sum_{p,u} A[(p,u),(i,j)] sino[p * nu + u]
void b1_back_launch(const B1Device& d, const float* sino, float* img, cudaStream_t s);
// Footprint evaluations the reference kernel performs for this geometry.
unsigned long long b1_count(const B1Device& d, cudaStream_t s);

}  // namespace sgd
