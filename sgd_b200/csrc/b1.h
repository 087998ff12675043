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
    int wcap = 16;                       // plane stride of the back kernel's staged windows (b1_back_plane)
    int wmax = 1;                        // widest bin window of a back-projection tile and view
    int* err = nullptr;                  // device flag: a bounded wait in a kernel gave up
    unsigned wait_limit = 1u << 22;      // polls of a back-projection staging wait before it gives up
};

// Plane strides the back kernel is built for, and its views per chunk at each
// (two at the widest planes, to stay within shared memory).
constexpr int kBackCaps[] = {16, 32, 48, 64, 96, 128, 192, 256, 320, 448, 640};
__host__ __device__ constexpr int b1_back_vc(int wcap) { return wcap <= 320 ? 4 : 2; }

// Tile bin windows of the back kernel; returns the widest.
int b1_back_windows(const FanGeometry& g, const std::vector<BinHomography>& hom, std::vector<int>& wins);
// Smallest plane stride that holds a window of `widest` bins and the null bin;
// fails when none does.
int b1_back_plane(int widest);
size_t b1_back_smem_bytes(int wcap);
void b1_prepare_device(int wcap);

// sino[p * nu + u] = sum_{i,j} A[(p,u),(i,j)] img[i * ny + j]; imgT is scratch of nx*ny floats.
void b1_forward_launch(const B1Device& d, const float* img, float* imgT, float* sino, cudaStream_t s);
// img[i * ny + j] = sum_{p,u} A[(p,u),(i,j)] sino[p * nu + u]
void b1_back_launch(const B1Device& d, const float* sino, float* img, cudaStream_t s);
// Footprint evaluations the reference kernel performs for this geometry.
unsigned long long b1_count(const B1Device& d, cudaStream_t s);

}  // namespace sgd
