// A_B1-compatible layer object: what b1_init returns to the caller.
#pragma once

#include <cuda_runtime.h>

#include "b1.h"
#include "fan_geometry.h"
#include "matrix_double.h"

namespace sgd {

// Device memory owned by a layer for the FP64 host entry points: the FP32
// image and sinogram, the transposed-image scratch of the forward kernel and
// pinned host staging.  Calls on one layer must not overlap.
struct Staging {
    float* d_img = nullptr;
    float* d_imgT = nullptr;
    float* d_sino = nullptr;
    float* h_img = nullptr;   // pinned
    float* h_sino = nullptr;  // pinned
    int* h_err = nullptr;     // pinned copy of the device error flag
};

class A_B1 {
public:
    FanGeometry geo;
    B1Device dev;
    Staging st;
    cudaStream_t stream = nullptr;
    int device = 0;
    unsigned long long count = 0;  // reference conv_count for this geometry

    A_B1(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
         const double* angles, const double* dz, const double* drho);
    ~A_B1();
    A_B1(const A_B1&) = delete;
    A_B1& operator=(const A_B1&) = delete;

    // layers/A_B1.hh:21-22 signatures.  vol holds the image in the host layout
    // x[ix*ny + iy]; proj the sinogram as [p][u].  `weight` is accepted and
    // ignored, as in the reference.
    void project(MatrixD& vol, MatrixD& proj, double weight);
    void back_project(MatrixD& vol, MatrixD& proj, double weight);

    // Device entry points (FP32, caller-owned device memory, caller's stream).
    void forward_dev(const float* d_img, float* d_sino, cudaStream_t s);
    void backward_dev(const float* d_sino, float* d_img, cudaStream_t s);

    // FP64 host entry points of the C ABI.
    void forward_host(double* b, const double* x);
    void backward_host(const double* b, double* x);

    // Raises (and clears) the device error flag set by a kernel whose bounded
    // wait gave up.  Synchronous; sync_device = false when the calls in
    // question ran on the layer's own stream and that was synchronised.
    void check_device_status(bool sync_device = true);

private:
    // Raises (and clears) the device error flag whose value e was read.
    void raise_device_error(int e);

    int* d_err_ = nullptr;
    int* d_wins_ = nullptr;
    float* d_rec_ = nullptr;
    float* d_strip_ = nullptr;
    BinHomography* d_hom_ = nullptr;
};

}  // namespace sgd
