// Layer object of the generic 2D fan-beam projectors (A_SF, B0, H0, Hl): what
// their *_init entry points return.  Owns the geometry tables, the FP64
// sinogram scratch of the forward kernel and the staging of the FP64 host
// entry points.  Calls on one layer must not overlap.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "csr_out.h"
#include "fan2d_params.h"
#include "fan_geometry.h"

namespace sgd {

// World-space box (with the basis support) covered by cells [i0, i1] x [j0, j1].
struct Box2 {
    double x0, x1, y0, y1;
};

class Proj2D {
public:
    virtual ~Proj2D();
    Proj2D(const Proj2D&) = delete;
    Proj2D& operator=(const Proj2D&) = delete;

    FanGeometry geo;
    Fan2DParams P;
    int device = 0;
    cudaStream_t stream = nullptr;
    unsigned long long count = 0;  // the reference's footprint-evaluation count (0 where it returns 0)
    float out_scale = 1.f;         // factor applied to every footprint (area), folded into the output

    // FP32 device entry points on a caller stream.  The forward accumulates in
    // the layer's FP64 sinogram scratch.
    virtual void forward_dev(const float* d_img, float* d_sino, cudaStream_t s) = 0;
    virtual void backward_dev(const float* d_sino, float* d_img, cudaStream_t s) = 0;

    // The layer's system matrix, rows p*nu + u, columns i*nj + j: the pairs
    // and footprints its kernels use, area factor included (csr_build.cuh).
    // Returns the entry count; copies out when `out` has a destination.
    virtual long long csr(const CsrOut& out) = 0;

    // FP64 host entry points: image x[i*nj + j], sinogram b[p*nu + u].
    void forward_host(double* b, const double* x);
    void backward_host(const double* b, double* x);

protected:
    Proj2D() = default;
    // Bin window [lo, hi] of world box b in view p for the forward tiles
    // (fan geometry by default; hi < lo when it misses).
    virtual void window(int p, const Box2& b, int& lo, int& hi) const;
    // Uploads tables, computes tile windows from `box`, allocates staging.
    template <class BoxFn>
    void finish_init(const std::vector<float>& view, int view_floats, const std::vector<float4>& bins, BoxFn box);

    float* d_view_ = nullptr;
    float4* d_bins_ = nullptr;
    int2* d_wins_ = nullptr;
    double* d_sino64_ = nullptr;
    float* d_img_ = nullptr;
    float* d_sino_ = nullptr;
    float* h_img_ = nullptr;
    float* h_sino_ = nullptr;
    size_t smem_fwd_ = 0;
};

// Bin window [lo, hi] of world box b in view p (corners through the view's
// homography, one bin of margin each side, clamped); hi < lo when it misses.
void box_window(const FanGeometry& g, int p, const Box2& b, int& lo, int& hi);

}  // namespace sgd
