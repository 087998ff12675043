// Layer object of the generic 2D fan-beam projectors (A_SF, B0, H0, Hl and the
// B1 reference-rounding mode): what their *_init entry points return.  Owns
// the geometry tables, the forward block strips, the back-projection tile
// windows and the staging of the FP64 host entry points.  Calls on one layer
// must not overlap.
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <vector>

#include "csr_out.h"
#include "fan2d_params.h"
#include "fan_geometry.h"

namespace sgd {

// How a basis's bin ranges sit on the cell grid: the ranges are floors of the
// continuous bin coordinate u = (h0 i + h1 j + h2) / (h3 i + h4 j + h5) of
// points within ri (along i) and rj (along j) index units of the cell (i, j).
struct RangeMap {
    double h[6];
    double ri, rj;
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

    // FP32 device entry points on a caller stream.
    virtual void forward_dev(const float* d_img, float* d_sino, cudaStream_t s) = 0;
    virtual void backward_dev(const float* d_sino, float* d_img, cudaStream_t s) = 0;

    // The layer's system matrix, rows p*nu + u, columns i*nj + j: the pairs
    // and footprints its kernels use, area factor included (csr_build.cuh).
    // Returns the entry count; copies out when `out` has a destination.
    virtual long long csr(const CsrOut& out) = 0;

    // FP64 host entry points: image x[i*nj + j], sinogram b[p*nu + u].
    void forward_host(double* b, const double* x);
    void backward_host(const double* b, double* x);

    // Status of the last back projections: 0, or -1 when a staged chunk did
    // not arrive within the bounded wait (those tiles were left unwritten).
    // Reading it synchronises the device (only the layer's stream when
    // sync_device is false) and clears the flag.
    int status(bool sync_device = true);

protected:
    Proj2D() = default;
    // The basis's range map of view p (cell-index space).
    virtual RangeMap range_map(int p) const = 0;
    // Uploads the view constants and basis table, builds the forward block
    // strips and the back tile windows from range_map, allocates staging.
    void finish_init(const std::vector<float>& view, const std::vector<float4>& bins);

    float* d_view_ = nullptr;
    float4* d_bins_ = nullptr;
    float4* d_strips_ = nullptr;
    int2* d_twin_ = nullptr;
    int* d_err_ = nullptr;
    float* d_img_ = nullptr;
    float* d_imgT_ = nullptr;  // the forward's line-major image copy
    double* d_part_ = nullptr;  // the forward's partial sums [kF2FwdParts][np][nu]
    double* d_out64_ = nullptr;  // the FP64 host entry points' output (allocated at their first call)
    void ensure_out64();
    float* d_sino_ = nullptr;
    float* h_img_ = nullptr;
    float* h_sino_ = nullptr;
};

// u = (h0 x + h1 y + h2) / (h3 x + h4 y + h5) of world point (x, y) in view p
// of a fan geometry, FP64.
void fan_world_hom(const FanGeometry& g, int p, double h[6]);

// The same map on the grid x = x0 + i dx, y = y0 + j dy.
RangeMap grid_range_map(const double hw[6], double x0, double dx, double y0, double dy, double ri, double rj);

// Host plan of the generic kernels for an ni x nj grid, np views of nu bins
// and the basis range map of each view: the forward block strips [np][nblk][2]
// (fan2d.cuh) and the back tile windows [tiles][np].  Every cell whose
// footprint (the bins of the points the map's radii cover) meets a block is a
// candidate of the block's strip, and every cell's footprint lies inside its
// tile's window.  Returns the widest window.
// `block`: bins per forward block (kF2Block for the 2D kernels).
int plan_fan2d(int ni, int nj, int np, int nu, const std::function<RangeMap(int)>& map, std::vector<float4>& strips,
               std::vector<int2>& twin, int block = kF2Block);

}  // namespace sgd
