// Batched B1 projector (b1_batch.cu): many fan-beam slices of different sizes
// in one persistent launch per direction, CUDA-graph capture, autotuned
// launch shape.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "b1_layer.h"

namespace sgd {

// One slice as the persistent kernels see it (device array, heaviest first).
struct B1Slice {
    const float4* rec;
    const float* strip;
    const BinHomography* hom;
    const int2* wins;
    long long img_off, sino_off;  // into the caller's arenas
    int nx, ny, np, nu, tiles_x;
    float dxdy;
};

class B1Batch {
public:
    B1Batch(int ns, const int* nx, const int* ny, const int* np, const int* nu, const double* dx, const double* dy,
            const double* du, const double* lsd, const double* lso, const double* const* angles);
    ~B1Batch();
    B1Batch(const B1Batch&) = delete;
    B1Batch& operator=(const B1Batch&) = delete;

    // arenas: slice k's image at img[img_off[k]], sinogram at sino[sino_off[k]]
    void forward(const float* img, float* sino, cudaStream_t s);
    void backward(const float* sino, float* img, cudaStream_t s);
    // Captures forward (img -> sino) and/or backward (sino_in -> img_out) on
    // the batch's own stream into a CUDA graph; replay() launches it.
    void capture(const float* img, float* sino, const float* sino_in, float* img_out);
    void replay(cudaStream_t s);
    // Loads the launch shape for this GPU and geometry from the cache, or
    // measures all variants and appends the best; returns 1 when loaded.
    int tune(const char* cache_path);
    // Must not overlap batch work in flight on any stream: it rewrites the
    // work-item table the persistent kernels read (it synchronises the
    // device first) and drops a captured graph.
    void set_variant(int fw, int vc);
    void check_status();
    // Polls of each back-projection staging wait before it gives up (the
    // failure path's test sets 0); drops a captured graph.
    void set_wait_limit(unsigned polls);

    int fw() const { return fw_; }
    int vc() const { return vc_; }
    const std::vector<long long>& img_off() const { return img_off_; }
    const std::vector<long long>& sino_off() const { return sino_off_; }

private:
    int resident(const void* fn, int threads, size_t smem) const;
    void release_graph();
    std::string cache_key() const;

    std::vector<std::unique_ptr<A_B1>> layers_;
    std::vector<int> order_, layer_of_;  // processing order; slice -> layer
    std::vector<long long> img_off_, sino_off_, fwd_start_, back_start_;
    std::string signature_, gpu_name_;
    int ns_ = 0, sms_ = 0, device_ = 0, max_nx_ = 0, max_ny_ = 0;
    int wmax_ = 1, wcap_ = 0;  // widest tile window over the slices; plane stride of the back kernel
    int fw_ = 8, vc_ = 4;
    unsigned wait_limit_ = 1u << 22;
    cudaStream_t stream_ = nullptr;
    B1Slice* d_slices_ = nullptr;
    long long* d_start_ = nullptr;  // [forward starts | backward starts]
    unsigned long long* d_counter_ = nullptr;
    int* d_err_ = nullptr;
    float* d_imgT_ = nullptr;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
};

}  // namespace sgd
