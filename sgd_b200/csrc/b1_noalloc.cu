// sgd_b1_forward_noalloc: the B1 forward projection without any device
// allocation during the call.
//
// Some callers cannot call cudaMalloc while they run: code living under
// another framework's memory pool that owns the device heap, or a real-time
// reconstruction loop where cudaMalloc's implicit device synchronisation is
// not allowed.  The regular device entry point (sgd_b1_forward_dev) needs a
// transposed copy of the image as scratch, which the layer allocates for
// itself at b1_init.  This entry point uses a fixed scratch array instead: a
// file-scope __device__ array of kNoAllocMaxPixels floats (4 MiB), which the
// driver places in every GPU's memory when it loads this library's device
// code and keeps until the process exits.  The caller passes the layer (made
// earlier by b1_init), the input image and the output sinogram, all on the
// device.
//
// Set-up: the first call on each device looks up the array's device address
// with cudaGetSymbolAddress (the host-side symbol is only a stand-in, not a
// device address) and caches it for that device; make that first call before
// any stream capture.  The cache lives as long as the process: a
// cudaDeviceReset destroys the context that owns the array (and every layer
// made in it), after which the cached address is stale, so the entry point
// is not to be called after a reset.  The image must be at most kNoAllocMaxPixels pixels.
// Every call shares the one array; a call overwrites all of the scratch it
// reads before reading it, so nothing needs clearing, but calls that overlap
// on the GPU (concurrent streams, or several host threads) race on it.
#include <cuda_runtime.h>

#include <mutex>

#include "b1_layer.h"
#include "common.h"

namespace {

constexpr size_t kNoAllocMaxPixels = size_t(1) << 20;  // 1024 x 1024 images
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float g_transpose_scratch[kNoAllocMaxPixels];

float* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

// Device address of g_transpose_scratch on the current device (looked up once
// per device, with that device current).
float* scratch_on_current_device() {
    int dev = -1;
    SGD_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) sgd::fail("sgd_b1_forward_noalloc: device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_transpose_scratch);
        if (e != cudaSuccess || !p)
            sgd::fail("sgd_b1_forward_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                      cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<float*>(p);
    }
    return g_scratch_addr[dev];
}

}  // namespace

extern "C" int sgd_b1_forward_noalloc(void* layer, const float* d_img, float* d_sino, void* stream) {
    return sgd::guarded_status([&] {
        if (!layer || !d_img || !d_sino) sgd::fail("sgd_b1_forward_noalloc: null argument");
        sgd::A_B1* L = static_cast<sgd::A_B1*>(layer);
        const size_t pixels = (size_t)L->dev.nx * L->dev.ny;
        if (pixels > kNoAllocMaxPixels)
            sgd::fail("sgd_b1_forward_noalloc: image of %d x %d = %zu pixels exceeds this entry point's fixed "
                      "scratch of %zu pixels; use sgd_b1_forward_dev",
                      L->dev.nx, L->dev.ny, pixels, kNoAllocMaxPixels);
        int dev = -1;
        SGD_CUDA(cudaGetDevice(&dev));
        if (dev != L->device)
            sgd::fail("sgd_b1_forward_noalloc: layer lives on device %d but device %d is current", L->device, dev);
        sgd::b1_forward_launch(L->dev, d_img, scratch_on_current_device(), d_sino,
                               static_cast<cudaStream_t>(stream));
    });
}
