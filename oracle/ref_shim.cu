// ORACLE — test/bench infrastructure only.  Compiled together with the
// reference's own sources into oracle/_ref/libnetwork.so; never part of the
// product.  Adds entry points the reference does not export, so that its
// kernels can be timed alone (device buffers already resident, no host
// transposes or copies): the reference-GPU bar in the benchmark notes.
#include <cuda_runtime.h>
#include "A_B1.hh"
#include "A_SF.hh"
#include "A_B0.hh"
#include "../utils/matrix_double.hh"

namespace {
template <class L>
float time_layer(L* layer, int nvol, int nproj, int reps, float* ms_back) {
    MatrixD vol(nvol, 1), proj(nproj, 1);
    vol.allocateMemory();
    proj.allocateMemory();
    for (int i = 0; i < nvol; ++i) *vol[i] = 1.0;
    for (int i = 0; i < nproj; ++i) *proj[i] = 1.0;
    vol.copyHostToDevice();
    proj.copyHostToDevice();
    layer->project(vol, proj, 1.0);  // warm-up
    layer->back_project(vol, proj, 1.0);
    cudaDeviceSynchronize();
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2);
    cudaEventRecord(e0);
    for (int r = 0; r < reps; ++r) layer->project(vol, proj, 1.0);
    cudaEventRecord(e1);
    for (int r = 0; r < reps; ++r) layer->back_project(vol, proj, 1.0);
    cudaEventRecord(e2);
    cudaEventSynchronize(e2);
    float f = 0.f, b = 0.f;
    cudaEventElapsedTime(&f, e0, e1);
    cudaEventElapsedTime(&b, e1, e2);
    cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2);
    if (ms_back) *ms_back = b / reps;
    return f / reps;
}
}  // namespace

extern "C" {
// Average milliseconds of one A_B1::project (returned) and one
// A_B1::back_project (*ms_back) over `reps` calls, kernels only.
float ref_b1_kernel_ms(A_B1* layer, int reps, float* ms_back) {
    GeoData* g = layer->geodata;
    return time_layer(layer, g->nxyz.x * g->nxyz.y, g->np * g->nuv.x, reps, ms_back);
}
float ref_sf_kernel_ms(A_SF* layer, int reps, float* ms_back) {
    GeoData* g = layer->geodata;
    return time_layer(layer, g->nxyz.x * g->nxyz.y, g->np * g->nuv.x, reps, ms_back);
}
float ref_b0_kernel_ms(A_B0* layer, int reps, float* ms_back) {
    GeoData* g = layer->geodata;
    return time_layer(layer, g->nxyz.x * g->nxyz.y, g->np * g->nuv.x, reps, ms_back);
}
}
