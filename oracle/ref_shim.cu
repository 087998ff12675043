// ORACLE — test/bench infrastructure only.  Compiled together with the
// reference's own sources into oracle/_ref/libnetwork.so; never part of the
// product.  Adds entry points the reference does not export, so that its
// kernels can be timed alone (device buffers already resident, no host
// transposes or copies): the reference-GPU bar in the benchmark notes.
#include <cuda_runtime.h>
#include "A_B1.hh"
#include "A_SF.hh"
#include "A_B0.hh"
#include "SF_projector.hh"
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

// SF_projector has no C entry points in the reference: these build its SF
// layer on the geometry b1_3d_init uses (layers/A_B1_3D.cu:686-694) and run
// SF::project / SF::back_project on FP64 host arrays x[(iz*ny+iy)*nx+ix],
// b[(p*nv+v)*nu+u] (through FP32 Matrix buffers, as the layer takes them).
extern "C" {
void* ref_sf3d_init(int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy, double dz, double du,
                    double dv, double lsd, double lso, double* angles) {
    GeoData* geo = new GeoData(nx, ny, nz, nu, nv, np, dx, dy, dz, du, dv);
    geo->geo_init_angles(lsd, lso, angles);
    geo->initialize_projection_matrix();
    return new SF(geo);
}
void ref_sf3d_destroy(SF* layer) {
    delete layer->geodata;
    delete layer;
}
int ref_sf3d_forward(SF* layer, const double* x, double* b, int trap) {
    GeoData* g = layer->geodata;
    const size_t nvol = (size_t)g->nxyz.x * g->nxyz.y * g->nxyz.z, nproj = (size_t)g->np * g->nuv.x * g->nuv.y;
    Matrix vol(nvol, 1), proj(nproj, 1);
    vol.allocateMemory();
    proj.allocateMemory();
    for (size_t i = 0; i < nvol; ++i) *vol[i] = (float)x[i];
    vol.copyHostToDevice();
    cudaMemset(proj(0), 0, nproj * sizeof(float));
    layer->project(vol, proj, 1.0, trap != 0);
    proj.copyDeviceToHost();
    for (size_t i = 0; i < nproj; ++i) b[i] = *proj[i];
    return (int)cudaDeviceSynchronize();
}
int ref_sf3d_backward(SF* layer, const double* b, double* x) {
    GeoData* g = layer->geodata;
    const size_t nvol = (size_t)g->nxyz.x * g->nxyz.y * g->nxyz.z, nproj = (size_t)g->np * g->nuv.x * g->nuv.y;
    Matrix vol(nvol, 1), proj(nproj, 1);
    vol.allocateMemory();
    proj.allocateMemory();
    for (size_t i = 0; i < nproj; ++i) *proj[i] = (float)b[i];
    proj.copyHostToDevice();
    cudaMemset(vol(0), 0, nvol * sizeof(float));
    layer->back_project(vol, proj, 1.0);
    vol.copyDeviceToHost();
    for (size_t i = 0; i < nvol; ++i) x[i] = *vol[i];
    return (int)cudaDeviceSynchronize();
}
}
