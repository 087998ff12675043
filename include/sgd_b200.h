/* C ABI of sgd_b200/libnetwork.so, the B200-native CT projector library.
 *
 * The first group of each projector keeps the reference's extern "C" names and
 * signatures (hqpwca/SGD, layers/A_*.hh / layers/A_*.cu) so that callers that
 * bind the reference's libnetwork.so (python/operators/operators.py through
 * ctypes) bind this library unchanged.  The second group is new: explicit
 * destruction, error text, and FP32 device-pointer entry points for callers
 * that keep images and sinograms on the GPU.
 *
 * Conventions (all entry points):
 *   image    x[ix*ny + iy]        (reference host layout, layers/A_B1.cu:621-623)
 *   sinogram b[p*nu + u]          (layers/A_B1.cu:639-641)
 *   angles   radians, one per view
 *   errors   never thrown across the ABI: a failing call returns NULL / -1
 *            (void reference functions return nothing) and sgd_last_error()
 *            gives the message of the last failure on the calling thread.
 *   threads  calls on one handle must not overlap; distinct handles are
 *            independent.
 */
#ifndef SGD_B200_H
#define SGD_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Message of the last failure on this thread (new; the reference has no
 * error reporting, utils/exception.hh throws across the ABI). */
const char* sgd_last_error(void);

/* ---- geometry --------------------------------------------------------------- */

/* New, host only: per-view 3x4 projection matrices pm (FP64, may be NULL) and
 * their index-space FP32 form pmi, 12 values per view, as the reference's
 * GeoData::initialize_projection_matrix builds them (utils/geo.cu:58-201,
 * after geo_init_angles :232-269).  dz_off/drho may be NULL.  0 / -1. */
int sgd_geometry_pmi(int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy, double dz, double du,
                     double dv, double lsd, double lso, const double* angles, const double* dz_off,
                     const double* drho, double* pm_out, float* pmi_out);

/* ---- B1 bilinear box-spline, 2D fan beam ---------------------------------- */

/* Replaces b1_init, layers/A_B1.hh:24 / layers/A_B1.cu:595-603.  dz and drho
 * may be NULL (the reference declares them with C++ default arguments; a C
 * caller must pass all twelve).  Returns NULL on failure. */
void* b1_init(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
              double* angles, double* dz, double* drho);

/* Replaces b1_forward_projection, layers/A_B1.hh:25 / layers/A_B1.cu:605-644:
 * b = A x (b overwritten).  Returns the reference's footprint-evaluation count
 * for this geometry (its conv_count), or -1 on failure. */
int b1_forward_projection(double* b, double* x, void* layer);

/* Replaces b1_backward_projection, layers/A_B1.hh:26 / layers/A_B1.cu:646-678:
 * x = A^T b (x overwritten). */
void b1_backward_projection(double* b, double* x, void* layer);

/* New: b1_backward_projection with a status (0 ok, -1 failure). */
int sgd_b1_backward_projection(double* b, double* x, void* layer);

/* New: frees a layer returned by b1_init (the reference never frees). */
void b1_destroy(void* layer);

/* New: FP32 device entry points on a caller's stream (cudaStream_t, NULL =
 * legacy default stream).  d_img: nx*ny floats, d_sino: np*nu floats, both
 * device memory.  The forward overwrites d_sino, the backward d_img.
 * Return 0 on success, -1 on failure. */
int sgd_b1_forward_dev(void* layer, const float* d_img, float* d_sino, void* stream);
int sgd_b1_backward_dev(void* layer, const float* d_sino, float* d_img, void* stream);

/* New: the reference's footprint-evaluation count for the layer's geometry. */
unsigned long long sgd_b1_count(void* layer);

/* New: synchronises and reports (0 / -1, then clears) a device-side failure of
 * an earlier *_dev call: a kernel's bounded wait for its shared-memory staging
 * gave up, and the output of that call was not written. */
int sgd_b1_status(void* layer);

/* New, with no counterpart in the reference: the B1 forward projection of
 * sgd_b1_forward_dev without any device allocation during the call, for
 * callers that cannot call cudaMalloc while they run (code under another
 * framework's memory pool that owns the device heap; real-time loops where
 * cudaMalloc's implicit synchronisation is not allowed).  Its scratch is a
 * fixed 4 MiB __device__ array that every GPU loading this library holds until
 * exit, so images are limited to 1,048,576 pixels (1024 x 1024); larger ones
 * are rejected with -1 and a message.  The first call on each device looks up
 * the array's address (make it before any stream capture).  All calls share
 * the array: calls that overlap on the GPU race.  The layer's device must be
 * current.  Returns 0 on success, -1 on failure. */
int sgd_b1_forward_noalloc(void* layer, const float* d_img, float* d_sino, void* stream);

/* ---- A_SF separable footprint (SF-TR), 2D fan beam -------------------------- */

/* Replace SF_init / SF_forward_projection / SF_backward_projection,
 * layers/A_SF.hh:23-25 / layers/A_SF.cu:395-479 (same layouts as B1).  The
 * forward returns 0 as the reference does (its SF kernels never count), -1
 * on failure. */
void* SF_init(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
              double* angles);
int SF_forward_projection(double* b, double* x, void* layer);
void SF_backward_projection(double* b, double* x, void* layer);
/* New: status-returning backward, destruction, device entry points, count. */
int sgd_SF_backward_projection(double* b, double* x, void* layer);
void SF_destroy(void* layer);
int sgd_SF_forward_dev(void* layer, const float* d_img, float* d_sino, void* stream);
int sgd_SF_backward_dev(void* layer, const float* d_sino, float* d_img, void* stream);
unsigned long long sgd_SF_count(void* layer);

/* ---- B0 pixel indicator, 2D fan beam ----------------------------------------- */

/* Replace b0_init / b0_forward_projection / b0_backward_projection,
 * layers/A_B0.hh:24-26 / layers/A_B0.cu:494-575 (same layouts as B1; the
 * forward returns the reference's footprint-evaluation count). */
void* b0_init(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
              double* angles, double* dz, double* drho);
int b0_forward_projection(double* b, double* x, void* layer);
void b0_backward_projection(double* b, double* x, void* layer);
/* New: status-returning backward, destruction, device entry points, count. */
int sgd_b0_backward_projection(double* b, double* x, void* layer);
void b0_destroy(void* layer);
int sgd_b0_forward_dev(void* layer, const float* d_img, float* d_sino, void* stream);
int sgd_b0_backward_dev(void* layer, const float* d_sino, float* d_img, void* stream);
unsigned long long sgd_b0_count(void* layer);

/* ---- H0 / Hl hexagonal lattices, 2D fan beam --------------------------------- */

/* Replace h0_init / hl_init (layers/A_H0.cu:555-563, layers/A_Hl.cu:569-577):
 * nl rows of nc sites (odd rows nc-1 sites, shifted half a site), site
 * spacing dt; host layout x[ic*nl + il], sinogram b[p*nu + u].  h0_init
 * reproduces the reference including its bin bounds at the 0.5 dt row pitch
 * and its extra skip test in the back projection; hl_init the Hl basis. */
void* h0_init(int nl, int nc, int np, int nu, double dt, double du, double lsd, double lso, double* angles,
              double* dz, double* drho);
void* hl_init(int nl, int nc, int np, int nu, double dt, double du, double lsd, double lso, double* angles,
              double* dz, double* drho);
/* Replace h0_/hl_forward_projection and _backward_projection
 * (layers/A_H0.cu:565-642, layers/A_Hl.cu:579-656).  The H0 forward returns
 * the reference's count (three per visited bin), Hl 0 as the reference. */
int h0_forward_projection(double* b, double* x, void* layer);
void h0_backward_projection(double* b, double* x, void* layer);
int hl_forward_projection(double* b, double* x, void* layer);
void hl_backward_projection(double* b, double* x, void* layer);
/* New: any hexagonal mode.  mode 0 = H0 with the true hexagon bounds and no
 * skip test (an exact adjoint pair), 1 = H0 as the reference (h0_init),
 * 2 = Hl (hl_init).  Use the h0_* entry points below on a mode-0 layer. */
void* sgd_hex_init(int mode, int nl, int nc, int np, int nu, double dt, double du, double lsd, double lso,
                   double* angles, double* dz, double* drho);
int sgd_h0_backward_projection(double* b, double* x, void* layer);
int sgd_hl_backward_projection(double* b, double* x, void* layer);
void h0_destroy(void* layer);
void hl_destroy(void* layer);
int sgd_h0_forward_dev(void* layer, const float* d_img, float* d_sino, void* stream);
int sgd_h0_backward_dev(void* layer, const float* d_sino, float* d_img, void* stream);
int sgd_hl_forward_dev(void* layer, const float* d_img, float* d_sino, void* stream);
int sgd_hl_backward_dev(void* layer, const float* d_sino, float* d_img, void* stream);
unsigned long long sgd_h0_count(void* layer);
unsigned long long sgd_hl_count(void* layer);

/* ---- A_B1_3D cone beam ---------------------------------------------------- */

/* Replace b1_3d_init / b1_3d_forward_projection / b1_3d_backward_projection,
 * layers/A_B1_3D.hh:24 / layers/A_B1_3D.cu:686-772: volume x[(iz*ny + iy)*nx
 * + ix], projections b[(p*nv + v)*nu + u].  Both kernels reproduce the
 * reference, whose backward is not the transpose of its forward (no
 * 2/width factor, single-bin ranges skipped, layers/A_B1_3D.cu:404,433,436).
 * The forward returns the reference's footprint-evaluation count (~0 on
 * failure). */
void* b1_3d_init(int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy, double dz, double du,
                 double dv, double lsd, double lso, double* angles);
unsigned long long b1_3d_forward_projection(double* b, double* x, void* layer);
void b1_3d_backward_projection(double* b, double* x, void* layer);
/* New: mode 0 = as b1_3d_init, mode 1 = the backward is the exact transpose of
 * the forward (the dot-product-consistent pair autograd uses). */
void* sgd_b1_3d_init(int mode, int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy, double dz,
                     double du, double dv, double lsd, double lso, double* angles);
int sgd_b1_3d_backward_projection(double* b, double* x, void* layer);
void b1_3d_destroy(void* layer);
int sgd_b1_3d_forward_dev(void* layer, const float* d_vol, float* d_proj, void* stream);
int sgd_b1_3d_backward_dev(void* layer, const float* d_proj, float* d_vol, void* stream);
unsigned long long sgd_b1_3d_count(void* layer);

/* ---- SF_projector: 3D separable footprint --------------------------------- */

/* New entry points for the class SF of layers/SF_projector.hh:9-23, which the
 * reference exposes only as a C++ Layer (SF::SF(GeoData*), SF::project,
 * SF::back_project, layers/SF_projector.cu:359-400); the geometry is that of
 * b1_3d_init (GeoData::geo_init_angles).  Layouts as A_B1_3D.
 * mode 0 reproduces the reference kernels: the forward accumulates the
 * footprint of every non-zero voxel without its value or amplitude, and bins
 * past the u edges wrap into neighbouring detector rows.  mode 1 applies the
 * voxel value and amplitude, drops out-of-detector bins, and its backward is
 * the exact transpose of its forward.  trap_v: SF-TT (trapezoid in v) in the
 * forward (the reference's `tt` argument); mode 1's backward follows it. */
void* sgd_sf3d_init(int mode, int trap_v, int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy,
                    double dz, double du, double dv, double lsd, double lso, double* angles);
int sgd_sf3d_forward_projection(double* b, double* x, void* layer);
int sgd_sf3d_backward_projection(double* b, double* x, void* layer);
void sgd_sf3d_destroy(void* layer);
int sgd_sf3d_forward_dev(void* layer, const float* d_vol, float* d_proj, void* stream);
int sgd_sf3d_backward_dev(void* layer, const float* d_proj, float* d_vol, void* stream);

/* ---- system matrices ------------------------------------------------------ */

/* Replace pixel_matrix_generation / bilinear_matrix_generation
 * (layers/A_B0.cu:449-492, layers/A_B1.cu:545-593; python/matrix_gen/
 * A_B0_project.py:16, A_B1_project.py:16): uniform angles 2 pi p / np
 * (geo_init_example, no 45-degree snap), triplets (row p*nu + u, column
 * i*ny + j, value) as three doubles each in spmat, row-major, values > 0
 * without the dx*dy factor, each generator's own footprint formula.  Built on
 * the GPU in O(entries) instead of one dense nu x nx*ny slab per view.
 * Returns the entry count; -1 (with sgd_last_error) when buffer_size entries
 * do not hold the matrix, where the reference asserts. */
int pixel_matrix_generation(int np, int nu, int nx, int ny, double dx, double dy, double du, double lsd, double lso,
                            double* spmat, int buffer_size);
int bilinear_matrix_generation(int np, int nu, int nx, int ny, double dx, double dy, double du, double lsd,
                               double lso, double* spmat, int buffer_size);
/* New: the system matrix of a layer as CSR (rowptr[np*nu + 1] int64, cols
 * int32, vals FP64; rows p*nu + u, columns in the layer's host layout), the
 * same pairs and FP32 footprints its kernels use, area factor included, so
 * that A x equals the layer's forward projection.  With all three outputs
 * null it only counts.  Returns the entry count, -1 on error (cap too small
 * included). */
long long sgd_b1_matrix_csr(void* layer, long long* rowptr, int* cols, double* vals, long long cap);
long long sgd_b0_matrix_csr(void* layer, long long* rowptr, int* cols, double* vals, long long cap);
long long sgd_SF_matrix_csr(void* layer, long long* rowptr, int* cols, double* vals, long long cap);
long long sgd_h0_matrix_csr(void* layer, long long* rowptr, int* cols, double* vals, long long cap);
long long sgd_hl_matrix_csr(void* layer, long long* rowptr, int* cols, double* vals, long long cap);

/* ---- measurement ---------------------------------------------------------- */

/* New (no reference counterpart): FP32 FMA throughput of the current GPU in
 * FLOP/s (FMA = 2 FLOPs), the roofline denominator of the projectors.
 * scratch: >= blocks floats of device memory.  Returns -1 on failure. */
double sgd_fp32_fma_rate(float* scratch, int blocks, int iters, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SGD_B200_H */
