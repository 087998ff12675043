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

/* New, host only: the 64-byte B1 footprint record of every (view, bin), as
 * the B1 kernels read them (np*nu*16 floats, layout [view][chunk][bin][4]):
 * the edge offsets ya = i*r0 + (j*r2 + r4), yb = i*r1 + (j*r3 + r5) of pixel
 * (i, j) on the line through its centre across the bin's central ray, in
 * units of the profile half-width a, and the constants of the closed-form
 * footprint (beta, beta, 1+beta, 1+beta, -beta^2/12 twice, 1/(12 beta^2)
 * twice, 1/a, a; beta = b/a) that replaces the reference's
 * linear_convolution_1d (layers/A_B1.cu:182-197, layers/spline_conv.hh:
 * 295-405).  Arguments as b1_init.  0 / -1. */
int sgd_b1_bin_records(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
                       const double* angles, const double* dz, const double* drho, float* rec_out);

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

/* New, for testing the failure path above: the polls each back-projection
 * staging wait makes before it gives up (default 4194304).  With 0 every
 * wait gives up at once: the kernel still waits, with the full limit, for the
 * copies it issued, leaves its tiles unwritten and sets the flag that
 * sgd_b1_status reports; restoring the default restores normal calls.
 * Returns 0, or -1 for a null layer. */
int sgd_b1_set_wait_limit(void* layer, unsigned polls);

/* New, with no counterpart in the reference: the B1 forward projection of
 * sgd_b1_forward_dev without any device allocation during the call, for
 * callers that cannot call cudaMalloc while they run (code under another
 * framework's memory pool that owns the device heap; real-time loops where
 * cudaMalloc's implicit synchronisation is not allowed).  Its scratch is a
 * fixed 4 MiB __device__ array that every GPU loading this library holds until
 * exit, so images are limited to 1,048,576 pixels (1024 x 1024); larger ones
 * are rejected with -1 and a message.  The first call on each device looks up
 * the array's address (make it before any stream capture) and keeps it for
 * the process: after a cudaDeviceReset, which invalidates both that address
 * and every layer, this entry point must not be called again.  All calls
 * share the array: calls that overlap on the GPU race.  The layer's device
 * must be current.  Returns 0 on success, -1 on failure. */
int sgd_b1_forward_noalloc(void* layer, const float* d_img, float* d_sino, void* stream);

/* New: B1 in the reference layer's FP32 rounding.  Same arguments, layouts
 * and count as b1_init / b1_forward_projection / b1_backward_projection
 * (layers/A_B1.cu:595-678), but the bin centres are stepped in FP32 from each
 * pixel's first bin and the edge-ray offsets come from the reference's FP32
 * intersections (layers/A_B1.cu:100-197), so the output stays within a few
 * units in the last place of the reference's own; the b1_* layer evaluates
 * the exact bin geometry instead.  Runs on the generic 2D kernels. */
void* sgd_b1ref_init(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
                     double* angles, double* dz, double* drho);
int sgd_b1ref_forward_projection(double* b, double* x, void* layer);
int sgd_b1ref_backward_projection(double* b, double* x, void* layer);
void sgd_b1ref_destroy(void* layer);
int sgd_b1ref_forward_dev(void* layer, const float* d_img, float* d_sino, void* stream);
int sgd_b1ref_backward_dev(void* layer, const float* d_sino, float* d_img, void* stream);
unsigned long long sgd_b1ref_count(void* layer);

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

/* New (the reference has only point-source geometry, utils/geo.cu:234): B0 in
 * parallel-beam geometry.  View angle beta: rays along (cos beta, sin beta),
 * detector axis (-sin beta, cos beta) through the isocentre, nu bins of pitch
 * du centred on it.  The handle takes the b0_* and sgd_b0_* calls above. */
void* sgd_b0_parallel_init(int nx, int ny, int np, int nu, double dx, double dy, double du, double* angles);

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

/* New, for every layer of the generic 2D kernels (SF, B0, B0 parallel, H0,
 * Hl, B1 reference rounding): synchronises the layer's stream and reports
 * (0 / -1 with sgd_last_error, then clears) a back projection whose bounded
 * wait for its shared-memory staging gave up; those tiles were left
 * unwritten.  The FP64 host entry points check it themselves. */
int sgd_proj2d_status(void* layer);
/* New, for testing that path: as sgd_b1_set_wait_limit, for these layers. */
int sgd_proj2d_set_wait_limit(void* layer, unsigned polls);

/* New, host only (no GPU needed): the plan of the generic 2D kernels for an
 * nx x ny grid of cells in the fan geometry of b1_init (np views at angles,
 * nu bins of pitch du, distances lsd, lso), cell (i, j) at x = x0 + i dx,
 * y = y0 + j dy, whose bin ranges come from points within ri (along i) and
 * rj (along j) cells of it: the forward's block strips, 8 floats per (view,
 * block of 32 bins), and the back projection's bin windows, 2 ints (first,
 * last) per (tile of 8 x 32 cells, view).  Returns the widest window in bins,
 * -1 on error. */
int sgd_fan2d_plan(int nx, int ny, int np, int nu, double x0, double dx, double y0, double dy, double ri, double rj,
                   double du, double lsd, double lso, const double* angles, float* strips, int* twin);

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

/* New: synchronises the device and reports (0 / -1 with sgd_last_error, then
 * clears) an A_B1_3D back projection on the *_dev entry point whose bounded
 * wait for its staged projection window gave up; those voxels were left
 * unwritten.  The FP64 host entry point checks it itself. */
int sgd_b1_3d_status(void* layer);
/* New: the polls an A_B1_3D back projection spends waiting for one staged
 * view before it gives up (default 4194304); applies to later calls. */
int sgd_b1_3d_set_wait_limit(void* layer, unsigned limit);

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
 * forward (the reference's `tt` argument); mode 1's backward follows it.
 * The FP64 host entry points round their inputs to FP32 as the reference's
 * SF class does; mode 1 returns its FP64 accumulators, mode 0 rounds its
 * output to FP32 as the reference does; the *_dev entry points are FP32.
 * Mode 1 needs a circular orbit (the detector's u row of every projection
 * matrix free of z, which geo_init_angles geometries are). */
void* sgd_sf3d_init(int mode, int trap_v, int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy,
                    double dz, double du, double dv, double lsd, double lso, double* angles);
int sgd_sf3d_forward_projection(double* b, double* x, void* layer);
int sgd_sf3d_backward_projection(double* b, double* x, void* layer);
void sgd_sf3d_destroy(void* layer);
int sgd_sf3d_forward_dev(void* layer, const float* d_vol, float* d_proj, void* stream);
int sgd_sf3d_backward_dev(void* layer, const float* d_proj, float* d_vol, void* stream);
/* New: as sgd_b1_3d_status, for mode 1's back projection (mode 0's has no
 * staged wait and always reports 0). */
int sgd_sf3d_status(void* layer);
/* New: the polls a mode-1 back projection spends waiting for one staged view
 * before it gives up (default 4194304); applies to later calls. */
int sgd_sf3d_set_wait_limit(void* layer, unsigned limit);

/* ---- batched B1: many slices per launch ----------------------------------- */

/* New (the reference launches per view and per slice, layers/A_B1.cu:514-524):
 * ns fan-beam slices, each with the arguments of b1_init (no dz/drho), in one
 * persistent launch per direction.  Device arenas hold slice k's image at
 * img_off[k] (layout i*ny + j) and its sinogram at sino_off[k] ([p][u]);
 * sgd_b1_batch_offsets fills both arrays (ns + 1 entries each, the last is
 * the arena length).  capture/replay record forward (img -> sino) and/or
 * backward (sino_in -> img_out) into a CUDA graph on fixed arenas.  tune
 * picks the launch shape (warps per forward item, views per staged chunk)
 * from the cache file or by timing every variant (then appends it); returns
 * 1 when loaded, 0 when measured, -1 on error. */
void* sgd_b1_batch_create(int ns, const int* nx, const int* ny, const int* np, const int* nu, const double* dx,
                          const double* dy, const double* du, const double* lsd, const double* lso,
                          const double* const* angles);
void sgd_b1_batch_destroy(void* batch);
int sgd_b1_batch_offsets(void* batch, long long* img_off, long long* sino_off);
int sgd_b1_batch_forward(void* batch, const float* d_img, float* d_sino, void* stream);
int sgd_b1_batch_backward(void* batch, const float* d_sino, float* d_img, void* stream);
int sgd_b1_batch_capture(void* batch, const float* d_img, float* d_sino, const float* d_sino_in, float* d_img_out);
int sgd_b1_batch_replay(void* batch, void* stream);
int sgd_b1_batch_tune(void* batch, const char* cache_path, int* fw, int* vc);
/* set_variant and tune rewrite the work-item table the persistent kernels
 * read: they synchronise the device first and must not be called while
 * another thread has batch work in flight. */
int sgd_b1_batch_set_variant(void* batch, int fw, int vc);
int sgd_b1_batch_status(void* batch);
/* New, for testing the failure path: as sgd_b1_set_wait_limit, for the
 * batch's back projection (drops a captured graph). */
int sgd_b1_batch_set_wait_limit(void* batch, unsigned polls);

/* ---- ASD-POCS and its phantom simulator ----------------------------------- */

/* New (the reference's optimizer/asd_pocs.cu is empty): ASD-POCS (Sidky and
 * Pan 2008: SART step, optional positivity, adaptive TV descent) over the slices of a
 * batch, every scalar per image on the device, one CUDA graph per iteration.
 * bind() takes the iterate and data arenas (the batch's layout) and the image
 * shapes and resets the adaptive state; history() returns (|Ax-b|, |dx_SART|,
 * |dx_TV|) per iteration and image for the first hist_cap iterations. */
void* sgd_asd_create(void* batch, float beta, float beta_red, float alpha, float alpha_red, float r_max, float eps,
                     int ng, int nonneg);
void sgd_asd_destroy(void* h);
int sgd_asd_bind(void* h, float* d_x, const float* d_b, const int* nx, const int* ny, int hist_cap);
int sgd_asd_reset(void* h);
int sgd_asd_run(void* h, int iters, void* stream);
int sgd_asd_history(void* h, float* out, int iters);
/* New: fan-beam sinograms of ellipse phantoms (closed-form chords averaged over
 * `sub` rays per bin); with i0 > 0, Poisson counts and b = 100 ln(i0/counts),
 * the noise model of python/FORBILD.py:355-390. */
int sgd_ellipse_sinograms(const double* ell, int nell, int ni, int np, int nu, double du, double lsd, double lso,
                          const double* angles, int sub, double i0, unsigned long long seed, float* d_out,
                          void* stream);

/* ---- warm-start CNN kernels ----------------------------------------------- */

/* New (no reference counterpart; layers/layer.hh:9-17 is an MLP scaffold):
 * 3x3 convolution, zero padding, NCHW FP32 activations, BF16 weights
 * [Cout][Cin][3][3], FP32 accumulation; input gradient (scratch: Cin*Cout*9
 * BF16), weight and bias gradients (accumulated into), ReLU backward, MSE
 * gradient, Adam on FP32 master weights with a BF16 copy. */
int sgd_conv3x3_forward(const float* in, const void* w_bf16, const float* bias, float* out, int N, int Cin, int Cout,
                        int H, int W, int relu, void* stream);
int sgd_conv3x3_backward_data(const float* gout, const void* w_bf16, void* scratch_bf16, float* gin, int N, int Cin,
                              int Cout, int H, int W, void* stream);
int sgd_conv3x3_backward_weight(const float* in, const float* gout, float* gw, float* gbias, int N, int Cin, int Cout,
                                int H, int W, void* stream);
int sgd_relu_backward(float* g, const float* out, long long n, void* stream);
int sgd_mse_grad(const float* y, const float* t, float* g, long long n, double* d_loss, void* stream);
int sgd_adam_step(float* w, void* w_bf16, const float* g, float* m, float* v, long long n, float lr, float b1,
                  float b2, float eps, int step, void* stream);
/* New: sgd_conv3x3_forward for 32 input and 32 output channels (the
 * network's middle layers) on the sm_100 tensor cores: an implicit GEMM per
 * 128-pixel row segment issued as tcgen05.mma with the accumulator in tensor
 * memory; each FP32 activation enters as three BF16 terms, so the products
 * are exact and the result is an FP32 accumulation as in the direct kernel.
 * Other channel counts: -1 with a message.  sgd_conv3x3_tc_status
 * synchronises the device and returns -1 (and clears the flag) if a tile's
 * MMAs never completed within the kernel's bounded wait. */
int sgd_conv3x3_forward_tc(const float* in, const void* w_bf16, const float* bias, float* out, int N, int Cin,
                           int Cout, int H, int W, int relu, void* stream);
int sgd_conv3x3_tc_status(void);

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
long long sgd_b1ref_matrix_csr(void* layer, long long* rowptr, int* cols, double* vals, long long cap);

/* ---- measurement ---------------------------------------------------------- */

/* New (no reference counterpart): FP32 FMA throughput of the current GPU in
 * FLOP/s (FMA = 2 FLOPs), the roofline denominator of the projectors.
 * scratch: >= blocks floats of device memory.  Returns -1 on failure. */
double sgd_fp32_fma_rate(float* scratch, int blocks, int iters, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SGD_B200_H */
