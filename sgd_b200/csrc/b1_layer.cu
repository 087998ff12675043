// A_B1 layer: tables, staging and the FP64 host paths around the B1 kernels.
// Reference: layers/A_B1.cu:480-541 (class) and :595-678 (C entry points).
#include "b1_layer.h"

#include <cstring>

#include "common.h"

namespace sgd {

namespace {

__global__ void vol_to_img_kernel(const double* __restrict__ vol, float* __restrict__ img, int nx, int ny) {
    // vol[j*nx + i] (reference device layout) -> img[i*ny + j]
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)nx * ny) return;
    const int i = (int)(e / ny), j = (int)(e - (long long)i * ny);
    img[e] = (float)vol[(size_t)j * nx + i];
}

__global__ void add_img_to_vol_kernel(const float* __restrict__ img, double* __restrict__ vol, int nx, int ny) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)nx * ny) return;
    const int i = (int)(e / ny), j = (int)(e - (long long)i * ny);
    vol[(size_t)j * nx + i] += (double)img[e];
}

__global__ void add_sino_to_umajor_kernel(const float* __restrict__ sino, double* __restrict__ proj, int np, int nu) {
    // sino[p*nu + u] -> proj[u*np + p] (+=), the forward layout of layers/A_B1.cu:161
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)np * nu) return;
    const int p = (int)(e / nu), u = (int)(e - (long long)p * nu);
    proj[(size_t)u * np + p] += (double)sino[e];
}

__global__ void f64_to_f32_kernel(const double* __restrict__ a, float* __restrict__ b, long long n) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) b[e] = (float)a[e];
}

inline unsigned blocks_for(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

A_B1::A_B1(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
           const double* angles, const double* dz, const double* drho) {
    geo.init(nx, ny, np, nu, dx, dy, du, lsd, lso, angles, dz, drho);
    SGD_CUDA(cudaGetDevice(&device));
    std::vector<float> rec, strip;
    std::vector<BinHomography> hom;
    b1_tables(geo, rec, strip);
    bin_homographies(geo, hom);
    SGD_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    SGD_CUDA(cudaMalloc(&d_rec_, rec.size() * sizeof(float)));
    SGD_CUDA(cudaMalloc(&d_strip_, strip.size() * sizeof(float)));
    SGD_CUDA(cudaMalloc(&d_hom_, hom.size() * sizeof(BinHomography)));
    SGD_CUDA(cudaMemcpy(d_rec_, rec.data(), rec.size() * sizeof(float), cudaMemcpyHostToDevice));
    SGD_CUDA(cudaMemcpy(d_strip_, strip.data(), strip.size() * sizeof(float), cudaMemcpyHostToDevice));
    SGD_CUDA(cudaMemcpy(d_hom_, hom.data(), hom.size() * sizeof(BinHomography), cudaMemcpyHostToDevice));
    dev.nx = nx; dev.ny = ny; dev.np = np; dev.nu = nu;
    dev.dxdy = (float)(dx * dy);
    dev.rec = d_rec_; dev.strip = d_strip_; dev.hom = d_hom_;
    std::vector<int> wins;
    dev.wmax = b1_back_windows(geo, hom, wins);
    dev.wcap = b1_back_plane(dev.wmax);
    SGD_CUDA(cudaMalloc(&d_wins_, wins.size() * sizeof(int)));
    SGD_CUDA(cudaMemcpy(d_wins_, wins.data(), wins.size() * sizeof(int), cudaMemcpyHostToDevice));
    dev.wins = d_wins_;
    SGD_CUDA(cudaMalloc(&d_err_, sizeof(int)));
    SGD_CUDA(cudaMemset(d_err_, 0, sizeof(int)));
    dev.err = d_err_;
    b1_prepare_device(dev.wcap);

    const size_t nimg = (size_t)nx * ny, nsino = (size_t)np * nu;
    SGD_CUDA(cudaMalloc(&st.d_img, nimg * sizeof(float)));
    SGD_CUDA(cudaMalloc(&st.d_imgT, nimg * sizeof(float)));
    SGD_CUDA(cudaMalloc(&st.d_sino, nsino * sizeof(float)));
    SGD_CUDA(cudaMallocHost(&st.h_img, nimg * sizeof(float)));
    SGD_CUDA(cudaMallocHost(&st.h_sino, nsino * sizeof(float)));
    SGD_CUDA(cudaMallocHost(&st.h_err, sizeof(int)));
    count = b1_count(dev, stream);
}

A_B1::~A_B1() {
    if (stream) cudaStreamSynchronize(stream);
    cudaFree(d_rec_);
    cudaFree(d_strip_);
    cudaFree(d_hom_);
    cudaFree(d_err_);
    cudaFree(d_wins_);
    cudaFree(st.d_img);
    cudaFree(st.d_imgT);
    cudaFree(st.d_sino);
    cudaFreeHost(st.h_img);
    cudaFreeHost(st.h_sino);
    cudaFreeHost(st.h_err);
    if (stream) cudaStreamDestroy(stream);
}

void A_B1::forward_dev(const float* d_img, float* d_sino, cudaStream_t s) {
    b1_forward_launch(dev, d_img, st.d_imgT, d_sino, s);
}

void A_B1::backward_dev(const float* d_sino, float* d_img, cudaStream_t s) { b1_back_launch(dev, d_sino, d_img, s); }

void A_B1::forward_host(double* b, const double* x) {
    const long long nimg = (long long)dev.nx * dev.ny, nsino = (long long)dev.np * dev.nu;
#pragma omp parallel for schedule(static) if (nimg > (1 << 16))
    for (long long e = 0; e < nimg; ++e) st.h_img[e] = (float)x[e];
    SGD_CUDA(cudaMemcpyAsync(st.d_img, st.h_img, nimg * sizeof(float), cudaMemcpyHostToDevice, stream));
    forward_dev(st.d_img, st.d_sino, stream);
    SGD_CUDA(cudaMemcpyAsync(st.h_sino, st.d_sino, nsino * sizeof(float), cudaMemcpyDeviceToHost, stream));
    SGD_CUDA(cudaMemcpyAsync(st.h_err, d_err_, sizeof(int), cudaMemcpyDeviceToHost, stream));
    SGD_CUDA(cudaStreamSynchronize(stream));
    raise_device_error(*st.h_err);
#pragma omp parallel for schedule(static) if (nsino > (1 << 16))
    for (long long e = 0; e < nsino; ++e) b[e] = (double)st.h_sino[e];
}

void A_B1::backward_host(const double* b, double* x) {
    const long long nimg = (long long)dev.nx * dev.ny, nsino = (long long)dev.np * dev.nu;
#pragma omp parallel for schedule(static) if (nsino > (1 << 16))
    for (long long e = 0; e < nsino; ++e) st.h_sino[e] = (float)b[e];
    SGD_CUDA(cudaMemcpyAsync(st.d_sino, st.h_sino, nsino * sizeof(float), cudaMemcpyHostToDevice, stream));
    backward_dev(st.d_sino, st.d_img, stream);
    SGD_CUDA(cudaMemcpyAsync(st.h_img, st.d_img, nimg * sizeof(float), cudaMemcpyDeviceToHost, stream));
    SGD_CUDA(cudaMemcpyAsync(st.h_err, d_err_, sizeof(int), cudaMemcpyDeviceToHost, stream));
    SGD_CUDA(cudaStreamSynchronize(stream));
    raise_device_error(*st.h_err);
#pragma omp parallel for schedule(static) if (nimg > (1 << 16))
    for (long long e = 0; e < nimg; ++e) x[e] = (double)st.h_img[e];
}

void A_B1::check_device_status(bool sync_device) {
    int e = 0;
    // the *_dev calls may have run on any of the caller's streams
    if (sync_device) SGD_CUDA(cudaDeviceSynchronize());
    SGD_CUDA(cudaMemcpy(&e, d_err_, sizeof(int), cudaMemcpyDeviceToHost));
    raise_device_error(e);
}

void A_B1::raise_device_error(int e) {
    if (e) {
        SGD_CUDA(cudaMemset(d_err_, 0, sizeof(int)));
        fail("B1 back projector: a shared-memory staging wait timed out; output not written");
    }
}

void A_B1::project(MatrixD& vol, MatrixD& proj, double /*weight*/) {
    // layers/A_B1.cu:512-525: vol on the device as [iy][ix], proj accumulated
    // on the device in the u-major layout [u][p].
    const long long nimg = (long long)dev.nx * dev.ny, nsino = (long long)dev.np * dev.nu;
    vol_to_img_kernel<<<blocks_for(nimg, 256), 256, 0, stream>>>(vol(0), st.d_img, dev.nx, dev.ny);
    SGD_LAUNCH_CHECK();
    forward_dev(st.d_img, st.d_sino, stream);
    add_sino_to_umajor_kernel<<<blocks_for(nsino, 256), 256, 0, stream>>>(st.d_sino, proj(0), dev.np, dev.nu);
    SGD_LAUNCH_CHECK();
    SGD_CUDA(cudaStreamSynchronize(stream));
    check_device_status(false);
}

void A_B1::back_project(MatrixD& vol, MatrixD& proj, double /*weight*/) {
    // layers/A_B1.cu:527-541: proj on the device as [p][u], vol accumulated as [iy][ix].
    const long long nimg = (long long)dev.nx * dev.ny, nsino = (long long)dev.np * dev.nu;
    f64_to_f32_kernel<<<blocks_for(nsino, 256), 256, 0, stream>>>(proj(0), st.d_sino, nsino);
    SGD_LAUNCH_CHECK();
    backward_dev(st.d_sino, st.d_img, stream);
    add_img_to_vol_kernel<<<blocks_for(nimg, 256), 256, 0, stream>>>(st.d_img, vol(0), dev.nx, dev.ny);
    SGD_LAUNCH_CHECK();
    SGD_CUDA(cudaStreamSynchronize(stream));
    check_device_status(false);
}

}  // namespace sgd
