// ASD-POCS on the GPU over a batch of fan-beam B1 slices, and a seeded
// ellipse-phantom sinogram simulator with Poisson noise to feed it.
//
// The reference's optimizer/asd_pocs.cu is empty; the algorithm is the
// adaptive-steepest-descent POCS of Sidky and Pan (Phys. Med. Biol. 53,
// 2008), per image:
//   x_prev = x
//   x += beta * A^T((b - A x) / R) / C          SART step, R = A 1, C = A^T 1
//   x = max(x, 0)                               positivity (optional)
//   dp = |x - x_prev|, x_res = x
//   dtvg = alpha * dp                           (first iteration only)
//   ng times: x -= dtvg * g / |g|, g = grad TV(x)
//   dg = |x - x_res|
//   if dg > r_max * dp and dd > eps: dtvg *= alpha_red
//   beta *= beta_red
// with dd = |A x - b| of the iterate entering the SART step.  Every scalar
// lives on the device (one slot per image) so that an iteration is a fixed
// launch sequence: it is captured once in a CUDA graph and replayed.
// Projections go through the persistent batched B1 kernels (b1_batch.cu).
#include <curand_kernel.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "b1_batch.h"
#include "common.h"

namespace sgd {

struct AsdParams {
    float beta = 1.0f, beta_red = 0.995f, alpha = 0.002f, alpha_red = 0.95f, r_max = 0.94f, eps = 0.0f;
    int ng = 20;
    int nonneg = 1;  // project onto x >= 0 after the SART step
};

namespace {

constexpr int kThreads = 256;

// per-image FP64 accumulators, index [slot * ni + image]; slots kN2.. kN2+ng-1
// hold |grad TV|^2 of each TV step
enum Slot { kDD = 0, kDP = 1, kDG = 2, kN2 = 3 };

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double s[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x < 32) {
        t = threadIdx.x < kThreads / 32 ? s[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    }
    __syncthreads();
    return t;  // valid in thread 0
}

// r = (b - Ax) / R on the sinograms; acc[kDD] += |b - Ax|^2.  blockIdx.y = image
__global__ void __launch_bounds__(kThreads) sart_residual_kernel(const float* __restrict__ b,
                                                                 const float* __restrict__ ax,
                                                                 const float* __restrict__ R, float* __restrict__ r,
                                                                 const long long* __restrict__ off, int ni,
                                                                 double* __restrict__ acc) {
    const int im = blockIdx.y;
    const long long o0 = off[im], n = off[im + 1] - o0;
    double s = 0.0;
    for (long long e = (long long)blockIdx.x * kThreads + threadIdx.x; e < n; e += (long long)gridDim.x * kThreads) {
        const float res = b[o0 + e] - ax[o0 + e];
        s += (double)res * res;
        const float w = R[o0 + e];
        r[o0 + e] = w > 1e-6f ? res / w : 0.f;
    }
    s = block_sum(s);
    if (threadIdx.x == 0) atomicAdd(&acc[kDD * ni + im], s);
}

// x = x + beta g / C (then max(., 0) when nonneg); acc[kDP] += |x - x_prev|^2
__global__ void __launch_bounds__(kThreads) sart_update_kernel(float* __restrict__ x, const float* __restrict__ g,
                                                               const float* __restrict__ C,
                                                               const float* __restrict__ x_prev,
                                                               const float* __restrict__ beta,
                                                               const long long* __restrict__ off, int ni,
                                                               int nonneg, double* __restrict__ acc) {
    const int im = blockIdx.y;
    const long long o0 = off[im], n = off[im + 1] - o0;
    const float bt = beta[im];
    double s = 0.0;
    for (long long e = (long long)blockIdx.x * kThreads + threadIdx.x; e < n; e += (long long)gridDim.x * kThreads) {
        const float w = C[o0 + e];
        float v = x[o0 + e] + (w > 1e-6f ? bt * g[o0 + e] / w : 0.f);
        if (nonneg) v = fmaxf(v, 0.f);
        const float d = v - x_prev[o0 + e];
        s += (double)d * d;
        x[o0 + e] = v;
    }
    s = block_sum(s);
    if (threadIdx.x == 0) atomicAdd(&acc[kDP * ni + im], s);
}

// Gradient of the isotropic TV (Sidky and Pan 2008, eq. 11) with eps = 1e-8
// and replicated edges, image layout x[i * ny + j]; acc[slot] += |grad|^2.
// shape[im] = (nx, ny).
__global__ void __launch_bounds__(kThreads) tv_grad_kernel(const float* __restrict__ x, float* __restrict__ gtv,
                                                           const long long* __restrict__ off,
                                                           const int2* __restrict__ shape, int ni, int slot,
                                                           double* __restrict__ acc) {
    const int im = blockIdx.y;
    const long long o0 = off[im];
    const int nx = shape[im].x, ny = shape[im].y;
    const float* X = x + o0;
    auto at = [&](int i, int j) {
        i = min(max(i, 0), nx - 1);
        j = min(max(j, 0), ny - 1);
        return __ldg(X + (size_t)i * ny + j);
    };
    constexpr float eps = 1e-8f;
    double s = 0.0;
    for (long long e = (long long)blockIdx.x * kThreads + threadIdx.x; e < (long long)nx * ny;
         e += (long long)gridDim.x * kThreads) {
        const int i = (int)(e / ny), j = (int)(e - (long long)i * ny);
        const float c = at(i, j);
        const float a1 = c - at(i - 1, j), a2 = c - at(i, j - 1);
        float g = (a1 + a2) * rsqrtf(eps + a1 * a1 + a2 * a2);
        const float xi = at(i + 1, j), b1 = xi - c, b2 = xi - at(i + 1, j - 1);
        g -= b1 * rsqrtf(eps + b1 * b1 + b2 * b2);
        const float xj = at(i, j + 1), c1 = xj - c, c2 = xj - at(i - 1, j + 1);
        g -= c1 * rsqrtf(eps + c1 * c1 + c2 * c2);
        gtv[o0 + e] = g;
        s += (double)g * g;
    }
    s = block_sum(s);
    if (threadIdx.x == 0) atomicAdd(&acc[slot * ni + im], s);
}

// x -= dtvg * g / |g|
__global__ void __launch_bounds__(kThreads) tv_step_kernel(float* __restrict__ x, const float* __restrict__ gtv,
                                                           const float* __restrict__ dtvg,
                                                           const long long* __restrict__ off, int ni, int slot,
                                                           const double* __restrict__ acc) {
    const int im = blockIdx.y;
    const long long o0 = off[im], n = off[im + 1] - o0;
    const double n2 = acc[slot * ni + im];
    if (!(n2 > 0.0)) return;
    const float f = (float)(dtvg[im] / sqrt(n2));
    for (long long e = (long long)blockIdx.x * kThreads + threadIdx.x; e < n; e += (long long)gridDim.x * kThreads)
        x[o0 + e] -= f * gtv[o0 + e];
}

// acc[slot] += |x - y|^2
__global__ void __launch_bounds__(kThreads) diff_norm_kernel(const float* __restrict__ x,
                                                             const float* __restrict__ y,
                                                             const long long* __restrict__ off, int ni, int slot,
                                                             double* __restrict__ acc) {
    const int im = blockIdx.y;
    const long long o0 = off[im], n = off[im + 1] - o0;
    double s = 0.0;
    for (long long e = (long long)blockIdx.x * kThreads + threadIdx.x; e < n; e += (long long)gridDim.x * kThreads) {
        const float d = x[o0 + e] - y[o0 + e];
        s += (double)d * d;
    }
    s = block_sum(s);
    if (threadIdx.x == 0) atomicAdd(&acc[slot * ni + im], s);
}

// Adaptive step sizes from this iteration's norms; clears the accumulators.
// iter[0] counts iterations; hist[(it * ni + image) * 3] records (dd, dp, dg)
// while it < hist_cap.
__global__ void asd_adapt_kernel(float* __restrict__ beta, float* __restrict__ dtvg, int* __restrict__ iter,
                                 double* __restrict__ acc, int nslots, int ni, AsdParams prm,
                                 float* __restrict__ hist, int hist_cap) {
    const int it = iter[0];
    for (int im = threadIdx.x; im < ni; im += blockDim.x) {
        const double dd = sqrt(acc[kDD * ni + im]), dp = sqrt(acc[kDP * ni + im]), dg = sqrt(acc[kDG * ni + im]);
        if (it == 0) dtvg[im] = (float)(prm.alpha * dp);
        if (dg > prm.r_max * dp && dd > prm.eps) dtvg[im] *= prm.alpha_red;
        beta[im] *= prm.beta_red;
        if (it < hist_cap) {
            hist[((size_t)it * ni + im) * 3 + 0] = (float)dd;
            hist[((size_t)it * ni + im) * 3 + 1] = (float)dp;
            hist[((size_t)it * ni + im) * 3 + 2] = (float)dg;
        }
        for (int s = 0; s < nslots; ++s) acc[s * ni + im] = 0.0;
    }
    __syncthreads();
    if (threadIdx.x == 0) iter[0] = it + 1;
}

__global__ void fill_kernel(float* a, long long n, float v) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) a[e] = v;
}

// ---- phantom sinogram simulator ---------------------------------------------

// Line integral of an ellipse phantom along the ray from (px, py) with unit
// direction (dx, dy): closed-form chords, each ellipse mapped to the unit
// circle.  ell: n x (cx, cy, a, b, phi, rho).
__device__ double ellipse_ray(const double* ell, int n, double px, double py, double dx, double dy) {
    double t = 0.0;
    for (int k = 0; k < n; ++k) {
        const double* e = ell + 6 * k;
        double s, c;
        sincos(e[4], &s, &c);
        const double ox = ((px - e[0]) * c + (py - e[1]) * s) / e[2];
        const double oy = (-(px - e[0]) * s + (py - e[1]) * c) / e[3];
        const double vx = (dx * c + dy * s) / e[2], vy = (-dx * s + dy * c) / e[3];
        const double vv = vx * vx + vy * vy;
        const double t0 = -(ox * vx + oy * vy) / vv;
        const double qx = ox + t0 * vx, qy = oy + t0 * vy;
        const double d2 = qx * qx + qy * qy;
        if (d2 < 1.0) t += e[5] * 2.0 * sqrt((1.0 - d2) / vv);
    }
    return t;
}

// One thread per (image, view, bin): the bin-averaged line integral over
// `sub` rays spread across the bin, then (i0 > 0) transmitted counts
// ~ Poisson(i0 exp(-L / 100)) and b = 100 ln(i0 / max(counts, 1)) (the scaling
// of python/FORBILD.py:355-390).  geo[view] = (src x, src y, dtv x, dtv y,
// puv x, puv y) in FP64.
__global__ void ellipse_sinogram_kernel(const double* __restrict__ ell, int nell, const double* __restrict__ geo,
                                        int ni, int np, int nu, int sub, double i0, unsigned long long seed,
                                        float* __restrict__ out) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ni * np * nu) return;
    const int im = (int)(t / ((long long)np * nu));
    const int p = (int)((t / nu) % np), u = (int)(t % nu);
    const double* g = geo + 6 * p;
    double L = 0.0;
    for (int k = 0; k < sub; ++k) {
        const double off = u - 0.5 * nu + (k + 0.5) / sub;
        const double qx = g[2] + g[4] * off, qy = g[3] + g[5] * off;
        const double dx = qx - g[0], dy = qy - g[1];
        const double len = sqrt(dx * dx + dy * dy);
        L += ellipse_ray(ell + (size_t)im * nell * 6, nell, g[0], g[1], dx / len, dy / len);
    }
    L /= sub;
    if (i0 > 0.0) {
        curandStatePhilox4_32_10_t st;
        curand_init(seed, (unsigned long long)t, 0, &st);
        const double lam = i0 * exp(-L / 100.0);
        const double c = (double)curand_poisson(&st, lam);
        L = 100.0 * log(i0 / fmax(c, 1.0));
    }
    out[t] = (float)L;
}

}  // namespace

class AsdPocs {
public:
    AsdPocs(B1Batch* batch, const AsdParams& prm) : B(batch), prm_(prm) {
        ni_ = (int)batch->img_off().size() - 1;
        const long long nimg = batch->img_off().back(), nsino = batch->sino_off().back();
        SGD_CUDA(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
        auto alloc = [&](float** p, long long n) { SGD_CUDA(cudaMalloc(p, std::max(1ll, n) * sizeof(float))); };
        alloc(&ax_, nsino); alloc(&r_, nsino); alloc(&R_, nsino);
        alloc(&g_, nimg); alloc(&C_, nimg); alloc(&xprev_, nimg); alloc(&xres_, nimg); alloc(&ones_, nimg);
        alloc(&beta_, ni_); alloc(&dtvg_, ni_);
        nslots_ = kN2 + prm.ng;
        SGD_CUDA(cudaMalloc(&acc_, (size_t)nslots_ * ni_ * sizeof(double)));
        SGD_CUDA(cudaMalloc(&iter_, sizeof(int)));
        SGD_CUDA(cudaMalloc(&off_img_, (ni_ + 1) * sizeof(long long)));
        SGD_CUDA(cudaMalloc(&off_sino_, (ni_ + 1) * sizeof(long long)));
        SGD_CUDA(cudaMalloc(&shape_, ni_ * sizeof(int2)));
        SGD_CUDA(cudaMemcpy(off_img_, batch->img_off().data(), (ni_ + 1) * sizeof(long long), cudaMemcpyHostToDevice));
        SGD_CUDA(cudaMemcpy(off_sino_, batch->sino_off().data(), (ni_ + 1) * sizeof(long long),
                            cudaMemcpyHostToDevice));
        for (int k = 0; k < ni_; ++k) {
            max_img_ = std::max(max_img_, batch->img_off()[k + 1] - batch->img_off()[k]);
            max_sino_ = std::max(max_sino_, batch->sino_off()[k + 1] - batch->sino_off()[k]);
        }
        // SART normalisations: R = A 1, C = A^T 1
        fill_kernel<<<(unsigned)((nimg + 255) / 256), 256, 0, s_>>>(ones_, nimg, 1.f);
        SGD_LAUNCH_CHECK();
        B->forward(ones_, R_, s_);
        fill_kernel<<<(unsigned)((nsino + 255) / 256), 256, 0, s_>>>(r_, nsino, 1.f);
        SGD_LAUNCH_CHECK();
        B->backward(r_, C_, s_);
        SGD_CUDA(cudaStreamSynchronize(s_));
        B->check_status();
    }
    ~AsdPocs() {
        if (s_) cudaStreamSynchronize(s_);
        release();
        for (float* p : {ax_, r_, R_, g_, C_, xprev_, xres_, ones_, beta_, dtvg_, hist_}) cudaFree(p);
        cudaFree(acc_); cudaFree(iter_); cudaFree(off_img_); cudaFree(off_sino_); cudaFree(shape_);
        if (s_) cudaStreamDestroy(s_);
    }

    // Binds the iterate x and the data b (device arenas in the batch's
    // layout) and the image shapes, resets the adaptive state, records
    // (dd, dp, dg) of the first hist_cap iterations, and captures one
    // iteration as a CUDA graph.
    void bind(float* x, const float* b, const int* nx, const int* ny, int hist_cap) {
        x_ = x;
        b_ = b;
        std::vector<int2> sh(ni_);
        for (int k = 0; k < ni_; ++k) sh[k] = make_int2(nx[k], ny[k]);
        SGD_CUDA(cudaMemcpy(shape_, sh.data(), ni_ * sizeof(int2), cudaMemcpyHostToDevice));
        hist_cap_ = std::max(0, hist_cap);
        cudaFree(hist_);
        hist_ = nullptr;
        SGD_CUDA(cudaMalloc(&hist_, std::max<size_t>(1, (size_t)hist_cap_ * ni_ * 3) * sizeof(float)));
        reset();
        release();
        SGD_CUDA(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
        try {
            iteration(s_);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(s_, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        SGD_CUDA(cudaStreamEndCapture(s_, &graph_));
        SGD_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
    }

    void reset() {
        std::vector<float> b0(ni_, prm_.beta), d0(ni_, 0.f);
        SGD_CUDA(cudaMemcpy(beta_, b0.data(), ni_ * sizeof(float), cudaMemcpyHostToDevice));
        SGD_CUDA(cudaMemcpy(dtvg_, d0.data(), ni_ * sizeof(float), cudaMemcpyHostToDevice));
        SGD_CUDA(cudaMemset(acc_, 0, (size_t)nslots_ * ni_ * sizeof(double)));
        SGD_CUDA(cudaMemset(iter_, 0, sizeof(int)));
    }

    void run(int iters, cudaStream_t s) {
        if (!exec_) fail("ASD-POCS: bind() first");
        for (int k = 0; k < iters; ++k) SGD_CUDA(cudaGraphLaunch(exec_, s));
    }

    void history(float* out, int n) {
        SGD_CUDA(cudaDeviceSynchronize());
        SGD_CUDA(cudaMemcpy(out, hist_, (size_t)std::min(n, hist_cap_) * ni_ * 3 * sizeof(float),
                            cudaMemcpyDeviceToHost));
    }

private:
    void iteration(cudaStream_t s) {
        const long long nimg = B->img_off().back();
        dim3 gi((unsigned)std::min<long long>(64, (max_img_ + kThreads - 1) / kThreads), ni_);
        dim3 gs((unsigned)std::min<long long>(64, (max_sino_ + kThreads - 1) / kThreads), ni_);
        SGD_CUDA(cudaMemcpyAsync(xprev_, x_, nimg * sizeof(float), cudaMemcpyDeviceToDevice, s));
        B->forward(x_, ax_, s);
        sart_residual_kernel<<<gs, kThreads, 0, s>>>(b_, ax_, R_, r_, off_sino_, ni_, acc_);
        SGD_LAUNCH_CHECK();
        B->backward(r_, g_, s);
        sart_update_kernel<<<gi, kThreads, 0, s>>>(x_, g_, C_, xprev_, beta_, off_img_, ni_, prm_.nonneg, acc_);
        SGD_LAUNCH_CHECK();
        SGD_CUDA(cudaMemcpyAsync(xres_, x_, nimg * sizeof(float), cudaMemcpyDeviceToDevice, s));
        for (int k = 0; k < prm_.ng; ++k) {
            tv_grad_kernel<<<gi, kThreads, 0, s>>>(x_, g_, off_img_, shape_, ni_, kN2 + k, acc_);
            SGD_LAUNCH_CHECK();
            tv_step_kernel<<<gi, kThreads, 0, s>>>(x_, g_, dtvg_, off_img_, ni_, kN2 + k, acc_);
            SGD_LAUNCH_CHECK();
        }
        diff_norm_kernel<<<gi, kThreads, 0, s>>>(x_, xres_, off_img_, ni_, kDG, acc_);
        SGD_LAUNCH_CHECK();
        asd_adapt_kernel<<<1, 64, 0, s>>>(beta_, dtvg_, iter_, acc_, nslots_, ni_, prm_, hist_, hist_cap_);
        SGD_LAUNCH_CHECK();
    }
    void release() {
        if (exec_) cudaGraphExecDestroy(exec_);
        if (graph_) cudaGraphDestroy(graph_);
        exec_ = nullptr;
        graph_ = nullptr;
    }

    B1Batch* B;
    AsdParams prm_;
    int ni_ = 0, nslots_ = 0, hist_cap_ = 0;
    long long max_img_ = 0, max_sino_ = 0;
    cudaStream_t s_ = nullptr;
    float* x_ = nullptr;
    const float* b_ = nullptr;
    float *ax_ = nullptr, *r_ = nullptr, *R_ = nullptr, *g_ = nullptr, *C_ = nullptr, *xprev_ = nullptr,
          *xres_ = nullptr, *ones_ = nullptr, *beta_ = nullptr, *dtvg_ = nullptr, *hist_ = nullptr;
    double* acc_ = nullptr;
    int* iter_ = nullptr;
    long long *off_img_ = nullptr, *off_sino_ = nullptr;
    int2* shape_ = nullptr;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
};

}  // namespace sgd

extern "C" {

void* sgd_asd_create(void* batch, float beta, float beta_red, float alpha, float alpha_red, float r_max, float eps,
                     int ng, int nonneg) {
    return sgd::guarded<void*>(nullptr, [&]() -> void* {
        if (!batch) sgd::fail("sgd_asd_create: null batch");
        if (ng < 0 || ng > 200) sgd::fail("sgd_asd_create: ng must be in [0, 200]");
        sgd::AsdParams p;
        p.beta = beta; p.beta_red = beta_red; p.alpha = alpha; p.alpha_red = alpha_red; p.r_max = r_max;
        p.eps = eps; p.ng = ng; p.nonneg = nonneg ? 1 : 0;
        return new sgd::AsdPocs(static_cast<sgd::B1Batch*>(batch), p);
    });
}

void sgd_asd_destroy(void* h) { delete static_cast<sgd::AsdPocs*>(h); }

int sgd_asd_bind(void* h, float* d_x, const float* d_b, const int* nx, const int* ny, int hist_cap) {
    return sgd::guarded_status([&] {
        if (!h || !d_x || !d_b || !nx || !ny) sgd::fail("sgd_asd_bind: null argument");
        static_cast<sgd::AsdPocs*>(h)->bind(d_x, d_b, nx, ny, hist_cap);
    });
}

int sgd_asd_reset(void* h) {
    return sgd::guarded_status([&] {
        if (!h) sgd::fail("sgd_asd_reset: null argument");
        static_cast<sgd::AsdPocs*>(h)->reset();
    });
}

int sgd_asd_run(void* h, int iters, void* stream) {
    return sgd::guarded_status([&] {
        if (!h) sgd::fail("sgd_asd_run: null argument");
        static_cast<sgd::AsdPocs*>(h)->run(iters, static_cast<cudaStream_t>(stream));
    });
}

int sgd_asd_history(void* h, float* out, int iters) {
    return sgd::guarded_status([&] {
        if (!h || !out) sgd::fail("sgd_asd_history: null argument");
        static_cast<sgd::AsdPocs*>(h)->history(out, iters);
    });
}

// Fan-beam sinograms [image][view][bin] of ni ellipse phantoms (nell ellipses
// each, (cx, cy, a, b, phi, rho) in mm) in the geometry of b1_init, bin
// averages of `sub` rays; with i0 > 0, Poisson transmission noise.
int sgd_ellipse_sinograms(const double* ell, int nell, int ni, int np, int nu, double du, double lsd, double lso,
                          const double* angles, int sub, double i0, unsigned long long seed, float* d_out,
                          void* stream) {
    return sgd::guarded_status([&] {
        if (!ell || !angles || !d_out || ni < 1 || np < 1 || nu < 1 || nell < 1 || sub < 1)
            sgd::fail("sgd_ellipse_sinograms: invalid argument");
        std::vector<double> geo(6 * (size_t)np);
        for (int p = 0; p < np; ++p) {
            const double c = std::cos(angles[p]), s = std::sin(angles[p]);
            // utils/geo.cu:232-269 without the 45-degree snap (a 1e-16 change)
            geo[6 * p + 0] = -lso * c; geo[6 * p + 1] = -lso * s;
            geo[6 * p + 2] = (lsd - lso) * c; geo[6 * p + 3] = (lsd - lso) * s;
            geo[6 * p + 4] = -du * s; geo[6 * p + 5] = du * c;
        }
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        double *d_ell = nullptr, *d_geo = nullptr;
        SGD_CUDA(cudaMallocAsync(&d_ell, (size_t)ni * nell * 6 * sizeof(double), st));
        SGD_CUDA(cudaMallocAsync(&d_geo, geo.size() * sizeof(double), st));
        SGD_CUDA(cudaMemcpyAsync(d_ell, ell, (size_t)ni * nell * 6 * sizeof(double), cudaMemcpyHostToDevice, st));
        SGD_CUDA(cudaMemcpyAsync(d_geo, geo.data(), geo.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        const long long n = (long long)ni * np * nu;
        sgd::ellipse_sinogram_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(d_ell, nell, d_geo, ni, np, nu,
                                                                                  sub, i0, seed, d_out);
        SGD_LAUNCH_CHECK();
        SGD_CUDA(cudaFreeAsync(d_ell, st));
        SGD_CUDA(cudaFreeAsync(d_geo, st));
        SGD_CUDA(cudaStreamSynchronize(st));
    });
}

}  // extern "C"
