// SF_projector: 3D separable-footprint (SF-TR, optionally SF-TT) cone-beam
// projector.  Reference: layers/SF_projector.cu:42-78 (gamma), :81-234
// (SF_project), :237-356 (SF_backproject), :359-400 (SF::project /
// back_project); it has no C entry points there.
//
// Per voxel (ix, iy, iz) and view, through the view's index-space matrix pmi:
// the four in-plane corners (ix +- 1/2, iy +- 1/2) at iz give a trapezoid
// us[0..3] in u; the voxel's z extent gives a rectangle vs[0..1] in v (SF-TR),
// or the corners (ix +- 1/2, iy) at iz +- 1/2 a trapezoid (SF-TT, forward
// only in the reference).  This projector takes bins as [i - 1/2, i + 1/2]
// (ranges ceil(us - 1/2), :165-166), unlike the 2D projectors.  Amplitudes:
//   forward   lsd^2 dy dz / (du dv) * (1/r^2) * 2/(trapezoid width) * 1/(v width)
//   backward  lsd dx / np          * (1/r)   * 2/(trapezoid width) * 1/(v width)
// with r the distance from the source to (dx (ix - nx/2), dy (iy - ny/2),
// dz (iz - nz/2)) (integer halves, :104-105).
//
// Reference behaviour (mode 0), reproduced for parity:
//   * the forward adds the footprint alone, without the voxel value or the
//     amplitude (C is computed and never used, :190-221): it projects the
//     indicator of the non-zero voxels;
//   * bin indices are not clamped, j * nu + i is only bounds-checked, so bins
//     beyond the u edges wrap into neighbouring rows (:216, :336).
//   * on the snapped 3pi/4 and -pi/4 views its index-space matrices degenerate
//     (utils/geo.cu:36-41) and voxels project onto spans of hundreds of bins;
//     here a voxel whose span exceeds twice the detector is skipped (the one
//     deviation: the reference visits those spans).
// Mode 1 ("fixed"): exact projection matrices on every view, the forward
// scales by the voxel value and amplitude and drops out-of-detector bins; the
// back projection is its exact transpose.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "common.h"
#include "fan_geometry.h"

namespace sgd {

namespace {

constexpr int kSFZ = 64;  // the reference's Z_SIZE (layers/SF_projector.hh:3)

struct SFGeo {
    int nx, ny, nz, np, nu, nv, trap, mode;
    double dx, dy, dz;
    const float* pmi;    // [np][12]
    const double* src;   // [np][3]
    const double* fwdf;  // [np] forward factor lsd^2 dy dz / (du dv) (times dx in mode 1)
    double backf;        // lsd dx / np
};

__device__ __forceinline__ void sort4f(float* a) {
    auto s2 = [](float& x, float& y) {
        if (x > y) {
            const float t = y;
            y = x;
            x = t;
        }
    };
    s2(a[0], a[1]);
    s2(a[2], a[3]);
    s2(a[0], a[2]);
    s2(a[1], a[3]);
    s2(a[1], a[2]);
}

// layers/SF_projector.cu:42-78
__device__ __forceinline__ float sf_gamma(float s1, float s2, const float* us) {
    float g = 0.0f, tmp, b1, b2;
    b1 = fmaxf(s1, us[0]);
    b2 = fminf(s2, us[1]);
    tmp = (b2 > b1) ? (1 / (2 * (us[1] - us[0]))) * ((b2 - us[0]) * (b2 - us[0]) - (b1 - us[0]) * (b1 - us[0])) : 0.0f;
    if (tmp == tmp) g += tmp;
    b1 = fmaxf(s1, us[1]);
    b2 = fminf(s2, us[2]);
    tmp = (b2 > b1) ? b2 - b1 : 0.0f;
    if (tmp == tmp) g += tmp;
    b1 = fmaxf(s1, us[2]);
    b2 = fminf(s2, us[3]);
    tmp = (b2 > b1) ? (1 / (2 * (us[3] - us[2]))) * ((b1 - us[3]) * (b1 - us[3]) - (b2 - us[3]) * (b2 - us[3])) : 0.0f;
    if (tmp == tmp) g += tmp;
    return g;
}

struct SFVoxel {
    float us[4], vs[4];
    int min_u, max_u, min_v, max_v;
    float C;  // amplitude (forward or backward normalisation)
};

// Returns 0: voxel contributes, 1: skip this voxel, 2: skip the rest of the
// thread's z chunk (the reference's `return`, :150, :286).
__device__ int sf_voxel(const SFGeo& G, const float* pm, const double* src, double factor, bool fwd, int ix, int iy,
                        int iz, SFVoxel& o) {
    const int nxh = G.nx / 2, nyh = G.ny / 2, nzh = G.nz / 2;
    const float pmv2 = pm[4] * ix + pm[5] * iy + pm[7];
    const float pmv3 = pm[8] * ix + pm[9] * iy + pm[11];
    const float signy1 = iy - 0.5f, signy2 = iy + 0.5f, signx1 = ix - 0.5f, signx2 = ix + 0.5f;
    const float u1 = pm[0] * signx1 + pm[1] * signy1 + pm[3], u2 = pm[8] * signx1 + pm[9] * signy1 + pm[11];
    const float u3 = pm[0] * signx2 + pm[1] * signy1 + pm[3], u4 = pm[8] * signx2 + pm[9] * signy1 + pm[11];
    const float u5 = pm[0] * signx1 + pm[1] * signy2 + pm[3], u6 = pm[8] * signx1 + pm[9] * signy2 + pm[11];
    const float u7 = pm[0] * signx2 + pm[1] * signy2 + pm[3], u8 = pm[8] * signx2 + pm[9] * signy2 + pm[11];
    const float signz1 = (iz - 0.5f), signz2 = (iz + 0.5f);
    float min_v, max_v;
    const bool trap = fwd && G.trap;
    if (!trap) {
        o.vs[0] = (pmv2 + pm[6] * signz1) / (pmv3 + pm[10] * signz1);
        min_v = ceilf(o.vs[0] - 0.5f);
        if (min_v >= G.nv) return 2;
        o.vs[1] = (pmv2 + pm[6] * signz2) / (pmv3 + pm[10] * signz2);
        max_v = ceilf(o.vs[1] - 0.5f);
        if (max_v < 0) return 1;
    } else {
        const float v1 = pm[4] * signx1 + pm[5] * iy + pm[7], v2 = pm[4] * signx2 + pm[5] * iy + pm[7];
        const float v3 = pm[8] * signx1 + pm[9] * iy + pm[11], v4 = pm[8] * signx2 + pm[9] * iy + pm[11];
        o.vs[0] = (v1 + pm[6] * signz1) / (v3 + pm[10] * signz1);
        o.vs[1] = (v1 + pm[6] * signz2) / (v3 + pm[10] * signz2);
        o.vs[2] = (v2 + pm[6] * signz1) / (v4 + pm[10] * signz1);
        o.vs[3] = (v2 + pm[6] * signz2) / (v4 + pm[10] * signz2);
        sort4f(o.vs);
        min_v = ceilf(o.vs[0] - 0.5f);
        max_v = ceilf(o.vs[3] - 0.5f);
        if ((max_v < 0) || (min_v >= G.nv)) return 1;
    }
    const double ddx = G.dx * (ix - nxh) - src[0], ddy = G.dy * (iy - nyh) - src[1], ddz = G.dz * (iz - nzh) - src[2];
    float weight = rsqrtf((float)(ddx * ddx + ddy * ddy + ddz * ddz));
    if (fwd) weight *= weight;
    o.us[0] = (u1 + pm[2] * iz) / (u2 + pm[10] * iz);
    o.us[1] = (u3 + pm[2] * iz) / (u4 + pm[10] * iz);
    o.us[2] = (u5 + pm[2] * iz) / (u6 + pm[10] * iz);
    o.us[3] = (u7 + pm[2] * iz) / (u8 + pm[10] * iz);
    sort4f(o.us);
    const float min_u = ceilf(o.us[0] - 0.5f), max_u = ceilf(o.us[3] - 0.5f);
    if ((max_u < 0) || (min_u >= G.nu)) return 1;
    const float tw = (2 / (((o.us[3] - o.us[0]) + (o.us[2] - o.us[1]))));
    // SF-TT amplitude: 2 / (sum of the trapezoid's parallel sides).  The
    // reference's expression (:194) groups it differently, but its forward
    // never applies the amplitude, so only the fixed mode reads this.
    if (trap)
        o.C = (float)(weight * factor * tw * (2 / ((o.vs[3] - o.vs[0]) + (o.vs[2] - o.vs[1]))));
    else
        o.C = (float)(weight * factor * tw * (1 / (o.vs[1] - o.vs[0])));
    // a voxel whose projection spans more bins than twice the detector (near
    // the source plane, or through a degenerate matrix) is skipped: its
    // footprint is meaningless and the loops below would run unbounded
    if (!(max_u - min_u <= 2.f * G.nu + 4.f) || !(max_v - min_v <= 2.f * G.nv + 4.f)) return 1;
    o.min_u = (int)min_u; o.max_u = (int)max_u; o.min_v = (int)min_v; o.max_v = (int)max_v;
    return 0;
}

__device__ __forceinline__ float sf_fv(const SFGeo& G, bool trap, const SFVoxel& o, int j) {
    if (trap) return sf_gamma(j - 0.5f, j + 0.5f, o.vs);
    return fmaxf(fminf(j + 0.5f, o.vs[1]) - fmaxf(j - 0.5f, o.vs[0]), 0);
}

// a thread per (ix, iy, z chunk of 64) and view (grid z = views); the volume
// is FP32 (device entry points) or FP64 (mode 1 host entry points)
template <typename TVol>
__global__ void __launch_bounds__(128) sf3d_forward_kernel(SFGeo G, const TVol* __restrict__ vol,
                                                           double* __restrict__ proj64) {
    const int ix = blockIdx.x * 16 + threadIdx.x, iy = blockIdx.y * 8 + threadIdx.y;
    const int chunks = (G.nz + kSFZ - 1) / kSFZ;
    const int p = blockIdx.z / chunks, zc = blockIdx.z % chunks;
    if (ix >= G.nx || iy >= G.ny || p >= G.np) return;
    const float* pm = G.pmi + 12 * (size_t)p;
    const double* src = G.src + 3 * (size_t)p;
    const int nuv = G.nu * G.nv;
    double* pp = proj64 + (size_t)p * nuv;
    const bool trap = G.trap != 0;
    for (int iz = zc * kSFZ; iz < min(G.nz, (zc + 1) * kSFZ); ++iz) {
        const TVol C0 = vol[((size_t)iz * G.ny + iy) * G.nx + ix];
        SFVoxel o;
        const int r = sf_voxel(G, pm, src, G.fwdf[p], true, ix, iy, iz, o);
        if (r == 2 && G.mode == 0) break;  // the reference leaves its z chunk (:150)
        if (r != 0 || C0 == TVol(0)) continue;  // o is only filled when r == 0
        // mode 1 multiplies in FP64 so that the back kernel's terms are the
        // same real numbers (an adjoint pair to FP64 accumulation)
        const double amp = (G.mode == 0) ? 1.0 : (double)o.C * (double)C0;
        for (int i = o.min_u; i <= o.max_u; ++i) {
            const float g = sf_gamma(i - 0.5f, i + 0.5f, o.us);
            if (G.mode == 1 && (i < 0 || i >= G.nu)) continue;
            for (int j = o.min_v; j <= o.max_v; ++j) {
                const float f2 = g * sf_fv(G, trap, o, j);
                const int idxv = j * G.nu + i;
                if (G.mode == 1 && (j < 0 || j >= G.nv)) continue;
                if (idxv < nuv && idxv >= 0 && f2 == f2 && f2 != 0.f) atomicAdd(pp + idxv, (double)f2 * amp);
            }
        }
    }
}

// mode 0: SF_backproject (rect in v); mode 1: exact transpose of the fixed
// forward.  FP32 in and out (device entry points) or FP64 (mode 1 host entry
// points, so that the pair stays an adjoint pair to FP64 rounding end to end)
template <typename TProj, typename TVol>
__global__ void __launch_bounds__(128) sf3d_back_kernel(SFGeo G, const TProj* __restrict__ proj,
                                                        TVol* __restrict__ vol) {
    const int ix = blockIdx.x * 16 + threadIdx.x, iy = blockIdx.y * 8 + threadIdx.y;
    const int iz = blockIdx.z;
    if (ix >= G.nx || iy >= G.ny) return;
    const int nuv = G.nu * G.nv;
    const bool trap = G.mode == 1 && G.trap != 0;
    const int z0 = iz - iz % kSFZ;
    double acc = 0.0;
    for (int p = 0; p < G.np; ++p) {
        const float* pm = G.pmi + 12 * (size_t)p;
        const double* src = G.src + 3 * (size_t)p;
        SFVoxel o;
        // The reference walks z in chunks of 64 and leaves the chunk at the
        // first voxel whose v range starts beyond the detector.  v is monotone
        // in z along a column, so that voxel is either the chunk's first or
        // this one: test both.
        if (G.mode == 0 && iz != z0) {
            const float pmv2 = pm[4] * ix + pm[5] * iy + pm[7], pmv3 = pm[8] * ix + pm[9] * iy + pm[11];
            const float v0 = (pmv2 + pm[6] * (z0 - 0.5f)) / (pmv3 + pm[10] * (z0 - 0.5f));
            if (ceilf(v0 - 0.5f) >= G.nv) continue;
        }
        const int r = sf_voxel(G, pm, src, G.mode == 0 ? G.backf : G.fwdf[p], G.mode == 1, ix, iy, iz, o);
        if (r != 0) continue;
        const TProj* pp = proj + (size_t)p * nuv;
        double sumV = 0.0;
        for (int i = o.min_u; i <= o.max_u; ++i) {
            if (G.mode == 1 && (i < 0 || i >= G.nu)) continue;
            const float g = sf_gamma(i - 0.5f, i + 0.5f, o.us);
            for (int j = o.min_v; j <= o.max_v; ++j) {
                if (G.mode == 1 && (j < 0 || j >= G.nv)) continue;
                const float f = g * sf_fv(G, trap, o, j);
                const int idxv = j * G.nu + i;
                if (idxv < nuv && idxv >= 0 && (G.mode == 0 || (f == f && f != 0.f)))
                    sumV += (double)pp[idxv] * (double)f;
            }
        }
        sumV *= (double)o.C;
        if (sumV == sumV) acc += sumV;
    }
    vol[((size_t)iz * G.ny + iy) * G.nx + ix] = (TVol)acc;
}

__global__ void sf3d_finish_kernel(const double* __restrict__ s64, float* __restrict__ s32, long long n) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) s32[e] = (float)s64[e];
}

}  // namespace

class SF3D {
public:
    SFGeo G{};
    int device = 0;
    cudaStream_t stream = nullptr;

    SF3D(int mode, int trap, int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy, double dz, double du,
         double dv, double lsd, double lso, const double* angles) {
        if (nx <= 0 || ny <= 0 || nz <= 0 || np <= 0 || nu <= 0 || nv <= 0) fail("invalid sizes");
        check_pitches({dx, dy, dz, du, dv});
        check_distances(lsd, lso);
        check_views(np, angles, nullptr, nullptr);
        SGD_CUDA(cudaGetDevice(&device));
        SGD_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        const std::vector<ViewFrame> fr = view_frames(np, lsd, lso, du, dv, angles, nullptr, nullptr);
        std::vector<float> pmi((size_t)np * 12);
        std::vector<double> src((size_t)np * 3), fwdf(np);
        for (int p = 0; p < np; ++p) {
            double pm[12];
            // mode 0 keeps the reference's matrices, degenerate views included;
            // the corrected pair projects through the exact ones
            if (mode == 0) reference_pmi(fr[p], nu / 2.0, nv / 2.0, nx, ny, nz, dx, dy, dz, pm, &pmi[12 * (size_t)p]);
            else exact_pmi(fr[p], nu / 2.0, nv / 2.0, nx, ny, nz, dx, dy, dz, &pmi[12 * (size_t)p]);
            for (int k = 0; k < 3; ++k) src[3 * p + k] = fr[p].src[k];
            const float flsd = (float)lsd;  // SF::project: float lsd (:362)
            // the reference's factor lsd^2 dy dz / (du dv) (:364) lacks the
            // voxel's third side: the corrected pair multiplies it in, so
            // that its forward carries the voxel's line integrals for any dx
            fwdf[p] = flsd * flsd * dy * dz / (du * dv) * (mode == 1 ? dx : 1.0);
        }
        SGD_CUDA(cudaMalloc(&d_pmi_, pmi.size() * sizeof(float)));
        SGD_CUDA(cudaMemcpy(d_pmi_, pmi.data(), pmi.size() * sizeof(float), cudaMemcpyHostToDevice));
        SGD_CUDA(cudaMalloc(&d_src_, src.size() * sizeof(double)));
        SGD_CUDA(cudaMemcpy(d_src_, src.data(), src.size() * sizeof(double), cudaMemcpyHostToDevice));
        SGD_CUDA(cudaMalloc(&d_fwdf_, fwdf.size() * sizeof(double)));
        SGD_CUDA(cudaMemcpy(d_fwdf_, fwdf.data(), fwdf.size() * sizeof(double), cudaMemcpyHostToDevice));
        G = SFGeo{nx, ny, nz, np, nu, nv, trap, mode, dx, dy, dz, d_pmi_, d_src_, d_fwdf_,
                  (double)(float)lsd * dx / np};
        const size_t nvol = (size_t)nx * ny * nz, nproj = (size_t)np * nu * nv;
        SGD_CUDA(cudaMalloc(&d_proj64_, nproj * sizeof(double)));
        SGD_CUDA(cudaMalloc(&d_vol_, nvol * sizeof(float)));
        SGD_CUDA(cudaMalloc(&d_proj_, nproj * sizeof(float)));
        SGD_CUDA(cudaMallocHost(&h_vol_, nvol * sizeof(float)));
        SGD_CUDA(cudaMallocHost(&h_proj_, nproj * sizeof(float)));
    }
    ~SF3D() {
        if (stream) cudaStreamSynchronize(stream);
        cudaFree(d_pmi_); cudaFree(d_src_); cudaFree(d_fwdf_); cudaFree(d_proj64_);
        cudaFree(d_vol_); cudaFree(d_proj_); cudaFreeHost(h_vol_); cudaFreeHost(h_proj_);
        cudaFree(d_vol64_); cudaFreeHost(h_vol64_); cudaFreeHost(h_proj64_);
        if (stream) cudaStreamDestroy(stream);
    }
    // FP64 host arrays: x[(iz*ny + iy)*nx + ix], b[(p*nv + v)*nu + u].  Mode 1
    // keeps FP64 from the host buffers through the kernels and back; mode 0
    // rounds through FP32 as the reference's SF class does.
    void forward_host(double* b, const double* x) {
        const long long nvol = (long long)G.nx * G.ny * G.nz, nproj = (long long)G.np * G.nu * G.nv;
        if (G.mode == 1) {
            ensure_fp64();
            std::memcpy(h_vol64_, x, nvol * sizeof(double));
            SGD_CUDA(cudaMemcpyAsync(d_vol64_, h_vol64_, nvol * sizeof(double), cudaMemcpyHostToDevice, stream));
            forward64(d_vol64_, stream);
            SGD_CUDA(cudaMemcpyAsync(h_proj64_, d_proj64_, nproj * sizeof(double), cudaMemcpyDeviceToHost, stream));
            SGD_CUDA(cudaStreamSynchronize(stream));
            std::memcpy(b, h_proj64_, nproj * sizeof(double));
            return;
        }
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < nvol; ++e) h_vol_[e] = (float)x[e];
        SGD_CUDA(cudaMemcpyAsync(d_vol_, h_vol_, nvol * sizeof(float), cudaMemcpyHostToDevice, stream));
        forward_dev(d_vol_, d_proj_, stream);
        SGD_CUDA(cudaMemcpyAsync(h_proj_, d_proj_, nproj * sizeof(float), cudaMemcpyDeviceToHost, stream));
        SGD_CUDA(cudaStreamSynchronize(stream));
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < nproj; ++e) b[e] = (double)h_proj_[e];
    }
    void backward_host(const double* b, double* x) {
        const long long nvol = (long long)G.nx * G.ny * G.nz, nproj = (long long)G.np * G.nu * G.nv;
        if (G.mode == 1) {
            ensure_fp64();
            std::memcpy(h_proj64_, b, nproj * sizeof(double));
            SGD_CUDA(cudaMemcpyAsync(d_proj64_, h_proj64_, nproj * sizeof(double), cudaMemcpyHostToDevice, stream));
            dim3 grid((G.nx + 15) / 16, (G.ny + 7) / 8, G.nz);
            sf3d_back_kernel<double, double><<<grid, dim3(16, 8), 0, stream>>>(G, d_proj64_, d_vol64_);
            SGD_LAUNCH_CHECK();
            SGD_CUDA(cudaMemcpyAsync(h_vol64_, d_vol64_, nvol * sizeof(double), cudaMemcpyDeviceToHost, stream));
            SGD_CUDA(cudaStreamSynchronize(stream));
            std::memcpy(x, h_vol64_, nvol * sizeof(double));
            return;
        }
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < nproj; ++e) h_proj_[e] = (float)b[e];
        SGD_CUDA(cudaMemcpyAsync(d_proj_, h_proj_, nproj * sizeof(float), cudaMemcpyHostToDevice, stream));
        backward_dev(d_proj_, d_vol_, stream);
        SGD_CUDA(cudaMemcpyAsync(h_vol_, d_vol_, nvol * sizeof(float), cudaMemcpyDeviceToHost, stream));
        SGD_CUDA(cudaStreamSynchronize(stream));
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < nvol; ++e) x[e] = (double)h_vol_[e];
    }
    // d_proj64_ = A vol (FP64 accumulation)
    template <typename TVol>
    void forward64(const TVol* vol, cudaStream_t s) {
        const long long n = (long long)G.np * G.nu * G.nv;
        SGD_CUDA(cudaMemsetAsync(d_proj64_, 0, n * sizeof(double), s));
        const int chunks = (G.nz + kSFZ - 1) / kSFZ;
        dim3 grid((G.nx + 15) / 16, (G.ny + 7) / 8, G.np * chunks);
        sf3d_forward_kernel<TVol><<<grid, dim3(16, 8), 0, s>>>(G, vol, d_proj64_);
        SGD_LAUNCH_CHECK();
    }
    void forward_dev(const float* vol, float* proj, cudaStream_t s) {
        const long long n = (long long)G.np * G.nu * G.nv;
        forward64(vol, s);
        sf3d_finish_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d_proj64_, proj, n);
        SGD_LAUNCH_CHECK();
    }
    void backward_dev(const float* proj, float* vol, cudaStream_t s) {
        dim3 grid((G.nx + 15) / 16, (G.ny + 7) / 8, G.nz);
        sf3d_back_kernel<float, float><<<grid, dim3(16, 8), 0, s>>>(G, proj, vol);
        SGD_LAUNCH_CHECK();
    }

private:
    void ensure_fp64() {
        if (d_vol64_) return;
        const size_t nvol = (size_t)G.nx * G.ny * G.nz, nproj = (size_t)G.np * G.nu * G.nv;
        SGD_CUDA(cudaMalloc(&d_vol64_, nvol * sizeof(double)));
        SGD_CUDA(cudaMallocHost(&h_vol64_, nvol * sizeof(double)));
        SGD_CUDA(cudaMallocHost(&h_proj64_, nproj * sizeof(double)));
    }
    double* d_vol64_ = nullptr;
    double* h_vol64_ = nullptr;
    double* h_proj64_ = nullptr;
    float* d_pmi_ = nullptr;
    double* d_src_ = nullptr;
    double* d_fwdf_ = nullptr;
    double* d_proj64_ = nullptr;
    float* d_vol_ = nullptr;
    float* d_proj_ = nullptr;
    float* h_vol_ = nullptr;
    float* h_proj_ = nullptr;
};

}  // namespace sgd

extern "C" {

void* sgd_sf3d_init(int mode, int trap_v, int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy,
                    double dz, double du, double dv, double lsd, double lso, double* angles) {
    return sgd::guarded<void*>(nullptr, [&]() -> void* {
        if (mode != 0 && mode != 1) sgd::fail("sgd_sf3d_init: mode must be 0 or 1");
        return new sgd::SF3D(mode, trap_v, nx, ny, nz, np, nu, nv, dx, dy, dz, du, dv, lsd, lso, angles);
    });
}
void sgd_sf3d_destroy(void* layer) { delete static_cast<sgd::SF3D*>(layer); }
int sgd_sf3d_forward_dev(void* layer, const float* d_vol, float* d_proj, void* stream) {
    return sgd::guarded_status([&] {
        if (!layer || !d_vol || !d_proj) sgd::fail("sgd_sf3d_forward_dev: null argument");
        static_cast<sgd::SF3D*>(layer)->forward_dev(d_vol, d_proj, static_cast<cudaStream_t>(stream));
    });
}
int sgd_sf3d_forward_projection(double* b, double* x, void* layer) {
    return sgd::guarded_status([&] {
        if (!layer || !b || !x) sgd::fail("sgd_sf3d_forward_projection: null argument");
        static_cast<sgd::SF3D*>(layer)->forward_host(b, x);
    });
}
int sgd_sf3d_backward_projection(double* b, double* x, void* layer) {
    return sgd::guarded_status([&] {
        if (!layer || !b || !x) sgd::fail("sgd_sf3d_backward_projection: null argument");
        static_cast<sgd::SF3D*>(layer)->backward_host(b, x);
    });
}
int sgd_sf3d_backward_dev(void* layer, const float* d_proj, float* d_vol, void* stream) {
    return sgd::guarded_status([&] {
        if (!layer || !d_vol || !d_proj) sgd::fail("sgd_sf3d_backward_dev: null argument");
        static_cast<sgd::SF3D*>(layer)->backward_dev(d_proj, d_vol, static_cast<cudaStream_t>(stream));
    });
}

}  // extern "C"
