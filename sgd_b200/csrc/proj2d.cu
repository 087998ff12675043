#include <algorithm>
#include <cmath>
#include <functional>
#include <limits>

#include "common.h"
#include "fan2d.cuh"
#include "proj2d.h"

namespace sgd {

void fan_world_hom(const FanGeometry& g, int p, double h[6]) {
    // s = cross(P - D, X - P) / cross(e, X - P) (the detector coordinate of the
    // ray P -> X in units of the bin pitch), u = s + nu/2
    const double px = g.src[2 * p], py = g.src[2 * p + 1];
    const double ax = px - g.dtv[2 * p], ay = py - g.dtv[2 * p + 1];
    const double ex = g.puv[2 * p], ey = g.puv[2 * p + 1];
    const double hn = 0.5 * g.nu;
    h[3] = -ey;
    h[4] = ex;
    h[5] = ey * px - ex * py;
    h[0] = -ay + hn * h[3];
    h[1] = ax + hn * h[4];
    h[2] = (ay * px - ax * py) + hn * h[5];
}

RangeMap grid_range_map(const double hw[6], double x0, double dx, double y0, double dy, double ri, double rj) {
    RangeMap m;
    m.h[0] = hw[0] * dx;
    m.h[1] = hw[1] * dy;
    m.h[2] = hw[0] * x0 + hw[1] * y0 + hw[2];
    m.h[3] = hw[3] * dx;
    m.h[4] = hw[4] * dy;
    m.h[5] = hw[3] * x0 + hw[4] * y0 + hw[5];
    m.ri = ri;
    m.rj = rj;
    return m;
}

namespace {

// Bin window of the cell box [i0, i1] x [j0, j1] widened by the map's radii:
// the extremes of a linear-fractional map over a box are at its corners (when
// the box lies on one side of the source line, D of one sign); one bin of
// margin each side for the FP32 rounding of the kernels' ranges; clamped.
void tile_window(const RangeMap& m, int nu, double i0, double i1, double j0, double j1, int& lo, int& hi) {
    i0 -= m.ri, i1 += m.ri, j0 -= m.rj, j1 += m.rj;
    double umin = 1e300, umax = -1e300;
    int pos = 0, neg = 0;
    for (double i : {i0, i1})
        for (double j : {j0, j1}) {
            const double D = m.h[3] * i + m.h[4] * j + m.h[5];
            (D > 0 ? pos : neg)++;
            const double u = (m.h[0] * i + m.h[1] * j + m.h[2]) / D;
            umin = std::min(umin, u);
            umax = std::max(umax, u);
        }
    if (pos && neg) {  // the box reaches the source line: every bin
        lo = 0;
        hi = nu - 1;
        return;
    }
    if (umax < -1.0 || umin > nu + 1.0) {
        lo = 0;
        hi = -1;
        return;
    }
    lo = std::max(0, (int)std::floor(umin) - 1);
    hi = std::min(nu - 1, (int)std::floor(umax) + 1);
}

// Forward strip of bins [b0, b1) along one choice of major axis: the minor
// coordinate of the points at u = U on major line m is alpha_U + beta_U m.
struct StripFit {
    bool ok = false;
    double aa = 0, ba = 0, ab = 0, bb = 0, margin = 0;
    long long cells = 0;
    int mlo = 0, mhi = -1;
};

StripFit fit_strip(const RangeMap& m, double U0, double U1, bool jmaj, int nmajor, int nminor) {
    StripFit f;
    // along a major line u runs monotonically from its pole (outside the grid,
    // on the source's line) to its value at infinity along the minor axis;
    // when that value falls inside the strip the two crossings need not
    // bracket the strip, and this axis is not used
    const double dmin = jmaj ? m.h[3] : m.h[4], nmin = jmaj ? m.h[0] : m.h[1];
    if (dmin != 0.0) {
        const double uinf = nmin / dmin;
        if (uinf > U0 - 1.0 && uinf < U1 + 1.0) return f;
    }
    double al[2], be[2];
    const double Us[2] = {U0, U1};
    for (int t = 0; t < 2; ++t) {
        const double U = Us[t];
        const double ci = m.h[0] - U * m.h[3], cj = m.h[1] - U * m.h[4], c0 = m.h[2] - U * m.h[5];
        // ci i + cj j + c0 = 0
        const double cmin = jmaj ? ci : cj, cmaj = jmaj ? cj : ci;
        const double scale = std::fabs(ci) + std::fabs(cj);
        if (!(std::fabs(cmin) > 1e-9 * scale)) return f;
        al[t] = -c0 / cmin;
        be[t] = -cmaj / cmin;
    }
    f.ok = true;
    f.aa = al[0], f.ba = be[0], f.ab = al[1], f.bb = be[1];
    const double rmin = jmaj ? m.ri : m.rj, rmaj = jmaj ? m.rj : m.ri;
    f.margin = rmin + rmaj * std::max(std::fabs(be[0]), std::fabs(be[1])) + 0.5;
    for (int k = 0; k < nmajor; ++k) {
        const double na = al[0] + be[0] * k, nb = al[1] + be[1] * k;
        const long long lo = std::max(0LL, (long long)std::ceil(std::min(na, nb) - f.margin));
        const long long hi = std::min((long long)nminor - 1, (long long)std::floor(std::max(na, nb) + f.margin));
        if (hi >= lo) {
            f.cells += hi - lo + 1;
            if (f.mhi < f.mlo) f.mlo = k;
            f.mhi = k;
        }
    }
    return f;
}

}  // namespace

int plan_fan2d(int ni, int nj, int np, int nu, const std::function<RangeMap(int)>& map, std::vector<float4>& strips,
               std::vector<int2>& twin, int block) {
    const int nblk = (nu + block - 1) / block;
    strips.assign((size_t)np * nblk * 2, make_float4(0.f, 0.f, 0.f, 0.f));
    const int ti = (ni + kF2TileI - 1) / kF2TileI, tj = (nj + kF2TileJ - 1) / kF2TileJ;
    twin.assign((size_t)ti * tj * np, make_int2(0, -1));
    int wmax = 1;
    for (int p = 0; p < np; ++p) {
        const RangeMap m = map(p);
        // forward block strips: the major axis whose lines cross the strip
        // with the fewest candidate cells
        for (int k = 0; k < nblk; ++k) {
            // half a bin of slack for the FP32 rounding of the kernels' ranges
            const double U0 = k * block - 0.5, U1 = std::min(nu, (k + 1) * block) + 0.5;
            const StripFit fj = fit_strip(m, U0, U1, true, nj, ni);
            const StripFit fi = fit_strip(m, U0, U1, false, ni, nj);
            if (!fj.ok && !fi.ok) fail("projector geometry: degenerate detector strip in view %d", p);
            const bool usej = fj.ok && (!fi.ok || fj.cells <= fi.cells);
            const StripFit& f = usej ? fj : fi;
            float4* s = &strips[((size_t)p * nblk + k) * 2];
            s[0] = make_float4(usej ? 1.f : 0.f, (float)f.aa, (float)f.ba, (float)f.ab);
            s[1] = make_float4((float)f.bb, (float)f.margin, (float)f.mlo, (float)f.mhi);
        }
        // back tile windows
        for (int a = 0; a < ti; ++a)
            for (int b = 0; b < tj; ++b) {
                int lo, hi;
                tile_window(m, nu, a * kF2TileI, std::min(ni, (a + 1) * kF2TileI) - 1, b * kF2TileJ,
                            std::min(nj, (b + 1) * kF2TileJ) - 1, lo, hi);
                twin[((size_t)a * tj + b) * np + p] = make_int2(lo, hi);
                wmax = std::max(wmax, hi - lo + 1);
            }
    }
    return wmax;
}

void Proj2D::finish_init(const std::vector<float>& view, const std::vector<float4>& bins) {
    SGD_CUDA(cudaGetDevice(&device));
    SGD_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    P.np = geo.np;
    P.nu = geo.nu;
    const int np = geo.np, nu = geo.nu;
    SGD_CUDA(cudaMalloc(&d_view_, view.size() * sizeof(float)));
    SGD_CUDA(cudaMemcpy(d_view_, view.data(), view.size() * sizeof(float), cudaMemcpyHostToDevice));
    P.view = d_view_;
    if (!bins.empty()) {
        SGD_CUDA(cudaMalloc(&d_bins_, bins.size() * sizeof(float4)));
        SGD_CUDA(cudaMemcpy(d_bins_, bins.data(), bins.size() * sizeof(float4), cudaMemcpyHostToDevice));
        P.bins = d_bins_;
    }

    std::vector<float4> strips;
    std::vector<int2> twin;
    P.wcap = plan_fan2d(P.ni, P.nj, np, nu, [this](int p) { return range_map(p); }, strips, twin);
    P.nblk = (nu + kF2Block - 1) / kF2Block;
    P.tiles_j = (P.nj + kF2TileJ - 1) / kF2TileJ;
    SGD_CUDA(cudaMalloc(&d_strips_, strips.size() * sizeof(float4)));
    SGD_CUDA(cudaMemcpy(d_strips_, strips.data(), strips.size() * sizeof(float4), cudaMemcpyHostToDevice));
    P.strips = d_strips_;
    SGD_CUDA(cudaMalloc(&d_twin_, twin.size() * sizeof(int2)));
    SGD_CUDA(cudaMemcpy(d_twin_, twin.data(), twin.size() * sizeof(int2), cudaMemcpyHostToDevice));
    P.twin = d_twin_;
    SGD_CUDA(cudaMalloc(&d_err_, sizeof(int)));
    SGD_CUDA(cudaMemset(d_err_, 0, sizeof(int)));
    P.err = d_err_;

    const size_t nimg = (size_t)P.ni * P.nj, nsino = (size_t)np * nu;
    SGD_CUDA(cudaMalloc(&d_img_, nimg * sizeof(float)));
    SGD_CUDA(cudaMalloc(&d_imgT_, nimg * sizeof(float)));
    P.imgT = d_imgT_;
    SGD_CUDA(cudaMalloc(&d_part_, kF2FwdParts * nsino * sizeof(double)));
    P.part = d_part_;
    SGD_CUDA(cudaMalloc(&d_sino_, nsino * sizeof(float)));
    SGD_CUDA(cudaMallocHost(&h_img_, nimg * sizeof(float)));
    SGD_CUDA(cudaMallocHost(&h_sino_, nsino * sizeof(float)));
}

Proj2D::~Proj2D() {
    if (stream) cudaStreamSynchronize(stream);
    cudaFree(d_view_);
    cudaFree(d_bins_);
    cudaFree(d_strips_);
    cudaFree(d_twin_);
    cudaFree(d_err_);
    cudaFree(d_img_);
    cudaFree(d_imgT_);
    cudaFree(d_part_);
    cudaFree(d_out64_);
    cudaFree(d_sino_);
    cudaFreeHost(h_img_);
    cudaFreeHost(h_sino_);
    if (stream) cudaStreamDestroy(stream);
}

int Proj2D::status(bool sync_device) {
    int h = 0;
    // the *_dev calls may have run on any of the caller's streams
    if (sync_device) SGD_CUDA(cudaDeviceSynchronize());
    SGD_CUDA(cudaMemcpyAsync(&h, d_err_, sizeof(int), cudaMemcpyDeviceToHost, stream));
    SGD_CUDA(cudaMemsetAsync(d_err_, 0, sizeof(int), stream));
    SGD_CUDA(cudaStreamSynchronize(stream));
    return h ? -1 : 0;
}

// The FP64 host entry points: inputs rounded to FP32 (the kernels' input
// type, as the reference's layers round them), outputs the kernels' FP64 sums
// (the FP32 *_dev outputs round them once more).
void Proj2D::forward_host(double* b, const double* x) {
    const long long nimg = (long long)P.ni * P.nj, nsino = (long long)P.np * P.nu;
#pragma omp parallel for schedule(static) if (nimg > (1 << 16))
    for (long long e = 0; e < nimg; ++e) h_img_[e] = (float)x[e];
    SGD_CUDA(cudaMemcpyAsync(d_img_, h_img_, nimg * sizeof(float), cudaMemcpyHostToDevice, stream));
    ensure_out64();
    P.out64 = d_out64_;
    forward_dev(d_img_, d_sino_, stream);
    P.out64 = nullptr;
    SGD_CUDA(cudaMemcpyAsync(b, d_out64_, nsino * sizeof(double), cudaMemcpyDeviceToHost, stream));
    SGD_CUDA(cudaStreamSynchronize(stream));
}

void Proj2D::backward_host(const double* b, double* x) {
    const long long nimg = (long long)P.ni * P.nj, nsino = (long long)P.np * P.nu;
#pragma omp parallel for schedule(static) if (nsino > (1 << 16))
    for (long long e = 0; e < nsino; ++e) h_sino_[e] = (float)b[e];
    SGD_CUDA(cudaMemcpyAsync(d_sino_, h_sino_, nsino * sizeof(float), cudaMemcpyHostToDevice, stream));
    ensure_out64();
    P.out64 = d_out64_;
    backward_dev(d_sino_, d_img_, stream);
    P.out64 = nullptr;
    SGD_CUDA(cudaMemcpyAsync(x, d_out64_, nimg * sizeof(double), cudaMemcpyDeviceToHost, stream));
    SGD_CUDA(cudaStreamSynchronize(stream));
    if (status(false) != 0) fail("back projection: a staged view chunk did not arrive (bounded wait); output incomplete");
}

void Proj2D::ensure_out64() {
    if (d_out64_) return;
    const size_t n = std::max((size_t)P.ni * P.nj, (size_t)P.np * P.nu);
    SGD_CUDA(cudaMalloc(&d_out64_, n * sizeof(double)));
}

}  // namespace sgd
