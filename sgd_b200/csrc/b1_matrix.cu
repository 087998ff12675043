// B1 system matrices on the GPU.
//
//   sgd_b1_matrix_csr            the matrix of a B1 layer: exactly the pairs and
//                                FP32 footprints its projection kernels use,
//                                times dx*dy (so A x equals b1_forward_projection).
//   bilinear_matrix_generation   the reference's generator (layers/A_B1.cu:
//                                355-427, 545-593): uniform angles without the
//                                45-degree snap (geo_init_example), no dx*dy,
//                                entries > 0, and its own footprint window.
//
// The generator evaluates the footprint over [y, y + vblur] with
// y = |a1 - o| negated when o lies clockwise of edge ray a (:411-415), i.e.
// y = -xa with xa the signed offset of a1 from o along the lateral direction
// (fan_geometry.h), and vblur = |xb - xa|.  Its window is [-xa, -xa + |xb - xa|]
// where the projection kernels integrate over [xa, xb]: the two agree only
// for pixels centred on edge ray a.  Its two early exits are kept: both edge
// crossings more than a pixel away from the centre along x and along y
// (:400-401), and |a1 - o| > 2 (vx + vy) + vblur (:407-408).
#include <climits>
#include <cmath>
#include <vector>

#include "b1_kernels.cuh"
#include "b1_layer.h"
#include "common.h"
#include "csr_build.cuh"
#include "hom.cuh"

namespace sgd {

namespace {

__device__ __forceinline__ B1Bin bin_record(const float4* rec, int p, int u, int nu) {
    const float4* q = rec + (size_t)p * 4 * nu + u;
    return B1Bin{__ldg(q), __ldg(q + nu), __ldg(q + 2 * nu), __ldg(q + 3 * nu)};
}

__device__ __forceinline__ void hom_of(const BinHomography* hom, int p, float* h) {
    const BinHomography H = hom[p];
    h[0] = H.n0; h[1] = H.n1; h[2] = H.n2; h[3] = H.d0; h[4] = H.d1; h[5] = H.d2;
}

// The projection kernels' pairs: bins of the +-1 pixel support, conv > 1e-7.
struct B1CsrVisit {
    const float4* rec;
    const BinHomography* hom;
    int nu;
    float scale;
    __device__ bool valid(int, int) const { return true; }
    template <class F>
    __device__ void visit(int p, int i, int j, F&& f) const {
        float h[6];
        hom_of(hom, p, h);
        const float fi = (float)i, fj = (float)j;
        int lo, hi;
        box_bins(h, fi - 1.f, fi + 1.f, fj - 1.f, fj + 1.f, nu, lo, hi);
        for (int u = lo; u <= hi; ++u) {
            const float conv = b1_conv(fi, fj, bin_record(rec, p, u, nu));
            if (conv > kConvEps) f(u, conv * scale);
        }
    }
};

// The reference generator's entries.  gen[p * nu + u] = (|n.x|, |n.y|,
// 2 (vx + vy), 0) with n the bin's lateral unit vector.
struct B1GenVisit {
    const float4* rec;
    const BinHomography* hom;
    const float4* gen;
    int nu;
    float dx, dy;
    __device__ bool valid(int, int) const { return true; }
    template <class F>
    __device__ void visit(int p, int i, int j, F&& f) const {
        float h[6];
        hom_of(hom, p, h);
        const float fi = (float)i, fj = (float)j;
        int lo, hi;
        box_bins(h, fi - 1.f, fi + 1.f, fj - 1.f, fj + 1.f, nu, lo, hi);
        lo = max(0, lo - 2);  // the shifted window reaches about one bin further
        hi = min(nu - 1, hi + 2);
        for (int u = lo; u <= hi; ++u) {
            const B1Bin r = bin_record(rec, p, u, nu);
            const float4 g = __ldg(gen + (size_t)p * nu + u);
            // edge offsets in units of a (ya, yb) for the footprint, in mm
            // (xa, xb) for the window tests
            const float ya = b1_xa(fi, b1_xa_inner(fj, r), r), yb = b1_xb(fi, b1_xb_inner(fj, r), r);
            const float a = r.q3.w, xa = ya * a, xb = yb * a;
            const float w = fabsf(xb - xa), m = fminf(fabsf(xa), fabsf(xb));
            if (m * g.x > dx && m * g.y > dy) continue;
            if (fabsf(xa) > g.z + w) continue;
            const float wy = fabsf(yb - ya);
            const float conv = b1_conv_x(-ya, -ya + wy, r);
            if (conv > 0.f) f(u, conv);
        }
    }
};

}  // namespace

long long b1_layer_csr(A_B1& L, const CsrOut& out) {
    const B1Device& d = L.dev;
    B1CsrVisit v{reinterpret_cast<const float4*>(d.rec), d.hom, d.nu, d.dxdy};
    return build_csr(v, d.np, d.nu, d.nx, d.ny, out, L.stream);
}

long long b1_generator(int np, int nu, int nx, int ny, double dx, double dy, double du, double lsd, double lso,
                       const CsrOut& out) {
    if (np < 1 || nu < 1 || nx < 1 || ny < 1) fail("bilinear_matrix_generation: invalid sizes");
    // geo_init_example(lsd, lso, 0.0f, PI*2 * (np-1)/np) (utils/geo.cu:209-230)
    const double pi = 3.14159265358979323846;
    const double end = pi * 2 * (np - 1) / np;
    const double dangle = np > 1 ? (end - (double)0.0f) / (np - 1) : 0.0;
    std::vector<double> ang(np);
    for (int p = 0; p < np; ++p) ang[p] = (double)0.0f + p * dangle;
    A_B1 L(nx, ny, np, nu, dx, dy, du, lsd, lso, ang.data(), nullptr, nullptr);
    const FanGeometry& g = L.geo;
    std::vector<float4> gen((size_t)np * nu);
    for (int p = 0; p < np; ++p)
        for (int u = 0; u < nu; ++u) {
            const double off = u - 0.5 * nu + 0.5;
            const double sx = g.dtv[2 * p] + g.puv[2 * p] * off, sy = g.dtv[2 * p + 1] + g.puv[2 * p + 1] * off;
            const double tx = sx - g.src[2 * p], ty = sy - g.src[2 * p + 1], len = std::sqrt(tx * tx + ty * ty);
            const double vx = dx * std::fabs(ty) / len, vy = dy * std::fabs(tx) / len;
            gen[(size_t)p * nu + u] = make_float4((float)(std::fabs(ty) / len), (float)(std::fabs(tx) / len),
                                                  (float)(2 * vx + 2 * vy), 0.f);
        }
    float4* d_gen = nullptr;
    SGD_CUDA(cudaMalloc(&d_gen, gen.size() * sizeof(float4)));
    long long n = -1;
    try {
        SGD_CUDA(cudaMemcpy(d_gen, gen.data(), gen.size() * sizeof(float4), cudaMemcpyHostToDevice));
        B1GenVisit v{reinterpret_cast<const float4*>(L.dev.rec), L.dev.hom, d_gen, nu, (float)dx, (float)dy};
        n = build_csr(v, np, nu, nx, ny, out, L.stream);
    } catch (...) {
        cudaFree(d_gen);
        throw;
    }
    cudaFree(d_gen);
    return n;
}

}  // namespace sgd

extern "C" {

long long sgd_b1_matrix_csr(void* layer, long long* rowptr, int* cols, double* vals, long long cap) {
    return sgd::guarded<long long>(-1, [&]() -> long long {
        if (!layer) sgd::fail("sgd_b1_matrix_csr: null layer");
        if ((rowptr || cols || vals) && !(rowptr && cols && vals)) sgd::fail("sgd_b1_matrix_csr: partial output");
        sgd::CsrOut out;
        out.rowptr = rowptr; out.cols = cols; out.vals = vals; out.cap = cap;
        return sgd::b1_layer_csr(*static_cast<sgd::A_B1*>(layer), out);
    });
}

int bilinear_matrix_generation(int np, int nu, int nx, int ny, double dx, double dy, double du, double lsd,
                               double lso, double* spmat, int buffer_size) {
    return sgd::guarded<int>(-1, [&]() -> int {
        if (!spmat || buffer_size < 0) sgd::fail("bilinear_matrix_generation: null or negative buffer");
        sgd::CsrOut out;
        out.triplets = spmat;
        out.cap = buffer_size;
        const long long n = sgd::b1_generator(np, nu, nx, ny, dx, dy, du, lsd, lso, out);
        if (n > INT_MAX) sgd::fail("bilinear_matrix_generation: %lld entries overflow int", n);
        return (int)n;
    });
}

}  // extern "C"
