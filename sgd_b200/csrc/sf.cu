// A_SF: separable-footprint (SF-TR) 2D fan-beam projector on the generic 2D
// kernels.  Reference: layers/A_SF.cu:48-84 (gamma_calculate), :87-225
// (forward), :228-334 (backward), :395-479 (C entry points).
//
// Per pixel and view the four pixel corners (i +- 1/2, j +- 1/2) are projected
// through the view's index-space matrix pmi (bit-identical to the reference's,
// fan_geometry.h) into bin coordinates, sorted into a trapezoid us[0..3]; the
// footprint in bin u is the trapezoid's integral over [u, u+1] (unit plateau)
// times dx / max(|sin t|, |cos t|), t the direction of the pixel centre from
// the source; bins with gamma <= 1e-7 are dropped as the reference drops them.
// The corners' divisions are fast (MUFU) divisions: a range end that one moves
// by an ulp across a bin edge adds or drops a bin whose integral is about
// k ulp^2, far below that threshold.  The integral over bin [u, u+1] is F(u +
// 1) - F(u) with F the trapezoid's cumulative area (the reference sums its
// three clipped pieces, layers/A_SF.cu:48-84: the same number up to an FP32
// rounding of F), so a walk over a cell's bins takes one F per bin.
#include <cmath>

#include "common.h"
#include "proj2d_impl.cuh"

namespace sgd {

struct SFBasis {
    static constexpr int kViewFloats = 16;
    // [0..5] pmi 0,1,3,8,9,11  [6] puv.x  [7] singular  [8] src.x  [9] src.y
    // [10] dx  [11] dy  [12] (nx-1)/2  [13] (ny-1)/2
    struct View {
        float pm0, pm1, pm3, pm8, pm9, pm11, puvx, singular, srcx, srcy, dx, dy, nx2, ny2;
    };
    static constexpr int kBinF4 = 0;
    struct Cell {
        float us[4];
        float weight;
        float r0, r1, r2;  // reciprocal widths of the ramp up, the plateau and the ramp down
        float F;           // the cumulative area left of the walk's next bin
        int lo, hi;
    };
    __device__ static void load_view(const float* v, View& V) {
        const float4* q = reinterpret_cast<const float4*>(v);
        const float4 a = q[0], b = q[1], c = q[2], d = q[3];
        V = View{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w, d.x, d.y};
    }
    __device__ static bool valid(int, int, const Fan2DParams&) { return true; }

    __device__ static void sort2(float& a, float& b) {
        if (a > b) {
            const float t = b;
            b = a;
            a = t;
        }
    }
    // layers/A_SF.cu:116-177
    __device__ static void setup(const View& V, int ix, int iy, const Fan2DParams& P, Cell& c) {
        const float signx1 = ix - 0.5f, signx2 = ix + 0.5f, signy1 = iy - 0.5f, signy2 = iy + 0.5f;
        float* us = c.us;
        us[0] = __fdividef(V.pm0 * signx1 + V.pm3 + V.pm1 * signy1, V.pm8 * signx1 + V.pm11 + V.pm9 * signy1);
        us[1] = __fdividef(V.pm0 * signx1 + V.pm3 + V.pm1 * signy2, V.pm8 * signx1 + V.pm11 + V.pm9 * signy2);
        us[2] = __fdividef(V.pm0 * signx2 + V.pm3 + V.pm1 * signy1, V.pm8 * signx2 + V.pm11 + V.pm9 * signy1);
        us[3] = __fdividef(V.pm0 * signx2 + V.pm3 + V.pm1 * signy2, V.pm8 * signx2 + V.pm11 + V.pm9 * signy2);
        if (V.singular != 0.f) {
            const float r = __fdividef(1.0f, V.puvx);
#pragma unroll
            for (int k = 0; k < 4; ++k) us[k] = (us[k] * 1.5f - 1.0f) * r;
        }
        sort2(us[0], us[1]);
        sort2(us[2], us[3]);
        sort2(us[0], us[2]);
        sort2(us[1], us[3]);
        sort2(us[1], us[2]);
        c.lo = min(max(0, (int)floorf(us[0])), P.nu - 1);
        c.hi = min(max(0, (int)floorf(us[3])), P.nu - 1);
        // dx / max(|sin t|, |cos t|) for t = atan2(X, Y) (:174-177) without
        // the trigonometry: |sin t| = |X| / r, |cos t| = |Y| / r
        const float X = V.dx * (ix - V.nx2) - V.srcx, Y = V.dy * (iy - V.ny2) - V.srcy;
        // (X = Y = 0, a cell centred on the source: atan2(0, 0) = 0, weight dx)
        const float r2 = dot2f(X, X, Y, Y);
        c.weight = r2 > 0.f ? V.dx * __fdividef(r2 * rsqrtf(r2), fmaxf(fabsf(X), fabsf(Y))) : V.dx;
        // the pieces' reciprocal widths, once per cell and view (fast
        // reciprocals; a zero width gives an infinite one, see area)
        c.r0 = __fdividef(1.0f, us[1] - us[0]);
        c.r1 = __fdividef(1.0f, us[2] - us[1]);
        c.r2 = __fdividef(1.0f, us[3] - us[2]);
    }
    // the cumulative area at the first bin the walk evaluates
    __device__ static void start(const View&, Cell& c, int u) { c.F = area(c, (float)u); }
    // the trapezoid's area left of s from each piece's covered fraction t
    // in [0, 1] (saturated products, on the FMA pipe): ramp up w01 t0^2 / 2,
    // plateau w12 t1, ramp down w23 t2 (2 - t2) / 2.  A zero-width piece has
    // an infinite reciprocal width; its fraction saturates to 0 or 1 (0 for
    // the NaN at its own end) and it adds zero width times that.
    __device__ static float area(const Cell& c, float s) {
        const float* us = c.us;
        const float t0 = __saturatef((s - us[0]) * c.r0);
        const float t1 = __saturatef((s - us[1]) * c.r1);
        const float t2 = __saturatef((s - us[2]) * c.r2);
        const float h01 = 0.5f * (us[1] - us[0]), w12 = us[2] - us[1], h23 = 0.5f * (us[3] - us[2]);
        return __fmaf_rn(h01 * t0, t0, __fmaf_rn(w12, t1, h23 * t2 * (2.0f - t2)));
    }
    __device__ static float value(const View&, Cell& c, int u, BinRef, const Fan2DParams&) {
        const float F1 = area(c, u + 1.0f);
        const float g = F1 - c.F;
        c.F = F1;
        // (the amplitude is finite, so the product is a number wherever g is)
        return g > 1e-7f ? c.weight * g : 0.f;
    }
    __device__ static void skip(const View&, Cell&) {}
};

namespace {

class SFLayer final : public Proj2D {
public:
    SFLayer(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
            const double* angles) {
        geo.init(nx, ny, np, nu, dx, dy, du, lsd, lso, angles, nullptr, nullptr);
        P.ni = nx;
        P.nj = ny;
        std::vector<float> view((size_t)np * SFBasis::kViewFloats, 0.f);
        for (int p = 0; p < np; ++p) {
            float* v = &view[(size_t)p * SFBasis::kViewFloats];
            const float* m = &geo.pmi[12 * (size_t)p];
            v[0] = m[0]; v[1] = m[1]; v[2] = m[3]; v[3] = m[8]; v[4] = m[9]; v[5] = m[11];
            const float puvx = (float)geo.frames[p].puv[0], puvy = (float)geo.frames[p].puv[1];
            v[6] = puvx;
            v[7] = (std::fabs(puvx - puvy) < 1e-7f) ? 1.f : 0.f;  // layers/A_SF.cu:119
            v[8] = (float)geo.frames[p].src[0];
            v[9] = (float)geo.frames[p].src[1];
            v[10] = (float)dx;
            v[11] = (float)dy;
            v[12] = (nx - 1) / 2.0f;
            v[13] = (ny - 1) / 2.0f;
        }
        finish_init(view, {});
        count = 0;  // the reference's SF kernels never count (layers/A_SF.cu:19)
    }
    void forward_dev(const float* img, float* sino, cudaStream_t s) override {
        fan2d_forward<SFBasis>(P, img, sino, 1.f, s);
    }
    long long csr(const CsrOut& out) override { return fan2d_csr<SFBasis>(P, 1.f, out, stream); }
    void backward_dev(const float* sino, float* img, cudaStream_t s) override {
        fan2d_back<SFBasis>(P, sino, img, 1.f, s);
    }

protected:
    // ranges from the corners at +-1/2
    RangeMap range_map(int p) const override {
        double hw[6];
        fan_world_hom(geo, p, hw);
        return grid_range_map(hw, geo.x0(), geo.dx, geo.y0(), geo.dy, 0.5, 0.5);
    }
};

}  // namespace

Proj2D* make_sf_layer(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
                      const double* angles) {
    return new SFLayer(nx, ny, np, nu, dx, dy, du, lsd, lso, angles);
}

}  // namespace sgd
