// B1 (bilinear) fan-beam projector in the reference's rounding, on the
// generic 2D kernels: the mode used where results must match the reference
// layer itself (layers/A_B1.cu) to the last few units in the last place rather
// than the exact footprint.
//
// The default B1 projector (b1.cu) evaluates the footprint from exact FP64
// bin geometry.  The reference instead positions each bin in FP32: its centre
// is dtv + puv (minu - nu/2 + 1/2) for the pixel's first bin minu, then
// stepped by `sx += puv.x` (layers/A_B1.cu:153-154, :160), and the edge-ray
// offsets come from FP32 intersections with the line through the pixel centre
// perpendicular to the central ray (:182-195), where positions of ~600 mm are
// differenced down to a fraction of a pixel.  That rounding moves its output
// about 1e-5 (rel-L2) from the exact footprint at 512^2 x 720 views.  This
// basis repeats those FP32 steps: the visited range from the four corners at
// +-1 through pmi (:100-151), the stepped bin centre and the two offsets are
// the reference's FP32 expressions, written in the same order so that the
// compiler forms the same operations.  The footprint of the two offsets is
// then the closed form of b1_kernels.cuh (the integral of the tri * tri
// profile between them over their distance), whose own FP32 error is far
// below the geometry's.  Entries with conv <= 1e-7 are dropped (:203).
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.h"
#include "proj2d_impl.cuh"

namespace sgd {

struct B1RefBasis {
    static constexpr int kViewFloats = 20;
    // [0..5] pmi 0,1,3,8,9,11 [6] puv.x [7] puv.y [8] singular [9] src.x [10] src.y
    // [11] dtv.x [12] dtv.y [13] dx [14] dy [15] 0.5 (nx-1) [16] 0.5 (ny-1)
    struct View {
        float pm0, pm1, pm3, pm8, pm9, pm11, puvx, puvy, singular, srcx, srcy, dtvx, dtvy, dx, dy, nx2, ny2;
    };
    // per bin (FP32): b, a, a+b, a-b | 1/a, 1/(2a^2), -b^2/(12a^2), 1/(12a^2b^2) | -1/(24a^2b^2), 0, 0, 0
    // with a = max(vx, vy), b = min(vx, vy) of the reference's per-bin
    // vectors (layers/A_B1.cu:429-478); b = 0 below 1e-7 (the single-triangle
    // limit, :52-55)
    static constexpr int kBinF4 = 3;
    struct Cell {
        float ox, oy, sx, sy;  // pixel centre; centre of the next bin of the walk (FP32 stepped)
        int lo, hi;
    };
    __device__ static void load_view(const float* v, View& V) {
        const float4* q = reinterpret_cast<const float4*>(v);
        const float4 a = q[0], b = q[1], c = q[2], d = q[3], e = q[4];
        V = View{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w, d.x, d.y, d.z, d.w, e.x};
    }
    __device__ static bool valid(int, int, const Fan2DParams&) { return true; }
    __device__ static void order(float& a, float& b) {
        if (a > b) {
            const float t = b;
            b = a;
            a = t;
        }
    }
    // layers/A_B1.cu:96-154
    __device__ static void setup(const View& V, int ix, int iy, const Fan2DParams& P, Cell& c) {
        c.ox = (ix - V.nx2) * V.dx;
        c.oy = (iy - V.ny2) * V.dy;
        const float x1 = ix - 1.0f, x2 = ix + 1.0f, y1 = iy - 1.0f, y2 = iy + 1.0f;
        float us[4];
        if (V.singular == 0.f) {
            us[0] = (V.pm0 * x1 + V.pm3 + V.pm1 * y1) / (V.pm8 * x1 + V.pm11 + V.pm9 * y1);
            us[1] = (V.pm0 * x1 + V.pm3 + V.pm1 * y2) / (V.pm8 * x1 + V.pm11 + V.pm9 * y2);
            us[2] = (V.pm0 * x2 + V.pm3 + V.pm1 * y1) / (V.pm8 * x2 + V.pm11 + V.pm9 * y1);
            us[3] = (V.pm0 * x2 + V.pm3 + V.pm1 * y2) / (V.pm8 * x2 + V.pm11 + V.pm9 * y2);
        } else {
            us[0] = ((V.pm0 * x1 + V.pm3 + V.pm1 * y1) / (V.pm8 * x1 + V.pm11 + V.pm9 * y1) * 1.5f - 1.0f) / V.puvx;
            us[1] = ((V.pm0 * x1 + V.pm3 + V.pm1 * y2) / (V.pm8 * x1 + V.pm11 + V.pm9 * y2) * 1.5f - 1.0f) / V.puvx;
            us[2] = ((V.pm0 * x2 + V.pm3 + V.pm1 * y1) / (V.pm8 * x2 + V.pm11 + V.pm9 * y1) * 1.5f - 1.0f) / V.puvx;
            us[3] = ((V.pm0 * x2 + V.pm3 + V.pm1 * y2) / (V.pm8 * x2 + V.pm11 + V.pm9 * y2) * 1.5f - 1.0f) / V.puvx;
        }
        order(us[0], us[1]);
        order(us[2], us[3]);
        order(us[0], us[2]);
        order(us[1], us[3]);
        order(us[1], us[2]);
        c.lo = min(max(0, (int)floorf(us[0])), P.nu - 1);
        c.hi = min(max(0, (int)floorf(us[3])), P.nu - 1);
        c.sx = V.dtvx + V.puvx * (c.lo - 0.5f * P.nu + 0.5f);
        c.sy = V.dtvy + V.puvy * (c.lo - 0.5f * P.nu + 0.5f);
    }
    __device__ static void skip(const View& V, Cell& c) {
        c.sx += V.puvx;
        c.sy += V.puvy;
    }
    __device__ static void start(const View&, Cell&, int) {}
    // Odd cumulative profile G of the unit-area tri(a) * tri(b) convolution
    // (fan_geometry.h: S(x) in closed form, every power a distance to a knot).
    __device__ static float G(float x, const float4& k0, const float4& k1, const float4& k2) {
        const float b = k0.x, a = k0.y, apb = k0.z, amb = k0.w;
        const float ax = fabsf(x);
        const float w = fmaxf(b - ax, 0.f), w2 = w * w, w4 = w2 * w2;
        const float sin_ = fmaf(k1.w, w4, fmaf(ax, fmaf(-ax, k1.y, k1.x), k1.z));
        const float p = fmaxf(apb - ax, 0.f), q = fmaxf(a - ax, 0.f);
        const float p2 = p * p, q2 = q * q;
        const float t = fmaf(p2, p2, fmaf(-2.f * q2, q2, -2.f * w4));
        const float sout = fmaf(k2.x, t, 0.5f);
        return copysignf(ax <= amb ? sin_ : sout, x);
    }
    // layers/A_B1.cu:182-203 for the bin at the walk's current centre
    __device__ static float value(const View& V, Cell& c, int, BinRef t, const Fan2DParams&) {
        const float sx = c.sx, sy = c.sy;
        skip(V, c);
        const float px = V.srcx, py = V.srcy, ox = c.ox, oy = c.oy;
        const float ax = sx - V.puvx * 0.5f;
        const float ay = sy - V.puvy * 0.5f;
        const float bx = sx + V.puvx * 0.5f;
        const float by = sy + V.puvy * 0.5f;
        // the reference's expressions; a*b + c*d as dot2f (first product fused)
        const float num = dot2f(ox - px, sx - px, oy - py, sy - py);
        const float ra = num / dot2f(ax - px, sx - px, ay - py, sy - py);
        const float rb = num / dot2f(bx - px, sx - px, by - py, sy - py);
        const float ax1 = px + (ax - px) * ra, ay1 = py + (ay - py) * ra;
        const float bx1 = px + (bx - px) * rb, by1 = py + (by - py) * rb;
        const float x1 = sqrtf(dot2f(ax1 - ox, ax1 - ox, ay1 - oy, ay1 - oy));
        const float x2 = sqrtf(dot2f(bx1 - ox, bx1 - ox, by1 - oy, by1 - oy));
        const float sgn = (dot2f(ax1 - ox, bx1 - ox, ay1 - oy, by1 - oy) > 0) ? 1.0f : -1.0f;
        const float xa = x1 * sgn;
        const float4 k0 = t[0], k1 = t[1], k2 = t[2];
        const float conv = fabsf(G(x2, k0, k1, k2) - G(xa, k0, k1, k2)) / fabsf(x2 - xa);
        return (conv > 1e-7f && conv == conv) ? conv : 0.f;
    }
};

namespace {

class B1RefLayer final : public Proj2D {
public:
    B1RefLayer(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
               const double* angles, const double* dz, const double* drho) {
        geo.init(nx, ny, np, nu, dx, dy, du, lsd, lso, angles, dz, drho);
        P.ni = nx;
        P.nj = ny;
        std::vector<float> view((size_t)np * B1RefBasis::kViewFloats, 0.f);
        std::vector<float4> bins((size_t)np * nu * B1RefBasis::kBinF4);
        for (int p = 0; p < np; ++p) {
            const ViewFrame& f = geo.frames[p];
            float* v = &view[(size_t)p * B1RefBasis::kViewFloats];
            const float* m = &geo.pmi[12 * (size_t)p];
            v[0] = m[0]; v[1] = m[1]; v[2] = m[3]; v[3] = m[8]; v[4] = m[9]; v[5] = m[11];
            const float puvx = (float)f.puv[0], puvy = (float)f.puv[1];
            v[6] = puvx;
            v[7] = puvy;
            v[8] = (std::fabs(puvx - puvy) < 1e-7f) ? 1.f : 0.f;  // layers/A_B1.cu:103
            v[9] = (float)f.src[0]; v[10] = (float)f.src[1];
            v[11] = (float)f.dtv[0]; v[12] = (float)f.dtv[1];
            v[13] = (float)dx; v[14] = (float)dy;
            v[15] = 0.5f * (nx - 1); v[16] = 0.5f * (ny - 1);
            // the reference's per-bin vectors (FP64, stored as FP32): the
            // pixel sides projected across the ray through the bin centre
            const double cx = f.dtv[0], cy = f.dtv[1], ux = f.puv[0], uy = f.puv[1], px = f.src[0], py = f.src[1];
            for (int u = 0; u < nu; ++u) {
                const double sx = cx + ux * (u - 0.5 * nu + 0.5), sy = cy + uy * (u - 0.5 * nu + 0.5);
                const double th = std::atan2(std::fabs(px - sx), std::fabs(py - sy));
                const float vx = (float)std::fabs(dx * std::cos(th)), vy = (float)std::fabs(dy * std::sin(th));
                float r[16];
                b1_profile_constants(std::max(vx, vy), std::min(vx, vy), r);
                const float b = r[6], a = r[8];
                float4* o = &bins[(size_t)p * B1RefBasis::kBinF4 * nu + u];  // planes of nu words
                o[0] = make_float4(b, a, r[10], (float)((double)a - (double)b));
                o[nu] = make_float4(r[12], r[13], r[14], r[15]);
                o[2 * nu] = make_float4(-0.5f * r[15], 0.f, 0.f, 0.f);
            }
        }
        finish_init(view, bins);
        out_scale = (float)dx * (float)dy;
        count = fan2d_count<B1RefBasis>(P, stream);
    }
    void forward_dev(const float* img, float* sino, cudaStream_t s) override {
        fan2d_forward<B1RefBasis>(P, img, sino, out_scale, s);
    }
    long long csr(const CsrOut& out) override { return fan2d_csr<B1RefBasis>(P, out_scale, out, stream); }
    void backward_dev(const float* sino, float* img, cudaStream_t s) override {
        fan2d_back<B1RefBasis>(P, sino, img, out_scale, s);
    }

protected:
    // ranges from the corners at +-1
    RangeMap range_map(int p) const override {
        double hw[6];
        fan_world_hom(geo, p, hw);
        return grid_range_map(hw, geo.x0(), geo.dx, geo.y0(), geo.dy, 1.0, 1.0);
    }
};

}  // namespace

Proj2D* make_b1ref_layer(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
                         const double* angles, const double* dz, const double* drho) {
    return new B1RefLayer(nx, ny, np, nu, dx, dy, du, lsd, lso, angles, dz, drho);
}

}  // namespace sgd
