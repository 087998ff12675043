// B0: pixel-indicator fan-beam projector on the generic 2D kernels.
// Reference: layers/A_B0.cu:20-35 (footprint), :123-229 (forward), :231-336
// (backward), :338-388 (per-bin vectors), :494-575 (C entry points).
//
// Per pixel and view the bin range comes from the pixel's four corners through
// pmi (bit-identical to the reference's); per bin, the footprint is the
// 3-direction box spline of layers/spline_conv.hh:239-293 with directions
// (vx, vy, vblur) at an offset y measured from the pixel corner, vblur being
// the bin's width at the pixel's depth.  The reference's FP32 geometry is
// kept (its FP32 stepping of the bin centre, sx += puv.x, :202, and the FP32
// products it forms); its FP64 per-bin vectors and the FP64 scalings of
// those products, whose results it rounds to FP32 for the spline, run in
// FP32 here (a difference of an ulp or two per value), the two divisions by
// the source-bin distance as products with its reciprocals.
#include <climits>
#include <cmath>
#include <vector>

#include "common.h"
#include "hom.cuh"
#include "proj2d_impl.cuh"
#include "spline3.cuh"

namespace sgd {

struct B0Basis {
    static constexpr int kViewFloats = 20;
    // [0..5] pmi 0,1,3,8,9,11 [6] puv.x [7] singular [8] src.x [9] src.y [10] dtv.x
    // [11] dtv.y [12] puv.y [13] dx [14] dy [15] (nx-1)/2 [16] (ny-1)/2
    struct View {
        float pm0, pm1, pm3, pm8, pm9, pm11, puvx, singular, srcx, srcy, dtvx, dtvy, puvy, dx, dy, nx2, ny2;
    };
    // per bin: vx, vy, a0s, sb0 | 1/lsp, 1/lsp^2, 1/x0, 1/x1 (x0 >= x1
    // = |vx|, |vy|; computed in FP64, stored in FP32: the reference's FP64
    // arithmetic on them ends in FP32 arguments of the spline)
    static constexpr int kBinF4 = 2;
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
    __device__ static void sort2(float& a, float& b) {
        if (a > b) {
            const float t = b;
            b = a;
            a = t;
        }
    }
    // layers/A_B0.cu:152-198.  The bin range is the reference's: the floors
    // of the extreme corner projections under IEEE division.  Fast
    // quotients (within 2 ulp of the IEEE ones) give the same floors unless an
    // extreme lies next to an integer; that case, a non-finite projection
    // and the singular views take the IEEE divisions.
    __device__ static void setup(const View& V, int ix, int iy, const Fan2DParams& P, Cell& c) {
        c.ox = (ix - V.nx2) * V.dx;
        c.oy = (iy - V.ny2) * V.dy;
        const float signx1 = ix - 0.5f, signx2 = ix + 0.5f, signy1 = iy - 0.5f, signy2 = iy + 0.5f;
        const float u1 = V.pm0 * signx1 + V.pm3, u2 = V.pm8 * signx1 + V.pm11;
        const float u3 = V.pm0 * signx2 + V.pm3, u4 = V.pm8 * signx2 + V.pm11;
        const float n0 = u1 + V.pm1 * signy1, d0 = u2 + V.pm9 * signy1;
        const float n1 = u1 + V.pm1 * signy2, d1 = u2 + V.pm9 * signy2;
        const float n2 = u3 + V.pm1 * signy1, d2 = u4 + V.pm9 * signy1;
        const float n3 = u3 + V.pm1 * signy2, d3 = u4 + V.pm9 * signy2;
        float lo_u, hi_u;
        bool ieee = V.singular != 0.f;
        if (!ieee) {
            const float q0 = __fdividef(n0, d0), q1 = __fdividef(n1, d1);
            const float q2 = __fdividef(n2, d2), q3 = __fdividef(n3, d3);
            lo_u = fminf(fminf(q0, q1), fminf(q2, q3));
            hi_u = fmaxf(fmaxf(q0, q1), fmaxf(q2, q3));
            ieee = !(fabsf((q0 + q1) + (q2 + q3)) < 1e30f) || near_integer(lo_u) || near_integer(hi_u);
        }
        if (ieee) {
            float us[4] = {n0 / d0, n1 / d1, n2 / d2, n3 / d3};
            if (V.singular != 0.f) {
#pragma unroll
                for (int k = 0; k < 4; ++k) us[k] = (us[k] * 1.5f - 1.0f) / V.puvx;
            }
            sort2(us[0], us[1]);
            sort2(us[2], us[3]);
            sort2(us[0], us[2]);
            sort2(us[1], us[3]);
            sort2(us[1], us[2]);
            lo_u = us[0];
            hi_u = us[3];
        }
        c.lo = min(max(0, (int)floorf(lo_u)), P.nu - 1);
        c.hi = min(max(0, (int)floorf(hi_u)), P.nu - 1);
        const float fl = (float)c.lo;
        c.sx = V.dtvx + V.puvx * (fl - 0.5f * P.nu + 0.5f);
        c.sy = V.dtvy + V.puvy * (fl - 0.5f * P.nu + 0.5f);
    }
    // layers/A_B0.cu:20-35
    __device__ static float conv1d(float y, float v1, float v2, float v3) { return box3(y, v1, v2, v3); }
    // the reference's FP32 stepping of the bin centre (layers/A_B0.cu:202)
    __device__ static void skip(const View& V, Cell& c) {
        c.sx += V.puvx;
        c.sy += V.puvy;
    }
    __device__ static void start(const View&, Cell&, int) {}
    __device__ static float value(const View& V, Cell& c, int, BinRef t, const Fan2DParams&) {
        const float sx = c.sx, sy = c.sy;
        skip(V, c);
        const float4 b0 = t[0], b1 = t[1];  // vx, vy, a0s, sb0 | 1/lsp, 1/lsp^2, 1/x0, 1/x1
        const float px = V.srcx, py = V.srcy;
        // layers/A_B0.cu:207-219: the FP32 products as the reference forms
        // them, its FP64 scalings in FP32
        const float r1 = dot2f(c.ox - px, sx - px, c.oy - py, sy - py) * b1.y;
        const float vblur = (b0.z + b0.w) * (-r1);
        const float x1 = sx - px, y1 = sy - py, x2 = c.ox - 0.5f * V.dx - px, y2 = c.oy + 0.5f * V.dy - py;
        const float y = fmaf(b0.z, r1, dot2f(x1, y2, -x2, y1) * b1.x);
        // the spline as the (vx, vy) trapezoid's CDF differenced over the
        // blur width (box3_by_cum; within ~1e-7 of the closed form)
        const float conv = box3_by_cum(-y, b0.x, b0.y, vblur, b1.z, b1.w);
        return (conv > 1e-7f && conv == conv) ? conv : 0.f;
    }
};

// B0 in parallel-beam geometry (no counterpart in the reference, whose
// geometry always has a point source, utils/geo.cu:234).  View angle beta:
// rays along (cos beta, sin beta), detector axis e = (-sin beta, cos beta)
// through the isocentre (the limit of the fan geometry as the source
// recedes), bin u covering s in [(u - nu/2) du, (u - nu/2 + 1) du].  A pixel
// indicator of dx x dy projects onto e as the convolution of boxes of widths
// a = dx |e.x| and b = dy |e.y|; averaged over a bin it is dx dy times the
// unit-area 3-direction box spline of widths (a, b, du) at the distance of the
// pixel centre's projection from the bin centre (exact, not a model).
struct B0ParBasis {
    static constexpr int kViewFloats = 12;
    // [0] e.x [1] e.y [2] a [3] b [4] du [5] x0 [6] y0 [7] dx [8] dy [9] nu/2
    struct View {
        float ex, ey, a, b, du, x0, y0, dx, dy, hnu;
    };
    static constexpr int kBinF4 = 0;
    struct Cell {
        float s;
        int lo, hi;
    };
    __device__ static void load_view(const float* v, View& V) {
        const float4* q = reinterpret_cast<const float4*>(v);
        const float4 a = q[0], b = q[1], c = q[2];
        V = View{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y};
    }
    __device__ static bool valid(int, int, const Fan2DParams&) { return true; }
    __device__ static void setup(const View& V, int i, int j, const Fan2DParams& P, Cell& c) {
        const float ox = fmaf((float)i, V.dx, V.x0), oy = fmaf((float)j, V.dy, V.y0);
        c.s = fmaf(ox, V.ex, oy * V.ey);
        const float h = 0.5f * (V.a + V.b);
        c.lo = max(0, (int)floorf((c.s - h) / V.du + V.hnu));
        c.hi = min(P.nu - 1, (int)floorf((c.s + h) / V.du + V.hnu));
    }
    __device__ static float value(const View& V, Cell& c, int u, BinRef, const Fan2DParams&) {
        const float t = c.s - ((float)u - V.hnu + 0.5f) * V.du;
        const float conv = B0Basis::conv1d(t + 0.5f * (V.a + V.b + V.du), V.a, V.b, V.du);
        return (conv > 1e-7f && conv == conv) ? conv : 0.f;
    }
    __device__ static void skip(const View&, Cell&) {}
    __device__ static void start(const View&, Cell&, int) {}
};

namespace {

class B0Layer final : public Proj2D {
public:
    B0Layer(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
            const double* angles, const double* dz, const double* drho) {
        geo.init(nx, ny, np, nu, dx, dy, du, lsd, lso, angles, dz, drho);
        P.ni = nx;
        P.nj = ny;
        std::vector<float> view((size_t)np * B0Basis::kViewFloats, 0.f);
        std::vector<float4> bins((size_t)np * nu * B0Basis::kBinF4);
        for (int p = 0; p < np; ++p) {
            const ViewFrame& f = geo.frames[p];
            float* v = &view[(size_t)p * B0Basis::kViewFloats];
            const float* m = &geo.pmi[12 * (size_t)p];
            v[0] = m[0]; v[1] = m[1]; v[2] = m[3]; v[3] = m[8]; v[4] = m[9]; v[5] = m[11];
            v[6] = (float)f.puv[0];
            v[7] = (std::fabs((float)f.puv[0] - (float)f.puv[1]) < 1e-7f) ? 1.f : 0.f;  // layers/A_B0.cu:161
            v[8] = (float)f.src[0]; v[9] = (float)f.src[1];
            v[10] = (float)f.dtv[0]; v[11] = (float)f.dtv[1];
            v[12] = (float)f.puv[1];
            v[13] = (float)dx; v[14] = (float)dy;
            v[15] = 0.5f * (nx - 1); v[16] = 0.5f * (ny - 1);
            // layers/A_B0.cu:338-388, FP64
            const double cx = f.dtv[0], cy = f.dtv[1], ux = f.puv[0], uy = f.puv[1], px = f.src[0], py = f.src[1];
            for (int u = 0; u < nu; ++u) {
                const double sx = cx + ux * (u - 0.5 * nu + 0.5), sy = cy + uy * (u - 0.5 * nu + 0.5);
                const double ax = sx - ux * 0.5, ay = sy - uy * 0.5, bx = sx + ux * 0.5, by = sy + uy * 0.5;
                const double lsp = std::sqrt((px - sx) * (px - sx) + (py - sy) * (py - sy));
                const double th = std::atan2(std::fabs(px - sx), std::fabs(py - sy));
                double vx = std::fabs(dx * std::cos(th)), vy = std::fabs(dy * std::sin(th));
                if (py < sy) vx = -vx;
                if (px < sx) vy = -vy;
                double a0s = std::fabs((sx - px) * (ay - py) - (ax - px) * (sy - py)) / lsp;
                double sb0 = std::fabs((sx - px) * (by - py) - (bx - px) * (sy - py)) / lsp;
                a0s /= ((ax - px) * (sx - px) + (ay - py) * (sy - py)) / (lsp * lsp);
                sb0 /= ((bx - px) * (sx - px) + (by - py) * (sy - py)) / (lsp * lsp);
                float4* o = &bins[(size_t)p * B0Basis::kBinF4 * nu + u];  // planes of nu words
                o[0] = make_float4((float)vx, (float)vy, (float)a0s, (float)sb0);
                // the (vx, vy) trapezoid's 1/x0 and 1/x1, x0 >= x1 the widths'
                // magnitudes (an infinite second one for a box, whose ramp is
                // empty)
                const float fx = std::fabs((float)vx), fy = std::fabs((float)vy);
                const float fx0 = std::max(fx, fy), fx1 = std::min(fx, fy);
                o[nu] = make_float4((float)(1.0 / lsp), (float)(1.0 / (lsp * lsp)), 1.0f / fx0, 1.0f / fx1);
            }
        }
        finish_init(view, bins);
        out_scale = (float)dx * (float)dy;
        count = fan2d_count<B0Basis>(P, stream);
    }
    void forward_dev(const float* img, float* sino, cudaStream_t s) override {
        fan2d_forward<B0Basis>(P, img, sino, out_scale, s);
    }
    long long csr(const CsrOut& out) override { return fan2d_csr<B0Basis>(P, out_scale, out, stream); }
    void backward_dev(const float* sino, float* img, cudaStream_t s) override {
        fan2d_back<B0Basis>(P, sino, img, out_scale, s);
    }

protected:
    // ranges from the corners at +-1/2
    RangeMap range_map(int p) const override {
        double hw[6];
        fan_world_hom(geo, p, hw);
        return grid_range_map(hw, geo.x0(), geo.dx, geo.y0(), geo.dy, 0.5, 0.5);
    }
};

class B0ParallelLayer final : public Proj2D {
public:
    B0ParallelLayer(int nx, int ny, int np, int nu, double dx, double dy, double du, const double* angles) {
        if (nx < 1 || ny < 1 || np < 1 || nu < 1) fail("b0 parallel: invalid sizes");
        check_pitches({dx, dy, du});
        check_views(np, angles, nullptr, nullptr);
        geo.nx = nx; geo.ny = ny; geo.np = np; geo.nu = nu;
        geo.dx = dx; geo.dy = dy; geo.du = du;
        P.ni = nx;
        P.nj = ny;
        ex_.resize(np);
        ey_.resize(np);
        std::vector<float> view((size_t)np * B0ParBasis::kViewFloats, 0.f);
        for (int p = 0; p < np; ++p) {
            ex_[p] = -std::sin(angles[p]);
            ey_[p] = std::cos(angles[p]);
            float* v = &view[(size_t)p * B0ParBasis::kViewFloats];
            v[0] = (float)ex_[p]; v[1] = (float)ey_[p];
            v[2] = (float)(dx * std::fabs(ex_[p])); v[3] = (float)(dy * std::fabs(ey_[p]));
            v[4] = (float)du;
            v[5] = (float)(-0.5 * (nx - 1) * dx); v[6] = (float)(-0.5 * (ny - 1) * dy);
            v[7] = (float)dx; v[8] = (float)dy; v[9] = 0.5f * nu;
        }
        finish_init(view, {});
        out_scale = (float)dx * (float)dy;
        count = fan2d_count<B0ParBasis>(P, stream);
    }
    void forward_dev(const float* img, float* sino, cudaStream_t s) override {
        fan2d_forward<B0ParBasis>(P, img, sino, out_scale, s);
    }
    long long csr(const CsrOut& out) override { return fan2d_csr<B0ParBasis>(P, out_scale, out, stream); }
    void backward_dev(const float* sino, float* img, cudaStream_t s) override {
        fan2d_back<B0ParBasis>(P, sino, img, out_scale, s);
    }

protected:
    // u = s / du + nu/2 with s = x e.x + y e.y: a map without a pole; ranges
    // from the corners at +-1/2
    RangeMap range_map(int p) const override {
        const double hw[6] = {ex_[p] / geo.du, ey_[p] / geo.du, 0.5 * geo.nu, 0.0, 0.0, 1.0};
        return grid_range_map(hw, -0.5 * (geo.nx - 1) * geo.dx, geo.dx, -0.5 * (geo.ny - 1) * geo.dy, geo.dy, 0.5,
                              0.5);
    }

private:
    std::vector<double> ex_, ey_;
};


// The reference's pixel_matrix_generation (layers/A_B0.cu:37-121, 449-492):
// per (view, bin) and pixel, in FP64 there, a1/b1 = the edge rays' crossings
// of the line through the pixel centre o perpendicular to the central ray,
// z = o + (-dx/2, dy/2) - NM (a corner shifted onto that line), y = |a1 - z|
// negated when z lies counter-clockwise of edge ray a, vblur = -|b1 - a1|,
// and the footprint conv1d(y, vx, vy, vblur) with the signs of vx, vy set
// by the view (:69-70); entries > 0, no dx*dy.  Here a1 - z = xa n + c with
// xa affine in the pixel indices (fan_geometry.h), so one bin's constants
// are 16 floats: [xa_i xa_j xa_0 xb_i][xb_j xb_0 n.x n.y][c.x c.y k_i k_j]
// [k_0 vx vy 0], k the cross product of ray a with z - source, affine too.
struct B0GenVisit {
    const float4* rec;  // [view][bin][4]
    const BinHomography* hom;
    int nu;
    float dx, dy;
    __device__ bool valid(int, int) const { return true; }
    template <class F>
    __device__ void visit(int p, int i, int j, F&& f) const {
        const BinHomography H = hom[p];
        const float h[6] = {H.n0, H.n1, H.n2, H.d0, H.d1, H.d2};
        const float fi = (float)i, fj = (float)j;
        int lo, hi;
        box_bins(h, fi - 1.f, fi + 1.f, fj - 1.f, fj + 1.f, nu, lo, hi);
        lo = max(0, lo - 1);
        hi = min(nu - 1, hi + 1);
        for (int u = lo; u <= hi; ++u) {
            const float4* q = rec + ((size_t)p * nu + u) * 4;
            const float4 q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2), q3 = __ldg(q + 3);
            const float xa = fmaf(fi, q0.x, fmaf(fj, q0.y, q0.z)), xb = fmaf(fi, q0.w, fmaf(fj, q1.x, q1.y));
            const float m = fminf(fabsf(xa), fabsf(xb));
            if (m * fabsf(q1.z) > dx && m * fabsf(q1.w) > dy) continue;  // :98-99
            const float ex = fmaf(xa, q1.z, q2.x), ey = fmaf(xa, q1.w, q2.y);
            float y = sqrtf(ex * ex + ey * ey);
            const float vblur = -fabsf(xb - xa);
            if (y > fabsf(q3.y) + fabsf(q3.z) + fabsf(vblur)) continue;  // :112-113
            if (fmaf(fi, q2.z, fmaf(fj, q2.w, q3.x)) > 0.f) y = -y;      // :115-116
            const float conv = B0Basis::conv1d(y, q3.y, q3.z, vblur);
            if (conv > 0.f) f(u, conv);
        }
    }
};

long long b0_generator(int np, int nu, int nx, int ny, double dx, double dy, double du, double lsd, double lso,
                       const CsrOut& out) {
    if (np < 1 || nu < 1 || nx < 1 || ny < 1) fail("pixel_matrix_generation: invalid sizes");
    // geo_init_example(lsd, lso, 0.0f, PI*2 * (np-1)/np) (utils/geo.cu:209-230)
    const double pi = 3.14159265358979323846;
    const double end = pi * 2 * (np - 1) / np;
    const double dangle = np > 1 ? (end - (double)0.0f) / (np - 1) : 0.0;
    std::vector<double> ang(np);
    for (int p = 0; p < np; ++p) ang[p] = (double)0.0f + p * dangle;
    FanGeometry g;
    g.init(nx, ny, np, nu, dx, dy, du, lsd, lso, ang.data(), nullptr, nullptr);
    std::vector<BinHomography> hom;
    bin_homographies(g, hom);
    std::vector<float4> rec((size_t)np * nu * 4);
    const double x0 = g.x0(), y0 = g.y0();
    for (int p = 0; p < np; ++p) {
        const double px = g.src[2 * p], py = g.src[2 * p + 1];
        const double ex = g.puv[2 * p], ey = g.puv[2 * p + 1];
        for (int u = 0; u < nu; ++u) {
            const double off = u - 0.5 * nu + 0.5;
            const double sx = g.dtv[2 * p] + ex * off, sy = g.dtv[2 * p + 1] + ey * off;
            const double ax = sx - 0.5 * ex, ay = sy - 0.5 * ey, bx = sx + 0.5 * ex, by = sy + 0.5 * ey;
            const double L = std::sqrt((sx - px) * (sx - px) + (sy - py) * (sy - py));
            const double tx = (sx - px) / L, ty = (sy - py) / L, nxv = -ty, nyv = tx;
            // lateral offsets of the edge crossings (as the B1 tables)
            const double ka = ((ax - px) * nxv + (ay - py) * nyv) / ((ax - px) * tx + (ay - py) * ty);
            const double kb = ((bx - px) * nxv + (by - py) * nyv) / ((bx - px) * tx + (by - py) * ty);
            const double mAx = ka * tx - nxv, mAy = ka * ty - nyv, mBx = kb * tx - nxv, mBy = kb * ty - nyv;
            // z = o + (-dx/2, dy/2) - NM (:93-98)
            const double om = -0.5 * dx * (px - sx) + 0.5 * dy * (py - sy);
            const double NMx = om * (px - sx) / (L * L), NMy = om * (py - sy) / (L * L);
            const double cx = 0.5 * dx + NMx, cy = -0.5 * dy + NMy;
            // cross(a - src, z - src) / |a - src|, affine in (i, j)
            const double Ax = ax - px, Ay = ay - py, An = std::sqrt(Ax * Ax + Ay * Ay);
            const double k0 = -Ay * dx / An, k1 = Ax * dy / An;
            const double kc = (Ax * (y0 + 0.5 * dy - NMy - py) - Ay * (x0 - 0.5 * dx - NMx - px)) / An;
            // signed profile directions (:66-70)
            double vx = std::fabs(dx * std::fabs(py - sy) / L), vy = std::fabs(dy * std::fabs(px - sx) / L);
            if (py < sy) vx = -vx;
            if (px < sx) vy = -vy;
            float4* r = &rec[((size_t)p * nu + u) * 4];
            r[0] = make_float4((float)(mAx * dx), (float)(mAy * dy), (float)((x0 - px) * mAx + (y0 - py) * mAy),
                               (float)(mBx * dx));
            r[1] = make_float4((float)(mBy * dy), (float)((x0 - px) * mBx + (y0 - py) * mBy), (float)nxv, (float)nyv);
            r[2] = make_float4((float)cx, (float)cy, (float)k0, (float)k1);
            r[3] = make_float4((float)kc, (float)vx, (float)vy, 0.f);
        }
    }
    cudaStream_t s = nullptr;
    float4* d_rec = nullptr;
    BinHomography* d_hom = nullptr;
    long long n = -1;
    try {
        SGD_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        SGD_CUDA(cudaMalloc(&d_rec, rec.size() * sizeof(float4)));
        SGD_CUDA(cudaMalloc(&d_hom, hom.size() * sizeof(BinHomography)));
        SGD_CUDA(cudaMemcpy(d_rec, rec.data(), rec.size() * sizeof(float4), cudaMemcpyHostToDevice));
        SGD_CUDA(cudaMemcpy(d_hom, hom.data(), hom.size() * sizeof(BinHomography), cudaMemcpyHostToDevice));
        n = build_csr(B0GenVisit{d_rec, d_hom, nu, (float)dx, (float)dy}, np, nu, nx, ny, out, s);
    } catch (...) {
        cudaFree(d_rec); cudaFree(d_hom);
        if (s) cudaStreamDestroy(s);
        throw;
    }
    cudaFree(d_rec); cudaFree(d_hom);
    cudaStreamDestroy(s);
    return n;
}
}  // namespace

Proj2D* make_b0_layer(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
                      const double* angles, const double* dz, const double* drho) {
    return new B0Layer(nx, ny, np, nu, dx, dy, du, lsd, lso, angles, dz, drho);
}

Proj2D* make_b0_parallel_layer(int nx, int ny, int np, int nu, double dx, double dy, double du,
                               const double* angles) {
    return new B0ParallelLayer(nx, ny, np, nu, dx, dy, du, angles);
}

}  // namespace sgd

extern "C" int pixel_matrix_generation(int np, int nu, int nx, int ny, double dx, double dy, double du, double lsd,
                                       double lso, double* spmat, int buffer_size) {
    return sgd::guarded<int>(-1, [&]() -> int {
        if (!spmat || buffer_size < 0) sgd::fail("pixel_matrix_generation: null or negative buffer");
        sgd::CsrOut out;
        out.triplets = spmat;
        out.cap = buffer_size;
        const long long n = sgd::b0_generator(np, nu, nx, ny, dx, dy, du, lsd, lso, out);
        if (n > INT_MAX) sgd::fail("pixel_matrix_generation: %lld entries overflow int", n);
        return (int)n;
    });
}
