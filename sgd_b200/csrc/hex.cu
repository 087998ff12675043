// Hexagonal-lattice projectors H0 (hexagon indicator) and Hl (hexagonal
// linear box spline) on the generic 2D kernels.
// Reference: layers/A_H0.cu:84-358, :555-643 and layers/A_Hl.cu:21-46,
// :168-368, :569-656.
//
// Lattice: nl rows (il) of nc sites (ic), odd rows one site shorter and
// shifted by half a site; site (ic, il) at
//     x = (ic - (nc-1)/2 [odd rows: (nc-2)/2]) * sqrt(3) dt,  y = (il - (nl-1)/2) * dy
// with dy = 1.5 dt for H0 and 0.5 dt for Hl (A_H0.cu:174-183, A_Hl.cu:184-193).
// Host layout x[ic*nl + il] (A_H0.cu:581-583): cell (i, j) = (ic, il).
//
// Per (site, view, bin) the footprint follows the reference's FP32 geometry
// (bin centre stepped in FP32 from the first bin, edge rays intersected with
// the line through the site perpendicular to the bin's central ray: offset y
// and blur width vblur in FP64) and evaluates
//   H0: the sum of three 3-direction box splines (vblur, va, vb), (vblur, vb,
//       vc), (vblur, vc, va) (layers/spline_conv.hh:244-293), each the
//       difference over the blur width of its pair's trapezoid CDF, FP32;
//   Hl: the 4-direction box spline (vblur, va, vb, vc) (A_Hl.cu:21-46,
//       FP64 divided differences of truncated cubes there): with all four
//       directions kept, the difference over the blur width of the
//       3-direction spline's CDF in closed form, FP32, from per-bin constants
//       (box4_hex_by_cum, spline3.cuh); otherwise, as the reference, FP64
//       divided differences with the directions below 1e-8 dropped;
// va, vb, vc = dt sin(theta + {0, 2pi/3, 4pi/3}) with theta the bin's ray
// direction (FP64, per view and bin on the host; the reference recomputes them
// per pair from the stepped FP32 bin centre, a difference far below 1e-6).
//
// Bin ranges.  Hl and "H0 reference-compatible" take the reference's six-vertex
// bounds through pmi (A_H0.cu:84-156), including H0's use of the 0.5 dt row
// pitch pmi was built with (h0_init, A_H0.cu:556) although its sites sit at
// 1.5 dt, so that off-centre rows lose footprint exactly as in the reference,
// and H0's extra skip test in the back projection (A_H0.cu:333-334).
// "H0 corrected" bounds the true hexagon of each site and has no skip test:
// the pair is then an exact transpose.
#include <algorithm>
#include <cmath>

#include "common.h"
#include "proj2d_impl.cuh"
#include "spline3.cuh"

namespace sgd {

enum HexMode : int { kH0Corrected = 0, kH0Reference = 1, kHl = 2 };

// M: the HexMode, fixed per kernel so that each compiles only its own path
template <int M>
struct HexBasis {
    static constexpr int kViewFloats = 28;
    // [0..5] pmi 0,1,3,8,9,11 [6] puv.x [7] puv.y [8] src.x [9] src.y [10] dtv.x [11] dtv.y
    // [12] dt [13] dx [14] dy [15] (nl-1)/2 [16] (nc-1)/2 [17] (nc-2)/2
    // [18..23] world homography n0 n1 n2 d0 d1 d2 (u = (n0 x + n1 y + n2)/(d0 x + d1 y + d2))
    // [24] mode [25] back (1 in the back projection's view table, for H0's skip test)
    struct View {
        float pm0, pm1, pm3, pm8, pm9, pm11, puvx, puvy, srcx, srcy, dtvx, dtvy, dt, dx, dy, nl2, nc2, nc3;
        float h0, h1, h2, h3, h4, h5;
        int mode, back;
    };
    // per bin FP32 (va, vb, vc, ...); H0 with the true bounds holds (va, vb,
    // beta_a, beta_b) (alpha_a, alpha_b), vc = -(va + vb) (the three lattice
    // directions sum to 0) and the exact edge-ray maps, the signed offset of
    // edge ray e from site O along the line through O perpendicular to the
    // bin's central ray being alpha_e . O + beta_e; Hl adds its 3-direction
    // spline's constants (box4_hex_by_cum): (va, vb, vc, GK2) (x1, x2, h, rp6)
    static constexpr int kBinF4 = M == kH0Reference ? 1 : 2;
    struct Cell {
        float ox, oy, sx, sy;  // site; centre of the next bin of the walk (FP32 stepped)
        int lo, hi;
    };
    __device__ static void load_view(const float* v, View& V) {
        const float4* q = reinterpret_cast<const float4*>(v);
        const float4 a = q[0], b = q[1], c = q[2], d = q[3], e = q[4], f = q[5], g = q[6];
        V = View{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w, d.x, d.y, d.z, d.w, e.x, e.y,
                 e.z, e.w, f.x, f.y, f.z, f.w, (int)g.x, (int)g.y};
    }
    // nc = P.nj? no: cells are (ic, il) with ic in [0, nc) along i, il in [0, nl) along j
    __device__ static bool valid(int ic, int il, const Fan2DParams& P) { return !((il & 1) && ic == P.ni - 1); }

    // layers/A_H0.cu:47-156 (first stage; the jittered and linearised stages
    // only apply to singular projections, which a source outside the field of
    // view never produces; a full scan stays as the last resort).  With every
    // vertex regular, fast quotients give the reference's floors unless an
    // extreme lies next to an integer (near_integer); that case and any
    // irregular vertex take the reference's IEEE divisions.
    __device__ static void pmi_bounds(const View& V, int ic, int il, int nu, int& lo, int& hi) {
        const float icc = (float)ic + ((il & 1) ? 0.5f : 0.0f), ilc = (float)il;
        const float offc[6] = {0.0f, +0.5f, +0.5f, 0.0f, -0.5f, -0.5f};
        const float offl[6] = {-2.0f, -1.0f, +1.0f, +2.0f, +1.0f, -1.0f};
        float num[6], den[6];
        float umin = 1e30f, umax = -1e30f;
        bool regular = true;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const float ix = icc + offc[k], iy = ilc + offl[k];
            num[k] = fmaf(V.pm0, ix, fmaf(V.pm1, iy, V.pm3));
            den[k] = fmaf(V.pm8, ix, fmaf(V.pm9, iy, V.pm11));
            regular = regular && fabsf(num[k]) < 1e30f && fabsf(den[k]) >= 1e-8f && fabsf(den[k]) < 1e30f;
            const float u = __fdividef(num[k], den[k]);
            umin = fminf(umin, u);
            umax = fmaxf(umax, u);
        }
        if (!regular || !(fabsf(umin) < 1e30f && fabsf(umax) < 1e30f) || near_integer(umin) || near_integer(umax)) {
            umin = 1e30f;
            umax = -1e30f;
            int nvalid = 0;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                if (!isfinite(num[k]) || !isfinite(den[k]) || fabsf(den[k]) < 1e-8f) continue;
                const float u = num[k] / den[k];
                if (!isfinite(u)) continue;
                umin = fminf(umin, u);
                umax = fmaxf(umax, u);
                ++nvalid;
            }
            if (nvalid < 2) {
                lo = 0;
                hi = nu - 1;
                return;
            }
        }
        lo = min(max(0, (int)floorf(umin)), nu - 1);
        hi = min(max(0, (int)floorf(umax)), nu - 1);
        if (hi < lo) hi = lo;
    }
    // bins of the true hexagon (vertices at distance dt from the site)
    __device__ static void true_bounds(const View& V, float ox, float oy, int nu, int& lo, int& hi) {
        const float hx = 0.8660254037844386f * V.dt, hy = 0.5f * V.dt;
        const float xs[6] = {ox, ox + hx, ox + hx, ox, ox - hx, ox - hx};
        const float ys[6] = {oy - V.dt, oy - hy, oy + hy, oy + V.dt, oy + hy, oy - hy};
        float umin = 1e30f, umax = -1e30f;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            // fast division: a range end it moves by an ulp across a bin edge
            // adds or drops a bin the hexagon barely touches (value ~ 0)
            const float u = __fdividef(fmaf(V.h0, xs[k], fmaf(V.h1, ys[k], V.h2)), fmaf(V.h3, xs[k], fmaf(V.h4, ys[k], V.h5)));
            umin = fminf(umin, u);
            umax = fmaxf(umax, u);
        }
        lo = min(max(0, (int)floorf(umin)), nu - 1);
        hi = min(max(0, (int)floorf(umax)), nu - 1);
    }
    __device__ static void setup(const View& V, int ic, int il, const Fan2DParams& P, Cell& c) {
        c.oy = (il - V.nl2) * V.dy;
        c.ox = ((il & 1) ? (ic - V.nc3) : (ic - V.nc2)) * V.dx;
        if (M == kH0Corrected)
            true_bounds(V, c.ox, c.oy, P.nu, c.lo, c.hi);
        else
            pmi_bounds(V, ic, il, P.nu, c.lo, c.hi);
        const float fl = (float)c.lo;
        c.sx = V.dtvx + V.puvx * (fl - 0.5f * P.nu + 0.5f);
        c.sy = V.dtvy + V.puvy * (fl - 0.5f * P.nu + 0.5f);
    }
    // layers/A_Hl.cu:21-46 with spline_conv.hh:151-229: divided differences of
    // truncated powers y+^(m-1), m = number of kept directions
    __device__ static double tp(double y, int m) {
        if (!(y > 0)) return 0.0;
        return m == 2 ? y : (m == 3 ? y * y : y * y * y);
    }
    __device__ static double conv4(double y, double h1, double h2, double h3, double h4) {
        double hs[4];
        int m = 0;
        if (fabs(h1) > 1e-8) hs[m++] = h1;
        if (fabs(h2) > 1e-8) hs[m++] = h2;
        if (fabs(h3) > 1e-8) hs[m++] = h3;
        if (fabs(h4) > 1e-8) hs[m++] = h4;
        if (m < 2) return 0.0;
        // Delta_{h_{m-1}} ... Delta_{h_0} of tp, nested as the reference nests
        // forward_difference_mx_1 (outermost difference over the last kept h)
        double v[16];
        const int n = 1 << m;
        for (int s = 0; s < n; ++s) {
            double yy = y;
            for (int k = m - 1; k >= 0; --k)
                if (s & (1 << (m - 1 - k))) yy = yy - hs[k];
            v[s] = tp(yy, m);
        }
        for (int k = 0; k < m; ++k) {  // innermost difference first: h_0
            const int bit = 1 << (m - 1 - k);
            for (int s = 0; s < n; ++s)
                if (!(s & bit)) v[s] = (v[s] - v[s | bit]) / hs[k];
        }
        return m == 2 ? v[0] : (m == 3 ? v[0] / 2.0 : v[0] / 6.0);
    }
    // the reference's FP32 stepping of the bin centre
    __device__ static void skip(const View& V, Cell& c) {
        c.sx += V.puvx;
        c.sy += V.puvy;
    }
    __device__ static void start(const View&, Cell&, int) {}
    __device__ static float value(const View& V, Cell& c, int, BinRef t, const Fan2DParams&) {
        if (M == kH0Corrected) {
            // the exact bin geometry (this mode is held to the FP64 replica,
            // not to the reference's FP32 rounding): two affine maps in place
            // of the edge-ray intersections, divisions and square roots
            const float4 w0 = t[0], w1 = t[1];
            const float xa = __fmaf_rn(w1.x, c.ox, __fmaf_rn(w1.y, c.oy, w0.z));
            const float xb = __fmaf_rn(w1.z, c.ox, __fmaf_rn(w1.w, c.oy, w0.w));
            const float conv = box3_sum3_by_cum(xa, fabsf(xb - xa), w0.x, w0.y, -(w0.x + w0.y));
            return (conv == conv && conv > 0.f) ? conv : 0.f;
        }
        const float sx = c.sx, sy = c.sy;
        skip(V, c);
        const float px = V.srcx, py = V.srcy, ox = c.ox, oy = c.oy;
        const float ax = sx - V.puvx * 0.5f, ay = sy - V.puvy * 0.5f;
        const float bx = sx + V.puvx * 0.5f, by = sy + V.puvy * 0.5f;
        const float num = dot2f(ox - px, sx - px, oy - py, sy - py);
        const float dena = dot2f(ax - px, sx - px, ay - py, sy - py);
        const float denb = dot2f(bx - px, sx - px, by - py, sy - py);
        // fast divisions: within two ulps of the reference's, on positions
        // whose own FP32 rounding is larger
        const float ra = __fdividef(num, dena), rb = __fdividef(num, denb);
        const float ax1 = px + (ax - px) * ra, ay1 = py + (ay - py) * ra;
        const float bx1 = px + (bx - px) * rb, by1 = py + (by - py) * rb;
        if (M == kH0Reference && V.back) {  // layers/A_H0.cu:331-334
            const float da = hypotf(ax1 - ox, ay1 - oy), db = hypotf(bx1 - ox, by1 - oy);
            if (da > V.dt && db > V.dt && (ax1 - ox) * (bx1 - ox) >= 0.0f && (ay1 - oy) * (by1 - oy) >= 0.0f)
                return 0.f;
        }
        // the edge rays' separation and the site's offset: the reference takes
        // FP64 square roots of these FP32 differences and gives the offset
        // the sign of the site's side of edge ray a.  Both vectors lie along
        // the central ray's counter-clockwise normal n = (-(sy - py), sx -
        // px) / |s - p|, and since edge ray a turns the same way as the
        // central ray (cross(a - p, n) > 0) the offset's projection on n
        // carries exactly that sign: the projections are the same lengths
        // to a few ulp, far below the FP32 geometry's own rounding
        const float dbx = bx1 - ax1, dby = by1 - ay1, dax = ax1 - ox, day = ay1 - oy;
        const float cx = sx - px, cy = sy - py, rn = rsqrtf(fmaf(cx, cx, cy * cy));
        const float fblur = -fabsf(dot2f(dby, cx, -dbx, cy)) * rn;
        const float fy = dot2f(day, cx, -dax, cy) * rn;
        const float4 w = t[0];
        const float va = w.x, vb = w.y, vc = w.z;
        if (M == kHl) {
            // all four directions kept (every bin but those whose ray makes a
            // lattice direction vanish): the blur direction integrated in
            // closed form, FP32; otherwise the reference's FP64 divided
            // differences with the vanishing directions dropped
            if (fabsf(fblur) > 1e-8f && fabsf(va) > 1e-8f && fabsf(vb) > 1e-8f && fabsf(vc) > 1e-8f) {
                const float4 k = t[1];
                const float conv = box4_hex_by_cum(fy, -fblur, k.x, k.y, k.z, k.w, w.w);
                return (conv == conv && conv > 0.f) ? conv : 0.f;
            }
            const double conv = conv4((double)fy, (double)fblur, (double)va, (double)vb, (double)vc);
            return (conv == conv && conv > 0.0) ? (float)conv : 0.f;
        }
        // the three splines as differences of their pairs' trapezoid CDFs
        // over the blur width (box3_sum3_by_cum; within 1e-6 of the three
        // closed forms at values up to 3/dt)
        const float conv = box3_sum3_by_cum(fy, -fblur, va, vb, vc);
        return (conv == conv && conv > 0.f) ? conv : 0.f;
    }
};

namespace {

const double kSqrt3 = 1.7320508075688772935274463415;
const double kPi = 3.14159265358979323846;

class HexLayer final : public Proj2D {
public:
    // nl rows, nc sites per row (the reference's h0_init/hl_init argument order)
    HexLayer(int mode, int nl, int nc, int np, int nu, double dt, double du, double lsd, double lso,
             const double* angles, const double* dz, const double* drho)
        : mode_(mode) {
        if (nl <= 0 || nc <= 1) fail("invalid hexagonal lattice nl=%d nc=%d", nl, nc);
        check_pitches({dt});
        // GeoData(nc, nl, 1, nu, 1, np, dt*sqrt3, dt*0.5, 1, du, 1), A_H0.cu:556 / A_Hl.cu:570
        geo.init(nc, nl, np, nu, dt * kSqrt3, dt * 0.5f, du, lsd, lso, angles, dz, drho);
        P.ni = nc;
        P.nj = nl;
        const float fdt = (float)(dt * 0.5f) * 2.0f;  // d3xyz.y * 2.0f (A_H0.cu:171)
        const float fdx = fdt * (float)kSqrt3;
        const float fdy = fdt * (mode == kHl ? 0.5f : 1.5f);
        constexpr int kVF = HexBasis<kHl>::kViewFloats;
        std::vector<float> view((size_t)np * kVF, 0.f);
        const int nw = mode == kH0Corrected ? HexBasis<kH0Corrected>::kBinF4
                       : mode == kHl        ? HexBasis<kHl>::kBinF4
                                            : HexBasis<kH0Reference>::kBinF4;
        std::vector<float4> bins((size_t)np * nu * nw);
        std::vector<BinHomography> hom;
        bin_homographies(geo, hom);
        for (int p = 0; p < np; ++p) {
            const ViewFrame& f = geo.frames[p];
            float* v = &view[(size_t)p * kVF];
            const float* m = &geo.pmi[12 * (size_t)p];
            v[0] = m[0]; v[1] = m[1]; v[2] = m[3]; v[3] = m[8]; v[4] = m[9]; v[5] = m[11];
            v[6] = (float)f.puv[0]; v[7] = (float)f.puv[1];
            v[8] = (float)f.src[0]; v[9] = (float)f.src[1];
            v[10] = (float)f.dtv[0]; v[11] = (float)f.dtv[1];
            v[12] = fdt; v[13] = fdx; v[14] = fdy;
            v[15] = 0.5f * (nl - 1); v[16] = 0.5f * (nc - 1); v[17] = 0.5f * (nc - 2);
            // world homography from the index one: x = x0 + i dx  =>  i = (x - x0)/dx
            const BinHomography& H = hom[p];
            const double ix = 1.0 / geo.dx, iy = 1.0 / geo.dy, x0 = geo.x0(), y0 = geo.y0();
            v[18] = (float)(H.n0 * ix); v[19] = (float)(H.n1 * iy); v[20] = (float)(H.n2 - H.n0 * x0 * ix - H.n1 * y0 * iy);
            v[21] = (float)(H.d0 * ix); v[22] = (float)(H.d1 * iy); v[23] = (float)(H.d2 - H.d0 * x0 * ix - H.d1 * y0 * iy);
            v[24] = (float)mode;
            v[25] = 0.f;
            // va, vb, vc per bin from the bin's ray direction as the reference
            // computes it (FP32 atan2 of the FP32 bin centre, FP64 sines)
            const float px = (float)f.src[0], py = (float)f.src[1];
            for (int u = 0; u < nu; ++u) {
                const float sx = (float)f.dtv[0] + (float)f.puv[0] * (u - 0.5f * nu + 0.5f);
                const float sy = (float)f.dtv[1] + (float)f.puv[1] * (u - 0.5f * nu + 0.5f);
                const float th = std::atan2(sx - px, sy - py);
                double o[3];
                o[0] = (double)fdt * std::sin((double)th);
                o[1] = (double)fdt * std::sin((double)th + 2.0 * kPi / 3.0);
                o[2] = (double)fdt * std::sin((double)th + 4.0 * kPi / 3.0);
                float4* w = &bins[(size_t)p * nw * nu + u];  // planes of nu words
                w[0] = make_float4((float)o[0], (float)o[1], (float)o[2], 0.f);
                if (mode == kHl) {
                    // the 3-direction spline's constants (FP64): magnitudes
                    // x0 >= x1 >= x2 with x0 = x1 + x2 (the directions sum to 0)
                    double a[3] = {std::fabs(o[0]), std::fabs(o[1]), std::fabs(o[2])};
                    std::sort(a, a + 3);
                    const double x1 = a[1], x2 = a[0], x0 = x1 + x2;
                    const double rp6 = 1.0 / (6.0 * x0 * x1 * x2);
                    w[0].w = (float)(0.5 - rp6 * x2 * x2 * x2);
                    w[nu] = make_float4((float)x1, (float)x2, (float)(1.0 / x0), (float)rp6);
                }
                if (mode == kH0Corrected) {
                    // exact edge-ray maps of bin u (FP64): central direction
                    // c = s - S, n its counter-clockwise normal; the edge ray
                    // S + t d_e meets the line O + r n at r = (O - S) . (k_e c -
                    // n), k_e = (d_e . n) / (d_e . c) (the reference's offset
                    // and sign convention, layers/A_H0.cu:215-241)
                    const double Sx = f.src[0], Sy = f.src[1];
                    const double t0 = u - 0.5 * nu + 0.5;
                    const double cx0 = f.dtv[0] + f.puv[0] * t0, cy0 = f.dtv[1] + f.puv[1] * t0;
                    const double cx = cx0 - Sx, cy = cy0 - Sy, cl = std::hypot(cx, cy);
                    const double nx_ = -cy / cl, ny_ = cx / cl;
                    double al[2][2], be[2];
                    for (int e = 0; e < 2; ++e) {
                        const double sgn = e == 0 ? -0.5 : 0.5;
                        const double dx_ = cx + sgn * f.puv[0], dy_ = cy + sgn * f.puv[1];
                        const double k = (dx_ * nx_ + dy_ * ny_) / (dx_ * cx + dy_ * cy);
                        al[e][0] = k * cx - nx_;
                        al[e][1] = k * cy - ny_;
                        be[e] = -(al[e][0] * Sx + al[e][1] * Sy);
                    }
                    w[0] = make_float4((float)o[0], (float)o[1], (float)be[0], (float)be[1]);
                    w[nu] = make_float4((float)al[0][0], (float)al[0][1], (float)al[1][0], (float)al[1][1]);
                }
            }
        }
        back_view_ = view;
        for (int p = 0; p < np; ++p) back_view_[(size_t)p * kVF + 25] = 1.f;
        dt_ = dt;
        finish_init(view, bins);
        SGD_CUDA(cudaMalloc(&d_back_view_, back_view_.size() * sizeof(float)));
        SGD_CUDA(cudaMemcpy(d_back_view_, back_view_.data(), back_view_.size() * sizeof(float),
                            cudaMemcpyHostToDevice));
        out_scale = fdx * fdy;  // area factor (double)dx * (double)dy of the reference
        // the reference's H0 counts footprint evaluations three per bin; Hl never counts
        count = (mode == kHl) ? 0 : 3 * dispatch([&](auto b) { return fan2d_count<decltype(b)>(P, stream); });
    }
    ~HexLayer() override { cudaFree(d_back_view_); }
    void forward_dev(const float* img, float* sino, cudaStream_t s) override {
        dispatch([&](auto b) { fan2d_forward<decltype(b)>(P, img, sino, out_scale, s); return 0ull; });
    }
    long long csr(const CsrOut& out) override {
        return (long long)dispatch([&](auto b) { return (unsigned long long)fan2d_csr<decltype(b)>(P, out_scale, out, stream); });
    }
    void backward_dev(const float* sino, float* img, cudaStream_t s) override {
        Fan2DParams Q = P;
        Q.view = d_back_view_;
        dispatch([&](auto b) { fan2d_back<decltype(b)>(Q, sino, img, out_scale, s); return 0ull; });
    }

protected:
    // f(HexBasis<mode>()) for the layer's mode
    template <class F>
    unsigned long long dispatch(F&& f) const {
        if (mode_ == kH0Corrected) return f(HexBasis<kH0Corrected>());
        if (mode_ == kH0Reference) return f(HexBasis<kH0Reference>());
        return f(HexBasis<kHl>());
    }
    // The sites' true footprints: the hexagon (H0, rows at 1.5 dt: vertices
    // within 1/2 + 1/2 site, odd-row shift and vertex, and dt = 2/3 row) or
    // the linear element (Hl, rows at 0.5 dt: within one site and 2 rows).
    // The reference-compatible H0 takes its bin ranges from vertices on the
    // 0.5 dt rows of pmi instead; bins outside the true footprint hold 0, so
    // planning by the true one keeps every non-zero pair of those ranges.
    RangeMap range_map(int p) const override {
        double hw[6];
        fan_world_hom(geo, p, hw);
        if (mode_ == kHl) return grid_range_map(hw, geo.x0(), geo.dx, geo.y0(), geo.dy, 1.0, 2.0);
        return grid_range_map(hw, geo.x0(), geo.dx, -0.5 * (P.nj - 1) * 1.5 * dt_, 1.5 * dt_, 1.0, 1.0);
    }

private:
    int mode_;
    double dt_ = 0;
    std::vector<float> back_view_;
    float* d_back_view_ = nullptr;
};

}  // namespace

Proj2D* make_hex_layer(int mode, int nl, int nc, int np, int nu, double dt, double du, double lsd, double lso,
                       const double* angles, const double* dz, const double* drho) {
    return new HexLayer(mode, nl, nc, np, nu, dt, du, lsd, lso, angles, dz, drho);
}

}  // namespace sgd
