// FP64 host geometry for the 2D fan-beam projectors and the per-(view, bin)
// tables the B1 kernels read.
//
// World frame (utils/geo.cu:232-269 of the reference): at angle beta = 0 the
// source sits at (-lso + drho, 0), the detector centre at (lsd - lso, 0) and the
// detector u-axis is (0, du); everything is rotated by beta about the origin.
// Pixel (i, j) has centre ((i - (nx-1)/2) dx, (j - (ny-1)/2) dy); bin u has
// centre D + e (u - nu/2 + 1/2) (layers/A_B1.cu:96-98, :153).
#pragma once

#include <vector>

namespace sgd {

struct FanGeometry {
    int nx = 0, ny = 0, np = 0, nu = 0;
    double dx = 1, dy = 1, du = 1, lsd = 0, lso = 0;
    std::vector<double> beta;            // per-view angle after the 45-degree snap
    std::vector<double> src, dtv, puv;   // per view, (x, y)

    // geo_init_angles of utils/geo.cu:232-269, including its snapping of
    // angles within 1e-7 of an odd multiple of 45 degrees.
    void init(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
              const double* angles, const double* dz, const double* drho);

    double x0() const { return -0.5 * (nx - 1) * dx; }
    double y0() const { return -0.5 * (ny - 1) * dy; }
};

// Per-view map from pixel-index coordinates (i, j) to the continuous bin
// coordinate u (floor(u) = bin index):
//   u = (n0 i + n1 j + n2) / (d0 i + d1 j + d2)
struct BinHomography {
    float n0, n1, n2, d0, d1, d2, pad0, pad1;
};
void bin_homographies(const FanGeometry& g, std::vector<BinHomography>& out);

// ---------------------------------------------------------------------------
// B1 (bilinear box-spline) footprint tables.
//
// For bin u of view p and pixel (i, j) the reference footprint
// (layers/A_B1.cu:182-197) is
//     conv = (G(xb) - G(xa)) / (xb - xa)
// where xa, xb are the signed lateral offsets, on the line through the pixel
// centre perpendicular to the bin's central ray, of the bin's two edge rays, and
// G is the odd extension of the cumulative profile S of the convolution of two
// unit-area triangles of half-widths a = max(vx, vy), b = min(vx, vy)
// (conv_2tri_1box_* of layers/spline_conv.hh:295-390).  xa, xb are affine in
// (i, j); S is a quartic on each of five intervals of |x|.  The table stores,
// per (view, bin):
//   [0..2]  xa = i*c[0] + j*c[1] + c[2]
//   [3..5]  xb = i*c[3] + j*c[4] + c[5]
//   [6..9]  the four interval ends k1 <= k2 <= k3 <= k4 of |x|
//   [10 + 6r .. 15 + 6r], r = 0..4: interval start kr and the Taylor
//           coefficients s0..s4 of S(kr + h) in h.
// ---------------------------------------------------------------------------
constexpr int kB1Rec = 40;

// Strip parameters for the detector-driven forward kernel: along the major
// axis index m, the two edge rays cross the minor axis at
//     alpha_a + beta_a m  and  alpha_b + beta_b m   (minor index units);
// [4] = 1 when the major axis is y (rows), 0 when it is x (columns).
constexpr int kStripRec = 8;

// S(kr + h) tables for profile half-widths a >= b (b <= 1e-7 selects the
// single-triangle limit, layers/A_B1.cu:52-55).  out[0..3] = k1..k4,
// out[4 + 6r + c] = (kr, s0, s1, s2, s3, s4).
void b1_profile_table(double a, double b, double* out);

void b1_tables(const FanGeometry& g, std::vector<float>& rec, std::vector<float>& strip);

}  // namespace sgd
