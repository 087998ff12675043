// FP64 host geometry for the 2D fan-beam projectors and the per-(view, bin)
// tables the B1 kernels read.
//
// World frame (utils/geo.cu:232-269 of the reference): at angle beta = 0 the
// source sits at (-lso + drho, 0), the detector centre at (lsd - lso, 0) and the
// detector u-axis is (0, du); everything is rotated by beta about the origin.
// Pixel (i, j) has centre ((i - (nx-1)/2) dx, (j - (ny-1)/2) dy); bin u has
// centre D + e (u - nu/2 + 1/2) (layers/A_B1.cu:96-98, :153).
#pragma once

#include <initializer_list>
#include <vector>

namespace sgd {

// Argument checks every layer runs before its first CUDA call, so that no
// NaN or infinity reaches the geometry tables (where it would turn into bin
// ranges): pitches positive and finite; 0 < lso < lsd, finite; angles present
// and, with the optional per-view offsets dz and drho, finite.  Each throws
// through fail() (the C entry points turn that into NULL / -1 and
// sgd_last_error()).
void check_pitches(std::initializer_list<double> pitches);
void check_distances(double lsd, double lso);
void check_views(int np, const double* angles, const double* dz, const double* drho);

// One view of a circular (fan or cone) geometry in 3D: source, detector
// centre, detector u step and v step (utils/geo.cu:232-269).
struct ViewFrame {
    double src[3], dtv[3], puv[3], pvv[3];
};

// geo_init_angles of utils/geo.cu:232-269: per-view rotation by beta (snapped
// to an exact odd multiple of 45 degrees within 1e-7, the test in long
// double), source offsets dz (along z) and drho (along the source axis).
std::vector<ViewFrame> view_frames(int np, double lsd, double lso, double du, double dv, const double* angles,
                                   const double* dz, const double* drho);

// The reference's 3x4 projection matrix of a view and its index-space FP32
// form (utils/geo.cu:58-161): pmi maps voxel indices (i, j, k, 1) to
// homogeneous detector coordinates (u w, v w, w), with uc = nu/2, vc = nv/2.
// The arithmetic is done in the same order as the reference so that pmi is
// bit-identical (the visited-bin ranges of the separable-footprint and 3D
// kernels are floors of pmi projections).
void reference_pmi(const ViewFrame& f, double uc, double vc, int nx, int ny, int nz, double dx, double dy,
                   double dz, double pm[12], float pmi[12]);

// The same index-space map built directly from the ray geometry in FP64 (the
// detector plane through dtv spanned by puv and pvv, uc = nu/2, vc = nv/2).
// It equals reference_pmi up to rounding except on the views where the
// reference's detector-alignment matrix is singular (puv.x == puv.y, the
// snapped 3pi/4 and -pi/4 views), where reference_pmi degenerates
// (utils/geo.cu:36-41 returns the identity) and this one does not.
void exact_pmi(const ViewFrame& f, double uc, double vc, int nx, int ny, int nz, double dx, double dy, double dz,
               float pmi[12]);

struct FanGeometry {
    int nx = 0, ny = 0, np = 0, nu = 0;
    double dx = 1, dy = 1, du = 1, lsd = 0, lso = 0;
    std::vector<double> beta;            // per-view angle after the 45-degree snap
    std::vector<double> src, dtv, puv;   // per view, (x, y)
    std::vector<ViewFrame> frames;       // per view, 3D (2D layers: nz = nv = 1, dz = dv = 1)
    std::vector<float> pmi;              // per view, 12 floats (reference_pmi)

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
// B1 (bilinear box-spline) footprint records.
//
// For bin u of view p and pixel (i, j) the reference footprint
// (layers/A_B1.cu:182-197) is
//     conv = (G(xb) - G(xa)) / (xb - xa)
// where xa, xb are the signed lateral offsets, on the line through the pixel
// centre perpendicular to the bin's central ray, of the bin's two edge rays, and
// G is the odd extension of the cumulative profile S of the convolution of two
// unit-area triangles of half-widths a = max(vx, vy), b = min(vx, vy)
// (conv_2tri_1box_* of layers/spline_conv.hh:295-390).  The records measure
// offsets in units of a: y = x / a, beta = b / a <= 1, and then
//     conv = (G(yb) - G(ya)) / (yb - ya) / a
// with, for y >= 0, w = (beta - y)+, p = (1 + beta - y)+, q = (1 - y)+:
//     S(y) = y - y^2/2 - beta^2/12 + w^4/(12 beta^2)          for 1 - y >= beta
//     S(y) = 1/2 + (q^4 + w^4 - p^4/2)/(12 beta^2)            otherwise
// (the first piece is the second plus (1 - beta - y)^4/(24 beta^2), which
// cancels badly as beta -> 0; every power in the pieces used is of a distance
// to a nearby knot, so FP32 keeps its accuracy).  b <= 1e-7 uses the
// single-triangle limit as the reference does (layers/A_B1.cu:52-55).  In
// units of a the polynomial's own coefficients are the constants 1 and -1/2,
// so a record needs four profile constants, each stored twice.  One 64-byte
// record per (view, bin), stored as four float4 chunks in the layout
// [view][chunk][bin] so that consecutive bins of one chunk are consecutive
// 16-byte words (shared-memory bank groups).  Every field pair is an operand
// pair of the packed-FP32 form of the footprint (b1_kernels.cuh), so a
// kernel builds none:
//   [0] [1]  i coefficients of ya, yb        ya = i*r[0] + (j*r[2] + r[4])
//   [2] [3]  j coefficients of ya, yb        yb = i*r[1] + (j*r[3] + r[5])
//   [4] [5]  constant terms of ya, yb
//   [6] [7]  beta, beta          [8] [9]  1+beta, 1+beta
//   [10] [11]  -beta^2/12 (twice)    [12] [13]  1/(12 beta^2) (twice; 0 for beta = 0)
//   [14] 1/a     [15] a (mm)
// ---------------------------------------------------------------------------
constexpr int kB1Rec = 16;

// Strip parameters for the detector-driven forward kernel: along the major
// axis index m, the two edge rays cross the minor axis at
//     alpha_a + beta_a m  and  alpha_b + beta_b m   (minor index units);
// [4] = 1 when the major axis is y (rows), 0 when it is x (columns).
constexpr int kStripRec = 8;

// Fills r[6..15] for profile half-widths a >= b in the original units (the
// layout of the reference-rounding mode's tables: b, b, a, a, a+b, a+b, 1/a,
// 1/(2a^2), -b^2/(12a^2), 1/(12a^2b^2)).
void b1_profile_constants(double a, double b, float* r);

// Fills r[6..15] of a B1 record (offsets in units of a, above) for profile
// half-widths a >= b.
void b1_unit_profile_constants(double a, double b, float* r);

void b1_tables(const FanGeometry& g, std::vector<float>& rec, std::vector<float>& strip);

}  // namespace sgd
