// ORACLE — test infrastructure only, never part of the product path.
//
// A CPU restatement of the hqpwca/SGD CT projector layer, used by the tests, by
// `__graft_entry__.smoke()` and by the CPU-baseline leg of `bench.py` as the
// checker for the CUDA kernels in `sgd_b200/`.  Nothing in `sgd_b200/` links,
// loads or calls this file.
//
// Two kinds of function live here:
//   * formula replicas: the reference kernel's arithmetic restated on the CPU,
//     with the same visited-bin ranges, thresholds and normalisations.  They
//     are templated on the arithmetic type: `double` gives the FP64 replica,
//     `float` an FP32 emulation of the reference kernel (without its FMA
//     contraction) that shows how far the reference's own FP32 rounding sits
//     from the FP64 replica;
//   * geometry: `utils/geo.cu` restated (rotation, 45-degree snapping,
//     3x4 projection matrix and its index-space FP32 form `pmi`).
//
// Each function cites the reference file:line it follows.  The parity of this
// restatement with the reference itself is pinned by fixtures produced by the
// reference library built from source and run on a B200 (tests/golden/).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <algorithm>
#include <atomic>
#include <type_traits>
#include <functional>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double kPI = 3.14159265358979323846;  // utils/geo.hh:7

// ---------------------------------------------------------------------------
// geometry: utils/geo.cu
// ---------------------------------------------------------------------------

// utils/geo.cu:3-28 (row-major a[x*y] times b[y*z], result written to b)
void multm(const double* a, double* b, int x, int y, int z) {
    std::vector<double> c(x * z);
    for (int i = 0; i < x; i++)
        for (int j = 0; j < z; j++) {
            double s = 0.0;
            for (int k = 0; k < y; k++) s += a[i * y + k] * b[k * z + j];
            c[i * z + j] = s;
        }
    for (int i = 0; i < x * z; i++) b[i] = c[i];
}

// utils/geo.cu:30-56: inverse of a 3x3, identity when |det| < 1e-10
void invert3(double* m) {
    double n[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double det = m[0] * ((m[4] * m[8]) - (m[5] * m[7])) - m[1] * ((m[3] * m[8]) - (m[5] * m[6])) +
                 m[2] * ((m[3] * m[7]) - (m[4] * m[6]));
    if (std::fabs(det) < 1e-10) {
        n[0] = 1, n[4] = 1, n[8] = 1;
    } else {
        n[0] = ((m[4] * m[8]) - (m[5] * m[7])) / det;
        n[1] = -1 * ((m[1] * m[8]) - (m[2] * m[7])) / det;
        n[2] = ((m[1] * m[5]) - (m[2] * m[4])) / det;
        n[3] = -1 * ((m[3] * m[8]) - (m[5] * m[6])) / det;
        n[4] = ((m[0] * m[8]) - (m[2] * m[6])) / det;
        n[5] = -1 * ((m[0] * m[5]) - (m[2] * m[3])) / det;
        n[6] = ((m[3] * m[7]) - (m[4] * m[6])) / det;
        n[7] = -1 * ((m[0] * m[7]) - (m[1] * m[6])) / det;
        n[8] = ((m[0] * m[4]) - (m[1] * m[3])) / det;
    }
    for (int i = 0; i < 9; i++) m[i] = n[i];
}

// utils/geo.cu:58-161
void projection_matrix(double* pm, float* pmi, const double* src, const double* dtv, const double* puv,
                       const double* pvv, double uc, double vc, int nx, int ny, int nz, double ddx,
                       double ddy, double ddz) {
    double norm[3], vec[3];
    norm[0] = puv[1] * pvv[2] - puv[2] * pvv[1];
    norm[1] = puv[2] * pvv[0] - puv[0] * pvv[2];
    norm[2] = puv[0] * pvv[1] - puv[1] * pvv[0];
    double k = 0.0;
    for (int i = 0; i < 3; i++) k += norm[i] * (dtv[i] - src[i]);
    for (int i = 0; i < 3; i++) vec[i] = src[i] - dtv[i] + (uc * puv[i]) + (vc * pvv[i]) + 1;
    double pm4[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    double trans[16] = {1, 0, 0, -src[0], 0, 1, 0, -src[1], 0, 0, 1, -src[2], 0, 0, 0, 1};
    multm(trans, pm4, 4, 4, 4);
    double divdot[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, norm[0], norm[1], norm[2], 0};
    multm(divdot, pm4, 4, 4, 4);
    double scale[16] = {k, 0, 0, 0, 0, k, 0, 0, 0, 0, k, 0, 0, 0, 0, 1};
    multm(scale, pm4, 4, 4, 4);
    double trans2[12] = {1, 0, 0, vec[0], 0, 1, 0, vec[1], 0, 0, 1, vec[2]};
    multm(trans2, pm4, 3, 4, 4);
    double align[9] = {puv[0], pvv[0], 1, puv[1], pvv[1], 1, puv[2], pvv[2], 1};
    invert3(align);
    multm(align, pm4, 3, 3, 4);
    for (int i = 0; i < 12; i++) pm[i] = pm4[i] / pm4[11];
    // geo.cu:141-160: the index-space form is computed in FP32
    float dx = (float)ddx, dy = (float)ddy, dz = (float)ddz;
    float ox = (nx - 1) * dx / 2.0f, oy = (ny - 1) * dy / 2.0f, oz = (nz - 1) * dz / 2.0f;
    pmi[0] = dx * pm[0]; pmi[1] = dy * pm[1]; pmi[2] = dz * pm[2];
    pmi[3] = pm[3] - ox * pm[0] - oy * pm[1] - oz * pm[2];
    pmi[4] = dx * pm[4]; pmi[5] = dy * pm[5]; pmi[6] = dz * pm[6];
    pmi[7] = pm[7] - ox * pm[4] - oy * pm[5] - oz * pm[6];
    pmi[8] = dx * pm[8]; pmi[9] = dy * pm[9]; pmi[10] = dz * pm[10];
    pmi[11] = pm[11] - ox * pm[8] - oy * pm[9] - oz * pm[10];
}

void rotate(const double* vec, double* res, double angle) {  // utils/geo.cu:203-207
    res[0] = vec[0] * std::cos(angle) - vec[1] * std::sin(angle);
    res[1] = vec[0] * std::sin(angle) + vec[1] * std::cos(angle);
    res[2] = vec[2];
}

struct Geo {
    int nx, ny, nz, nu, nv, np;
    double dx, dy, dz, du, dv;
    std::vector<double> src, dtv, puv, pvv, pm;
    std::vector<float> pmi;
};

// utils/geo.cu:232-269 (mode 0, per-view angles with 45-degree snapping) and
// utils/geo.cu:209-230 (mode 1, uniform angles without snapping), followed by
// utils/geo.cu:188-201 (projection matrices).
void build_geo(Geo& g, double lsd, double lso, const double* angles, const double* dzs,
               const double* drho) {
    int np = g.np;
    g.src.assign(3 * np, 0.0); g.dtv.assign(3 * np, 0.0);
    g.puv.assign(3 * np, 0.0); g.pvv.assign(3 * np, 0.0);
    g.pm.assign(12 * np, 0.0); g.pmi.assign(12 * np, 0.0f);
    double src0[3] = {-lso, 0.0, 0.0};
    double dtv0[3] = {lsd - lso, 0.0, 0.0};
    double puv0[3] = {0.0, g.du, 0.0};
    double pvv0[3] = {0.0, 0.0, g.dv};
    for (int i = 0; i < np; ++i) {
        long double beta = angles[i];
        double s[3] = {src0[0], src0[1], 0.0};
        if (dzs) s[2] = dzs[i];
        if (drho) s[0] = src0[0] + drho[i];
        if (std::fabs(std::sin(beta) - std::cos(beta)) < 1e-7L)
            beta = (std::sin(beta) > 0) ? kPI / 4 : -kPI * 3 / 4;
        else if (std::fabs(std::sin(beta) + std::cos(beta)) < 1e-7L)
            beta = (std::sin(beta) > 0) ? kPI * 3 / 4 : -kPI / 4;
        double b = (double)beta;
        rotate(s, &g.src[3 * i], b);
        rotate(dtv0, &g.dtv[3 * i], b);
        rotate(puv0, &g.puv[3 * i], b);
        rotate(pvv0, &g.pvv[3 * i], b);
    }
    for (int p = 0; p < np; ++p)
        projection_matrix(&g.pm[12 * p], &g.pmi[12 * p], &g.src[3 * p], &g.dtv[3 * p], &g.puv[3 * p],
                          &g.pvv[3 * p], g.nu / 2.0, g.nv / 2.0, g.nx, g.ny, g.nz, g.dx, g.dy, g.dz);
}

// ---------------------------------------------------------------------------
// box-spline closed forms: layers/spline_conv.hh
// ---------------------------------------------------------------------------

// FLOP-counting scalar: every +, -, *, /, sqrt on it adds one to the counter
// (comparisons, abs, min/max are not counted).  Used once to freeze the
// algorithmic work of the reference formulas for the roofline.
struct CountedF {
    double v;
    static thread_local long long flops;
    CountedF(double x = 0.0) : v(x) {}
    explicit operator double() const { return v; }
};
thread_local long long CountedF::flops = 0;
inline CountedF operator+(CountedF a, CountedF b) { ++CountedF::flops; return a.v + b.v; }
inline CountedF operator-(CountedF a, CountedF b) { ++CountedF::flops; return a.v - b.v; }
inline CountedF operator*(CountedF a, CountedF b) { ++CountedF::flops; return a.v * b.v; }
inline CountedF operator/(CountedF a, CountedF b) { ++CountedF::flops; return a.v / b.v; }
inline CountedF operator-(CountedF a) { return -a.v; }
inline CountedF& operator+=(CountedF& a, CountedF b) { ++CountedF::flops; a.v += b.v; return a; }
inline bool operator<(CountedF a, CountedF b) { return a.v < b.v; }
inline bool operator>(CountedF a, CountedF b) { return a.v > b.v; }
inline bool operator<=(CountedF a, CountedF b) { return a.v <= b.v; }
inline bool operator>=(CountedF a, CountedF b) { return a.v >= b.v; }
inline bool operator==(CountedF a, CountedF b) { return a.v == b.v; }
inline CountedF sqrt(CountedF a) { ++CountedF::flops; return std::sqrt(a.v); }
inline CountedF fabs(CountedF a) { return std::fabs(a.v); }
inline CountedF floor(CountedF a) { return std::floor(a.v); }
inline CountedF max(CountedF a, CountedF b) { return a.v > b.v ? a : b; }
inline CountedF min(CountedF a, CountedF b) { return a.v < b.v ? a : b; }
using std::sqrt;
using std::fabs;
using std::floor;
using std::max;
using std::min;

template <class T> inline void sort2(T& a, T& b) { if (a > b) std::swap(a, b); }  // :6-14
template <class T> inline void sort4(T* u) {  // :25-39
    sort2(u[0], u[1]); sort2(u[2], u[3]); sort2(u[0], u[2]); sort2(u[1], u[3]); sort2(u[1], u[2]);
}

// layers/spline_conv.hh:295-332 (b <= a - b)
template <class T> T conv_2tri_1box_ag2b(T a, T b, T x) {
    T a3 = a * a * a, ab2 = a * b * b, b3 = b * b * b;
    T k1 = (6 * a * a * b * b);
    T sum = 0;
    if (x <= b) return (x * (12 * ab2 - 4 * b3 - 4 * b * x * x + x * x * x)) / (2 * k1);
    sum += ((12 * a - 7 * b) * b) / (12 * a * a);
    if (x <= a - b) return sum + (-2 * a * b + b * b + 2 * a * x - x * x) / (2 * a * a);
    sum += T(0.5) - b / a;
    if (x <= a)
        return sum + ((a - b - x) * (a3 - 13 * b3 + 9 * b * b * x - 3 * b * x * x - x * x * x -
                                     3 * a * a * (b + x) - 3 * a * (b - x) * (3 * b + x))) / (4 * k1);
    sum += (13 * b * b) / (24 * a * a);
    if (x < a + b)
        return sum + ((x - a) * (a + 2 * b - x) * (a * a + 2 * a * b + 2 * b * b - 2 * (a + b) * x + x * x)) /
                         (4 * k1);
    return sum + b * b / (24 * a * a);
}

// layers/spline_conv.hh:334-370 (b > a - b)
template <class T> T conv_2tri_1box_al2b(T a, T b, T x) {
    T a3 = a * a * a, a2b = a * a * b, ab2 = a * b * b, b3 = b * b * b;
    T k1 = (6 * a * a * b * b), k2 = a - b;
    T sum = 0;
    if (x <= a - b) return (x * (12 * ab2 - 4 * b3 - 4 * b * x * x + x * x * x)) / (2 * k1);
    sum += ((a - b) * (a3 - 7 * a2b + 23 * ab2 - 9 * b3)) / (2 * k1);
    if (x <= b)
        return sum + (((x - a + b) * (a3 - 11 * a2b + 43 * ab2 - 17 * b3 + (5 * a - 13 * b) * k2 * x -
                                      (a + 7 * b) * x * x + 3 * x * x * x)) / (4 * k1));
    sum += (((2 * b - a) * (a3 - 6 * a2b + 24 * ab2 - 8 * b3)) / (4 * k1));
    if (x <= a)
        return sum + (((b - x) * (4 * a3 - 3 * b3 + b * b * x - 5 * b * x * x - x * x * x - 6 * a * a * (3 * b + x) +
                                  4 * a * (b * b + 4 * b * x + x * x))) / (4 * k1));
    sum += (((b - a) * (a3 - 7 * a2b + 5 * ab2 - 3 * b3)) / (4 * k1));
    if (x < a + b)
        return sum + ((x - a) * (a + 2 * b - x) * (a * a + 2 * a * b + 2 * b * b - 2 * (a + b) * x + x * x)) /
                         (4 * k1);
    return sum + b * b / (24 * a * a);
}

// layers/spline_conv.hh:372-390
template <class T> T fast_2tri_1box_spline(T a, T b, T x1, T x2) {
    bool side = (x1 * x2) > T(0);
    x1 = fabs(x1), x2 = fabs(x2);
    T s1, s2;
    if (b <= a - b) { s1 = conv_2tri_1box_ag2b(a, b, x1); s2 = conv_2tri_1box_ag2b(a, b, x2); }
    else { s1 = conv_2tri_1box_al2b(a, b, x1); s2 = conv_2tri_1box_al2b(a, b, x2); }
    return side ? fabs(s1 - s2) : (s1 + s2);
}

// layers/spline_conv.hh:393-405
template <class T> T fast_1tri_1box_spline(T a, T x1, T x2) {
    bool side = (x1 * x2) > T(0);
    x1 = fabs(x1), x2 = fabs(x2);
    T s1 = (x1 >= a) ? T(0.5) : (x1 / a - (x1 * x1) / (2 * a * a));
    T s2 = (x2 >= a) ? T(0.5) : (x2 / a - (x2 * x2) / (2 * a * a));
    return side ? fabs(s1 - s2) : (s1 + s2);
}

// layers/A_B1.cu:48-59
template <class T> T b1_linear_convolution_1d(T x1, T x2, T a, T b) {
    if (b > T(1e-7f)) return fast_2tri_1box_spline<T>(a, b, x1, x2) / fabs(x2 - x1);
    return fast_1tri_1box_spline<T>(a, x1, x2) / fabs(x2 - x1);
}

// ---------------------------------------------------------------------------
// visited bin range (every 2D kernel, e.g. layers/A_B1.cu:120-151): the corners
// (ix+-h, iy+-h) projected through pmi in FP32, sorted, floored and clamped.
// ---------------------------------------------------------------------------
template <class T = float>
inline void bin_range(const float* pm, float puvx, bool singular, float sx1, float sx2, float sy1, float sy2,
                      int nu, int& minu, int& maxu, float* us_out = nullptr) {
    T us[4];
    T xs[4] = {sx1, sx1, sx2, sx2};
    T ys[4] = {sy1, sy2, sy1, sy2};
    for (int k = 0; k < 4; ++k) {
        T num, den;
        if constexpr (std::is_same<T, float>::value) {
            // the reference's FP32 expression as its compiler contracts it
            // into fused multiply-adds: (pm0 x + pm3) + pm1 y
            num = (T)std::fmaf(pm[1], (float)ys[k], std::fmaf(pm[0], (float)xs[k], pm[3]));
            den = (T)std::fmaf(pm[9], (float)ys[k], std::fmaf(pm[8], (float)xs[k], pm[11]));
        } else {
            num = T(pm[0]) * xs[k] + T(pm[3]) + T(pm[1]) * ys[k];
            den = T(pm[8]) * xs[k] + T(pm[11]) + T(pm[9]) * ys[k];
        }
        us[k] = num / den;
        if (singular) us[k] = (us[k] * T(1.5f) - T(1.0f)) / T(puvx);
    }
    sort4(us);
    minu = std::min(std::max(0, (int)(double)floor(us[0])), nu - 1);
    maxu = std::min(std::max(0, (int)(double)floor(us[3])), nu - 1);
    if (us_out) for (int k = 0; k < 4; ++k) us_out[k] = (float)(double)us[k];
}

// ---------------------------------------------------------------------------
// B1 (bilinear) fan-beam projector: layers/A_B1.cu
// ---------------------------------------------------------------------------

// per-(view,bin) vx, vy in FP32: layers/A_B1.cu:429-478
void b1_vectors(const Geo& g, std::vector<float>& vecs) {
    int np = g.np, nu = g.nu;
    vecs.assign((size_t)2 * np * nu, 0.0f);
    for (int p = 0; p < np; ++p) {
        double cx = g.dtv[3 * p], cy = g.dtv[3 * p + 1];
        double ux = g.puv[3 * p], uy = g.puv[3 * p + 1];
        double px = g.src[3 * p], py = g.src[3 * p + 1];
        for (int u = 0; u < nu; ++u) {
            double sx = cx + ux * (u - 0.5 * nu + 0.5), sy = cy + uy * (u - 0.5 * nu + 0.5);
            double theta = std::atan2(std::fabs(px - sx), std::fabs(py - sy));
            vecs[(size_t)p * nu * 2 + u] = (float)std::fabs(g.dx * std::cos(theta));
            vecs[(size_t)p * nu * 2 + nu + u] = (float)std::fabs(g.dy * std::sin(theta));
        }
    }
}

// The per-(pixel,view) body shared by b1_forward_projection (layers/A_B1.cu:62-208)
// and b1_backward_projection (:211-353).  `visit(u, conv)` is called for every
// bin the reference keeps (conv > 1e-7, :203 and :347).  Returns the number of
// footprint evaluations (the reference's conv_count increments, :50).
template <class T, class Visit>
long long b1_pixel_view(const Geo& g, const float* vecs_p, int p, int ix, int iy, Visit visit) {
    int nx = g.nx, ny = g.ny, nu = g.nu;
    float dx = (float)g.dx, dy = (float)g.dy;
    const float* pm = &g.pmi[12 * p];
    float srcx = (float)g.src[3 * p], srcy = (float)g.src[3 * p + 1];
    float puvx = (float)g.puv[3 * p], puvy = (float)g.puv[3 * p + 1];
    float dtvx = (float)g.dtv[3 * p], dtvy = (float)g.dtv[3 * p + 1];
    bool singular = std::fabs(puvx - puvy) < 1e-7f;  // :103
    float fox = (ix - 0.5f * (nx - 1)) * dx;       // :96
    float foy = (iy - 0.5f * (ny - 1)) * dy;       // :98
    int minu, maxu;
    // :100-151 (the range always runs in FP32, except under op counting)
    if (std::is_same<T, CountedF>::value)
        bin_range<CountedF>(pm, puvx, singular, ix - 1.0f, ix + 1.0f, iy - 1.0f, iy + 1.0f, nu, minu, maxu);
    else
        bin_range<float>(pm, puvx, singular, ix - 1.0f, ix + 1.0f, iy - 1.0f, iy + 1.0f, nu, minu, maxu);
    T ox = fox, oy = foy, px = srcx, py = srcy;
    long long cnt = 0;
    for (int u = minu; u <= maxu; ++u) {
        T off = T(u) - T(0.5f) * nu + T(0.5f);
        T sx = T(dtvx) + T(puvx) * off, sy = T(dtvy) + T(puvy) * off;  // :153-154, :160
        T vx = vecs_p[u], vy = vecs_p[nu + u];                         // :163-164
        T ax = sx - T(puvx) * T(0.5f), ay = sy - T(puvy) * T(0.5f);   // :182-185
        T bx = sx + T(puvx) * T(0.5f), by = sy + T(puvy) * T(0.5f);
        T num = (ox - px) * (sx - px) + (oy - py) * (sy - py);
        T ra = num / ((ax - px) * (sx - px) + (ay - py) * (sy - py));  // :187-188
        T rb = num / ((bx - px) * (sx - px) + (by - py) * (sy - py));
        T ax1 = px + (ax - px) * ra, ay1 = py + (ay - py) * ra;      // :189-190
        T bx1 = px + (bx - px) * rb, by1 = py + (by - py) * rb;
        T x1 = sqrt((ax1 - ox) * (ax1 - ox) + (ay1 - oy) * (ay1 - oy));  // :192-193
        T x2 = sqrt((bx1 - ox) * (bx1 - ox) + (by1 - oy) * (by1 - oy));
        T sgn = ((ax1 - ox) * (bx1 - ox) + (ay1 - oy) * (by1 - oy) > T(0)) ? T(1) : T(-1);  // :195
        T conv = b1_linear_convolution_1d<T>(x1 * sgn, x2, max(vx, vy), min(vx, vy));  // :197
        ++cnt;
        if (conv == conv && conv > T(1e-7f)) visit(u, (double)conv);
    }
    return cnt;
}

template <class T>
long long b1_forward(const Geo& g, const std::vector<float>& vecs, const double* x, double* b) {
    int nx = g.nx, ny = g.ny, nu = g.nu, np = g.np;
    double dxy = (double)(float)g.dx * (double)(float)g.dy;
    std::memset(b, 0, sizeof(double) * (size_t)np * nu);
    long long total = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : total)
    for (int p = 0; p < np; ++p) {
        double* bp = b + (size_t)p * nu;
        const float* vp = &vecs[(size_t)p * nu * 2];
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                double C = x[(size_t)ix * ny + iy];  // host layout x[ix*ny+iy], A_B1.cu:621-623
                total += b1_pixel_view<T>(g, vp, p, ix, iy, [&](int u, double conv) { bp[u] += conv * C * dxy; });
            }
    }
    return total;
}

template <class T>
void b1_backward(const Geo& g, const std::vector<float>& vecs, const double* b, double* x) {
    int nx = g.nx, ny = g.ny, nu = g.nu, np = g.np;
    double dxy = (double)(float)g.dx * (double)(float)g.dy;
#pragma omp parallel for schedule(dynamic)
    for (int ix = 0; ix < nx; ++ix)
        for (int iy = 0; iy < ny; ++iy) {
            double acc = 0.0;
            for (int p = 0; p < np; ++p) {
                const double* bp = b + (size_t)p * nu;
                const float* vp = &vecs[(size_t)p * nu * 2];
                double val = 0.0;  // :304, one partial per view, :351
                b1_pixel_view<T>(g, vp, p, ix, iy, [&](int u, double conv) { val += conv * bp[u] * dxy; });
                acc += val;
            }
            x[(size_t)ix * ny + iy] = acc;
        }
}

// ---------------------------------------------------------------------------
// A_SF separable footprint (SF-TR) fan-beam projector: layers/A_SF.cu
// ---------------------------------------------------------------------------

// layers/A_SF.cu:48-84
template <class T> T sf_gamma(T s1, T s2, const T* us) {
    T g = 0, tmp, b1, b2;
    b1 = max(s1, us[0]); b2 = min(s2, us[1]);
    tmp = (b2 > b1) ? (T(1) / (T(2) * (us[1] - us[0]))) * ((b2 - us[0]) * (b2 - us[0]) - (b1 - us[0]) * (b1 - us[0])) : T(0);
    if (tmp == tmp) g += tmp;
    b1 = max(s1, us[1]); b2 = min(s2, us[2]);
    tmp = (b2 > b1) ? b2 - b1 : T(0);
    if (tmp == tmp) g += tmp;
    b1 = max(s1, us[2]); b2 = min(s2, us[3]);
    tmp = (b2 > b1) ? (T(1) / (T(2) * (us[3] - us[2]))) * ((b1 - us[3]) * (b1 - us[3]) - (b2 - us[3]) * (b2 - us[3])) : T(0);
    if (tmp == tmp) g += tmp;
    return g;
}

// Per-(pixel, view) body of SF_forward_projection (layers/A_SF.cu:87-225) and
// SF_backward_projection (:228-334): visit(u, weight*gamma) for kept bins.
// chord: the amplitude is the pixel's chord along the ray through its centre,
// min(dx/|sin|, dy/|cos|), instead of the reference's dx/max(|sin|, |cos|)
// (equal for square pixels).
template <class T, class Visit>
void sf_pixel_view(const Geo& g, int p, int ix, int iy, Visit visit, bool chord = false) {
    int nx = g.nx, ny = g.ny, nu = g.nu;
    float dx = (float)g.dx, dy = (float)g.dy;
    const float* pm = &g.pmi[12 * p];
    float srcx = (float)g.src[3 * p], srcy = (float)g.src[3 * p + 1];
    float puvx = (float)g.puv[3 * p], puvy = (float)g.puv[3 * p + 1];
    bool singular = std::fabs(puvx - puvy) < 1e-7f;            // :119
    float nx2 = (nx - 1) / 2.0f, ny2 = (ny - 1) / 2.0f;        // :101
    int minu, maxu;
    float usf[4];
    bin_range<float>(pm, puvx, singular, ix - 0.5f, ix + 0.5f, iy - 0.5f, iy + 0.5f, nu, minu, maxu, usf);  // :116-167
    T us[4] = {usf[0], usf[1], usf[2], usf[3]};
    T theta = std::atan2((double)(dx * (ix - nx2) - srcx), (double)(dy * (iy - ny2) - srcy));  // :174
    T st = std::fabs(std::sin((double)theta)), ct = std::fabs(std::cos((double)theta));
    T weight = chord ? min(T(dx) / st, T(dy) / ct) : T(dx) / max(st, ct);  // :177
    for (int u = minu; u <= maxu; ++u) {
        T gm = sf_gamma<T>(T(u), T(u) + T(1), us);              // :209
        T val = weight * gm;
        if (val == val && gm > T(1e-7f)) visit(u, (double)val);  // :214
    }
}

// ---------------------------------------------------------------------------
// B0 pixel-indicator fan-beam projector: layers/A_B0.cu
// ---------------------------------------------------------------------------

// layers/spline_conv.hh:52-58 (descending sort)
template <class T> inline void sort2d(T& a, T& b) { if (a < b) std::swap(a, b); }

// layers/spline_conv.hh:239-293: value of the 3-direction box spline at x for
// |directions| sorted in descending order
template <class T> T univariate3dir_fast3(T x, const T* xi) {
    T h = T(1) / xi[0];
    T p = xi[0] * xi[1] * xi[2];
    T K0 = (xi[0] - xi[1] - xi[2]) / T(2), K1 = (xi[0] - xi[1] + xi[2]) / T(2);
    T K2 = (xi[0] + xi[1] - xi[2]) / T(2), K3 = (xi[0] + xi[1] + xi[2]) / T(2);
    if (x >= K3) return T(0);
    if (x >= K2) return T(0.5f) * (K3 - x) * (K3 - x) / p;
    if (x >= K1) return ((xi[0] + xi[1]) / T(2) - x) * xi[2] / p;
    if (x < -K0) return h - (K0 * K0 + x * x) / p;
    if (x < K0) return h;
    return h - T(0.5f) * (K0 - x) * (K0 - x) / p;
}
template <class T> T univariate3dir_fast2(T x, const T* xi) {
    return max(T(0), min(T(1) / xi[0], ((xi[0] + xi[1]) / T(2) - x) / (xi[0] * xi[1])));
}

// layers/A_B0.cu:20-35
template <class T> T b0_linear_convolution_1d(T y, T v1, T v2, T v3) {
    T vs[3];
    y = fabs(y - (v1 + v2 + v3) / T(2));
    vs[0] = fabs(v1), vs[1] = fabs(v2), vs[2] = fabs(v3);
    sort2d(vs[1], vs[2]); sort2d(vs[0], vs[1]); sort2d(vs[1], vs[2]);
    if (vs[2] > T(1e-7f)) return univariate3dir_fast3<T>(y, vs);
    return univariate3dir_fast2<T>(y, vs);
}

// per-(view, bin) vx, vy, a0s, sb0, lsp in FP64: layers/A_B0.cu:338-388
void b0_vectors(const Geo& g, std::vector<double>& vecs) {
    int np = g.np, nu = g.nu;
    vecs.assign((size_t)5 * np * nu, 0.0);
    for (int p = 0; p < np; ++p) {
        double cx = g.dtv[3 * p], cy = g.dtv[3 * p + 1], ux = g.puv[3 * p], uy = g.puv[3 * p + 1];
        double px = g.src[3 * p], py = g.src[3 * p + 1];
        for (int u = 0; u < nu; ++u) {
            double sx = cx + ux * (u - 0.5 * nu + 0.5), sy = cy + uy * (u - 0.5 * nu + 0.5);
            double ax = sx - ux * 0.5, ay = sy - uy * 0.5, bx = sx + ux * 0.5, by = sy + uy * 0.5;
            double lsp = std::sqrt((px - sx) * (px - sx) + (py - sy) * (py - sy));
            double theta = std::atan2(std::fabs(px - sx), std::fabs(py - sy));
            double vx = std::fabs(g.dx * std::cos(theta)), vy = std::fabs(g.dy * std::sin(theta));
            if (py < sy) vx = -vx;
            if (px < sx) vy = -vy;
            double a0s = std::fabs((sx - px) * (ay - py) - (ax - px) * (sy - py)) / lsp;
            double sb0 = std::fabs((sx - px) * (by - py) - (bx - px) * (sy - py)) / lsp;
            a0s /= ((ax - px) * (sx - px) + (ay - py) * (sy - py)) / (lsp * lsp);
            sb0 /= ((bx - px) * (sx - px) + (by - py) * (sy - py)) / (lsp * lsp);
            double* v = &vecs[(size_t)p * nu * 5];
            v[u] = vx; v[nu + u] = vy; v[2 * nu + u] = a0s; v[3 * nu + u] = sb0; v[4 * nu + u] = lsp;
        }
    }
}

// Per-(pixel, view) body of b0_forward_projection (layers/A_B0.cu:123-229)
// and b0_backward_projection (:231-336).  visit(u, conv*dx*dy) for kept bins;
// returns the evaluation count (the reference's conv_count).
template <class T, class Visit>
long long b0_pixel_view(const Geo& g, const double* vp, int p, int ix, int iy, Visit visit) {
    int nx = g.nx, ny = g.ny, nu = g.nu;
    float dx = (float)g.dx, dy = (float)g.dy;
    float nx2 = 0.5f * (nx - 1), ny2 = 0.5f * (ny - 1);
    const float* pm = &g.pmi[12 * p];
    float srcx = (float)g.src[3 * p], srcy = (float)g.src[3 * p + 1];
    float puvx = (float)g.puv[3 * p], puvy = (float)g.puv[3 * p + 1];
    float dtvx = (float)g.dtv[3 * p], dtvy = (float)g.dtv[3 * p + 1];
    bool singular = std::fabs(puvx - puvy) < 1e-7f;
    float fox = (ix - nx2) * dx, foy = (iy - ny2) * dy;          // :152-153
    int minu, maxu;
    bin_range<float>(pm, puvx, singular, ix - 0.5f, ix + 0.5f, iy - 0.5f, iy + 0.5f, nu, minu, maxu);  // :158-195
    T ox = fox, oy = foy, px = srcx, py = srcy;
    T cx = ox - T(0.5f * dx), cy = oy + T(0.5f * dy);         // pixel corner, :213
    long long cnt = 0;
    for (int u = minu; u <= maxu; ++u) {
        T off = T(u) - T(0.5f) * nu + T(0.5f);
        T sx = T(dtvx) + T(puvx) * off, sy = T(dtvy) + T(puvy) * off;  // :197-198, :202
        T vx = vp[u], vy = vp[nu + u], a0s = vp[2 * nu + u], sb0 = vp[3 * nu + u], lsp = vp[4 * nu + u];
        T r1 = ((ox - px) * (sx - px) + (oy - py) * (sy - py)) / (lsp * lsp);  // :211
        T vblur = (a0s + sb0) * (-r1);
        T y = ((sx - px) * (cy - py) - (cx - px) * (sy - py)) / lsp;       // :213
        y = y + a0s * r1;
        T conv = b0_linear_convolution_1d<T>(-y, vx, vy, vblur);             // :219
        ++cnt;
        if (conv == conv && conv > T(1e-7f)) visit(u, (double)conv * (double)dx * (double)dy);  // :223-225
    }
    return cnt;
}

// ---------------------------------------------------------------------------
// Hexagonal lattices: H0 (layers/A_H0.cu) and Hl (layers/A_Hl.cu)
// ---------------------------------------------------------------------------
const double kSQRT3 = 1.7320508075688772935274463415;

// layers/A_Hl.cu:21-46 with layers/spline_conv.hh:151-229, on any scalar
// type (the FLOP counter runs it on CountedF)
template <class T> T hl_conv_t(T y, T h1, T h2, T h3, T h4) {
    T hs[4];
    int m = 0;
    if (std::fabs((double)h1) > 1e-8) hs[m++] = h1;
    if (std::fabs((double)h2) > 1e-8) hs[m++] = h2;
    if (std::fabs((double)h3) > 1e-8) hs[m++] = h3;
    if (std::fabs((double)h4) > 1e-8) hs[m++] = h4;
    if (m < 2) return T(0);
    std::function<T(T, int)> D = [&](T yy, int k) -> T {
        if (k < 0) return yy > T(0) ? (m == 2 ? yy : (m == 3 ? yy * yy : yy * yy * yy)) : T(0);
        return (D(yy, k - 1) - D(yy - hs[k], k - 1)) / hs[k];
    };
    T v = D(y, m - 1);
    return m == 2 ? v : (m == 3 ? v / T(2) : v / T(6));
}

double hl_linear_convolution_1d(double y, double h1, double h2, double h3, double h4) {
    double hs[4];
    int m = 0;
    if (std::fabs(h1) > 1e-8) hs[m++] = h1;
    if (std::fabs(h2) > 1e-8) hs[m++] = h2;
    if (std::fabs(h3) > 1e-8) hs[m++] = h3;
    if (std::fabs(h4) > 1e-8) hs[m++] = h4;
    if (m < 2) return 0.0;
    // recursive divided difference: D(y, k) over hs[0..k]
    std::function<double(double, int)> D = [&](double yy, int k) -> double {
        if (k < 0) return yy > 0 ? (m == 2 ? yy : (m == 3 ? yy * yy : yy * yy * yy)) : 0.0;
        return (D(yy, k - 1) - D(yy - hs[k], k - 1)) / hs[k];
    };
    double v = D(y, m - 1);
    return m == 2 ? v : (m == 3 ? v / 2.0 : v / 6.0);
}

// mode 0: H0 with the true hexagon bounds, 1: H0 as the reference (pmi bounds
// at the 0.5 dt row pitch, skip test in the back projection), 2: Hl.
// visit(u, conv*dx*dy) for kept bins; returns the evaluation count.
template <class T, class Visit>
long long hex_site_view(const Geo& g, int mode, bool back, int p, int ic, int il, Visit visit) {
    int nc = g.nx, nl = g.ny, nu = g.nu;
    float dt = (float)g.dy * 2.0f;                         // A_H0.cu:171
    float dx = dt * (float)kSQRT3;
    float dy = dt * (mode == 2 ? 0.5f : 1.5f);
    float nl2 = 0.5f * (nl - 1), nc2 = 0.5f * (nc - 1), nc3 = 0.5f * (nc - 2);
    float foy = (il - nl2) * dy;
    float fox = ((il & 1) ? (ic - nc3) : (ic - nc2)) * dx;
    const float* pm = &g.pmi[12 * p];
    float srcx = (float)g.src[3 * p], srcy = (float)g.src[3 * p + 1];
    float puvx = (float)g.puv[3 * p], puvy = (float)g.puv[3 * p + 1];
    float dtvx = (float)g.dtv[3 * p], dtvy = (float)g.dtv[3 * p + 1];
    int minu, maxu;
    if (mode == 0) {
        // true hexagon, FP64 through the exact detector mapping
        double px = g.src[3 * p], py = g.src[3 * p + 1], Dx = g.dtv[3 * p], Dy = g.dtv[3 * p + 1];
        double ex = g.puv[3 * p], ey = g.puv[3 * p + 1];
        double hx = 0.8660254037844386 * dt, hy = 0.5 * dt;
        double xs[6] = {fox, fox + hx, fox + hx, (double)fox, fox - hx, fox - hx};
        double ys[6] = {foy - (double)dt, foy - hy, foy + hy, foy + (double)dt, foy + hy, foy - hy};
        double umin = 1e300, umax = -1e300;
        for (int k = 0; k < 6; ++k) {
            double wx = xs[k] - px, wy = ys[k] - py;
            double u = ((px - Dx) * wy - (py - Dy) * wx) / (ex * wy - ey * wx) + 0.5 * nu;
            umin = std::min(umin, u); umax = std::max(umax, u);
        }
        minu = std::min(std::max(0, (int)std::floor(umin)), nu - 1);
        maxu = std::min(std::max(0, (int)std::floor(umax)), nu - 1);
    } else {
        // layers/A_H0.cu:84-156 (first stage)
        float icc = (float)ic + ((il & 1) ? 0.5f : 0.0f), ilc = (float)il;
        const float offc[6] = {0.0f, +0.5f, +0.5f, 0.0f, -0.5f, -0.5f};
        const float offl[6] = {-2.0f, -1.0f, +1.0f, +2.0f, +1.0f, -1.0f};
        float umin = 1e30f, umax = -1e30f;
        for (int k = 0; k < 6; ++k) {
            float ix = icc + offc[k], iy = ilc + offl[k];
            float num = std::fmaf(pm[0], ix, std::fmaf(pm[1], iy, pm[3]));
            float den = std::fmaf(pm[8], ix, std::fmaf(pm[9], iy, pm[11]));
            float u = num / den;
            umin = std::min(umin, u); umax = std::max(umax, u);
        }
        minu = std::min(std::max(0, (int)std::floor(umin)), nu - 1);
        maxu = std::min(std::max(0, (int)std::floor(umax)), nu - 1);
        if (maxu < minu) maxu = minu;
    }
    T ox = fox, oy = foy, px = srcx, py = srcy;
    long long cnt = 0;
    for (int u = minu; u <= maxu; ++u) {
        T off = T(u) - T(0.5f) * nu + T(0.5f);
        T sx = T(dtvx) + T(puvx) * off, sy = T(dtvy) + T(puvy) * off;
        T ax = sx - T(puvx) * T(0.5f), ay = sy - T(puvy) * T(0.5f);
        T bx = sx + T(puvx) * T(0.5f), by = sy + T(puvy) * T(0.5f);
        T num = (ox - px) * (sx - px) + (oy - py) * (sy - py);
        T ra = num / ((ax - px) * (sx - px) + (ay - py) * (sy - py));
        T rb = num / ((bx - px) * (sx - px) + (by - py) * (sy - py));
        T ax1 = px + (ax - px) * ra, ay1 = py + (ay - py) * ra;
        T bx1 = px + (bx - px) * rb, by1 = py + (by - py) * rb;
        if (mode == 1 && back) {  // A_H0.cu:331-334
            T da = std::hypot((double)(ax1 - ox), (double)(ay1 - oy)), db = std::hypot((double)(bx1 - ox), (double)(by1 - oy));
            if (da > T(dt) && db > T(dt) && (ax1 - ox) * (bx1 - ox) >= T(0) && (ay1 - oy) * (by1 - oy) >= T(0)) continue;
        }
        double theta = std::atan2((double)(sx - px), (double)(sy - py));
        double va = (double)dt * std::sin(theta);
        double vb = (double)dt * std::sin(theta + 2.0 * kPI / 3.0);
        double vc = (double)dt * std::sin(theta + 4.0 * kPI / 3.0);
        double vblur = -std::sqrt((double)((bx1 - ax1) * (bx1 - ax1) + (by1 - ay1) * (by1 - ay1)));
        double y = std::sqrt((double)((ax1 - ox) * (ax1 - ox) + (ay1 - oy) * (ay1 - oy)));
        if ((ay - py) * (ox - px) < (oy - py) * (ax - px)) y = -y;
        double conv;
        if (mode == 2) {
            if (std::is_same<T, CountedF>::value)
                conv = (double)hl_conv_t<T>(T(y), T(vblur), T(va), T(vb), T(vc));
            else
                conv = hl_linear_convolution_1d(y, vblur, va, vb, vc);
        } else {
            conv = (double)b0_linear_convolution_1d<T>(T(y), T(vblur), T(va), T(vb)) +
                   (double)b0_linear_convolution_1d<T>(T(y), T(vblur), T(vb), T(vc)) +
                   (double)b0_linear_convolution_1d<T>(T(y), T(vblur), T(vc), T(va));
            cnt += 3;
        }
        if (conv == conv && conv > 0.0) visit(u, conv * (double)dx * (double)dy);
    }
    return cnt;
}

// ---------------------------------------------------------------------------
// A_B1_3D cone beam: layers/A_B1_3D.cu
// ---------------------------------------------------------------------------

// mode 0: forward as the reference (:82-312); mode 1: backward as the
// reference (:314-531); mode 2: backward as the exact transpose of the
// forward.  visit(u, v, weight) for every kept (u, v) of voxel (ix, iy, iz)
// in view p; returns the footprint-evaluation count (forward).
template <class T, class Visit>
long long b1_3d_voxel_view(const Geo& g, const float* vecs_p, int mode, int p, int ix, int iy, int iz, Visit visit) {
    int nx = g.nx, ny = g.ny, nz = g.nz, nu = g.nu, nv = g.nv;
    float dx = (float)g.dx, dy = (float)g.dy, dz = (float)g.dz;
    const float* pm = &g.pmi[12 * p];
    float srcx = (float)g.src[3 * p], srcy = (float)g.src[3 * p + 1], srcz = (float)g.src[3 * p + 2];
    float puvx = (float)g.puv[3 * p], puvy = (float)g.puv[3 * p + 1];
    float dtvx = (float)g.dtv[3 * p], dtvy = (float)g.dtv[3 * p + 1];
    bool singular = std::fabs(puvx - puvy) < 1e-7f;
    float fox = (ix - 0.5f * (nx - 1)) * dx, foy = (iy - 0.5f * (ny - 1)) * dy, foz = (iz - 0.5f * (nz - 1)) * dz;
    float sx1 = ix - 1.0f, sx2 = ix + 1.0f, sy1 = iy - 1.0f, sy2 = iy + 1.0f;
    // FP32 ranges as the reference computes them (with its contractions)
    auto U = [&](float x, float y) {
        float n = std::fmaf(pm[1], y, pm[0] * x) + pm[3], d = std::fmaf(pm[9], y, pm[8] * x) + pm[11];
        float u = n / d;
        return singular ? (u * 1.5f - 1.0f) / puvx : u;
    };
    float us[4] = {U(sx1, sy1), U(sx2, sy1), U(sx1, sy2), U(sx2, sy2)};
    sort4(us);
    int minu = std::min(std::max(0, (int)std::floor(us[0])), nu - 1);
    int maxu = std::min(std::max(0, (int)std::floor(us[3])), nu - 1);
    if (mode == 1 && minu >= maxu) return 0;
    float v1 = std::fmaf(pm[5], (float)iy, pm[4] * sx1) + pm[7], v2 = std::fmaf(pm[5], (float)iy, pm[4] * sx2) + pm[7];
    float v3 = std::fmaf(pm[9], (float)iy, pm[8] * sx1) + pm[11], v4 = std::fmaf(pm[9], (float)iy, pm[8] * sx2) + pm[11];
    auto V = [&](float a, float b, float z) {
        float v = std::fmaf(pm[6], z, a) / std::fmaf(pm[10], z, b);
        return singular ? (v * 1.5f - 1.0f) / puvy : v;
    };
    float sz1 = iz - 0.5f, sz2 = iz + 0.5f;
    float vsf[4] = {V(v1, v3, sz1), V(v1, v3, sz2), V(v2, v4, sz1), V(v2, v4, sz2)};
    sort4(vsf);
    if (vsf[0] >= nv) return -1;  // the reference returns for the rest of its z chunk
    int minv = std::min(std::max(0, (int)std::floor(vsf[0])), nv - 1);
    int maxv = std::min(std::max(0, (int)std::floor(vsf[3])), nv - 1);
    if (mode == 1 && minv >= maxv) return 0;
    T ox = fox, oy = foy, oz = foz, px = srcx, py = srcy, pz = srcz;
    T vs[4] = {vsf[0], vsf[1], vsf[2], vsf[3]};
    T weight = sqrt(((ox - px) * (ox - px) + (oy - py) * (oy - py) + (oz - pz) * (oz - pz)) /
                    ((ox - px) * (ox - px) + (oy - py) * (oy - py)));
    T C = T(dx) * T(dy) * T(dz) * weight;
    if (mode != 1) C = C * (T(2) / ((vs[3] - vs[0]) + (vs[2] - vs[1])));
    long long cnt = 0;
    for (int u = minu; u <= maxu; ++u) {
        T off = T(u) - T(0.5f) * nu + T(0.5f);
        T sx = T(dtvx) + T(puvx) * off, sy = T(dtvy) + T(puvy) * off;
        T vx = vecs_p[u], vy = vecs_p[nu + u];
        T ax = sx - T(puvx) * T(0.5f), ay = sy - T(puvy) * T(0.5f), bx = sx + T(puvx) * T(0.5f), by = sy + T(puvy) * T(0.5f);
        T num = (ox - px) * (sx - px) + (oy - py) * (sy - py);
        T ra = num / ((ax - px) * (sx - px) + (ay - py) * (sy - py));
        T rb = num / ((bx - px) * (sx - px) + (by - py) * (sy - py));
        T ax1 = px + (ax - px) * ra, ay1 = py + (ay - py) * ra, bx1 = px + (bx - px) * rb, by1 = py + (by - py) * rb;
        T x1 = sqrt((ax1 - ox) * (ax1 - ox) + (ay1 - oy) * (ay1 - oy));
        T x2 = sqrt((bx1 - ox) * (bx1 - ox) + (by1 - oy) * (by1 - oy));
        T sgn = ((ax1 - ox) * (bx1 - ox) + (ay1 - oy) * (by1 - oy) > T(0)) ? T(1) : T(-1);
        T conv = b1_linear_convolution_1d<T>(x1 * sgn, x2, max(vx, vy), min(vx, vy));
        ++cnt;
        if (mode == 1) { if (!(conv == conv && conv > T(1e-7f))) continue; }
        else if (!(conv * C == conv * C)) continue;
        for (int j = minv; j <= maxv; ++j) {
            T gm = sf_gamma<T>(T(j), T(j) + T(1), vs);
            if (gm > T(1e-7f)) visit(u, j, (double)(conv * C * gm));
        }
    }
    return cnt;
}

// Index-space projection matrices built directly from the ray geometry in
// FP64 (detector plane through dtv spanned by puv, pvv; u = offset/du + nu/2),
// replacing pmi: equal to it except on the views where utils/geo.cu:36-41
// degenerates (puv.x == puv.y).  Used by the corrected SF_projector mode.
void exact_pmi_geo(Geo& g) {
    auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    for (int p = 0; p < g.np; ++p) {
        const double *S = &g.src[3 * p], *D = &g.dtv[3 * p], *eu = &g.puv[3 * p], *ev = &g.pvv[3 * p];
        const double n[3] = {eu[1] * ev[2] - eu[2] * ev[1], eu[2] * ev[0] - eu[0] * ev[2], eu[0] * ev[1] - eu[1] * ev[0]};
        double SD[3], DS[3];
        for (int k = 0; k < 3; ++k) { SD[k] = S[k] - D[k]; DS[k] = D[k] - S[k]; }
        const double uu = dot(eu, eu), vv = dot(ev, ev);
        double rows[3][4];
        for (int k = 0; k < 3; ++k) {
            rows[0][k] = dot(eu, SD) / uu * n[k] + dot(n, DS) * eu[k] / uu;
            rows[1][k] = dot(ev, SD) / vv * n[k] + dot(n, DS) * ev[k] / vv;
            rows[2][k] = n[k];
        }
        for (int r = 0; r < 3; ++r) rows[r][3] = -(rows[r][0] * S[0] + rows[r][1] * S[1] + rows[r][2] * S[2]);
        for (int k = 0; k < 4; ++k) {
            rows[0][k] += 0.5 * g.nu * rows[2][k];
            rows[1][k] += 0.5 * g.nv * rows[2][k];
        }
        const double x0 = -0.5 * (g.nx - 1) * g.dx, y0 = -0.5 * (g.ny - 1) * g.dy, z0 = -0.5 * (g.nz - 1) * g.dz;
        double m[12];
        for (int r = 0; r < 3; ++r) {
            m[4 * r] = rows[r][0] * g.dx;
            m[4 * r + 1] = rows[r][1] * g.dy;
            m[4 * r + 2] = rows[r][2] * g.dz;
            m[4 * r + 3] = rows[r][3] + rows[r][0] * x0 + rows[r][1] * y0 + rows[r][2] * z0;
        }
        for (int k = 0; k < 12; ++k) g.pmi[12 * p + k] = (float)(m[k] / m[11]);
    }
}

// ---------------------------------------------------------------------------
// SF_projector 3D separable footprint: layers/SF_projector.cu
// ---------------------------------------------------------------------------

// One voxel (ix, iy, iz) in view p.  fwd: the forward's amplitude (1/r^2,
// lsd^2 dy dz / (du dv)) and, with trap, the SF-TT v trapezoid
// (:81-234); otherwise the backward's (1/r, lsd dx / np, :237-356).
// mode 0 visits exactly the bins the reference visits (unclamped u, wrap into
// neighbouring rows through j * nu + i, :216, :336) with the footprint alone
// in the forward (the reference never applies C or the voxel value there,
// :190-221); mode 1 keeps in-detector bins only and multiplies by the
// amplitude.  visit(index into the view's nu*nv plane, weight).
// Returns -1 when the reference leaves the rest of its z chunk (:150, :286),
// 0 when the voxel is skipped, 1 when it was visited.
template <class T, class Visit>
int sf3d_voxel_view(const Geo& g, double lsd, int mode, bool fwd, bool trap, int p, int ix, int iy, int iz,
                    Visit visit) {
    const int nu = g.nu, nv = g.nv, nuv = nu * nv;
    const float* pm = &g.pmi[12 * p];
    // FP32 corner projections as the kernel computes them (ranges and skips)
    auto lin = [&](int r, float x, float y) { return std::fmaf(pm[4 * r + 1], y, pm[4 * r] * x) + pm[4 * r + 3]; };
    const float sx1 = ix - 0.5f, sx2 = ix + 0.5f, sy1 = iy - 0.5f, sy2 = iy + 0.5f;
    const float sz1 = iz - 0.5f, sz2 = iz + 0.5f;
    T vs[4];
    float min_v, max_v;
    if (!(fwd && trap)) {
        const float a = lin(1, (float)ix, (float)iy), b = lin(2, (float)ix, (float)iy);
        const float v0 = std::fmaf(pm[6], sz1, a) / std::fmaf(pm[10], sz1, b);
        min_v = std::ceil(v0 - 0.5f);
        if (min_v >= nv) return -1;
        const float v1 = std::fmaf(pm[6], sz2, a) / std::fmaf(pm[10], sz2, b);
        max_v = std::ceil(v1 - 0.5f);
        if (max_v < 0) return 0;
        vs[0] = v0; vs[1] = v1;
    } else {
        const float a1 = lin(1, sx1, (float)iy), a2 = lin(1, sx2, (float)iy);
        const float b1 = lin(2, sx1, (float)iy), b2 = lin(2, sx2, (float)iy);
        float v[4] = {std::fmaf(pm[6], sz1, a1) / std::fmaf(pm[10], sz1, b1),
                      std::fmaf(pm[6], sz2, a1) / std::fmaf(pm[10], sz2, b1),
                      std::fmaf(pm[6], sz1, a2) / std::fmaf(pm[10], sz1, b2),
                      std::fmaf(pm[6], sz2, a2) / std::fmaf(pm[10], sz2, b2)};
        sort4(v);
        min_v = std::ceil(v[0] - 0.5f);
        max_v = std::ceil(v[3] - 0.5f);
        if (max_v < 0 || min_v >= nv) return 0;
        for (int k = 0; k < 4; ++k) vs[k] = v[k];
    }
    float uf[4] = {std::fmaf(pm[2], (float)iz, lin(0, sx1, sy1)) / std::fmaf(pm[10], (float)iz, lin(2, sx1, sy1)),
                   std::fmaf(pm[2], (float)iz, lin(0, sx2, sy1)) / std::fmaf(pm[10], (float)iz, lin(2, sx2, sy1)),
                   std::fmaf(pm[2], (float)iz, lin(0, sx1, sy2)) / std::fmaf(pm[10], (float)iz, lin(2, sx1, sy2)),
                   std::fmaf(pm[2], (float)iz, lin(0, sx2, sy2)) / std::fmaf(pm[10], (float)iz, lin(2, sx2, sy2))};
    sort4(uf);
    const float min_u = std::ceil(uf[0] - 0.5f), max_u = std::ceil(uf[3] - 0.5f);
    if (max_u < 0 || min_u >= nu) return 0;
    // spans wider than twice the detector (degenerate projections): skipped, as the kernels do
    if (!(max_u - min_u <= 2.f * nu + 4.f) || !(max_v - min_v <= 2.f * nv + 4.f)) return 0;
    T us[4] = {uf[0], uf[1], uf[2], uf[3]};
    // :173 / :300 with the integer halves of :104-105
    const double ddx = g.dx * (ix - g.nx / 2) - g.src[3 * p], ddy = g.dy * (iy - g.ny / 2) - g.src[3 * p + 1];
    const double ddz = g.dz * (iz - g.nz / 2) - g.src[3 * p + 2];
    T w = T(1) / sqrt(T(ddx * ddx + ddy * ddy + ddz * ddz));
    const double flsd = (double)(float)lsd;  // float lsd = *lsds[p] (:362, :384)
    T C;
    const T tw = T(2) / ((us[3] - us[0]) + (us[2] - us[1]));
    if (fwd) {
        // :364; the corrected pair (mode 1) multiplies in the missing dx
        const double factor =
            (double)((float)flsd * (float)flsd) * g.dy * g.dz / (g.du * g.dv) * (mode == 1 ? g.dx : 1.0);
        C = w * w * T(factor) * tw * (trap ? T(2) / ((vs[3] - vs[0]) + (vs[2] - vs[1])) : T(1) / (vs[1] - vs[0]));
    } else {
        C = w * T(flsd * g.dx / g.np) * tw * (T(1) / (vs[1] - vs[0]));
    }
    const T amp = (mode == 0 && fwd) ? T(1) : C;
    for (int i = (int)min_u; i <= (int)max_u; ++i) {
        if (mode == 1 && (i < 0 || i >= nu)) continue;
        const T gu = sf_gamma<T>(T(i) - T(0.5), T(i) + T(0.5), us);
        for (int j = (int)min_v; j <= (int)max_v; ++j) {
            if (mode == 1 && (j < 0 || j >= nv)) continue;
            const T fv = (fwd && trap) ? sf_gamma<T>(T(j) - T(0.5), T(j) + T(0.5), vs)
                                       : max(min(T(j) + T(0.5), vs[1]) - max(T(j) - T(0.5), vs[0]), T(0));
            const long long idx = (long long)j * nu + i;
            if (idx >= 0 && idx < nuv) visit((int)idx, (double)(gu * fv * amp));
        }
    }
    return 1;
}

// ---------------------------------------------------------------------------
// exact FP64 projectors: layers/Ref_projector.cu, python/matrix_gen/*_ref_project.py
// ---------------------------------------------------------------------------

// Parameter interval [t0, t1] of the line a + t d inside the box [lo, hi]
// (slab method); false when the line misses it.  Replaces the six face tests
// of lineInBox (layers/Ref_projector.cu:99-154), which gather the crossing
// points with a 1e-13 tolerance and return |max - min| of them.
bool line_box(const double* a, const double* d, const double* lo, const double* hi, int dim, double& t0,
              double& t1) {
    t0 = -INFINITY; t1 = INFINITY;
    for (int k = 0; k < dim; ++k) {
        if (d[k] == 0.0) {
            if (a[k] < lo[k] || a[k] > hi[k]) return false;
            continue;
        }
        double ta = (lo[k] - a[k]) / d[k], tb = (hi[k] - a[k]) / d[k];
        if (ta > tb) std::swap(ta, tb);
        t0 = std::max(t0, ta); t1 = std::min(t1, tb);
    }
    return t1 > t0;
}

// Chord length of the line through p1 and p2 inside the box [c1, c1 + d]
// (layers/Ref_projector.cu:99-154, in FP64 throughout; the reference returns
// sqrtf of it, FP32 precision).
double chord3(const double* p1, const double* p2, const double* c1, const double* d) {
    double dir[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]};
    double hi[3] = {c1[0] + d[0], c1[1] + d[1], c1[2] + d[2]};
    double t0, t1;
    if (!line_box(p1, dir, c1, hi, 3, t0, t1)) return 0.0;
    return (t1 - t0) * std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
}

// Line integral, in mm, of a 2D pixel basis centred at o along the line from
// s through q: kind 0 the pixel indicator of size dx x dy (the A_B0 model),
// kind 1 the bilinear hat (1 - |x|/dx)+ (1 - |y|/dy)+ (the A_B1 model).  For
// the hat the line is cut at the hat's cell edges; on each piece the
// integrand is a product of two affine functions of the arc length, so
// Simpson's rule is exact there.
double pixel_line_integral(int kind, const double* s, const double* q, const double* o, double dx, double dy) {
    double d[2] = {q[0] - s[0], q[1] - s[1]};
    const double len = std::sqrt(d[0] * d[0] + d[1] * d[1]);
    d[0] /= len; d[1] /= len;
    const double hx = kind == 0 ? 0.5 * dx : dx, hy = kind == 0 ? 0.5 * dy : dy;
    double lo[2] = {o[0] - hx, o[1] - hy}, hi[2] = {o[0] + hx, o[1] + hy};
    double t0, t1;
    if (!line_box(s, d, lo, hi, 2, t0, t1)) return 0.0;
    if (kind == 0) return t1 - t0;
    double cut[4];
    int nc = 0;
    cut[nc++] = t0;
    for (int k = 0; k < 2; ++k)
        if (d[k] != 0.0) {
            double t = (o[k] - s[k]) / d[k];
            if (t > t0 && t < t1) cut[nc++] = t;
        }
    cut[nc++] = t1;
    std::sort(cut, cut + nc);
    auto h = [&](double t) {
        double x = s[0] + t * d[0] - o[0], y = s[1] + t * d[1] - o[1];
        return std::max(0.0, 1.0 - std::fabs(x) / dx) * std::max(0.0, 1.0 - std::fabs(y) / dy);
    };
    double sum = 0.0;
    for (int k = 0; k + 1 < nc; ++k) {
        double a = cut[k], b = cut[k + 1];
        sum += (b - a) / 6.0 * (h(a) + 4.0 * h(0.5 * (a + b)) + h(b));
    }
    return sum;
}

// Adaptive Simpson with Richardson's correction (q + (q - v)/15), the scheme
// of simpson_layer (layers/Ref_projector.cu:156-214) in one dimension.
template <class F>
double adaptive_simpson(F f, double a, double b, double fa, double fm, double fb, double whole, double eps,
                        int depth) {
    const double m = 0.5 * (a + b), lm = 0.5 * (a + m), rm = 0.5 * (m + b);
    const double flm = f(lm), frm = f(rm);
    const double left = (m - a) / 6.0 * (fa + 4.0 * flm + fm), right = (b - m) / 6.0 * (fm + 4.0 * frm + fb);
    const double q = left + right;
    if (depth <= 0 || std::fabs(q - whole) <= 15.0 * eps) return q + (q - whole) / 15.0;
    return adaptive_simpson(f, a, m, fa, flm, fm, left, 0.5 * eps, depth - 1) +
           adaptive_simpson(f, m, b, fm, frm, fb, right, 0.5 * eps, depth - 1);
}

template <class F>
double integrate(F f, double a, double b, double eps) {
    const double fa = f(a), fm = f(0.5 * (a + b)), fb = f(b);
    return adaptive_simpson(f, a, b, fa, fm, fb, (b - a) / 6.0 * (fa + 4.0 * fm + fb), eps, 40);
}

// Integral over [0, 1] of an integrand whose kinks lie at `cuts` (where the
// ray passes the basis function's breakpoints): each smooth piece is
// integrated separately, so the adaptive rule never stops early on a
// coincidental agreement across a kink.
template <class F>
double integrate_pieces(F f, std::vector<double> cuts, double eps) {
    cuts.push_back(0.0);
    cuts.push_back(1.0);
    std::sort(cuts.begin(), cuts.end());
    double sum = 0.0;
    for (size_t k = 0; k + 1 < cuts.size(); ++k) {
        const double a = std::max(0.0, cuts[k]), b = std::min(1.0, cuts[k + 1]);
        if (b > a) sum += integrate(f, a, b, eps * (b - a));
    }
    return sum;
}

// Breakpoints of a pixel basis centred at o: the corners of the indicator
// (kind 0) or the 3 x 3 grid of the hat's cell corners (kind 1).
inline void basis_breakpoints(int kind, const double* o, double dx, double dy, std::vector<double>& px,
                              std::vector<double>& py) {
    px.clear();
    py.clear();
    if (kind == 0) {
        for (int a = -1; a <= 1; a += 2)
            for (int b = -1; b <= 1; b += 2) { px.push_back(o[0] + 0.5 * a * dx); py.push_back(o[1] + 0.5 * b * dy); }
    } else {
        for (int a = -1; a <= 1; ++a)
            for (int b = -1; b <= 1; ++b) { px.push_back(o[0] + a * dx); py.push_back(o[1] + b * dy); }
    }
}

// geo_init_example (utils/geo.cu:209-230) with the arguments the matrix
// generators pass (start 0, end 2 pi (np - 1)/np, layers/A_B1.cu:547): uniform
// angles without the 45-degree snap.  (np = 1 divides 0 by 0 there; it is
// taken as the single angle 0 here.)
void build_geo_example(Geo& g, double lsd, double lso) {
    const int np = g.np;
    g.src.assign(3 * np, 0.0); g.dtv.assign(3 * np, 0.0);
    g.puv.assign(3 * np, 0.0); g.pvv.assign(3 * np, 0.0);
    const double end = kPI * 2 * (np - 1) / np;
    const double dangle = np > 1 ? (end - (double)0.0f) / (np - 1) : 0.0;
    double src0[3] = {-lso, 0.0, 0.0}, dtv0[3] = {lsd - lso, 0.0, 0.0};
    double puv0[3] = {0.0, g.du, 0.0}, pvv0[3] = {0.0, 0.0, g.dv};
    for (int i = 0; i < np; ++i) {
        const double beta = (double)0.0f + i * dangle;
        rotate(src0, &g.src[3 * i], beta);
        rotate(dtv0, &g.dtv[3 * i], beta);
        rotate(puv0, &g.puv[3 * i], beta);
        rotate(pvv0, &g.pvv[3 * i], beta);
    }
}

// One (view, bin) row of the generators' dense slab: bilinear_matrix_generate
// (layers/A_B1.cu:355-427, kind 1) or b0_matrix_generate (layers/A_B0.cu:
// 37-121, kind 0).  FP64 geometry; the footprint in T (float: the reference,
// whose FP64 arguments meet its float-only linear_convolution_1d).
// visit(col, value) for every entry with value > 0, in column order.
template <class T, class Visit>
void generator_row(const Geo& g, int kind, int p, int iu, Visit visit) {
    const int nx = g.nx, ny = g.ny, nu = g.nu;
    const double nx2 = 0.5 * (nx - 1), ny2 = 0.5 * (ny - 1), dx = g.dx, dy = g.dy;
    const double px = g.src[3 * p], py = g.src[3 * p + 1];
    const double sx = g.dtv[3 * p] + g.puv[3 * p] * (iu - 0.5 * nu + 0.5);
    const double sy = g.dtv[3 * p + 1] + g.puv[3 * p + 1] * (iu - 0.5 * nu + 0.5);
    const double ax = sx - g.puv[3 * p] * 0.5, ay = sy - g.puv[3 * p + 1] * 0.5;
    const double bx = sx + g.puv[3 * p] * 0.5, by = sy + g.puv[3 * p + 1] * 0.5;
    const double theta = std::atan2(std::fabs(px - sx), std::fabs(py - sy));
    const double sint = std::sin(theta), cost = std::cos(theta);
    double vx = dx * cost, vy = dy * sint;
    if (kind == 0) {
        vx = std::fabs(vx); vy = std::fabs(vy);
        if (py < sy) vx = -vx;
        if (px < sx) vy = -vy;
    }
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            const double ox = (i - nx2) * dx, oy = (j - ny2) * dy;
            const double num = (ox - px) * (sx - px) + (oy - py) * (sy - py);
            const double ra = num / ((ax - px) * (sx - px) + (ay - py) * (sy - py));
            const double rb = num / ((bx - px) * (sx - px) + (by - py) * (sy - py));
            const double ax1 = px + (ax - px) * ra, ay1 = py + (ay - py) * ra;
            const double bx1 = px + (bx - px) * rb, by1 = py + (by - py) * rb;
            if (std::fabs(ax1 - ox) > dx && std::fabs(bx1 - ox) > dx && std::fabs(ay1 - oy) > dy &&
                std::fabs(by1 - oy) > dy)
                continue;
            T conv;
            if (kind == 1) {
                const double vblur = std::sqrt((bx1 - ax1) * (bx1 - ax1) + (by1 - ay1) * (by1 - ay1));
                double y = std::sqrt((ax1 - ox) * (ax1 - ox) + (ay1 - oy) * (ay1 - oy));
                if (y > 2 * std::fabs(vx) + 2 * std::fabs(vy) + std::fabs(vblur)) continue;
                if ((ay - py) * (ox - px) > (oy - py) * (ax - px)) y = -y;
                conv = b1_linear_convolution_1d<T>(T(y), T(y + vblur), T(std::max(vx, vy)), T(std::min(vx, vy)));
            } else {
                const double om = -0.5 * dx * (px - sx) + 0.5 * dy * (py - sy);
                const double l2 = (sx - px) * (sx - px) + (sy - py) * (sy - py);
                const double zx = ox - 0.5 * dx - om * (px - sx) / l2, zy = oy + 0.5 * dy - om * (py - sy) / l2;
                const double vblur = -std::sqrt((bx1 - ax1) * (bx1 - ax1) + (by1 - ay1) * (by1 - ay1));
                double y = std::sqrt((ax1 - zx) * (ax1 - zx) + (ay1 - zy) * (ay1 - zy));
                if (y > std::fabs(vx) + std::fabs(vy) + std::fabs(vblur)) continue;
                if ((ay - py) * (zx - px) < (zy - py) * (ax - px)) y = -y;
                conv = b0_linear_convolution_1d<T>(T(y), T(vx), T(vy), T(vblur));
            }
            if (conv > T(0)) visit(i * ny + j, (double)conv);
        }
}

Geo make_geo(int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy, double dz, double du,
             double dv) {
    Geo g;
    g.nx = nx; g.ny = ny; g.nz = nz; g.np = np; g.nu = nu; g.nv = nv;
    g.dx = dx; g.dy = dy; g.dz = dz; g.du = du; g.dv = dv;
    return g;
}

}  // namespace

extern "C" {

// Geometry tables exactly as utils/geo.cu builds them (2D inits use nz = nv = 1,
// dz = dv = 1, layers/A_B1.cu:596).
void oracle_geometry(int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy, double dz, double du,
                     double dv, double lsd, double lso, const double* angles, const double* dzs,
                     const double* drho, double* src, double* dtv, double* puv, double* pvv, double* pm,
                     float* pmi) {
    Geo g = make_geo(nx, ny, nz, np, nu, nv, dx, dy, dz, du, dv);
    build_geo(g, lsd, lso, angles, dzs, drho);
    std::memcpy(src, g.src.data(), sizeof(double) * 3 * np);
    std::memcpy(dtv, g.dtv.data(), sizeof(double) * 3 * np);
    std::memcpy(puv, g.puv.data(), sizeof(double) * 3 * np);
    std::memcpy(pvv, g.pvv.data(), sizeof(double) * 3 * np);
    std::memcpy(pm, g.pm.data(), sizeof(double) * 12 * np);
    std::memcpy(pmi, g.pmi.data(), sizeof(float) * 12 * np);
}

// b1_forward_projection / b1_backward_projection (layers/A_B1.cu:605-678) with the
// same host layouts: x[ix*ny+iy], b[p*nu+u].  precision: 0 = FP64 replica,
// 1 = FP32 emulation.  dz/drho may be null.  Returns the footprint-evaluation count.
long long oracle_b1_forward(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd,
                            double lso, const double* angles, const double* dzs, const double* drho,
                            const double* x, double* b, int precision) {
    Geo g = make_geo(nx, ny, 1, np, nu, 1, dx, dy, 1, du, 1);
    build_geo(g, lsd, lso, angles, dzs, drho);
    std::vector<float> vecs;
    b1_vectors(g, vecs);
    return precision ? b1_forward<float>(g, vecs, x, b) : b1_forward<double>(g, vecs, x, b);
}

void oracle_b1_backward(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
                        const double* angles, const double* dzs, const double* drho, const double* b, double* x,
                        int precision) {
    Geo g = make_geo(nx, ny, 1, np, nu, 1, dx, dy, 1, du, 1);
    build_geo(g, lsd, lso, angles, dzs, drho);
    std::vector<float> vecs;
    b1_vectors(g, vecs);
    if (precision) b1_backward<float>(g, vecs, b, x); else b1_backward<double>(g, vecs, b, x);
}

// b1_3d_forward_projection / b1_3d_backward_projection (layers/A_B1_3D.cu:
// 696-772): volume x[(iz*ny + iy)*nx + ix], projections b[(p*nv + v)*nu + u].
// back_mode 1: the reference's backward, 2: exact transpose of the forward.
unsigned long long oracle_b1_3d_forward(int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy,
                                        double dz, double du, double dv, double lsd, double lso, const double* angles,
                                        const double* x, double* b) {
    Geo g = make_geo(nx, ny, nz, np, nu, nv, dx, dy, dz, du, dv);
    build_geo(g, lsd, lso, angles, nullptr, nullptr);
    std::vector<float> vecs;
    b1_vectors(g, vecs);
    std::memset(b, 0, sizeof(double) * (size_t)np * nu * nv);
    long long total = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : total)
    for (int p = 0; p < np; ++p) {
        double* bp = b + (size_t)p * nu * nv;
        const float* vp = &vecs[(size_t)p * nu * 2];
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix)
                for (int z0 = 0; z0 < nz; z0 += 32)
                    for (int iz = z0; iz < std::min(nz, z0 + 32); ++iz) {
                        double C = x[((size_t)iz * ny + iy) * nx + ix];
                        long long n = b1_3d_voxel_view<double>(g, vp, 0, p, ix, iy, iz, [&](int u, int v, double w) {
                            bp[(size_t)v * nu + u] += w * C;
                        });
                        if (n < 0) break;
                        total += n;
                    }
    }
    return (unsigned long long)total;
}

void oracle_b1_3d_backward(int back_mode, int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy,
                           double dz, double du, double dv, double lsd, double lso, const double* angles,
                           const double* b, double* x) {
    Geo g = make_geo(nx, ny, nz, np, nu, nv, dx, dy, dz, du, dv);
    build_geo(g, lsd, lso, angles, nullptr, nullptr);
    std::vector<float> vecs;
    b1_vectors(g, vecs);
    std::memset(x, 0, sizeof(double) * (size_t)nx * ny * nz);
#pragma omp parallel for schedule(dynamic) collapse(2)
    for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix)
            for (int p = 0; p < np; ++p) {
                const double* bp = b + (size_t)p * nu * nv;
                const float* vp = &vecs[(size_t)p * nu * 2];
                for (int z0 = 0; z0 < nz; z0 += 32)
                    for (int iz = z0; iz < std::min(nz, z0 + 32); ++iz) {
                        double acc = 0.0;
                        long long n = b1_3d_voxel_view<double>(g, vp, back_mode, p, ix, iy, iz, [&](int u, int v, double w) {
                            acc += w * bp[(size_t)v * nu + u];
                        });
                        if (n < 0) break;
                        x[((size_t)iz * ny + iy) * nx + ix] += acc;
                    }
            }
}

// SF::project / SF::back_project (layers/SF_projector.cu:359-400) over all
// views: volume x[(iz*ny + iy)*nx + ix], projections b[(p*nv + v)*nu + u].
// mode 0 reproduces the reference kernels, mode 1 the corrected forward and
// its exact transpose (trap selects SF-TT in v for mode-1 backward too).
void oracle_sf3d_forward(int mode, int trap, int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy,
                         double dz, double du, double dv, double lsd, double lso, const double* angles,
                         const double* x, double* b) {
    Geo g = make_geo(nx, ny, nz, np, nu, nv, dx, dy, dz, du, dv);
    build_geo(g, lsd, lso, angles, nullptr, nullptr);
    if (mode == 1) exact_pmi_geo(g);
    std::memset(b, 0, sizeof(double) * (size_t)np * nu * nv);
#pragma omp parallel for schedule(dynamic)
    for (int p = 0; p < np; ++p) {
        double* bp = b + (size_t)p * nu * nv;
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix)
                for (int z0 = 0; z0 < nz; z0 += 64)
                    for (int iz = z0; iz < std::min(nz, z0 + 64); ++iz) {
                        const double C = x[((size_t)iz * ny + iy) * nx + ix];
                        // the reference reads the voxel after the v tests (:170-171)
                        int r = sf3d_voxel_view<double>(g, lsd, mode, true, trap != 0, p, ix, iy, iz,
                                                        [&](int idx, double w) {
                                                            if (C != 0) bp[idx] += mode == 0 ? w : w * C;
                                                        });
                        if (r < 0 && mode == 0) break;
                    }
    }
}

void oracle_sf3d_backward(int mode, int trap, int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy,
                          double dz, double du, double dv, double lsd, double lso, const double* angles,
                          const double* b, double* x) {
    Geo g = make_geo(nx, ny, nz, np, nu, nv, dx, dy, dz, du, dv);
    build_geo(g, lsd, lso, angles, nullptr, nullptr);
    if (mode == 1) exact_pmi_geo(g);
    std::memset(x, 0, sizeof(double) * (size_t)nx * ny * nz);
#pragma omp parallel for schedule(dynamic) collapse(2)
    for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix)
            for (int p = 0; p < np; ++p) {
                const double* bp = b + (size_t)p * nu * nv;
                for (int z0 = 0; z0 < nz; z0 += 64)
                    for (int iz = z0; iz < std::min(nz, z0 + 64); ++iz) {
                        double acc = 0.0;
                        int r = sf3d_voxel_view<double>(g, lsd, mode, mode == 1, trap != 0, p, ix, iy, iz,
                                                        [&](int idx, double w) { acc += w * bp[idx]; });
                        if (r < 0 && mode == 0) break;
                        x[((size_t)iz * ny + iy) * nx + ix] += acc;
                    }
            }
}

// Exact fan-beam system matrix of the pixel-indicator (kind 0) or bilinear
// (kind 1) basis, dense, M[(p*nu + u)*(nx*ny) + ix*ny + iy]: the line
// integral of the basis function along the ray from the source to each point
// of bin u, averaged over the bin (python/matrix_gen/A_B0_ref_project.py:
// 137-193, A_B1_ref_project.py:83-139, with scipy's quad replaced by the
// adaptive Simpson above to a relative tolerance `tol`).  Bin u spans
// dtv + puv (u - nu/2 + t), t in [0, 1] (layers/A_B1.cu:153); pixel centres
// ((i - (nx-1)/2) dx, (j - (ny-1)/2) dy).  The integrand has kinks where the
// ray meets pixel corners; the adaptive rule resolves them.
void oracle_exact_fan2d_matrix(int kind, int nx, int ny, int np, int nu, double dx, double dy, double du,
                               double lsd, double lso, const double* angles, const double* dzs, const double* drho,
                               double tol, double* M) {
    Geo g = make_geo(nx, ny, 1, np, nu, 1, dx, dy, 1, du, 1);
    build_geo(g, lsd, lso, angles, dzs, drho);
    const size_t ncol = (size_t)nx * ny;
    std::memset(M, 0, sizeof(double) * ncol * np * nu);
    const double reach = kind == 0 ? 0.5 * std::hypot(dx, dy) : std::hypot(dx, dy);
#pragma omp parallel for schedule(dynamic) collapse(2)
    for (int p = 0; p < np; ++p)
        for (int u = 0; u < nu; ++u) {
            const double* s = &g.src[3 * p];
            const double* dt = &g.dtv[3 * p];
            const double* pu = &g.puv[3 * p];
            double* row = M + ((size_t)p * nu + u) * ncol;
            double e0[2], e1[2];
            for (int k = 0; k < 2; ++k) {
                e0[k] = dt[k] + pu[k] * (u - 0.5 * nu) - s[k];
                e1[k] = dt[k] + pu[k] * (u - 0.5 * nu + 1.0) - s[k];
            }
            const double n0 = std::hypot(e0[0], e0[1]), n1 = std::hypot(e1[0], e1[1]);
            for (int ix = 0; ix < nx; ++ix)
                for (int iy = 0; iy < ny; ++iy) {
                    const double o[2] = {(ix - 0.5 * (nx - 1)) * dx, (iy - 0.5 * (ny - 1)) * dy};
                    const double r[2] = {o[0] - s[0], o[1] - s[1]};
                    // signed distances of the centre from the two edge rays:
                    // outside the wedge by more than the support radius -> 0
                    const double c0 = (e0[0] * r[1] - e0[1] * r[0]) / n0, c1 = (e1[0] * r[1] - e1[1] * r[0]) / n1;
                    if ((c0 > reach && c1 > reach) || (c0 < -reach && c1 < -reach)) continue;
                    auto f = [&](double t) {
                        double q[2] = {dt[0] + pu[0] * (u - 0.5 * nu + t), dt[1] + pu[1] * (u - 0.5 * nu + t)};
                        return pixel_line_integral(kind, s, q, o, dx, dy);
                    };
                    // bin parameter of the ray through each breakpoint C:
                    // cross(D - S + e (off + t), C - S) = 0
                    std::vector<double> bx, by, cuts;
                    basis_breakpoints(kind, o, dx, dy, bx, by);
                    const double off = u - 0.5 * nu;
                    for (size_t k = 0; k < bx.size(); ++k) {
                        const double cx = bx[k] - s[0], cy = by[k] - s[1];
                        const double den = pu[0] * cy - pu[1] * cx;
                        if (den == 0.0) continue;
                        const double t = -((dt[0] - s[0]) * cy - (dt[1] - s[1]) * cx) / den - off;
                        if (t > 0.0 && t < 1.0) cuts.push_back(t);
                    }
                    const double scale = kind == 0 ? std::hypot(dx, dy) : std::max(dx, dy);
                    row[(size_t)ix * ny + iy] = integrate_pieces(f, cuts, tol * scale);
                }
        }
}

// Exact fan-beam system matrix of the hexagon indicator, the basis of H0
// (layers/A_H0.cu:158-256): site (ic, il) of the lattice at
// ((ic - (nc-1)/2 [odd rows: (nc-2)/2]) sqrt(3) dt, (il - (nl-1)/2) 1.5 dt)
// (:174-183; odd rows hold nc - 1 sites), a regular hexagon of circumradius dt
// with vertices at 30 + 60 k degrees (the union of the three rhombi spanned
// by the directions at -90, 30 and 150 degrees whose X-rays the kernel sums,
// :229-245).  Entry: the chord length through the hexagon along the ray from
// the source to each point of bin u, averaged over the bin, exact per piece
// between the rays through the vertices (the chord is linear in between).
// Dense, M[(p*nu + u)*(nc*nl) + ic*nl + il]; absent sites stay 0.
void oracle_exact_hex_matrix(int nl, int nc, int np, int nu, double dt, double du, double lsd, double lso,
                             const double* angles, double tol, double* M) {
    Geo g = make_geo(nc, nl, 1, np, nu, 1, dt * std::sqrt(3.0), dt * 0.5, 1, du, 1);
    build_geo(g, lsd, lso, angles, nullptr, nullptr);
    const size_t ncol = (size_t)nc * nl;
    std::memset(M, 0, sizeof(double) * ncol * np * nu);
    const double sdx = dt * std::sqrt(3.0), sdy = 1.5 * dt;
    double vx[6], vy[6];
    for (int k = 0; k < 6; ++k) {
        vx[k] = dt * std::cos(kPI / 6 + k * kPI / 3);
        vy[k] = dt * std::sin(kPI / 6 + k * kPI / 3);
    }
    // chord of the hexagon at o along the line s -> q (Cyrus-Beck clipping
    // against its six edges, counter-clockwise)
    auto chord = [&](const double* s, const double* q, const double* o) {
        double d[2] = {q[0] - s[0], q[1] - s[1]};
        const double len = std::hypot(d[0], d[1]);
        d[0] /= len; d[1] /= len;
        double t0 = -1e300, t1 = 1e300;
        for (int k = 0; k < 6; ++k) {
            const double ax = o[0] + vx[k], ay = o[1] + vy[k];
            const double ex = vx[(k + 1) % 6] - vx[k], ey = vy[(k + 1) % 6] - vy[k];
            // inside: cross(e, X - A) >= 0
            const double num = ex * (s[1] - ay) - ey * (s[0] - ax);
            const double den = ex * d[1] - ey * d[0];
            if (den == 0.0) {
                if (num < 0) return 0.0;
                continue;
            }
            const double t = -num / den;
            if (den > 0) t0 = std::max(t0, t);
            else t1 = std::min(t1, t);
        }
        return t1 > t0 ? t1 - t0 : 0.0;
    };
#pragma omp parallel for schedule(dynamic) collapse(2)
    for (int p = 0; p < np; ++p)
        for (int u = 0; u < nu; ++u) {
            const double* s = &g.src[3 * p];
            const double* dtv = &g.dtv[3 * p];
            const double* pu = &g.puv[3 * p];
            double* row = M + ((size_t)p * nu + u) * ncol;
            double e0[2], e1[2];
            for (int k = 0; k < 2; ++k) {
                e0[k] = dtv[k] + pu[k] * (u - 0.5 * nu) - s[k];
                e1[k] = dtv[k] + pu[k] * (u - 0.5 * nu + 1.0) - s[k];
            }
            const double n0 = std::hypot(e0[0], e0[1]), n1 = std::hypot(e1[0], e1[1]);
            for (int ic = 0; ic < nc; ++ic)
                for (int il = 0; il < nl; ++il) {
                    if ((il & 1) && ic == nc - 1) continue;
                    const double o[2] = {(ic - ((il & 1) ? 0.5 * (nc - 2) : 0.5 * (nc - 1))) * sdx,
                                         (il - 0.5 * (nl - 1)) * sdy};
                    const double r[2] = {o[0] - s[0], o[1] - s[1]};
                    const double c0 = (e0[0] * r[1] - e0[1] * r[0]) / n0, c1 = (e1[0] * r[1] - e1[1] * r[0]) / n1;
                    if ((c0 > dt && c1 > dt) || (c0 < -dt && c1 < -dt)) continue;
                    auto f = [&](double t) {
                        const double q[2] = {dtv[0] + pu[0] * (u - 0.5 * nu + t), dtv[1] + pu[1] * (u - 0.5 * nu + t)};
                        return chord(s, q, o);
                    };
                    std::vector<double> cuts;
                    const double off = u - 0.5 * nu;
                    for (int k = 0; k < 6; ++k) {
                        const double cx = o[0] + vx[k] - s[0], cy = o[1] + vy[k] - s[1];
                        const double den = pu[0] * cy - pu[1] * cx;
                        if (den == 0.0) continue;
                        const double t = -((dtv[0] - s[0]) * cy - (dtv[1] - s[1]) * cx) / den - off;
                        if (t > 0.0 && t < 1.0) cuts.push_back(t);
                    }
                    row[(size_t)ic * nl + il] = integrate_pieces(f, cuts, tol * 2.0 * dt);
                }
        }
}

// Exact fan-beam system matrix of the hexagonal linear element, the basis of
// Hl (layers/A_Hl.cu:168-266): sites on the lattice of H0 with rows 0.5 dt
// apart (:184-193), each carrying the Courant hat of the triangular lattice
// (value 1 at the site, 0 at its six neighbours at distance dt, linear on the
// six triangles): h(X) = max(0, 1 - |X - o|_hex) with |.|_hex the gauge of the
// hexagon of circumradius dt and vertices at 30 + 60 k degrees.  The kernel
// evaluates its X-ray as the univariate box spline of the three lattice
// directions (:21-46).  Entry: the line integral of h along the ray from the
// source to each point of bin u, averaged over the bin; along a ray h is
// linear between the crossings of the six spokes and six edges, across the
// bin the integral is smooth between the rays through the centre and the
// vertices, so each piece is integrated exactly.
// Dense, M[(p*nu + u)*(nc*nl) + ic*nl + il]; absent sites stay 0.
void oracle_exact_hl_matrix(int nl, int nc, int np, int nu, double dt, double du, double lsd, double lso,
                            const double* angles, double tol, double* M) {
    Geo g = make_geo(nc, nl, 1, np, nu, 1, dt * std::sqrt(3.0), dt * 0.5, 1, du, 1);
    build_geo(g, lsd, lso, angles, nullptr, nullptr);
    const size_t ncol = (size_t)nc * nl;
    std::memset(M, 0, sizeof(double) * ncol * np * nu);
    const double sdx = dt * std::sqrt(3.0), sdy = 0.5 * dt, apo = 0.5 * std::sqrt(3.0) * dt;
    double vx[7], vy[7], mx[6], my[6];
    for (int k = 0; k < 6; ++k) {
        vx[k] = dt * std::cos(kPI / 6 + k * kPI / 3);
        vy[k] = dt * std::sin(kPI / 6 + k * kPI / 3);
        mx[k] = std::cos(k * kPI / 3);  // edge normals, between the vertices
        my[k] = std::sin(k * kPI / 3);
    }
    vx[6] = vy[6] = 0.0;  // the centre
    auto hat = [&](double x, double y) {
        double gauge = 0.0;
        for (int k = 0; k < 6; ++k) gauge = std::max(gauge, (x * mx[k] + y * my[k]) / apo);
        return std::max(0.0, 1.0 - gauge);
    };
    // line integral of the hat at o along s -> q: Simpson on the pieces
    // between the crossings of the spokes (centre to vertex) and edges
    auto line = [&](const double* s, const double* q, const double* o) {
        double d[2] = {q[0] - s[0], q[1] - s[1]};
        const double len = std::hypot(d[0], d[1]);
        d[0] /= len; d[1] /= len;
        const double ax = s[0] - o[0], ay = s[1] - o[1];
        // the hexagon's extent along the ray
        double t0 = -1e300, t1 = 1e300;
        for (int k = 0; k < 6; ++k) {
            const double num = apo - (ax * mx[k] + ay * my[k]), den = d[0] * mx[k] + d[1] * my[k];
            if (den == 0.0) {
                if (num < 0) return 0.0;
                continue;
            }
            const double t = num / den;
            if (den > 0) t1 = std::min(t1, t);
            else t0 = std::max(t0, t);
        }
        if (!(t1 > t0)) return 0.0;
        double cut[8];
        int nc2 = 0;
        cut[nc2++] = t0;
        for (int k = 0; k < 6; ++k) {  // spoke k: o + r (vx, vy), r in [0, 1]
            const double den = d[0] * vy[k] - d[1] * vx[k];
            if (den == 0.0) continue;
            const double t = (ay * vx[k] - ax * vy[k]) / den;
            if (t > t0 && t < t1 && nc2 < 7) cut[nc2++] = t;
        }
        cut[nc2++] = t1;
        std::sort(cut, cut + nc2);
        double sum = 0.0;
        for (int k = 0; k + 1 < nc2; ++k) {
            const double a = cut[k], b = cut[k + 1], m = 0.5 * (a + b);
            sum += (b - a) / 6.0 * (hat(ax + a * d[0], ay + a * d[1]) + 4.0 * hat(ax + m * d[0], ay + m * d[1]) +
                                    hat(ax + b * d[0], ay + b * d[1]));
        }
        return sum;
    };
#pragma omp parallel for schedule(dynamic) collapse(2)
    for (int p = 0; p < np; ++p)
        for (int u = 0; u < nu; ++u) {
            const double* s = &g.src[3 * p];
            const double* dtv = &g.dtv[3 * p];
            const double* pu = &g.puv[3 * p];
            double* row = M + ((size_t)p * nu + u) * ncol;
            double e0[2], e1[2];
            for (int k = 0; k < 2; ++k) {
                e0[k] = dtv[k] + pu[k] * (u - 0.5 * nu) - s[k];
                e1[k] = dtv[k] + pu[k] * (u - 0.5 * nu + 1.0) - s[k];
            }
            const double n0 = std::hypot(e0[0], e0[1]), n1 = std::hypot(e1[0], e1[1]);
            for (int ic = 0; ic < nc; ++ic)
                for (int il = 0; il < nl; ++il) {
                    if ((il & 1) && ic == nc - 1) continue;
                    const double o[2] = {(ic - ((il & 1) ? 0.5 * (nc - 2) : 0.5 * (nc - 1))) * sdx,
                                         (il - 0.5 * (nl - 1)) * sdy};
                    const double r[2] = {o[0] - s[0], o[1] - s[1]};
                    const double c0 = (e0[0] * r[1] - e0[1] * r[0]) / n0, c1 = (e1[0] * r[1] - e1[1] * r[0]) / n1;
                    if ((c0 > dt && c1 > dt) || (c0 < -dt && c1 < -dt)) continue;
                    auto f = [&](double t) {
                        const double q[2] = {dtv[0] + pu[0] * (u - 0.5 * nu + t), dtv[1] + pu[1] * (u - 0.5 * nu + t)};
                        return line(s, q, o);
                    };
                    std::vector<double> cuts;
                    const double off = u - 0.5 * nu;
                    for (int k = 0; k < 7; ++k) {
                        const double cx = o[0] + vx[k] - s[0], cy = o[1] + vy[k] - s[1];
                        const double den = pu[0] * cy - pu[1] * cx;
                        if (den == 0.0) continue;
                        const double t = -((dtv[0] - s[0]) * cy - (dtv[1] - s[1]) * cx) / den - off;
                        if (t > 0.0 && t < 1.0) cuts.push_back(t);
                    }
                    row[(size_t)ic * nl + il] = integrate_pieces(f, cuts, tol * dt);
                }
        }
}

// Exact parallel-beam system matrix of the pixel-indicator (kind 0) or
// bilinear (kind 1) basis, dense, M[(p*nu + u)*(nx*ny) + ix*ny + iy]: for
// view angle beta the rays run along (cos beta, sin beta) and bin u covers
// the lateral coordinate s in [(u - nu/2) du, (u - nu/2 + 1) du] along
// (-sin beta, cos beta); the line integral of the basis function averaged
// over the bin by adaptive Simpson (tolerance `tol` relative).  The
// reference has no parallel geometry; this is the checker of the
// parallel-beam B0 layer.
void oracle_exact_parallel_matrix(int kind, int nx, int ny, int np, int nu, double dx, double dy, double du,
                                  const double* angles, double tol, double* M) {
    const size_t ncol = (size_t)nx * ny;
    std::memset(M, 0, sizeof(double) * ncol * np * nu);
    const double reach = kind == 0 ? 0.5 * std::hypot(dx, dy) : std::hypot(dx, dy);
    const double far = 1e4 * (nx * dx + ny * dy);
#pragma omp parallel for schedule(dynamic) collapse(2)
    for (int p = 0; p < np; ++p)
        for (int u = 0; u < nu; ++u) {
            const double rx = std::cos(angles[p]), ry = std::sin(angles[p]), ex = -ry, ey = rx;
            const double s0 = (u - 0.5 * nu) * du, s1 = s0 + du;
            double* row = M + ((size_t)p * nu + u) * ncol;
            for (int ix = 0; ix < nx; ++ix)
                for (int iy = 0; iy < ny; ++iy) {
                    const double o[2] = {(ix - 0.5 * (nx - 1)) * dx, (iy - 0.5 * (ny - 1)) * dy};
                    const double so = o[0] * ex + o[1] * ey;
                    if (so + reach < s0 || so - reach > s1) continue;
                    auto f = [&](double t) {
                        const double s = s0 + t * du;
                        const double a[2] = {s * ex - far * rx, s * ey - far * ry};
                        const double b[2] = {s * ex + far * rx, s * ey + far * ry};
                        return pixel_line_integral(kind, a, b, o, dx, dy);
                    };
                    std::vector<double> bx, by, cuts;
                    basis_breakpoints(kind, o, dx, dy, bx, by);
                    for (size_t k = 0; k < bx.size(); ++k) {
                        const double t = (bx[k] * ex + by[k] * ey - s0) / du;
                        if (t > 0.0 && t < 1.0) cuts.push_back(t);
                    }
                    const double scale = kind == 0 ? std::hypot(dx, dy) : std::max(dx, dy);
                    row[(size_t)ix * ny + iy] = integrate_pieces(f, cuts, tol * scale);
                }
        }
}

// Ref_project_Simpson (layers/Ref_projector.cu:217-367) over a whole volume:
// for every non-zero voxel (x[(iz*ny + iy)*nx + ix]) and view, the detector
// cells its eight corners project onto (ranges ceil(u - 1/2), as SF) receive
// the voxel value times the chord length of the voxel box along the ray from
// the source to points of the cell, averaged over the cell with the 3 x 3
// Simpson rule (adaptive = 0, :330-361) or with the adaptive rule of
// simpson_layer (adaptive = 1: 5 x 5 composite against 3 x 3, Richardson
// correction, recursion into quarter cells to `max_depth`, :156-214).  The
// reference runs voxel (0, 0, z < 64) of views 0, 15, 35, 45 only and takes
// sqrtf of the FP64 chord; this restatement covers every voxel and view in
// FP64.  Cell (i, j) is centred at dtv + (i - nu/2) puv + (j - nv/2) pvv.
void oracle_ref_simpson_3d(int adaptive, int max_depth, double eps, int nx, int ny, int nz, int np, int nu, int nv,
                           double dx, double dy, double dz, double du, double dv, double lsd, double lso,
                           const double* angles, const double* x, double* b) {
    Geo g = make_geo(nx, ny, nz, np, nu, nv, dx, dy, dz, du, dv);
    build_geo(g, lsd, lso, angles, nullptr, nullptr);
    std::memset(b, 0, sizeof(double) * (size_t)np * nu * nv);
    const double d3[3] = {dx, dy, dz};
#pragma omp parallel for schedule(dynamic)
    for (int p = 0; p < np; ++p) {
        const double* s = &g.src[3 * p];
        const double* dt = &g.dtv[3 * p];
        const double* pu = &g.puv[3 * p];
        const double* pv = &g.pvv[3 * p];
        const double* pm = &g.pm[12 * p];
        double* bp = b + (size_t)p * nu * nv;
        for (int iz = 0; iz < nz; ++iz)
            for (int iy = 0; iy < ny; ++iy)
                for (int ix = 0; ix < nx; ++ix) {
                    const double C = x[((size_t)iz * ny + iy) * nx + ix];
                    if (C == 0) continue;
                    const double c1[3] = {-(nx * dx) / 2 + ix * dx, -(ny * dy) / 2 + iy * dy, -(nz * dz) / 2 + iz * dz};
                    // detector coordinates of the eight corners (world-space pm)
                    double umin = INFINITY, umax = -INFINITY, vmin = INFINITY, vmax = -INFINITY;
                    for (int k = 0; k < 8; ++k) {
                        const double w[3] = {c1[0] + (k & 1) * dx, c1[1] + ((k >> 1) & 1) * dy,
                                             c1[2] + ((k >> 2) & 1) * dz};
                        const double h = pm[8] * w[0] + pm[9] * w[1] + pm[10] * w[2] + pm[11];
                        const double uu = (pm[0] * w[0] + pm[1] * w[1] + pm[2] * w[2] + pm[3]) / h;
                        const double vv = (pm[4] * w[0] + pm[5] * w[1] + pm[6] * w[2] + pm[7]) / h;
                        umin = std::min(umin, uu); umax = std::max(umax, uu);
                        vmin = std::min(vmin, vv); vmax = std::max(vmax, vv);
                    }
                    const int i0 = std::max(0, (int)std::ceil(umin - 0.5)), i1 = std::min(nu - 1, (int)std::ceil(umax - 0.5));
                    const int j0 = std::max(0, (int)std::ceil(vmin - 0.5)), j1 = std::min(nv - 1, (int)std::ceil(vmax - 0.5));
                    for (int i = i0; i <= i1; ++i)
                        for (int j = j0; j <= j1; ++j) {
                            double M[3], U[3], V[3];
                            for (int k = 0; k < 3; ++k) {
                                M[k] = dt[k] + (i - 0.5 * nu) * pu[k] + (j - 0.5 * nv) * pv[k];
                                U[k] = 0.5 * pu[k]; V[k] = 0.5 * pv[k];
                            }
                            auto chord = [&](double a, double c) {
                                double q[3] = {M[0] + a * U[0] + c * V[0], M[1] + a * U[1] + c * V[1],
                                               M[2] + a * U[2] + c * V[2]};
                                return chord3(s, q, c1, d3);
                            };
                            double val;
                            if (!adaptive) {
                                val = (chord(-1, -1) + chord(1, -1) + chord(-1, 1) + chord(1, 1) +
                                       4 * (chord(0, -1) + chord(-1, 0) + chord(1, 0) + chord(0, 1)) + 16 * chord(0, 0)) / 36;
                            } else {
                                std::function<double(double, double, double, int)> layer =
                                    [&](double a, double c, double hsz, int depth) -> double {
                                    // 5 x 5 samples at steps hsz/2 around (a, c), cell half-size hsz
                                    double t[5][5];
                                    for (int r = 0; r < 5; ++r)
                                        for (int q = 0; q < 5; ++q)
                                            t[r][q] = chord(a + (r - 2) * 0.5 * hsz, c + (q - 2) * 0.5 * hsz);
                                    const double v3 = (t[0][0] + t[0][4] + t[4][0] + t[4][4] +
                                                       4 * (t[0][2] + t[2][0] + t[2][4] + t[4][2]) + 16 * t[2][2]) / 36;
                                    double q5 = 0;
                                    const double wv[5] = {1, 4, 2, 4, 1};
                                    for (int r = 0; r < 5; ++r)
                                        for (int q = 0; q < 5; ++q) q5 += wv[r] * wv[q] * t[r][q];
                                    q5 /= 144;
                                    if (std::fabs(q5 - v3) <= eps || depth <= 0) return q5 + (q5 - v3) / 15;
                                    const double hh = 0.5 * hsz;
                                    return 0.25 * (layer(a - hh, c - hh, hh, depth - 1) + layer(a + hh, c - hh, hh, depth - 1) +
                                                   layer(a - hh, c + hh, hh, depth - 1) + layer(a + hh, c + hh, hh, depth - 1));
                                };
                                val = layer(0, 0, 1.0, max_depth);
                            }
                            bp[(size_t)j * nu + i] += C * val;
                        }
                }
    }
}

// pixel_matrix_generation (kind 0, layers/A_B0.cu:449-492) and
// bilinear_matrix_generation (kind 1, layers/A_B1.cu:545-593): COO triplets
// (row p*nu + u, col i*ny + j, value) in row-major order over all views, no
// dx*dy factor, entries > 0.  precision 1 evaluates the footprint in float as
// the reference does, 0 in FP64.  Writes at most `cap` entries; returns nnz.
long long oracle_matrix_generation(int kind, int np, int nu, int nx, int ny, double dx, double dy, double du,
                                   double lsd, double lso, int precision, long long cap, long long* rows,
                                   int* cols, double* vals) {
    Geo g = make_geo(nx, ny, 1, np, nu, 1, dx, dy, 0, du, 0);
    build_geo_example(g, lsd, lso);
    std::vector<long long> cnt((size_t)np * nu, 0);
#pragma omp parallel for schedule(dynamic) collapse(2)
    for (int p = 0; p < np; ++p)
        for (int u = 0; u < nu; ++u) {
            long long c = 0;
            auto count = [&](int, double) { ++c; };
            if (precision) generator_row<float>(g, kind, p, u, count); else generator_row<double>(g, kind, p, u, count);
            cnt[(size_t)p * nu + u] = c;
        }
    std::vector<long long> off(cnt.size() + 1, 0);
    for (size_t r = 0; r < cnt.size(); ++r) off[r + 1] = off[r] + cnt[r];
#pragma omp parallel for schedule(dynamic) collapse(2)
    for (int p = 0; p < np; ++p)
        for (int u = 0; u < nu; ++u) {
            long long k = off[(size_t)p * nu + u];
            const long long row = (long long)p * nu + u;
            auto put = [&](int col, double v) {
                if (k < cap) { rows[k] = row; cols[k] = col; vals[k] = v; }
                ++k;
            };
            if (precision) generator_row<float>(g, kind, p, u, put); else generator_row<double>(g, kind, p, u, put);
        }
    return off.back();
}

// b0_forward_projection / b0_backward_projection (layers/A_B0.cu:504-575),
// same host layouts as B1.  FP64 replica (precision 0) or FP32 (1).
long long oracle_b0_forward(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
                            const double* angles, const double* dzs, const double* drho, const double* x, double* b,
                            int precision) {
    Geo g = make_geo(nx, ny, 1, np, nu, 1, dx, dy, 1, du, 1);
    build_geo(g, lsd, lso, angles, dzs, drho);
    std::vector<double> vecs;
    b0_vectors(g, vecs);
    std::memset(b, 0, sizeof(double) * (size_t)np * nu);
    long long total = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : total)
    for (int p = 0; p < np; ++p) {
        double* bp = b + (size_t)p * nu;
        const double* vp = &vecs[(size_t)p * nu * 5];
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                double C = x[(size_t)ix * ny + iy];
                auto visit = [&](int u, double v) { bp[u] += v * C; };
                total += precision ? b0_pixel_view<float>(g, vp, p, ix, iy, visit)
                                   : b0_pixel_view<double>(g, vp, p, ix, iy, visit);
            }
    }
    return total;
}

void oracle_b0_backward(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
                        const double* angles, const double* dzs, const double* drho, const double* b, double* x,
                        int precision) {
    Geo g = make_geo(nx, ny, 1, np, nu, 1, dx, dy, 1, du, 1);
    build_geo(g, lsd, lso, angles, dzs, drho);
    std::vector<double> vecs;
    b0_vectors(g, vecs);
#pragma omp parallel for schedule(dynamic)
    for (int ix = 0; ix < nx; ++ix)
        for (int iy = 0; iy < ny; ++iy) {
            double acc = 0.0;
            for (int p = 0; p < np; ++p) {
                const double* bp = b + (size_t)p * nu;
                const double* vp = &vecs[(size_t)p * nu * 5];
                double val = 0.0;
                auto visit = [&](int u, double v) { val += v * bp[u]; };
                if (precision) b0_pixel_view<float>(g, vp, p, ix, iy, visit);
                else b0_pixel_view<double>(g, vp, p, ix, iy, visit);
                acc += val;
            }
            x[(size_t)ix * ny + iy] = acc;
        }
}

// h0_/hl_ forward and backward (layers/A_H0.cu:565-642, layers/A_Hl.cu:579-656):
// nl rows of nc sites, host layout x[ic*nl + il], b[p*nu + u]; mode as
// hex_site_view.  GeoData(nc, nl, 1, nu, 1, np, dt*sqrt3, dt*0.5, 1, du, 1).
long long oracle_hex_forward(int mode, int nl, int nc, int np, int nu, double dt, double du, double lsd, double lso,
                             const double* angles, const double* x, double* b, int precision) {
    Geo g = make_geo(nc, nl, 1, np, nu, 1, dt * kSQRT3, dt * 0.5f, 1, du, 1);
    build_geo(g, lsd, lso, angles, nullptr, nullptr);
    std::memset(b, 0, sizeof(double) * (size_t)np * nu);
    long long total = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : total)
    for (int p = 0; p < np; ++p) {
        double* bp = b + (size_t)p * nu;
        for (int ic = 0; ic < nc; ++ic)
            for (int il = 0; il < nl; ++il) {
                if ((il & 1) && ic == nc - 1) continue;
                double C = x[(size_t)ic * nl + il];
                auto visit = [&](int u, double v) { bp[u] += v * C; };
                total += precision ? hex_site_view<float>(g, mode, false, p, ic, il, visit)
                                   : hex_site_view<double>(g, mode, false, p, ic, il, visit);
            }
    }
    return total;
}

void oracle_hex_backward(int mode, int nl, int nc, int np, int nu, double dt, double du, double lsd, double lso,
                         const double* angles, const double* b, double* x, int precision) {
    Geo g = make_geo(nc, nl, 1, np, nu, 1, dt * kSQRT3, dt * 0.5f, 1, du, 1);
    build_geo(g, lsd, lso, angles, nullptr, nullptr);
#pragma omp parallel for schedule(dynamic)
    for (int ic = 0; ic < nc; ++ic)
        for (int il = 0; il < nl; ++il) {
            double acc = 0.0;
            if (!((il & 1) && ic == nc - 1))
                for (int p = 0; p < np; ++p) {
                    const double* bp = b + (size_t)p * nu;
                    double val = 0.0;
                    auto visit = [&](int u, double v) { val += v * bp[u]; };
                    if (precision) hex_site_view<float>(g, mode, true, p, ic, il, visit);
                    else hex_site_view<double>(g, mode, true, p, ic, il, visit);
                    acc += val;
                }
            x[(size_t)ic * nl + il] = acc;
        }
}

// SF_forward_projection / SF_backward_projection (layers/A_SF.cu:406-479),
// same host layouts as B1.  FP64 replica (precision 0) or FP32 (1).
// precision: 0 FP64 replica, 1 FP32, 2 FP64 with the chord amplitude
// (sf_pixel_view), not a reference behaviour: the model-error check of the
// reference's amplitude on non-square pixels.
void oracle_sf_forward(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
                       const double* angles, const double* x, double* b, int precision) {
    Geo g = make_geo(nx, ny, 1, np, nu, 1, dx, dy, 1, du, 1);
    build_geo(g, lsd, lso, angles, nullptr, nullptr);
    std::memset(b, 0, sizeof(double) * (size_t)np * nu);
#pragma omp parallel for schedule(dynamic)
    for (int p = 0; p < np; ++p) {
        double* bp = b + (size_t)p * nu;
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                double C = x[(size_t)ix * ny + iy];
                auto visit = [&](int u, double v) { bp[u] += v * C; };
                if (precision == 1) sf_pixel_view<float>(g, p, ix, iy, visit);
                else sf_pixel_view<double>(g, p, ix, iy, visit, precision == 2);
            }
    }
}

void oracle_sf_backward(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
                        const double* angles, const double* b, double* x, int precision) {
    Geo g = make_geo(nx, ny, 1, np, nu, 1, dx, dy, 1, du, 1);
    build_geo(g, lsd, lso, angles, nullptr, nullptr);
#pragma omp parallel for schedule(dynamic)
    for (int ix = 0; ix < nx; ++ix)
        for (int iy = 0; iy < ny; ++iy) {
            double acc = 0.0;
            for (int p = 0; p < np; ++p) {
                const double* bp = b + (size_t)p * nu;
                double val = 0.0;
                auto visit = [&](int u, double v) { val += v * bp[u]; };
                if (precision) sf_pixel_view<float>(g, p, ix, iy, visit); else sf_pixel_view<double>(g, p, ix, iy, visit);
                acc += val;
            }
            x[(size_t)ix * ny + iy] = acc;
        }
}

// Rows of the B1 system matrix for the views listed in `views` (the entries the
// reference's kernels produce, FP64 replica), as COO triplets in row-major
// order: row = k*nu + u for the k-th listed view, col = ix*ny + iy (the column
// convention of layers/A_B1.cu:580-582).  Writes at most `cap` entries and
// returns the count needed (call again with a larger buffer if it exceeds cap).
long long oracle_b1_matrix(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd,
                           double lso, const double* angles, const int* views, int nviews, long long cap,
                           int* rows, int* cols, double* vals) {
    Geo g = make_geo(nx, ny, 1, np, nu, 1, dx, dy, 1, du, 1);
    build_geo(g, lsd, lso, angles, nullptr, nullptr);
    std::vector<float> vecs;
    b1_vectors(g, vecs);
    double dxy = (double)(float)g.dx * (double)(float)g.dy;
    long long n = 0;
    for (int k = 0; k < nviews; ++k) {
        int p = views[k];
        const float* vp = &vecs[(size_t)p * nu * 2];
        std::vector<std::vector<std::pair<int, double>>> byrow(nu);
        for (int ix = 0; ix < nx; ++ix)
            for (int iy = 0; iy < ny; ++iy)
                b1_pixel_view<double>(g, vp, p, ix, iy, [&](int u, double conv) {
                    byrow[u].push_back({ix * ny + iy, conv * dxy});
                });
        for (int u = 0; u < nu; ++u)
            for (auto& e : byrow[u]) {
                if (n < cap) { rows[n] = k * nu + u; cols[n] = e.first; vals[n] = e.second; }
                ++n;
            }
    }
    return n;
}

// Algorithmic FLOPs of the reference B1 formula on this geometry, counted over
// `nviews` views spread evenly over the scan: out[0] = FLOPs of the bin-range
// step per pixel-view, out[1] = FLOPs per footprint evaluation (forward body,
// layers/A_B1.cu:120-206, without the accumulation), out[2] = evaluations per
// pixel-view.
void oracle_b1_flops(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
                     const double* angles, int nviews, double* out) {
    Geo g = make_geo(nx, ny, 1, np, nu, 1, dx, dy, 1, du, 1);
    build_geo(g, lsd, lso, angles, nullptr, nullptr);
    std::vector<float> vecs;
    b1_vectors(g, vecs);
    long long range_flops = 0, eval_flops = 0, evals = 0, pv = 0;
    for (int k = 0; k < nviews; ++k) {
        int p = (int)((long long)k * np / nviews);
        const float* vp = &vecs[(size_t)p * nu * 2];
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                // range alone
                CountedF::flops = 0;
                int minu, maxu;
                bin_range<CountedF>(&g.pmi[12 * p], (float)g.puv[3 * p], std::fabs((float)g.puv[3 * p] - (float)g.puv[3 * p + 1]) < 1e-7f,
                                    ix - 1.0f, ix + 1.0f, iy - 1.0f, iy + 1.0f, nu, minu, maxu);
                long long r = CountedF::flops;
                CountedF::flops = 0;
                long long n = b1_pixel_view<CountedF>(g, vp, p, ix, iy, [](int, double) {});
                range_flops += r;
                eval_flops += CountedF::flops - r;
                evals += n;
                ++pv;
            }
    }
    out[0] = (double)range_flops / pv;
    out[1] = evals ? (double)eval_flops / evals : 0.0;
    out[2] = (double)evals / pv;
}


// Algorithmic FLOPs of the reference formulas of the other 2D projectors,
// counted (+, -, *, /, sqrt) on the path taken over `nviews` evenly spread
// views of every cell: kind 1 A_SF (layers/A_SF.cu:96-225), 2 A_B0
// (layers/A_B0.cu:140-229), 3 A_H0 (layers/A_H0.cu:158-256, the six-vertex
// bound of :84-156 counted as 6 x (4 + 4 + 1)), 4 A_Hl (layers/A_Hl.cu:
// 168-266 with the divided differences of :21-46).  out[0] = FLOPs per
// cell-view (bin range, per-cell terms and every footprint evaluation),
// out[1] = bins visited per cell-view.  For the lattices, nx x ny = nl rows x
// nc sites and dx is the site spacing dt.
void oracle_fan2d_flops(int kind, int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd,
                        double lso, const double* angles, int nviews, double* out) {
    const bool hex = kind == 3 || kind == 4;
    const int nl = nx, nc = ny;
    Geo g = hex ? make_geo(nc, nl, 1, np, nu, 1, dx * kSQRT3, dx * 0.5f, 1, du, 1)
                : make_geo(nx, ny, 1, np, nu, 1, dx, dy, 1, du, 1);
    build_geo(g, lsd, lso, angles, nullptr, nullptr);
    std::vector<double> b0v;
    if (kind == 2) b0_vectors(g, b0v);
    long long total = 0, bins = 0, cells = 0;
    for (int k = 0; k < nviews; ++k) {
        int p = (int)((long long)k * np / nviews);
        const float* pm = &g.pmi[12 * p];
        const float puvx = (float)g.puv[3 * p];
        const bool singular = std::fabs(puvx - (float)g.puv[3 * p + 1]) < 1e-7f;
        for (int i = 0; i < g.nx; ++i)
            for (int j = 0; j < g.ny; ++j) {
                if (hex && (j & 1) && i == g.nx - 1) continue;
                CountedF::flops = 0;
                long long n = 0;
                if (kind == 1 || kind == 2) {
                    int lo, hi;
                    bin_range<CountedF>(pm, puvx, singular, i - 0.5f, i + 0.5f, j - 0.5f, j + 0.5f, g.nu, lo, hi);
                    n = hi - lo + 1;
                    if (kind == 1)
                        sf_pixel_view<CountedF>(g, p, i, j, [](int, double) {});
                    else
                        b0_pixel_view<CountedF>(g, &b0v[(size_t)p * g.nu * 5], p, i, j, [](int, double) {});
                } else {
                    const long long c = hex_site_view<CountedF>(g, kind == 3 ? 1 : 2, false, p, i, j,
                                                                [](int, double) {});
                    CountedF::flops += 54;
                    n = kind == 3 ? c / 3 : 0;
                    if (kind == 4) {  // Hl does not count: bins of the six-vertex range
                        float icc = (float)i + ((j & 1) ? 0.5f : 0.0f);
                        const float oc[6] = {0.0f, 0.5f, 0.5f, 0.0f, -0.5f, -0.5f};
                        const float ol[6] = {-2.0f, -1.0f, 1.0f, 2.0f, 1.0f, -1.0f};
                        float umin = 1e30f, umax = -1e30f;
                        for (int v = 0; v < 6; ++v) {
                            const float u = std::fmaf(pm[0], icc + oc[v], std::fmaf(pm[1], j + ol[v], pm[3])) /
                                            std::fmaf(pm[8], icc + oc[v], std::fmaf(pm[9], j + ol[v], pm[11]));
                            umin = std::min(umin, u);
                            umax = std::max(umax, u);
                        }
                        const int lo = std::min(std::max(0, (int)std::floor(umin)), g.nu - 1);
                        const int hi = std::min(std::max(0, (int)std::floor(umax)), g.nu - 1);
                        n = std::max(hi, lo) - lo + 1;
                    }
                }
                total += CountedF::flops;
                bins += n;
                ++cells;
            }
    }
    out[0] = cells ? (double)total / cells : 0.0;
    out[1] = cells ? (double)bins / cells : 0.0;
}


// Algorithmic FLOPs of the reference's cone-beam formulas, counted (+, -, *,
// /, sqrt) on the path taken over `nviews` evenly spread views and the voxels
// whose ix and iy are multiples of `stride` (every iz): kind 1 the A_B1_3D
// forward (layers/A_B1_3D.cu:82-312: bin ranges, per-voxel weight and axial
// trapezoid, per u the edge-ray footprint, per (u, v) the trapezoid
// integral), kind 2 the SF_projector forward (layers/SF_projector.cu:81-234,
// its amplitude and in-detector bins as the corrected pair evaluates them).
// out[0] = FLOPs per voxel-view, out[1] = (u, v) bins visited per voxel-view.
void oracle_cone_flops(int kind, int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy, double dz,
                       double du, double dv, double lsd, double lso, const double* angles, int nviews, int stride,
                       double* out) {
    Geo g = make_geo(nx, ny, nz, np, nu, nv, dx, dy, dz, du, dv);
    build_geo(g, lsd, lso, angles, nullptr, nullptr);
    std::vector<float> vecs;
    if (kind == 1) b1_vectors(g, vecs);
    if (kind == 2) exact_pmi_geo(g);
    long long total = 0, bins = 0, vv = 0;
    for (int k = 0; k < nviews; ++k) {
        const int p = (int)((long long)k * np / nviews);
        for (int iy = 0; iy < ny; iy += stride)
            for (int ix = 0; ix < nx; ix += stride)
                for (int iz = 0; iz < nz; ++iz) {
                    CountedF::flops = 0;
                    long long n = 0;
                    if (kind == 1)
                        b1_3d_voxel_view<CountedF>(g, &vecs[(size_t)p * nu * 2], 0, p, ix, iy, iz,
                                                   [&](int, int, double) { ++n; });
                    else
                        sf3d_voxel_view<CountedF>(g, lsd, 1, true, false, p, ix, iy, iz, [&](int, double) { ++n; });
                    total += CountedF::flops;
                    bins += n;
                    ++vv;
                }
    }
    out[0] = vv ? (double)total / vv : 0.0;
    out[1] = vv ? (double)bins / vv : 0.0;
}

}  // extern "C"
