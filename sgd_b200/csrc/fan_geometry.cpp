#include "fan_geometry.h"

#include <algorithm>
#include <cmath>

#include "common.h"

namespace sgd {

namespace {
const double kPI = 3.14159265358979323846;

inline double cross(double ax, double ay, double bx, double by) { return ax * by - ay * bx; }
}  // namespace

void check_pitches(std::initializer_list<double> pitches) {
    for (double d : pitches)
        if (!(d > 0) || !std::isfinite(d)) fail("pixel, voxel and bin pitches must be positive and finite (got %g)", d);
}

void check_distances(double lsd, double lso) {
    if (!(lso > 0) || !(lsd > lso) || !std::isfinite(lsd)) fail("need 0 < lso < lsd (lso=%g lsd=%g)", lso, lsd);
}

void check_views(int np, const double* angles, const double* dz, const double* drho) {
    if (!angles) fail("angles pointer is null");
    for (int p = 0; p < np; ++p) {
        if (!std::isfinite(angles[p])) fail("angle of view %d is not finite", p);
        if (dz && !std::isfinite(dz[p])) fail("dz of view %d is not finite", p);
        if (drho && !std::isfinite(drho[p])) fail("drho of view %d is not finite", p);
    }
}

std::vector<ViewFrame> view_frames(int np, double lsd, double lso, double du, double dv, const double* angles,
                                   const double* dz, const double* drho) {
    std::vector<ViewFrame> out(np);
    for (int p = 0; p < np; ++p) {
        long double b = angles[p];
        if (std::fabs(std::sin(b) - std::cos(b)) < 1e-7L)
            b = (std::sin(b) > 0) ? kPI / 4 : -kPI * 3 / 4;
        else if (std::fabs(std::sin(b) + std::cos(b)) < 1e-7L)
            b = (std::sin(b) > 0) ? kPI * 3 / 4 : -kPI / 4;
        const double bb = (double)b, c = std::cos(bb), s = std::sin(bb);
        const double v[4][3] = {{-lso + (drho ? drho[p] : 0.0), 0.0, dz ? dz[p] : 0.0},
                                {lsd - lso, 0.0, 0.0},
                                {0.0, du, 0.0},
                                {0.0, 0.0, dv}};
        double* dst[4] = {out[p].src, out[p].dtv, out[p].puv, out[p].pvv};
        for (int k = 0; k < 4; ++k) {  // rotation about z, utils/geo.cu:203-207
            dst[k][0] = v[k][0] * c - v[k][1] * s;
            dst[k][1] = v[k][0] * s + v[k][1] * c;
            dst[k][2] = v[k][2];
        }
    }
    return out;
}

namespace {
// out = a (r x n) times b (n x 4), row-major, sums in index order from 0.0
void mat_mul(const double* a, int r, int n, const double* b, double* out) {
    double t[16];
    for (int i = 0; i < r; ++i)
        for (int j = 0; j < 4; ++j) {
            double acc = 0.0;
            for (int k = 0; k < n; ++k) acc += a[i * n + k] * b[k * 4 + j];
            t[i * 4 + j] = acc;
        }
    for (int i = 0; i < r * 4; ++i) out[i] = t[i];
}
}  // namespace

void reference_pmi(const ViewFrame& f, double uc, double vc, int nx, int ny, int nz, double ddx, double ddy,
                   double ddz, double pm[12], float pmi[12]) {
    const double *src = f.src, *dtv = f.dtv, *puv = f.puv, *pvv = f.pvv;
    // detector normal, and k = n . (D - S): source-to-detector distance along n
    const double n[3] = {puv[1] * pvv[2] - puv[2] * pvv[1], puv[2] * pvv[0] - puv[0] * pvv[2],
                         puv[0] * pvv[1] - puv[1] * pvv[0]};
    double k = 0.0;
    for (int i = 0; i < 3; ++i) k += n[i] * (dtv[i] - src[i]);
    double off[3];
    for (int i = 0; i < 3; ++i) off[i] = src[i] - dtv[i] + (uc * puv[i]) + (vc * pvv[i]) + 1;
    // X -> X - S, -> (X - S, n.(X - S)), scaled by k, shifted to detector
    // corner coordinates, then expressed in the (puv, pvv, 1) basis
    double m[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    const double t1[16] = {1, 0, 0, -src[0], 0, 1, 0, -src[1], 0, 0, 1, -src[2], 0, 0, 0, 1};
    mat_mul(t1, 4, 4, m, m);
    const double t2[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, n[0], n[1], n[2], 0};
    mat_mul(t2, 4, 4, m, m);
    const double t3[16] = {k, 0, 0, 0, 0, k, 0, 0, 0, 0, k, 0, 0, 0, 0, 1};
    mat_mul(t3, 4, 4, m, m);
    const double t4[12] = {1, 0, 0, off[0], 0, 1, 0, off[1], 0, 0, 1, off[2]};
    mat_mul(t4, 3, 4, m, m);
    // inverse of B = [puv pvv 1] by cofactors; identity when |det| < 1e-10
    // (views at odd multiples of 45 degrees, utils/geo.cu:36-41)
    const double B[9] = {puv[0], pvv[0], 1, puv[1], pvv[1], 1, puv[2], pvv[2], 1};
    double Bi[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    const double det = B[0] * ((B[4] * B[8]) - (B[5] * B[7])) - B[1] * ((B[3] * B[8]) - (B[5] * B[6])) +
                       B[2] * ((B[3] * B[7]) - (B[4] * B[6]));
    if (!(std::fabs(det) < 1e-10)) {
        Bi[0] = ((B[4] * B[8]) - (B[5] * B[7])) / det;
        Bi[1] = -1 * ((B[1] * B[8]) - (B[2] * B[7])) / det;
        Bi[2] = ((B[1] * B[5]) - (B[2] * B[4])) / det;
        Bi[3] = -1 * ((B[3] * B[8]) - (B[5] * B[6])) / det;
        Bi[4] = ((B[0] * B[8]) - (B[2] * B[6])) / det;
        Bi[5] = -1 * ((B[0] * B[5]) - (B[2] * B[3])) / det;
        Bi[6] = ((B[3] * B[7]) - (B[4] * B[6])) / det;
        Bi[7] = -1 * ((B[0] * B[7]) - (B[1] * B[6])) / det;
        Bi[8] = ((B[0] * B[4]) - (B[1] * B[3])) / det;
    }
    mat_mul(Bi, 3, 3, m, m);
    for (int i = 0; i < 12; ++i) pm[i] = m[i] / m[11];
    // index space: X = (i dx - ox, j dy - oy, k dz - oz), origin offsets in FP32
    const float dx = (float)ddx, dy = (float)ddy, dz = (float)ddz;
    const float ox = (nx - 1) * dx / 2.0f, oy = (ny - 1) * dy / 2.0f, oz = (nz - 1) * dz / 2.0f;
    for (int r = 0; r < 3; ++r) {
        const double* q = pm + 4 * r;
        pmi[4 * r + 0] = dx * q[0];
        pmi[4 * r + 1] = dy * q[1];
        pmi[4 * r + 2] = dz * q[2];
        pmi[4 * r + 3] = q[3] - ox * q[0] - oy * q[1] - oz * q[2];
    }
}

void FanGeometry::init(int nx_, int ny_, int np_, int nu_, double dx_, double dy_, double du_, double lsd_,
                       double lso_, const double* angles, const double* dz, const double* drho) {
    if (nx_ <= 0 || ny_ <= 0 || np_ <= 0 || nu_ <= 0) fail("invalid sizes nx=%d ny=%d np=%d nu=%d", nx_, ny_, np_, nu_);
    check_pitches({dx_, dy_, du_});
    check_distances(lsd_, lso_);
    check_views(np_, angles, dz, drho);
    nx = nx_; ny = ny_; np = np_; nu = nu_;
    dx = dx_; dy = dy_; du = du_; lsd = lsd_; lso = lso_;
    beta.resize(np); src.resize(2 * np); dtv.resize(2 * np); puv.resize(2 * np);
    for (int p = 0; p < np; ++p) {
        // utils/geo.cu:241-257: the snap test runs in long double.
        long double b = angles[p];
        if (std::fabs(std::sin(b) - std::cos(b)) < 1e-7L)
            b = (std::sin(b) > 0) ? kPI / 4 : -kPI * 3 / 4;
        else if (std::fabs(std::sin(b) + std::cos(b)) < 1e-7L)
            b = (std::sin(b) > 0) ? kPI * 3 / 4 : -kPI / 4;
        double bb = (double)b;
        double c = std::cos(bb), s = std::sin(bb);
        double sx = -lso + (drho ? drho[p] : 0.0);
        beta[p] = bb;
        src[2 * p] = sx * c;                 // rotate((sx, 0), beta)
        src[2 * p + 1] = sx * s;
        dtv[2 * p] = (lsd - lso) * c;
        dtv[2 * p + 1] = (lsd - lso) * s;
        puv[2 * p] = -du * s;                // rotate((0, du), beta)
        puv[2 * p + 1] = du * c;
    }
    // 2D layers use nz = nv = 1 and dz = dv = 1 (layers/A_B1.cu:596)
    frames = view_frames(np, lsd, lso, du, 1.0, angles, dz, drho);
    pmi.resize(12 * (size_t)np);
    for (int p = 0; p < np; ++p) {
        double pm[12];
        reference_pmi(frames[p], nu / 2.0, 0.5, nx, ny, 1, dx, dy, 1.0, pm, &pmi[12 * (size_t)p]);
    }
}

void bin_homographies(const FanGeometry& g, std::vector<BinHomography>& out) {
    out.resize(g.np);
    for (int p = 0; p < g.np; ++p) {
        double px = g.src[2 * p], py = g.src[2 * p + 1];
        double Dx = g.dtv[2 * p], Dy = g.dtv[2 * p + 1];
        double ex = g.puv[2 * p], ey = g.puv[2 * p + 1];
        // s = cross(P - D, X - P) / cross(e, X - P), X = (x0 + i dx, y0 + j dy);
        // u = s + nu/2.
        double ax = px - Dx, ay = py - Dy;
        // cross(a, X - P) = ax (Xy - py) - ay (Xx - px)
        double n0 = -ay * g.dx, n1 = ax * g.dy, n2 = ax * (g.y0() - py) - ay * (g.x0() - px);
        double d0 = -ey * g.dx, d1 = ex * g.dy, d2 = ex * (g.y0() - py) - ey * (g.x0() - px);
        double h = 0.5 * g.nu;
        BinHomography& H = out[p];
        H.n0 = (float)(n0 + h * d0);
        H.n1 = (float)(n1 + h * d1);
        H.n2 = (float)(n2 + h * d2);
        H.d0 = (float)d0;
        H.d1 = (float)d1;
        H.d2 = (float)d2;
        H.pad0 = H.pad1 = 0.f;
    }
}

void b1_profile_constants(double a, double b, float* r) {
    if (b <= 1e-7) b = 0.0;  // single-triangle limit
    r[6] = r[7] = (float)b;
    r[8] = r[9] = (float)a;
    r[10] = r[11] = (float)(a + b);
    r[12] = (float)(1.0 / a);
    r[13] = (float)(1.0 / (2.0 * a * a));
    r[14] = -(float)(b * b / (12.0 * a * a));
    r[15] = b > 0 ? (float)(1.0 / (12.0 * a * a * b * b)) : 0.f;
}

void b1_unit_profile_constants(double a, double b, float* r) {
    if (b <= 1e-7) b = 0.0;  // single-triangle limit
    const double beta = b / a;
    r[6] = r[7] = (float)beta;
    r[8] = r[9] = (float)(1.0 + beta);
    r[10] = r[11] = (float)(-beta * beta / 12.0);
    r[12] = r[13] = beta > 0 ? (float)(1.0 / (12.0 * beta * beta)) : 0.f;
    r[14] = (float)(1.0 / a);
    r[15] = (float)a;
}

void b1_tables(const FanGeometry& g, std::vector<float>& rec, std::vector<float>& strip) {
    const int np = g.np, nu = g.nu;
    rec.assign((size_t)np * nu * kB1Rec, 0.f);
    strip.assign((size_t)np * nu * kStripRec, 0.f);
    const double x0 = g.x0(), y0 = g.y0();
    for (int p = 0; p < np; ++p) {
        const double px = g.src[2 * p], py = g.src[2 * p + 1];
        const double Dx = g.dtv[2 * p], Dy = g.dtv[2 * p + 1];
        const double ex = g.puv[2 * p], ey = g.puv[2 * p + 1];
        for (int u = 0; u < nu; ++u) {
            const double off = u - 0.5 * nu + 0.5;
            const double sx = Dx + ex * off, sy = Dy + ey * off;
            const double ax = sx - 0.5 * ex, ay = sy - 0.5 * ey;
            const double bx = sx + 0.5 * ex, by = sy + 0.5 * ey;
            double dxr = sx - px, dyr = sy - py;
            const double L = std::sqrt(dxr * dxr + dyr * dyr);
            const double tx = dxr / L, ty = dyr / L;  // central-ray unit vector
            const double nxv = -ty, nyv = tx;         // lateral unit vector
            // edge ray slopes relative to the central ray: k = ((E-P).n) / ((E-P).t)
            const double ka = ((ax - px) * nxv + (ay - py) * nyv) / ((ax - px) * tx + (ay - py) * ty);
            const double kb = ((bx - px) * nxv + (by - py) * nyv) / ((bx - px) * tx + (by - py) * ty);
            // x_E(O) = t k_E - q = (O - P).(k_E t - n)
            const double mAx = ka * tx - nxv, mAy = ka * ty - nyv;
            const double mBx = kb * tx - nxv, mBy = kb * ty - nyv;
            // profile half-widths (layers/A_B1.cu:429-478): vx = |dx cos(theta)|,
            // vy = |dy sin(theta)| with theta = atan2(|px - sx|, |py - sy|);
            // offsets are stored in units of a
            const double vx = std::fabs(g.dx * ty), vy = std::fabs(g.dy * tx);
            const double a = std::max(vx, vy);
            float r[kB1Rec];
            r[0] = (float)(mAx * g.dx / a);
            r[1] = (float)(mBx * g.dx / a);
            r[2] = (float)(mAy * g.dy / a);
            r[3] = (float)(mBy * g.dy / a);
            r[4] = (float)(((x0 - px) * mAx + (y0 - py) * mAy) / a);
            r[5] = (float)(((x0 - px) * mBx + (y0 - py) * mBy) / a);
            b1_unit_profile_constants(a, std::min(vx, vy), r);
            for (int q = 0; q < 4; ++q)
                for (int k = 0; k < 4; ++k) rec[(((size_t)p * 4 + q) * nu + u) * 4 + k] = r[4 * q + k];

            // strip of the bin in index space for the forward kernel
            float* s = &strip[((size_t)p * nu + u) * kStripRec];
            const bool ydom = std::fabs(ty) >= std::fabs(tx);
            if (ydom) {
                // i(j) where the edge ray crosses row j: x = px + (y - py) (Ex - px)/(Ey - py)
                const double sa = (ax - px) / (ay - py), sb = (bx - px) / (by - py);
                s[0] = (float)((px + (y0 - py) * sa - x0) / g.dx);
                s[1] = (float)(sa * g.dy / g.dx);
                s[2] = (float)((px + (y0 - py) * sb - x0) / g.dx);
                s[3] = (float)(sb * g.dy / g.dx);
            } else {
                const double sa = (ay - py) / (ax - px), sb = (by - py) / (bx - px);
                s[0] = (float)((py + (x0 - px) * sa - y0) / g.dy);
                s[1] = (float)(sa * g.dx / g.dy);
                s[2] = (float)((py + (x0 - px) * sb - y0) / g.dy);
                s[3] = (float)(sb * g.dx / g.dy);
            }
            s[4] = ydom ? 1.f : 0.f;
        }
    }
}

void exact_pmi(const ViewFrame& f, double uc, double vc, int nx, int ny, int nz, double dx, double dy, double dz,
               float pmi[12]) {
    const double* S = f.src;
    const double* D = f.dtv;
    const double* eu = f.puv;
    const double* ev = f.pvv;
    const double n[3] = {eu[1] * ev[2] - eu[2] * ev[1], eu[2] * ev[0] - eu[0] * ev[2], eu[0] * ev[1] - eu[1] * ev[0]};
    auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    const double uu = dot(eu, eu), vv = dot(ev, ev);
    double SD[3], DS[3];
    for (int k = 0; k < 3; ++k) { SD[k] = S[k] - D[k]; DS[k] = -SD[k]; }
    // ray S -> X meets the detector at P = S + t (X - S), t = n.(D - S) / n.(X - S):
    // (P - D).e/|e|^2 times w = n.(X - S) is linear in X
    double rows[3][4];
    for (int k = 0; k < 3; ++k) {
        rows[0][k] = dot(eu, SD) / uu * n[k] + dot(n, DS) * eu[k] / uu;
        rows[1][k] = dot(ev, SD) / vv * n[k] + dot(n, DS) * ev[k] / vv;
        rows[2][k] = n[k];
    }
    for (int r = 0; r < 3; ++r) rows[r][3] = -(rows[r][0] * S[0] + rows[r][1] * S[1] + rows[r][2] * S[2]);
    for (int k = 0; k < 4; ++k) {
        rows[0][k] += uc * rows[2][k];
        rows[1][k] += vc * rows[2][k];
    }
    // voxel indices -> world: x = (i - (nx-1)/2) dx, ...
    const double x0 = -0.5 * (nx - 1) * dx, y0 = -0.5 * (ny - 1) * dy, z0 = -0.5 * (nz - 1) * dz;
    double m[12];
    for (int r = 0; r < 3; ++r) {
        m[4 * r + 0] = rows[r][0] * dx;
        m[4 * r + 1] = rows[r][1] * dy;
        m[4 * r + 2] = rows[r][2] * dz;
        m[4 * r + 3] = rows[r][3] + rows[r][0] * x0 + rows[r][1] * y0 + rows[r][2] * z0;
    }
    for (int k = 0; k < 12; ++k) pmi[k] = (float)(m[k] / m[11]);
}

}  // namespace sgd
