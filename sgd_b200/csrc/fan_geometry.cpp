#include "fan_geometry.h"

#include <algorithm>
#include <cmath>

#include "common.h"

namespace sgd {

namespace {
const double kPI = 3.14159265358979323846;

inline double cross(double ax, double ay, double bx, double by) { return ax * by - ay * bx; }
}  // namespace

void FanGeometry::init(int nx_, int ny_, int np_, int nu_, double dx_, double dy_, double du_, double lsd_,
                       double lso_, const double* angles, const double* /*dz*/, const double* drho) {
    if (nx_ <= 0 || ny_ <= 0 || np_ <= 0 || nu_ <= 0) fail("invalid sizes nx=%d ny=%d np=%d nu=%d", nx_, ny_, np_, nu_);
    if (!(dx_ > 0) || !(dy_ > 0) || !(du_ > 0)) fail("pixel and bin pitches must be positive");
    if (!(lso_ > 0) || !(lsd_ > lso_)) fail("need 0 < lso < lsd (lso=%g lsd=%g)", lso_, lsd_);
    if (!angles) fail("angles pointer is null");
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
    r[6] = (float)a;
    r[7] = (float)b;
    r[8] = (float)(a + b);
    r[9] = (float)(a - b);
    r[10] = (float)(1.0 / a);
    r[11] = (float)(1.0 / (2.0 * a * a));
    r[12] = (float)(b * b / (12.0 * a * a));
    r[13] = b > 0 ? (float)(1.0 / (12.0 * a * a * b * b)) : 0.f;
    r[14] = b > 0 ? (float)(1.0 / (24.0 * a * a * b * b)) : 0.f;
    r[15] = 0.f;
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
            float r[kB1Rec];
            r[0] = (float)(mAx * g.dx);
            r[1] = (float)(mAy * g.dy);
            r[2] = (float)((x0 - px) * mAx + (y0 - py) * mAy);
            r[3] = (float)(mBx * g.dx);
            r[4] = (float)(mBy * g.dy);
            r[5] = (float)((x0 - px) * mBx + (y0 - py) * mBy);
            // profile half-widths (layers/A_B1.cu:429-478): vx = |dx cos(theta)|,
            // vy = |dy sin(theta)| with theta = atan2(|px - sx|, |py - sy|)
            const double vx = std::fabs(g.dx * ty), vy = std::fabs(g.dy * tx);
            b1_profile_constants(std::max(vx, vy), std::min(vx, vy), r);
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

}  // namespace sgd
