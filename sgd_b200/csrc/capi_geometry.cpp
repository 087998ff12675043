// Host-only geometry entry point (no GPU needed): the per-view projection
// matrices the kernels use, for inspection and for the CPU tests.
#include <cstring>

#include "common.h"
#include "fan_geometry.h"

extern "C" int sgd_geometry_pmi(int nx, int ny, int nz, int np, int nu, int nv, double dx, double dy, double dz,
                                double du, double dv, double lsd, double lso, const double* angles,
                                const double* dz_off, const double* drho, double* pm_out, float* pmi_out) {
    return sgd::guarded_status([&] {
        if (np <= 0 || !angles || !pmi_out) sgd::fail("sgd_geometry_pmi: bad arguments");
        const std::vector<sgd::ViewFrame> f = sgd::view_frames(np, lsd, lso, du, dv, angles, dz_off, drho);
        for (int p = 0; p < np; ++p) {
            double pm[12];
            sgd::reference_pmi(f[p], nu / 2.0, nv / 2.0, nx, ny, nz, dx, dy, dz, pm, pmi_out + 12 * (size_t)p);
            if (pm_out) std::memcpy(pm_out + 12 * (size_t)p, pm, sizeof(pm));
        }
    });
}

extern "C" int sgd_b1_bin_records(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd,
                                  double lso, const double* angles, const double* dz, const double* drho,
                                  float* rec_out) {
    return sgd::guarded_status([&] {
        if (!rec_out) sgd::fail("sgd_b1_bin_records: null output");
        sgd::FanGeometry g;
        g.init(nx, ny, np, nu, dx, dy, du, lsd, lso, angles, dz, drho);
        std::vector<float> rec, strip;
        sgd::b1_tables(g, rec, strip);
        std::memcpy(rec_out, rec.data(), rec.size() * sizeof(float));
    });
}
