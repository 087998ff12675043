// extern "C" entry points of the generic 2D projectors (A_SF, B0, H0, Hl).
// Names and signatures of the reference ones are kept; see include/sgd_b200.h.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "common.h"
#include "proj2d.h"

namespace sgd {
Proj2D* make_sf_layer(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
                      const double* angles);
Proj2D* make_b0_layer(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
                      const double* angles, const double* dz, const double* drho);
Proj2D* make_b0_parallel_layer(int nx, int ny, int np, int nu, double dx, double dy, double du,
                               const double* angles);
Proj2D* make_hex_layer(int mode, int nl, int nc, int np, int nu, double dt, double du, double lsd, double lso,
                       const double* angles, const double* dz, const double* drho);
Proj2D* make_b1ref_layer(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
                         const double* angles, const double* dz, const double* drho);
}

using sgd::Proj2D;

namespace {
int fwd_host(double* b, double* x, void* layer, const char* what) {
    return sgd::guarded<int>(-1, [&]() -> int {
        if (!layer || !b || !x) sgd::fail("%s: null argument", what);
        Proj2D* L = static_cast<Proj2D*>(layer);
        L->forward_host(b, x);
        return (int)L->count;
    });
}
int bwd_host(double* b, double* x, void* layer, const char* what) {
    return sgd::guarded_status([&] {
        if (!layer || !b || !x) sgd::fail("%s: null argument", what);
        static_cast<Proj2D*>(layer)->backward_host(b, x);
    });
}
int fwd_dev(void* layer, const float* img, float* sino, void* stream, const char* what) {
    return sgd::guarded_status([&] {
        if (!layer || !img || !sino) sgd::fail("%s: null argument", what);
        static_cast<Proj2D*>(layer)->forward_dev(img, sino, static_cast<cudaStream_t>(stream));
    });
}
int bwd_dev(void* layer, const float* sino, float* img, void* stream, const char* what) {
    return sgd::guarded_status([&] {
        if (!layer || !img || !sino) sgd::fail("%s: null argument", what);
        static_cast<Proj2D*>(layer)->backward_dev(sino, img, static_cast<cudaStream_t>(stream));
    });
}
long long matrix_csr(void* layer, long long* rowptr, int* cols, double* vals, long long cap, const char* what) {
    return sgd::guarded<long long>(-1, [&]() -> long long {
        if (!layer) sgd::fail("%s: null layer", what);
        if ((rowptr || cols || vals) && !(rowptr && cols && vals)) sgd::fail("%s: partial output", what);
        sgd::CsrOut out;
        out.rowptr = rowptr; out.cols = cols; out.vals = vals; out.cap = cap;
        return static_cast<Proj2D*>(layer)->csr(out);
    });
}
}  // namespace

extern "C" {

void* SF_init(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
              double* angles) {
    return sgd::guarded<void*>(nullptr, [&]() -> void* {
        return sgd::make_sf_layer(nx, ny, np, nu, dx, dy, du, lsd, lso, angles);
    });
}
int SF_forward_projection(double* b, double* x, void* layer) { return fwd_host(b, x, layer, "SF_forward_projection"); }
void SF_backward_projection(double* b, double* x, void* layer) { bwd_host(b, x, layer, "SF_backward_projection"); }
int sgd_SF_backward_projection(double* b, double* x, void* layer) {
    return bwd_host(b, x, layer, "SF_backward_projection");
}
void SF_destroy(void* layer) { delete static_cast<Proj2D*>(layer); }
int sgd_SF_forward_dev(void* layer, const float* d_img, float* d_sino, void* stream) {
    return fwd_dev(layer, d_img, d_sino, stream, "sgd_SF_forward_dev");
}
int sgd_SF_backward_dev(void* layer, const float* d_sino, float* d_img, void* stream) {
    return bwd_dev(layer, d_sino, d_img, stream, "sgd_SF_backward_dev");
}
unsigned long long sgd_SF_count(void* layer) { return layer ? static_cast<Proj2D*>(layer)->count : 0ull; }

void* b0_init(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
              double* angles, double* dz, double* drho) {
    return sgd::guarded<void*>(nullptr, [&]() -> void* {
        return sgd::make_b0_layer(nx, ny, np, nu, dx, dy, du, lsd, lso, angles, dz, drho);
    });
}
int b0_forward_projection(double* b, double* x, void* layer) { return fwd_host(b, x, layer, "b0_forward_projection"); }
void b0_backward_projection(double* b, double* x, void* layer) { bwd_host(b, x, layer, "b0_backward_projection"); }
int sgd_b0_backward_projection(double* b, double* x, void* layer) {
    return bwd_host(b, x, layer, "b0_backward_projection");
}
void b0_destroy(void* layer) { delete static_cast<Proj2D*>(layer); }
int sgd_b0_forward_dev(void* layer, const float* d_img, float* d_sino, void* stream) {
    return fwd_dev(layer, d_img, d_sino, stream, "sgd_b0_forward_dev");
}
int sgd_b0_backward_dev(void* layer, const float* d_sino, float* d_img, void* stream) {
    return bwd_dev(layer, d_sino, d_img, stream, "sgd_b0_backward_dev");
}
unsigned long long sgd_b0_count(void* layer) { return layer ? static_cast<Proj2D*>(layer)->count : 0ull; }

void* sgd_hex_init(int mode, int nl, int nc, int np, int nu, double dt, double du, double lsd, double lso,
                   double* angles, double* dz, double* drho) {
    return sgd::guarded<void*>(nullptr, [&]() -> void* {
        if (mode < 0 || mode > 2) sgd::fail("sgd_hex_init: mode must be 0, 1 or 2");
        return sgd::make_hex_layer(mode, nl, nc, np, nu, dt, du, lsd, lso, angles, dz, drho);
    });
}
void* h0_init(int nl, int nc, int np, int nu, double dt, double du, double lsd, double lso, double* angles,
              double* dz, double* drho) {
    return sgd_hex_init(1, nl, nc, np, nu, dt, du, lsd, lso, angles, dz, drho);
}
void* hl_init(int nl, int nc, int np, int nu, double dt, double du, double lsd, double lso, double* angles,
              double* dz, double* drho) {
    return sgd_hex_init(2, nl, nc, np, nu, dt, du, lsd, lso, angles, dz, drho);
}
int h0_forward_projection(double* b, double* x, void* layer) { return fwd_host(b, x, layer, "h0_forward_projection"); }
void h0_backward_projection(double* b, double* x, void* layer) { bwd_host(b, x, layer, "h0_backward_projection"); }
int hl_forward_projection(double* b, double* x, void* layer) { return fwd_host(b, x, layer, "hl_forward_projection"); }
void hl_backward_projection(double* b, double* x, void* layer) { bwd_host(b, x, layer, "hl_backward_projection"); }
int sgd_h0_backward_projection(double* b, double* x, void* layer) {
    return bwd_host(b, x, layer, "h0_backward_projection");
}
int sgd_hl_backward_projection(double* b, double* x, void* layer) {
    return bwd_host(b, x, layer, "hl_backward_projection");
}
void h0_destroy(void* layer) { delete static_cast<Proj2D*>(layer); }
void hl_destroy(void* layer) { delete static_cast<Proj2D*>(layer); }
int sgd_h0_forward_dev(void* layer, const float* d_img, float* d_sino, void* stream) {
    return fwd_dev(layer, d_img, d_sino, stream, "sgd_h0_forward_dev");
}
int sgd_h0_backward_dev(void* layer, const float* d_sino, float* d_img, void* stream) {
    return bwd_dev(layer, d_sino, d_img, stream, "sgd_h0_backward_dev");
}
int sgd_hl_forward_dev(void* layer, const float* d_img, float* d_sino, void* stream) {
    return fwd_dev(layer, d_img, d_sino, stream, "sgd_hl_forward_dev");
}
int sgd_hl_backward_dev(void* layer, const float* d_sino, float* d_img, void* stream) {
    return bwd_dev(layer, d_sino, d_img, stream, "sgd_hl_backward_dev");
}
unsigned long long sgd_h0_count(void* layer) { return layer ? static_cast<Proj2D*>(layer)->count : 0ull; }
unsigned long long sgd_hl_count(void* layer) { return layer ? static_cast<Proj2D*>(layer)->count : 0ull; }

// B0 in parallel-beam geometry; the handle takes the b0_* / sgd_b0_* calls.
void* sgd_b0_parallel_init(int nx, int ny, int np, int nu, double dx, double dy, double du, double* angles) {
    return sgd::guarded<void*>(nullptr, [&]() -> void* {
        return sgd::make_b0_parallel_layer(nx, ny, np, nu, dx, dy, du, angles);
    });
}

// B1 in the reference's FP32 rounding (b1ref.cu).
void* sgd_b1ref_init(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
                     double* angles, double* dz, double* drho) {
    return sgd::guarded<void*>(nullptr, [&]() -> void* {
        return sgd::make_b1ref_layer(nx, ny, np, nu, dx, dy, du, lsd, lso, angles, dz, drho);
    });
}
int sgd_b1ref_forward_projection(double* b, double* x, void* layer) {
    return fwd_host(b, x, layer, "sgd_b1ref_forward_projection");
}
int sgd_b1ref_backward_projection(double* b, double* x, void* layer) {
    return bwd_host(b, x, layer, "sgd_b1ref_backward_projection");
}
void sgd_b1ref_destroy(void* layer) { delete static_cast<Proj2D*>(layer); }
int sgd_b1ref_forward_dev(void* layer, const float* d_img, float* d_sino, void* stream) {
    return fwd_dev(layer, d_img, d_sino, stream, "sgd_b1ref_forward_dev");
}
int sgd_b1ref_backward_dev(void* layer, const float* d_sino, float* d_img, void* stream) {
    return bwd_dev(layer, d_sino, d_img, stream, "sgd_b1ref_backward_dev");
}
unsigned long long sgd_b1ref_count(void* layer) { return layer ? static_cast<Proj2D*>(layer)->count : 0ull; }
long long sgd_b1ref_matrix_csr(void* layer, long long* rowptr, int* cols, double* vals, long long cap) {
    return matrix_csr(layer, rowptr, cols, vals, cap, "sgd_b1ref_matrix_csr");
}

// Host-only plan of the generic kernels for a grid of nx x ny cells in the
// fan geometry of b1_init (np views at `angles`, nu bins of pitch du, source
// and detector distances lso, lsd): cell (i, j) at x = x0 + i dx,
// y = y0 + j dy, with bin ranges from points within ri, rj cells of it.
// Strips [np][ceil(nu/32)][8] floats, windows [tiles][np][2] ints (tiles of
// 8 x 32 cells).  Returns the widest window, or -1 (sgd_last_error()).
int sgd_fan2d_plan(int nx, int ny, int np, int nu, double x0, double dx, double y0, double dy, double ri, double rj,
                   double du, double lsd, double lso, const double* angles, float* strips, int* twin) {
    return sgd::guarded<int>(-1, [&]() -> int {
        if (!angles || !strips || !twin) sgd::fail("sgd_fan2d_plan: null argument");
        if (!(ri >= 0.0) || !(rj >= 0.0)) sgd::fail("sgd_fan2d_plan: negative reach");
        sgd::FanGeometry g;
        g.init(nx, ny, np, nu, dx, dy, du, lsd, lso, angles, nullptr, nullptr);
        std::vector<float4> st;
        std::vector<int2> tw;
        const int w = sgd::plan_fan2d(nx, ny, np, nu, [&](int p) {
            double hw[6];
            sgd::fan_world_hom(g, p, hw);
            return sgd::grid_range_map(hw, x0, dx, y0, dy, ri, rj);
        }, st, tw);
        std::memcpy(strips, st.data(), st.size() * sizeof(float4));
        std::memcpy(twin, tw.data(), tw.size() * sizeof(int2));
        return w;
    });
}

int sgd_proj2d_set_wait_limit(void* layer, unsigned polls) {
    return sgd::guarded_status([&] {
        if (!layer) sgd::fail("sgd_proj2d_set_wait_limit: null layer");
        static_cast<Proj2D*>(layer)->P.wait_limit = polls;
    });
}

int sgd_proj2d_status(void* layer) {
    return sgd::guarded_status([&] {
        if (!layer) sgd::fail("sgd_proj2d_status: null layer");
        if (static_cast<Proj2D*>(layer)->status() != 0)
            sgd::fail("back projection: a staged view chunk did not arrive within the bounded wait; "
                      "the affected tiles were left unwritten");
    });
}

long long sgd_SF_matrix_csr(void* layer, long long* rowptr, int* cols, double* vals, long long cap) {
    return matrix_csr(layer, rowptr, cols, vals, cap, "sgd_SF_matrix_csr");
}
long long sgd_b0_matrix_csr(void* layer, long long* rowptr, int* cols, double* vals, long long cap) {
    return matrix_csr(layer, rowptr, cols, vals, cap, "sgd_b0_matrix_csr");
}
long long sgd_h0_matrix_csr(void* layer, long long* rowptr, int* cols, double* vals, long long cap) {
    return matrix_csr(layer, rowptr, cols, vals, cap, "sgd_h0_matrix_csr");
}
long long sgd_hl_matrix_csr(void* layer, long long* rowptr, int* cols, double* vals, long long cap) {
    return matrix_csr(layer, rowptr, cols, vals, cap, "sgd_hl_matrix_csr");
}

}  // extern "C"
