// extern "C" entry points of the B1 projector.  Names and signatures of the
// reference ones are kept (layers/A_B1.hh:23-27); see include/sgd_b200.h.
#include <cuda_runtime.h>

#include "b1_layer.h"
#include "common.h"

using sgd::A_B1;

extern "C" {

const char* sgd_last_error() { return sgd::last_error(); }

void* b1_init(int nx, int ny, int np, int nu, double dx, double dy, double du, double lsd, double lso,
              double* angles, double* dz, double* drho) {
    return sgd::guarded<void*>(nullptr, [&]() -> void* {
        return new A_B1(nx, ny, np, nu, dx, dy, du, lsd, lso, angles, dz, drho);
    });
}

void b1_destroy(void* layer) { delete static_cast<A_B1*>(layer); }

int b1_forward_projection(double* b, double* x, void* layer) {
    return sgd::guarded<int>(-1, [&]() -> int {
        if (!layer || !b || !x) sgd::fail("b1_forward_projection: null argument");
        A_B1* L = static_cast<A_B1*>(layer);
        L->forward_host(b, x);
        return (int)L->count;
    });
}

void b1_backward_projection(double* b, double* x, void* layer) {
    sgd::guarded_status([&] {
        if (!layer || !b || !x) sgd::fail("b1_backward_projection: null argument");
        static_cast<A_B1*>(layer)->backward_host(b, x);
    });
}

int sgd_b1_backward_projection(double* b, double* x, void* layer) {
    return sgd::guarded_status([&] {
        if (!layer || !b || !x) sgd::fail("sgd_b1_backward_projection: null argument");
        static_cast<A_B1*>(layer)->backward_host(b, x);
    });
}

int sgd_b1_forward_dev(void* layer, const float* d_img, float* d_sino, void* stream) {
    return sgd::guarded_status([&] {
        if (!layer || !d_img || !d_sino) sgd::fail("sgd_b1_forward_dev: null argument");
        static_cast<A_B1*>(layer)->forward_dev(d_img, d_sino, static_cast<cudaStream_t>(stream));
    });
}

int sgd_b1_backward_dev(void* layer, const float* d_sino, float* d_img, void* stream) {
    return sgd::guarded_status([&] {
        if (!layer || !d_img || !d_sino) sgd::fail("sgd_b1_backward_dev: null argument");
        static_cast<A_B1*>(layer)->backward_dev(d_sino, d_img, static_cast<cudaStream_t>(stream));
    });
}

int sgd_b1_status(void* layer) {
    return sgd::guarded_status([&] {
        if (!layer) sgd::fail("sgd_b1_status: null layer");
        static_cast<A_B1*>(layer)->check_device_status();
    });
}

int sgd_b1_set_wait_limit(void* layer, unsigned polls) {
    return sgd::guarded_status([&] {
        if (!layer) sgd::fail("sgd_b1_set_wait_limit: null layer");
        static_cast<A_B1*>(layer)->dev.wait_limit = polls;
    });
}

unsigned long long sgd_b1_count(void* layer) {
    return layer ? static_cast<A_B1*>(layer)->count : 0ull;
}

}  // extern "C"
