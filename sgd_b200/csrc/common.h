// Shared host-side helpers: error reporting across the C ABI, CUDA checks.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdarg>
#include <string>
#include <stdexcept>

namespace sgd {

// Failures never cross the C ABI as C++ exceptions (ctypes would abort).  Each
// entry point catches sgd::Error, stores its text for sgd_last_error() and
// returns a sentinel.
struct Error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void set_last_error(const std::string& msg);
const char* last_error();

[[noreturn]] inline void fail(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    throw Error(buf);
}

inline void check_cuda(cudaError_t e, const char* what, const char* file, int line) {
    if (e != cudaSuccess) fail("%s failed at %s:%d: %s", what, file, line, cudaGetErrorString(e));
}

#define SGD_CUDA(call) ::sgd::check_cuda((call), #call, __FILE__, __LINE__)
#define SGD_LAUNCH_CHECK() ::sgd::check_cuda(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)

// Runs `body`; on sgd::Error (or any std::exception) records the message and
// returns `sentinel`.
template <class R, class F>
R guarded(R sentinel, F&& body) {
    try {
        return body();
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return sentinel;
    }
}

template <class F>
int guarded_status(F&& body) {
    try {
        body();
        return 0;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return -1;
    }
}

}  // namespace sgd
