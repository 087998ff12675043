// Host + device FP64 buffer with the interface of the reference's MatrixD
// (utils/matrix_double.hh:7-36): operator[] is the host pointer, operator()
// the device pointer.  Kept so C++ callers of project/back_project
// (SGD.cu:176-187, Bilinear.cu:25-39 in the reference) compile against this
// library by including reference_compat.h, which names the classes in the
// global namespace as the reference does.  Errors throw sgd::Error instead of
// NNException.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <memory>

namespace sgd {

struct Shape {
    size_t x, y;
    Shape(size_t x_ = 1, size_t y_ = 1) : x(x_), y(y_) {}
};

class MatrixD {
public:
    Shape shape;
    std::shared_ptr<double> data_device;
    std::shared_ptr<double> data_host;

    MatrixD(size_t x_dim = 1, size_t y_dim = 1);
    explicit MatrixD(Shape s);

    void allocateMemory();
    void allocateCudaMemory();
    void allocateHostMemory();
    void allocateMemoryIfNotAllocated(Shape s);
    void setCudaMemory(double* ptr);   // borrowed, not freed
    void setHostMemory(double* ptr);   // borrowed, not freed
    void copyHostToDevice();
    void copyDeviceToHost();

    double* operator[](int index) { return data_host.get() + index; }
    const double* operator[](int index) const { return data_host.get() + index; }
    double* operator()(int index) { return data_device.get() + index; }
    const double* operator()(int index) const { return data_device.get() + index; }

    size_t size() const { return shape.x * shape.y; }

private:
    bool device_allocated = false;
    bool host_allocated = false;
};

}  // namespace sgd
