#include "matrix_double.h"

#include "common.h"

namespace sgd {

MatrixD::MatrixD(size_t x_dim, size_t y_dim) : shape(x_dim, y_dim) {}
MatrixD::MatrixD(Shape s) : shape(s) {}

void MatrixD::allocateCudaMemory() {
    if (device_allocated) return;
    double* p = nullptr;
    SGD_CUDA(cudaMalloc(&p, size() * sizeof(double)));
    data_device = std::shared_ptr<double>(p, [](double* q) { cudaFree(q); });
    device_allocated = true;
}

void MatrixD::allocateHostMemory() {
    if (host_allocated) return;
    data_host = std::shared_ptr<double>(new double[size()], [](double* q) { delete[] q; });
    host_allocated = true;
}

void MatrixD::allocateMemory() {
    allocateCudaMemory();
    allocateHostMemory();
}

void MatrixD::allocateMemoryIfNotAllocated(Shape s) {
    if (!device_allocated && !host_allocated) {
        shape = s;
        allocateMemory();
    }
}

void MatrixD::setCudaMemory(double* ptr) {
    if (device_allocated) return;
    data_device = std::shared_ptr<double>(ptr, [](double*) {});
    device_allocated = true;
}

void MatrixD::setHostMemory(double* ptr) {
    if (host_allocated) return;
    data_host = std::shared_ptr<double>(ptr, [](double*) {});
    host_allocated = true;
}

void MatrixD::copyHostToDevice() {
    if (!(device_allocated && host_allocated)) fail("MatrixD: copy to unallocated device memory");
    SGD_CUDA(cudaMemcpy(data_device.get(), data_host.get(), size() * sizeof(double), cudaMemcpyHostToDevice));
}

void MatrixD::copyDeviceToHost() {
    if (!(device_allocated && host_allocated)) fail("MatrixD: copy to unallocated host memory");
    SGD_CUDA(cudaMemcpy(data_host.get(), data_device.get(), size() * sizeof(double), cudaMemcpyDeviceToHost));
}

}  // namespace sgd
