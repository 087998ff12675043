// Non-template parts of the GPU system-matrix builder (csr_build.cuh).
#include "csr_build.cuh"

namespace sgd {

__global__ void csr_triplets_kernel(const unsigned long long* key, const float* val, long long n, long long ncols,
                                    long long row0, double* out) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const unsigned long long kk = key[k];
    const long long row = (long long)(kk / (unsigned long long)ncols), col = (long long)(kk % (unsigned long long)ncols);
    out[3 * k] = (double)(row0 + row);
    out[3 * k + 1] = (double)col;
    out[3 * k + 2] = (double)val[k];
}

__global__ void csr_split_kernel(const unsigned long long* key, const float* val, long long n, long long ncols,
                                 int* cols, double* vals) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    cols[k] = (int)(key[k] % (unsigned long long)ncols);
    vals[k] = (double)val[k];
}

// rowptr[r] = base + (first entry whose row is >= r), r = 0..nrows.
__global__ void csr_rowptr_kernel(const unsigned long long* key, long long n, long long ncols, long long nrows,
                                  long long base, long long* rowptr) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r > nrows) return;
    const unsigned long long target = (unsigned long long)r * (unsigned long long)ncols;
    long long lo = 0, hi = n;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (key[mid] < target) lo = mid + 1;
        else hi = mid;
    }
    rowptr[r] = base + lo;
}

CsrScratch::~CsrScratch() {
    for (void* p : p_)
        if (p) cudaFree(p);
}

void* CsrScratch::get(int slot, size_t bytes, cudaStream_t s) {
    if (bytes == 0) bytes = 1;
    if (n_[slot] < bytes) {
        if (p_[slot]) {
            SGD_CUDA(cudaStreamSynchronize(s));
            SGD_CUDA(cudaFree(p_[slot]));
            p_[slot] = nullptr;
            n_[slot] = 0;
        }
        SGD_CUDA(cudaMalloc(&p_[slot], bytes));
        n_[slot] = bytes;
    }
    return p_[slot];
}

}  // namespace sgd
