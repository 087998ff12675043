// GPU system-matrix builder: the sparse matrix of a 2D projector, row-major
// (row p*nu + u, column = cell index i*nj + j), built from the same footprint
// code the projector kernels run.
//
// Voxel-driven and batched over views.  A visitor V supplies
//   __device__ bool valid(int i, int j) const
//   template <class F> __device__ void visit(int p, int i, int j, F&& f) const
//       calling f(u, value) for every entry of cell (i, j) in view p, u ascending.
// Per batch of views: a count kernel (one thread per (view, cell)), an
// exclusive scan of the counts, an emit kernel writing (key, value) with
// key = (batch-local row) * ncols + column, a radix sort by key (columns
// ascending within rows, rows ascending: the order of the reference's
// generators, layers/A_B1.cu:576-588), then the batch is converted on the
// device to the caller's format and copied out.  Batches cover disjoint,
// increasing row ranges, so their concatenation is sorted.
#pragma once

#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "common.h"
#include "csr_out.h"

namespace sgd {

template <class V>
__global__ void csr_count_kernel(V vis, int p0, int nvb, int ni, int nj, unsigned long long* cnt) {
    const long long ncell = (long long)ni * nj;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ncell * nvb) return;
    const int pl = (int)(t / ncell);
    const long long cell = t - (long long)pl * ncell;
    const int i = (int)(cell / nj), j = (int)(cell - (long long)i * nj);
    unsigned long long n = 0;
    if (vis.valid(i, j)) vis.visit(p0 + pl, i, j, [&](int, float) { ++n; });
    cnt[t] = n;
}

template <class V>
__global__ void csr_emit_kernel(V vis, int p0, int nvb, int ni, int nj, int nu, const unsigned long long* off,
                                unsigned long long* key, float* val) {
    const long long ncell = (long long)ni * nj;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ncell * nvb) return;
    const int pl = (int)(t / ncell);
    const long long cell = t - (long long)pl * ncell;
    const int i = (int)(cell / nj), j = (int)(cell - (long long)i * nj);
    if (!vis.valid(i, j)) return;
    unsigned long long k = off[t];
    const unsigned long long rowbase = (unsigned long long)pl * nu;
    vis.visit(p0 + pl, i, j, [&](int u, float v) {
        key[k] = (rowbase + (unsigned long long)u) * (unsigned long long)ncell + (unsigned long long)cell;
        val[k] = v;
        ++k;
    });
}

__global__ void csr_triplets_kernel(const unsigned long long* key, const float* val, long long n, long long ncols,
                                    long long row0, double* out);
__global__ void csr_split_kernel(const unsigned long long* key, const float* val, long long n, long long ncols,
                                 int* cols, double* vals);
__global__ void csr_rowptr_kernel(const unsigned long long* key, long long n, long long ncols, long long nrows,
                                  long long base, long long* rowptr);

// Scratch of one build, reused across batches.
class CsrScratch {
public:
    ~CsrScratch();
    void* get(int slot, size_t bytes, cudaStream_t s);

private:
    void* p_[8] = {};
    size_t n_[8] = {};
};

// Views per batch: about 2^25 (view, cell) items.
inline int csr_batch_views(long long ncell, int np) {
    return (int)std::max<long long>(1, std::min<long long>(np, (1ll << 25) / std::max<long long>(1, ncell)));
}

template <class V>
long long build_csr(const V& vis, int np, int nu, int ni, int nj, const CsrOut& out, cudaStream_t s) {
    const long long ncell = (long long)ni * nj;
    const int vb = csr_batch_views(ncell, np);
    CsrScratch sc;
    auto count_batch = [&](int p0, int nvb, unsigned long long* cnt) {
        const long long items = ncell * nvb;
        csr_count_kernel<V><<<(unsigned)((items + 255) / 256), 256, 0, s>>>(vis, p0, nvb, ni, nj, cnt);
        SGD_LAUNCH_CHECK();
    };
    // pass 1: entries per batch
    std::vector<long long> bn;
    long long total = 0;
    for (int p0 = 0; p0 < np; p0 += vb) {
        const int nvb = std::min(vb, np - p0);
        const long long items = ncell * nvb;
        auto* cnt = static_cast<unsigned long long*>(sc.get(0, items * 8, s));
        auto* sum = static_cast<unsigned long long*>(sc.get(1, 8, s));
        count_batch(p0, nvb, cnt);
        size_t tb = 0;
        SGD_CUDA(cub::DeviceReduce::Sum(nullptr, tb, cnt, sum, items, s));
        SGD_CUDA(cub::DeviceReduce::Sum(sc.get(2, tb, s), tb, cnt, sum, items, s));
        unsigned long long h = 0;
        SGD_CUDA(cudaMemcpyAsync(&h, sum, 8, cudaMemcpyDeviceToHost, s));
        SGD_CUDA(cudaStreamSynchronize(s));
        bn.push_back((long long)h);
        total += (long long)h;
    }
    if (out.counting()) return total;
    if (total > out.cap) fail("matrix has %lld entries, the output holds %lld", total, out.cap);
    if (out.rowptr) out.rowptr[0] = 0;
    // pass 2: emit, sort, convert, copy out
    int bits = 1;
    while (bits < 64 && ((unsigned long long)vb * nu * (unsigned long long)ncell) >> bits) ++bits;
    long long done = 0;
    int b = 0;
    for (int p0 = 0; p0 < np; p0 += vb, ++b) {
        const int nvb = std::min(vb, np - p0);
        const long long items = ncell * nvb, n = bn[b];
        if (n == 0) {
            if (out.rowptr)
                for (long long r = 0; r < (long long)nvb * nu; ++r) out.rowptr[(long long)p0 * nu + r + 1] = done;
            continue;
        }
        auto* cnt = static_cast<unsigned long long*>(sc.get(0, items * 8, s));
        auto* off = static_cast<unsigned long long*>(sc.get(1, items * 8, s));
        auto* k0 = static_cast<unsigned long long*>(sc.get(3, n * 8, s));
        auto* k1 = static_cast<unsigned long long*>(sc.get(4, n * 8, s));
        auto* v0 = static_cast<float*>(sc.get(5, n * 4, s));
        auto* v1 = static_cast<float*>(sc.get(6, n * 4, s));
        count_batch(p0, nvb, cnt);
        size_t tb = 0;
        SGD_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, off, items, s));
        SGD_CUDA(cub::DeviceScan::ExclusiveSum(sc.get(2, tb, s), tb, cnt, off, items, s));
        csr_emit_kernel<V><<<(unsigned)((items + 255) / 256), 256, 0, s>>>(vis, p0, nvb, ni, nj, nu, off, k0, v0);
        SGD_LAUNCH_CHECK();
        SGD_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, k0, k1, v0, v1, n, 0, bits, s));
        SGD_CUDA(cub::DeviceRadixSort::SortPairs(sc.get(2, tb, s), tb, k0, k1, v0, v1, n, 0, bits, s));
        const unsigned g = (unsigned)((n + 255) / 256);
        if (out.triplets) {
            auto* t = static_cast<double*>(sc.get(7, n * 24, s));
            csr_triplets_kernel<<<g, 256, 0, s>>>(k1, v1, n, ncell, (long long)p0 * nu, t);
            SGD_LAUNCH_CHECK();
            SGD_CUDA(cudaMemcpyAsync(out.triplets + 3 * done, t, n * 24, cudaMemcpyDeviceToHost, s));
        } else {
            auto* c = static_cast<int*>(sc.get(7, n * 4, s));
            auto* v = static_cast<double*>(sc.get(3, n * 8, s));  // k0 is free after the sort
            csr_split_kernel<<<g, 256, 0, s>>>(k1, v1, n, ncell, c, v);
            SGD_LAUNCH_CHECK();
            const long long nrows = (long long)nvb * nu;
            auto* rp = static_cast<long long*>(sc.get(5, (nrows + 1) * 8, s));  // v0 is free too
            csr_rowptr_kernel<<<(unsigned)((nrows + 256) / 256), 256, 0, s>>>(k1, n, ncell, nrows, done, rp);
            SGD_LAUNCH_CHECK();
            SGD_CUDA(cudaMemcpyAsync(out.cols + done, c, n * 4, cudaMemcpyDeviceToHost, s));
            SGD_CUDA(cudaMemcpyAsync(out.vals + done, v, n * 8, cudaMemcpyDeviceToHost, s));
            SGD_CUDA(cudaMemcpyAsync(out.rowptr + (long long)p0 * nu + 1, rp + 1, nrows * 8, cudaMemcpyDeviceToHost,
                                     s));
        }
        SGD_CUDA(cudaStreamSynchronize(s));
        done += n;
    }
    return total;
}

}  // namespace sgd
