// Batched B1 projection of many fan-beam slices of different sizes and
// geometries: one persistent launch per direction, captured in a CUDA graph,
// with its launch shape chosen by an autotuner whose results are cached.
//
// A batch owns one B1 layer (tables) per distinct slice geometry and reads
// arenas: slice k's image at img_off[k] (host layout i*ny + j) and its
// sinogram at sino_off[k] ([p][u]) of caller-provided device arrays.  The
// persistent kernels run a grid of (CTAs per SM x SMs) CTAs that take work
// items from a global counter:
//   forward  an item is FW consecutive (view, bin) rows of one slice, one warp
//            per row (b1_forward_row);
//   backward an item is one 32x8 tile of one slice (b1_back_tile), the CTA's
//            mbarriers carrying their phase across items.
// Items are ordered by slice, heaviest slices (most views) first, so that the
// uneven tail is made of light items.  The reference has no batched path: it
// launches per view (layers/A_B1.cu:514-524).
//
// Tuned: FW (warps per forward item, 4/8/16) and VC (views per staged chunk
// of the backward, 2/4/8).  The tuner times every variant on the batch itself
// (CUDA events, zero inputs) and appends the winner to a text cache keyed by
// GPU name, SM count and the batch's geometry signature.
#include "b1_batch.h"

#include <algorithm>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>
#include <string>

#include "b1_body.cuh"
#include "common.h"

namespace sgd {

namespace {

__device__ __forceinline__ int find_slice(const long long* start, int ns, long long item) {
    int lo = 0, hi = ns - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <int FW>
__global__ void __launch_bounds__(FW * 32, 32 / FW)
b1_forward_batch_kernel(const B1Slice* __restrict__ sl, const long long* __restrict__ start, int ns, long long total,
                        const float* __restrict__ img, const float* __restrict__ imgT, float* __restrict__ sino,
                        unsigned long long* __restrict__ counter) {
    __shared__ long long s_item;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = (long long)atomicAdd(counter, 1ull);
        __syncthreads();
        const long long item = s_item;
        if (item >= total) return;
        const int k = find_slice(start, ns, item);
        const B1Slice S = sl[k];
        const long long gw = (item - start[k]) * FW + warp;
        if (gw < (long long)S.np * S.nu)
            b1_forward_row(S.rec, S.strip, img + S.img_off, imgT + S.img_off, sino + S.sino_off, S.nx, S.ny, S.nu,
                           S.dxdy, gw, lane);
    }
}

template <int VC, int WCAP>
__global__ void __launch_bounds__(kBackThreads, 7)
b1_back_batch_kernel(const B1Slice* __restrict__ sl, const long long* __restrict__ start, int ns, long long total,
                     const float* __restrict__ sino, float* __restrict__ img, unsigned long long* __restrict__ counter,
                     int* __restrict__ err, uint32_t wait_limit) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ long long s_item;
    if (threadIdx.x == 0) {
        uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    uint32_t use0 = 0, use1 = 0;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = (long long)atomicAdd(counter, 1ull);
        __syncthreads();
        const long long item = s_item;
        if (item >= total) return;
        const int k = find_slice(start, ns, item);
        const B1Slice S = sl[k];
        const int t = (int)(item - start[k]);
        const int bx = t % S.tiles_x, by = t / S.tiles_x;
        if (!b1_back_tile<VC, WCAP>(S.rec, S.hom, S.wins + (size_t)t * S.np, sino + S.sino_off, img + S.img_off,
                                    S.nx, S.ny, S.np, S.nu, S.dxdy, err, wait_limit, by * kBackTI, bx * kBackTJ,
                                    smem, use0, use1))
            return;
    }
}

// in[r * cols + c] -> out[c * rows + r] for every slice (blockIdx.z)
__global__ void batch_transpose_kernel(const B1Slice* __restrict__ sl, const float* __restrict__ in,
                                       float* __restrict__ out) {
    const B1Slice S = sl[blockIdx.z];
    const int rows = S.nx, cols = S.ny;
    if ((int)blockIdx.x * 32 >= cols || (int)blockIdx.y * 32 >= rows) return;
    const float* a = in + S.img_off;
    float* b = out + S.img_off;
    __shared__ float t[32][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    for (int q = threadIdx.y; q < 32; q += 8) {
        const int r = blockIdx.y * 32 + q;
        if (r < rows && c < cols) t[q][threadIdx.x] = a[(size_t)r * cols + c];
    }
    __syncthreads();
    const int r = blockIdx.y * 32 + threadIdx.x;
    for (int q = threadIdx.y; q < 32; q += 8) {
        const int cc = blockIdx.x * 32 + q;
        if (r < rows && cc < cols) b[(size_t)cc * rows + r] = t[threadIdx.x][q];
    }
}

constexpr int kFWs[3] = {4, 8, 16};
constexpr int kVCs[3] = {2, 4, 8};
// Plane strides of the batch's back kernels (staged windows of every slice).
constexpr int kBatchCaps[] = {48, 64, 96, 128, 256};
constexpr size_t kSmemMax = 227 * 1024;

// Dynamic shared memory of the back kernel for vc views per chunk and plane
// stride wcap (b1_back_smem).
constexpr size_t batch_back_smem(int vc, int wcap) {
    return (size_t)(16 + 3 * vc * 8 + 3 * vc * 32) + (size_t)2 * vc * kBackPlanes * wcap * 16;
}

// Calls f(kernel, dynamic shared memory bytes) for views per chunk vc and
// plane stride wcap; fails for a combination that does not fit in shared
// memory (eight views of 256-bin windows).
template <class F>
void with_batch_back_kernel(int vc, int wcap, F&& f) {
    if (batch_back_smem(vc, wcap) > kSmemMax)
        fail("B1 batch: %d views per chunk of %d-bin windows exceed shared memory", vc, wcap);
#define SGD_B1_BATCH_CASE(V, W)                                                      \
    if (vc == V && wcap == W) {                                                      \
        static_assert(b1_back_smem<V, W>() == batch_back_smem(V, W), "smem formula"); \
        f(b1_back_batch_kernel<V, W>, b1_back_smem<V, W>());                         \
        return;                                                                      \
    }
    SGD_B1_BATCH_CASE(2, 48) SGD_B1_BATCH_CASE(2, 64) SGD_B1_BATCH_CASE(2, 96) SGD_B1_BATCH_CASE(2, 128)
    SGD_B1_BATCH_CASE(2, 256) SGD_B1_BATCH_CASE(4, 48) SGD_B1_BATCH_CASE(4, 64) SGD_B1_BATCH_CASE(4, 96)
    SGD_B1_BATCH_CASE(4, 128) SGD_B1_BATCH_CASE(4, 256) SGD_B1_BATCH_CASE(8, 48) SGD_B1_BATCH_CASE(8, 64)
    SGD_B1_BATCH_CASE(8, 96) SGD_B1_BATCH_CASE(8, 128)
#undef SGD_B1_BATCH_CASE
    fail("B1 batch: no back kernel for %d views per chunk and %d-bin windows", vc, wcap);
}

}  // namespace

B1Batch::B1Batch(int ns, const int* nx, const int* ny, const int* np, const int* nu, const double* dx,
                 const double* dy, const double* du, const double* lsd, const double* lso,
                 const double* const* angles) {
    if (ns < 1) fail("B1 batch: no slices");
    SGD_CUDA(cudaGetDevice(&device_));
    SGD_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    cudaDeviceProp prop;
    SGD_CUDA(cudaGetDeviceProperties(&prop, device_));
    sms_ = prop.multiProcessorCount;
    gpu_name_ = prop.name;
    // heaviest slices first: backward tile cost ~ views, forward row cost ~ image side
    order_.resize(ns);
    std::iota(order_.begin(), order_.end(), 0);
    std::stable_sort(order_.begin(), order_.end(), [&](int a, int b) {
        return (long long)np[a] * std::max(nx[a], ny[a]) > (long long)np[b] * std::max(nx[b], ny[b]);
    });
    // slices with identical geometry share one layer (tables)
    auto same = [&](int a, int b) {
        return nx[a] == nx[b] && ny[a] == ny[b] && np[a] == np[b] && nu[a] == nu[b] && dx[a] == dx[b] &&
               dy[a] == dy[b] && du[a] == du[b] && lsd[a] == lsd[b] && lso[a] == lso[b] &&
               std::memcmp(angles[a], angles[b], sizeof(double) * np[a]) == 0;
    };
    std::ostringstream sig;
    img_off_.assign(ns + 1, 0);
    sino_off_.assign(ns + 1, 0);
    layer_of_.assign(ns, -1);
    for (int k = 0; k < ns; ++k) {
        if (!angles[k]) fail("B1 batch: slice %d has no angles", k);
        for (int q = 0; q < k && layer_of_[k] < 0; ++q)
            if (same(k, q)) layer_of_[k] = layer_of_[q];
        if (layer_of_[k] < 0) {
            layer_of_[k] = (int)layers_.size();
            layers_.emplace_back(new A_B1(nx[k], ny[k], np[k], nu[k], dx[k], dy[k], du[k], lsd[k], lso[k],
                                          angles[k], nullptr, nullptr));
        }
        img_off_[k + 1] = img_off_[k] + (long long)nx[k] * ny[k];
        sino_off_[k + 1] = sino_off_[k] + (long long)np[k] * nu[k];
        sig << nx[k] << 'x' << ny[k] << 'x' << np[k] << 'x' << nu[k] << ';';
    }
    signature_ = sig.str();
    ns_ = ns;
    std::vector<B1Slice> host(ns);
    fwd_start_.assign(ns + 1, 0);
    back_start_.assign(ns + 1, 0);
    for (int q = 0; q < ns; ++q) {
        const int k = order_[q];
        const B1Device& d = layers_[layer_of_[k]]->dev;
        B1Slice& S = host[q];
        S.rec = reinterpret_cast<const float4*>(d.rec);
        S.strip = d.strip;
        S.hom = d.hom;
        S.wins = reinterpret_cast<const int2*>(d.wins);
        S.img_off = img_off_[k];
        S.sino_off = sino_off_[k];
        S.nx = d.nx; S.ny = d.ny; S.np = d.np; S.nu = d.nu;
        S.tiles_x = (d.ny + kBackTJ - 1) / kBackTJ;
        S.dxdy = d.dxdy;
        wmax_ = std::max(wmax_, d.wmax);
        back_start_[q + 1] = back_start_[q] + (long long)S.tiles_x * ((d.nx + kBackTI - 1) / kBackTI);
        max_nx_ = std::max(max_nx_, d.nx);
        max_ny_ = std::max(max_ny_, d.ny);
    }
    wcap_ = 0;
    for (int c : kBatchCaps)
        if (wmax_ + 1 <= c) {
            wcap_ = c;
            break;
        }
    if (!wcap_) fail("B1 batch: a tile's bin window of %d bins is too wide (at most %d)", wmax_, kBatchCaps[4] - 1);
    SGD_CUDA(cudaMalloc(&d_slices_, ns * sizeof(B1Slice)));
    SGD_CUDA(cudaMemcpy(d_slices_, host.data(), ns * sizeof(B1Slice), cudaMemcpyHostToDevice));
    SGD_CUDA(cudaMalloc(&d_start_, 2 * (ns + 1) * sizeof(long long)));
    SGD_CUDA(cudaMalloc(&d_counter_, 2 * sizeof(unsigned long long)));
    SGD_CUDA(cudaMalloc(&d_err_, sizeof(int)));
    SGD_CUDA(cudaMemset(d_err_, 0, sizeof(int)));
    SGD_CUDA(cudaMalloc(&d_imgT_, std::max(1ll, img_off_[ns]) * sizeof(float)));
    for (int vc : kVCs) {
        if (batch_back_smem(vc, wcap_) > kSmemMax) continue;
        with_batch_back_kernel(vc, wcap_, [](auto kern, size_t smem) {
            SGD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            SGD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                          cudaSharedmemCarveoutMaxShared));
        });
    }
    set_variant(8, 4);
}

B1Batch::~B1Batch() {
    if (stream_) cudaStreamSynchronize(stream_);
    release_graph();
    cudaFree(d_slices_);
    cudaFree(d_start_);
    cudaFree(d_counter_);
    cudaFree(d_err_);
    cudaFree(d_imgT_);
    if (stream_) cudaStreamDestroy(stream_);
}

void B1Batch::set_variant(int fw, int vc) {
    if (fw != 4 && fw != 8 && fw != 16) fail("B1 batch: forward warps %d not in {4, 8, 16}", fw);
    if (vc != 2 && vc != 4 && vc != 8) fail("B1 batch: views per chunk %d not in {2, 4, 8}", vc);
    with_batch_back_kernel(vc, wcap_, [](auto, size_t) {});  // fails when the windows do not fit
    // the start table below is read by persistent kernels that may still be
    // running on the caller's or the batch's stream: let them finish first
    SGD_CUDA(cudaDeviceSynchronize());
    fw_ = fw;
    vc_ = vc;
    for (int q = 0; q < ns_; ++q) {
        const B1Device& d = layers_[layer_of_[order_[q]]]->dev;
        fwd_start_[q + 1] = fwd_start_[q] + ((long long)d.np * d.nu + fw - 1) / fw;
    }
    std::vector<long long> st(2 * (ns_ + 1));
    std::copy(fwd_start_.begin(), fwd_start_.end(), st.begin());
    std::copy(back_start_.begin(), back_start_.end(), st.begin() + ns_ + 1);
    SGD_CUDA(cudaMemcpy(d_start_, st.data(), st.size() * sizeof(long long), cudaMemcpyHostToDevice));
    release_graph();  // a captured graph holds the old launch shape
}

int B1Batch::resident(const void* fn, int threads, size_t smem) const {
    int n = 0;
    SGD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, smem));
    return std::max(1, n);
}

void B1Batch::forward(const float* img, float* sino, cudaStream_t s) {
    SGD_CUDA(cudaMemsetAsync(d_counter_, 0, sizeof(unsigned long long), s));
    dim3 tb(32, 8), tg((max_ny_ + 31) / 32, (max_nx_ + 31) / 32, ns_);
    batch_transpose_kernel<<<tg, tb, 0, s>>>(d_slices_, img, d_imgT_);
    SGD_LAUNCH_CHECK();
    const long long total = fwd_start_[ns_];
    auto launch = [&](auto kern, int fw) {
        const int grid = sms_ * resident((const void*)kern, fw * 32, 0);
        kern<<<grid, fw * 32, 0, s>>>(d_slices_, d_start_, ns_, total, img, d_imgT_, sino, d_counter_);
    };
    if (fw_ == 4) launch(b1_forward_batch_kernel<4>, 4);
    else if (fw_ == 8) launch(b1_forward_batch_kernel<8>, 8);
    else launch(b1_forward_batch_kernel<16>, 16);
    SGD_LAUNCH_CHECK();
}

void B1Batch::backward(const float* sino, float* img, cudaStream_t s) {
    SGD_CUDA(cudaMemsetAsync(d_counter_ + 1, 0, sizeof(unsigned long long), s));
    const long long total = back_start_[ns_];
    const long long* bstart = d_start_ + ns_ + 1;
    auto launch = [&](auto kern, size_t smem) {
        const int grid = sms_ * resident((const void*)kern, kBackThreads, smem);
        kern<<<grid, kBackThreads, smem, s>>>(d_slices_, bstart, ns_, total, sino, img, d_counter_ + 1, d_err_,
                                              wait_limit_);
    };
    with_batch_back_kernel(vc_, wcap_, launch);
    SGD_LAUNCH_CHECK();
}

void B1Batch::check_status() {
    SGD_CUDA(cudaDeviceSynchronize());
    int e = 0;
    SGD_CUDA(cudaMemcpy(&e, d_err_, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        SGD_CUDA(cudaMemset(d_err_, 0, sizeof(int)));
        fail("B1 batch back projection: a staged chunk did not arrive (bounded wait expired)");
    }
}

void B1Batch::set_wait_limit(unsigned polls) {
    wait_limit_ = polls;
    release_graph();  // a captured graph holds the old kernel argument
}

void B1Batch::release_graph() {
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    exec_ = nullptr;
    graph_ = nullptr;
}

void B1Batch::capture(const float* img, float* sino, const float* sino_in, float* img_out) {
    release_graph();
    SGD_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    try {
        if (img && sino) forward(img, sino, stream_);
        if (sino_in && img_out) backward(sino_in, img_out, stream_);
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(stream_, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    SGD_CUDA(cudaStreamEndCapture(stream_, &graph_));
    SGD_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
}

void B1Batch::replay(cudaStream_t s) {
    if (!exec_) fail("B1 batch: no captured graph");
    SGD_CUDA(cudaGraphLaunch(exec_, s));
}

std::string B1Batch::cache_key() const {
    std::ostringstream k;
    k << gpu_name_ << '|' << sms_ << '|' << signature_;
    std::string s = k.str();
    for (char& c : s)
        if (c == ' ') c = '_';
    return s;
}

int B1Batch::tune(const char* cache_path) {
    const std::string key = cache_key();
    if (cache_path && *cache_path) {
        std::ifstream in(cache_path);
        std::string k;
        int fw = 0, vc = 0;
        while (in >> k >> fw >> vc)
            if (k == key && batch_back_smem(vc, wcap_) <= kSmemMax) {  // an entry this build can run
                set_variant(fw, vc);
                return 1;
            }
    }
    // time every variant on zero inputs (the set of visited pairs does not
    // depend on the values)
    float *img = nullptr, *sino = nullptr;
    SGD_CUDA(cudaMalloc(&img, std::max(1ll, img_off_[ns_]) * sizeof(float)));
    SGD_CUDA(cudaMalloc(&sino, std::max(1ll, sino_off_[ns_]) * sizeof(float)));
    SGD_CUDA(cudaMemset(img, 0, img_off_[ns_] * sizeof(float)));
    SGD_CUDA(cudaMemset(sino, 0, sino_off_[ns_] * sizeof(float)));
    cudaEvent_t e0, e1;
    SGD_CUDA(cudaEventCreate(&e0));
    SGD_CUDA(cudaEventCreate(&e1));
    auto time_ms = [&](auto&& run) {
        run();  // warm-up
        float best = 1e30f;
        for (int r = 0; r < 3; ++r) {
            SGD_CUDA(cudaEventRecord(e0, stream_));
            run();
            SGD_CUDA(cudaEventRecord(e1, stream_));
            SGD_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            SGD_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            best = std::min(best, ms);
        }
        return best;
    };
    int best_fw = 8, best_vc = 4;
    float tf = 1e30f, tb = 1e30f;
    for (int fw : kFWs) {
        set_variant(fw, vc_);
        const float t = time_ms([&] { forward(img, sino, stream_); });
        if (t < tf) { tf = t; best_fw = fw; }
    }
    for (int vc : kVCs) {
        if (batch_back_smem(vc, wcap_) > kSmemMax) continue;
        set_variant(best_fw, vc);
        const float t = time_ms([&] { backward(sino, img, stream_); });
        if (t < tb) { tb = t; best_vc = vc; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(img);
    cudaFree(sino);
    check_status();
    set_variant(best_fw, best_vc);
    if (cache_path && *cache_path) {
        std::ofstream out(cache_path, std::ios::app);
        out << key << ' ' << best_fw << ' ' << best_vc << '\n';
    }
    return 0;
}

}  // namespace sgd

extern "C" {

void* sgd_b1_batch_create(int ns, const int* nx, const int* ny, const int* np, const int* nu, const double* dx,
                          const double* dy, const double* du, const double* lsd, const double* lso,
                          const double* const* angles) {
    return sgd::guarded<void*>(nullptr, [&]() -> void* {
        if (!nx || !ny || !np || !nu || !dx || !dy || !du || !lsd || !lso || !angles)
            sgd::fail("sgd_b1_batch_create: null argument");
        return new sgd::B1Batch(ns, nx, ny, np, nu, dx, dy, du, lsd, lso, angles);
    });
}

void sgd_b1_batch_destroy(void* batch) { delete static_cast<sgd::B1Batch*>(batch); }

int sgd_b1_batch_offsets(void* batch, long long* img_off, long long* sino_off) {
    return sgd::guarded_status([&] {
        if (!batch || !img_off || !sino_off) sgd::fail("sgd_b1_batch_offsets: null argument");
        const auto* b = static_cast<sgd::B1Batch*>(batch);
        std::copy(b->img_off().begin(), b->img_off().end(), img_off);
        std::copy(b->sino_off().begin(), b->sino_off().end(), sino_off);
    });
}

int sgd_b1_batch_forward(void* batch, const float* d_img, float* d_sino, void* stream) {
    return sgd::guarded_status([&] {
        if (!batch || !d_img || !d_sino) sgd::fail("sgd_b1_batch_forward: null argument");
        static_cast<sgd::B1Batch*>(batch)->forward(d_img, d_sino, static_cast<cudaStream_t>(stream));
    });
}

int sgd_b1_batch_backward(void* batch, const float* d_sino, float* d_img, void* stream) {
    return sgd::guarded_status([&] {
        if (!batch || !d_img || !d_sino) sgd::fail("sgd_b1_batch_backward: null argument");
        static_cast<sgd::B1Batch*>(batch)->backward(d_sino, d_img, static_cast<cudaStream_t>(stream));
    });
}

int sgd_b1_batch_capture(void* batch, const float* d_img, float* d_sino, const float* d_sino_in, float* d_img_out) {
    return sgd::guarded_status([&] {
        if (!batch) sgd::fail("sgd_b1_batch_capture: null batch");
        static_cast<sgd::B1Batch*>(batch)->capture(d_img, d_sino, d_sino_in, d_img_out);
    });
}

int sgd_b1_batch_replay(void* batch, void* stream) {
    return sgd::guarded_status([&] {
        if (!batch) sgd::fail("sgd_b1_batch_replay: null batch");
        static_cast<sgd::B1Batch*>(batch)->replay(static_cast<cudaStream_t>(stream));
    });
}

int sgd_b1_batch_tune(void* batch, const char* cache_path, int* fw, int* vc) {
    return sgd::guarded<int>(-1, [&]() -> int {
        if (!batch) sgd::fail("sgd_b1_batch_tune: null batch");
        auto* b = static_cast<sgd::B1Batch*>(batch);
        const int loaded = b->tune(cache_path);
        if (fw) *fw = b->fw();
        if (vc) *vc = b->vc();
        return loaded;
    });
}

int sgd_b1_batch_set_variant(void* batch, int fw, int vc) {
    return sgd::guarded_status([&] {
        if (!batch) sgd::fail("sgd_b1_batch_set_variant: null batch");
        static_cast<sgd::B1Batch*>(batch)->set_variant(fw, vc);
    });
}

int sgd_b1_batch_set_wait_limit(void* batch, unsigned polls) {
    return sgd::guarded_status([&] {
        if (!batch) sgd::fail("sgd_b1_batch_set_wait_limit: null batch");
        static_cast<sgd::B1Batch*>(batch)->set_wait_limit(polls);
    });
}

int sgd_b1_batch_status(void* batch) {
    return sgd::guarded_status([&] {
        if (!batch) sgd::fail("sgd_b1_batch_status: null batch");
        static_cast<sgd::B1Batch*>(batch)->check_status();
    });
}

}  // extern "C"
