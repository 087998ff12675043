// Bodies of the B1 projection kernels, shared by the single-geometry kernels
// (b1.cu) and the persistent batched kernels (b1_batch.cu).
//
//   b1_forward_row   detector-driven: one warp per (view, bin).  Lanes split
//                    the lines (major axis) the bin's ray strip crosses; each
//                    lane evaluates the footprint of the few pixels of its line
//                    inside the strip (packed-pair form, b1_kernels.cuh), and
//                    the warp reduces with shuffles.  The sinogram value is
//                    written once, no atomics.
//   b1_back_tile     voxel-driven: one thread per pixel of a 32x8 tile.  Per
//                    chunk of VC views the CTA stages the bin window its tile
//                    projects onto in shared memory: the 64-byte footprint
//                    records by TMA bulk copies, the sinogram values by plain
//                    loads.  A ring of kStages buffers with a full and an
//                    empty mbarrier each replaces CTA-wide barriers: warp 0
//                    stages chunk c + kStages - 1 once every thread has
//                    released it, and each warp runs on as soon as its next
//                    chunk is full.  Each thread accumulates over all views
//                    in registers and writes its pixel once, no atomics.
//
// Reference: layers/A_B1.cu:62-208 (forward, one launch per view, FP64
// atomics) and :211-353 (backward).
#pragma once

#include <cstdint>

#include "b1_kernels.cuh"
#include "fan_geometry.h"
#include "hom.cuh"
#include "tma.cuh"

namespace sgd {

constexpr int kBackTI = 8;    // tile extent along i (x)
constexpr int kBackTJ = 32;   // tile extent along j (y): contiguous in memory
constexpr int kBackThreads = kBackTI * kBackTJ;
constexpr uint32_t kWaitLimit = 1u << 22;
constexpr int kStages = 3;    // staging ring depth of the back projection

// kStages full + kStages empty mbarriers | kStages x VC windows | kStages x VC
// homographies, then the staged records and sinogram windows
template <int VC>
__host__ __device__ constexpr int b1_header_bytes() {
    return 16 * kStages + kStages * VC * 8 + kStages * VC * 32;
}

template <int VC>
__host__ __device__ constexpr size_t b1_back_smem(int wcap) {
    return b1_header_bytes<VC>() + (size_t)kStages * VC * wcap * (sizeof(B1Bin) + sizeof(float));
}

// Thread 0, once per CTA before its first tile: full barriers expect the 32
// lanes of the staging warp (and the TMA bytes), empty barriers every thread.
__device__ __forceinline__ void b1_back_init(unsigned char* smem) {
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
    for (int s = 0; s < kStages; ++s) {
        mbar_init(&bars[s], 32);
        mbar_init(&bars[kStages + s], kBackThreads);
    }
    fence_mbar_init();
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Records are float4 chunks laid out [view][chunk][bin] (fan_geometry.h).
__device__ __forceinline__ B1Bin load_bin(const float4* rec, int p, int u, int nu) {
    const float4* q = rec + (size_t)p * 4 * nu + u;
    return B1Bin{__ldg(q), __ldg(q + nu), __ldg(q + 2 * nu), __ldg(q + 3 * nu)};
}

// Candidate minor indices of major line m: the strip between the edge rays over
// the lines m-1..m+1 a pixel's support covers, widened by the +-1 pixel support
// along the minor axis.
__device__ __forceinline__ void strip_span(const float4& st, float aa, float ab, float fm, int nmin, int& nlo,
                                           int& nhi) {
    const float fa = fmaf(st.y, fm, st.x);
    const float fb = fmaf(st.w, fm, st.z);
    const float lo = fminf(fa - aa, fb - ab) - 1.0f;
    const float hi = fmaxf(fa + aa, fb + ab) + 1.0f;
    nlo = max(0, (int)ceilf(lo));
    nhi = min(nmin - 1, (int)floorf(hi));
}

// Sinogram value of row gw = p * nu + u.  img (i, j) at img[i * ny + j];
// imgT (i, j) at imgT[j * nx + i].
__device__ __forceinline__ void b1_forward_row(const float4* __restrict__ rec, const float* __restrict__ strip,
                                               const float* __restrict__ img, const float* __restrict__ imgT,
                                               float* __restrict__ sino, int nx, int ny, int nu, float dxdy,
                                               long long gw, int lane) {
    const int p = (int)(gw / nu), u = (int)(gw - (long long)p * nu);
    const B1Pair k = b1_pair(load_bin(rec, p, u, nu));
    const float4 st = __ldg(reinterpret_cast<const float4*>(strip + gw * kStripRec));
    const bool ydom = __ldg(strip + gw * kStripRec + 4) > 0.5f;
    const float aa = fabsf(st.y), ab = fabsf(st.w);

    // FP32 sums within a line (a few terms), FP64 across lines and lanes: the
    // forward and back kernels then round the same products to within FP64
    // accumulation error, which the dot-product adjoint test needs.
    double acc = 0.0;
    if (ydom) {
        // rows j = m, candidate columns i = n; the j terms are hoisted
        for (int m = lane; m < ny; m += 32) {
            const float fm = (float)m;
            int nlo, nhi;
            strip_span(st, aa, ab, fm, nx, nlo, nhi);
            const float2 inner = b1_inner2(pair(fm), k);
            float row = 0.f;
            float2 fn = pair((float)nlo);
            const float* sp = img + (size_t)nlo * ny + m;
            for (int n = nlo; n <= nhi; ++n, fn = __fadd2_rn(fn, pair(1.0f)), sp += ny) {
                const float conv = b1_conv_pair(b1_edges2(fn, inner, k), k);
                if (conv > kConvEps) row = fmaf(conv, __ldg(sp), row);
            }
            acc += (double)row;
        }
    } else {
        // columns i = m, candidate rows j = n
        for (int m = lane; m < nx; m += 32) {
            const float2 fm = pair((float)m);
            int nlo, nhi;
            strip_span(st, aa, ab, fm.x, ny, nlo, nhi);
            float row = 0.f;
            float2 fn = pair((float)nlo);
            const float* sp = imgT + (size_t)nlo * nx + m;
            for (int n = nlo; n <= nhi; ++n, fn = __fadd2_rn(fn, pair(1.0f)), sp += nx) {
                const float conv = b1_conv_pair(b1_edges2(fm, b1_inner2(fn, k), k), k);
                if (conv > kConvEps) row = fmaf(conv, __ldg(sp), row);
            }
            acc += (double)row;
        }
    }
    acc = warp_sum(acc);
    if (lane == 0) sino[gw] = (float)acc * dxdy;
}

// Back projection of the 32x8 tile at (i0, j0).  twin[p] = (lo, hi): bins of
// view p the tile's pixels can touch (host-computed, conservative; fits in
// wcap).  The ring's mbarriers (b1_back_init) carry their phases across the
// tiles of a persistent CTA: gseq counts the chunks this CTA started before
// this tile (chunk g uses stage g % kStages, phase (g / kStages) & 1).
// Returns false, with *err set and the tile unwritten, when a wait gave up
// (bounded); the copies in flight are awaited (bounded) first.
template <int VC>
__device__ __forceinline__ bool b1_back_tile(const float4* __restrict__ rec, const BinHomography* __restrict__ hom,
                                             const int2* __restrict__ twin, const float* __restrict__ sino,
                                             float* __restrict__ img, int nx, int ny, int np, int nu, int wcap,
                                             float dxdy, int* __restrict__ err, int i0, int j0, unsigned char* smem,
                                             volatile int& s_abort, uint32_t& gseq) {
    constexpr int kHeader = b1_header_bytes<VC>();
    static_assert(kHeader % 16 == 0, "staged records must start 16-byte aligned");
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);                             // [kStages]
    uint64_t* empty = full + kStages;                                              // [kStages]
    int* win = reinterpret_cast<int*>(smem + 16 * kStages);                          // [kStages][VC][2]
    float* hs = reinterpret_cast<float*>(smem + 16 * kStages + kStages * VC * 8);   // [kStages][VC][8]
    float4* srec = reinterpret_cast<float4*>(smem + kHeader);                       // [kStages][VC][4][wcap]
    float* ssino = reinterpret_cast<float*>(srec + kStages * VC * 4 * wcap);        // [kStages][VC][wcap]

    // each warp covers an 8 (j) x 4 (i) block of the 32 x 8 tile, so that its
    // lanes read few distinct bins of a view
    const int tid = threadIdx.x, w = tid >> 5, l = tid & 31;
    const int i = i0 + 4 * (w >> 2) + (l >> 3), j = j0 + 8 * (w & 3) + (l & 7);
    const float fi = (float)i, fj = (float)j;
    const int nchunks = (np + VC - 1) / VC;

    // Warp 0 stages chunk c once every thread released the stage's previous
    // contents: lane v < VC the window, homography and records (TMA) of view
    // c * VC + v, all lanes the sinogram windows.  Every lane arrives on the
    // full barrier after its own shared-memory writes.  The outcome is
    // warp-uniform.
    auto produce = [&](int c) -> bool {
        const uint32_t g = gseq + (uint32_t)c;
        const int s = (int)(g % kStages);
        const bool freed =
            g < (uint32_t)kStages || mbar_wait_or_abort(&empty[s], (g / kStages - 1) & 1u, kWaitLimit, &s_abort);
        if (!__all_sync(0xffffffffu, freed)) return false;
        const int p = c * VC + l;
        int2 lh = make_int2(0, -1);
        uint32_t bytes = 0;
        if (l < VC) {
            if (p < np) {
                lh = __ldg(twin + p);
                const BinHomography H = hom[p];
                float* h = hs + (s * VC + l) * 8;
                h[0] = H.n0; h[1] = H.n1; h[2] = H.n2; h[3] = H.d0; h[4] = H.d1; h[5] = H.d2;
            }
            win[(s * VC + l) * 2] = lh.x;
            win[(s * VC + l) * 2 + 1] = lh.y;
            if (lh.y >= lh.x) bytes = (uint32_t)(lh.y - lh.x + 1) * sizeof(B1Bin);
        }
#pragma unroll
        for (int v = 0; v < VC; ++v) {
            const int lo = __shfl_sync(0xffffffffu, lh.x, v), hi = __shfl_sync(0xffffffffu, lh.y, v);
            const float* sp = sino + (size_t)(c * VC + v) * nu + lo;
            float* dp = ssino + (s * VC + v) * wcap;
            for (int k = l; k <= hi - lo; k += 32) dp[k] = __ldg(sp + k);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
        if (l == 0) mbar_arrive_expect_tx(&full[s], bytes);
        else mbar_arrive(&full[s]);
        __syncwarp();
        if (l < VC && lh.y >= lh.x) {
            fence_proxy_async_smem();
            const uint32_t n = (uint32_t)(lh.y - lh.x + 1) * 16u;
            for (int q = 0; q < 4; ++q)
                bulk_copy_g2s(srec + ((s * VC + l) * 4 + q) * wcap, rec + ((size_t)p * 4 + q) * nu + lh.x, n,
                              &full[s]);
        }
        return true;
    };

    __syncthreads();  // s_abort and the previous tile settled
    int produced = 0;  // warp 0: chunks staged so far
    if (w == 0) {
        const int first = min(kStages - 1, nchunks);
        while (produced < first && produce(produced)) ++produced;
        if (produced < first && l == 0) {
            s_abort = 1;
            atomicExch(err, 1);
        }
    }

    // Control flow stays warp-uniform (warp 0 runs warp-collective staging
    // inside the loop): abort flags and wait outcomes are voted per warp.
    double acc = 0.0;  // FP32 within a chunk (a few tens of terms), FP64 across chunks
    int c = 0;
    for (; c < nchunks; ++c) {
        if (__any_sync(0xffffffffu, s_abort != 0)) break;
        if (w == 0 && produced == c + kStages - 1 && produced < nchunks) {
            if (!produce(produced)) {
                if (l == 0) {
                    s_abort = 1;
                    atomicExch(err, 1);
                }
                break;
            }
            ++produced;
        }
        const uint32_t g = gseq + (uint32_t)c;
        const int s = (int)(g % kStages);
        const bool ready = mbar_wait_or_abort(&full[s], (g / kStages) & 1u, kWaitLimit, &s_abort);
        if (!__all_sync(0xffffffffu, ready)) {
            if (l == 0) {
                s_abort = 1;
                atomicExch(err, 1);
            }
            break;
        }
        if (i < nx && j < ny) {
            // per view, this pixel's bins: trip counts differ by at most one
            // bin between the lanes of a warp.  (A single flat loop over all
            // the chunk's (view, bin) pairs, switching views per lane,
            // measured 1.38x slower at 512^2 x 720 views: the warp ran the
            // switch on most iterations.)  The bin loop is not unrolled:
            // unrolled, it spills at the 48 registers five CTAs per SM allow.
            float csum = 0.f;
#pragma unroll
            for (int v = 0; v < VC; ++v) {
                const int lo = win[(s * VC + v) * 2], hi = win[(s * VC + v) * 2 + 1];
                if (hi < lo) continue;
                int a, b;
                box_bins(hs + (s * VC + v) * 8, fi - 1.f, fi + 1.f, fj - 1.f, fj + 1.f, nu, a, b);
                a = max(a, lo);
                b = min(b, hi);
                const float4* rb = srec + (s * VC + v) * 4 * wcap - lo;
                const float* sb = ssino + (s * VC + v) * wcap - lo;
#pragma unroll 1
                for (int u = a; u <= b; ++u) {
                    const B1Bin r{rb[u], rb[u + wcap], rb[u + 2 * wcap], rb[u + 3 * wcap]};
                    const float conv = b1_conv(fi, fj, r);
                    if (conv > kConvEps) csum = fmaf(conv, sb[u], csum);
                }
            }
            acc += (double)csum;
        }
        mbar_arrive(&empty[s]);
    }
    // after a give-up: wait (bounded) for the copies still in flight into this
    // CTA's shared memory (chunks warp 0 staged but did not consume)
    if (w == 0 && l == 0)
        for (int k = c; k < produced; ++k) {
            const uint32_t g = gseq + (uint32_t)k;
            mbar_wait_bounded(&full[g % kStages], (g / kStages) & 1u, kWaitLimit);
        }
    __syncthreads();  // every thread agrees on the outcome
    if (s_abort) return false;
    gseq += (uint32_t)nchunks;
    if (i < nx && j < ny) img[(size_t)i * ny + j] = (float)acc * dxdy;
    return true;
}

}  // namespace sgd
