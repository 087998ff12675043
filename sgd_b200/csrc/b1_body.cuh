// Bodies of the B1 projection kernels, shared by the single-geometry kernels
// (b1.cu) and the persistent batched kernels (b1_batch.cu).
//
//   b1_forward_row   detector-driven: one warp per (view, bin).  Lanes split
//                    the lines (major axis) the bin's ray strip crosses; each
//                    lane evaluates the footprint of the few pixels of its line
//                    inside the strip (packed-pair form, b1_kernels.cuh), and
//                    the warp reduces with shuffles.  The sinogram value is
//                    written once, no atomics.
//   b1_back_tile     voxel-driven: two pixels per thread (rows i and i + 4)
//                    of a 32x8 tile, 128 threads.  Per
//                    chunk of VC views the CTA stages the bin window its tile
//                    projects onto in shared memory: the 64-byte footprint
//                    records by TMA bulk copies completed on an mbarrier
//                    (double-buffered, the next chunk in flight while this one
//                    is evaluated), the sinogram values by plain loads, as five
//                    planes of 16-byte words per view whose stride WCAP is a
//                    compile-time constant (one address per evaluation, the
//                    five loads at fixed offsets from it), closed by a null
//                    bin whose footprint is zero.  Each thread evaluates a
//                    bin's two edges as one packed-FP32 pair (the record's
//                    operand pairs as staged), accumulates over all views in
//                    registers and writes its pixel once, no atomics.
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
constexpr int kBackThreads = kBackTI * kBackTJ / 2;  // two pixels per thread
constexpr uint32_t kWaitLimit = 1u << 22;

// 2 mbarriers | 3 x VC windows | 3 x VC homographies, then the staged planes
template <int VC>
__host__ __device__ constexpr int b1_header_bytes() {
    return 16 + 3 * VC * 8 + 3 * VC * 32;
}

// Staged planes per view: the four record chunks; the sinogram value of a
// bin replaces the staged copy of its record's last field (a, which the
// projection does not read), so one 16-byte load brings both.
constexpr int kBackPlanes = 4;

// Shared memory of the back tile: two chunk slots of VC views, each view
// kBackPlanes planes of WCAP 16-byte words.  A view's window of bins must
// leave room for the null bin: widest window + 1 <= WCAP.
template <int VC, int WCAP>
__host__ __device__ constexpr size_t b1_back_smem() {
    return b1_header_bytes<VC>() + (size_t)2 * VC * kBackPlanes * WCAP * 16;
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
                const float xv = __ldg(sp);  // issued before the footprint math, which hides its latency
                const float conv = b1_conv_pair(b1_edges2(fn, inner, k), k);
                if (conv > kConvEps) row = fmaf(conv, xv, row);
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
                const float xv = __ldg(sp);
                const float conv = b1_conv_pair(b1_edges2(fm, b1_inner2(fn, k), k), k);
                if (conv > kConvEps) row = fmaf(conv, xv, row);
            }
            acc += (double)row;
        }
    }
    acc = warp_sum(acc);
    if (lane == 0) sino[gw] = (float)acc * dxdy;
}

// Back projection of the 32x8 tile at (i0, j0).  twin[p] = (lo, hi): bins of
// view p the tile's pixels can touch (host-computed, conservative; at most
// WCAP - 1 of them).  The CTA's two mbarriers (at the start of smem) are
// initialised by the caller; use0/use1 count the phases barriers 0/1
// completed before this tile, so that a persistent CTA can run many tiles on
// the same barriers.  Returns false, with *err set and the tile unwritten,
// when a staged chunk never arrived (bounded wait); the CTA's barriers are
// then out of step and it must not run further tiles.
// wait_limit: polls of each staging wait before it gives up (kWaitLimit in
// production; a test sets 0 to take the failure path).
template <int VC, int WCAP>
__device__ __forceinline__ bool b1_back_tile(const float4* __restrict__ rec, const BinHomography* __restrict__ hom,
                                             const int2* __restrict__ twin, const float* __restrict__ sino,
                                             float* __restrict__ img, int nx, int ny, int np, int nu, float dxdy,
                                             int* __restrict__ err, uint32_t wait_limit, int i0, int j0,
                                             unsigned char* smem, uint32_t& use0,
                                             uint32_t& use1) {
    constexpr int kHeader = b1_header_bytes<VC>();
    static_assert(kHeader % 16 == 0, "staged records must start 16-byte aligned");
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem);           // [2]
    int* win = reinterpret_cast<int*>(smem + 16);                   // [3][VC][2]
    float* hs = reinterpret_cast<float*>(smem + 16 + 3 * VC * 8);  // [3][VC][8]
    float4* srec = reinterpret_cast<float4*>(smem + kHeader);      // [2][VC][kBackPlanes][WCAP]

    // warp w covers columns j0 + 8w .. + 7 of rows i0 .. i0 + 3 (pixel A) and
    // of rows i0 + 4 .. i0 + 7 (pixel B): 8 x 4 blocks whose lanes read few
    // distinct bins of a view.  Each quarter-warp (the lanes of one shared
    // memory wavefront of 16-byte loads) takes a 2 x 4 block of it, whose
    // bins span fewer 16-byte words than a row of 8 pixels would
    const int tid = threadIdx.x, w = tid >> 5, l = tid & 31;
    const int quarter = l >> 3, r = l & 7;
    const int i = i0 + 2 * (quarter >> 1) + (r >> 2), j = j0 + 8 * w + 4 * (quarter & 1) + (r & 3), iB = i + 4;
    const float fi = (float)i, fj = (float)j, fiB = (float)iB;
    const float2 fi2 = pair(fi), fj2 = pair(fj), fiB2 = pair(fiB);
    const int nchunks = (np + VC - 1) / VC;
    auto parity = [&](int c) { return (((c & 1) ? use1 : use0) + (uint32_t)(c >> 1)) & 1u; };

    // stage chunk c: windows and homographies (read after the next barrier),
    // the null bin after each window, and footprint records by TMA, lane v of
    // warp 0 taking view v; sinogram values by all threads
    auto stage = [&](int c) {
        const int st = c & 1, slot = c % 3;
        if (w == 0) {
            const int p = c * VC + l;
            int2 lh = make_int2(0, -1);
            uint32_t bytes = 0;
            if (l < VC) {
                if (p < np) {
                    lh = __ldg(twin + p);
                    const BinHomography H = hom[p];
                    float* h = hs + (slot * VC + l) * 8;
                    h[0] = H.n0; h[1] = H.n1; h[2] = H.n2; h[3] = H.d0; h[4] = H.d1; h[5] = H.d2;
                    h[6] = fabsf(H.d0) + fabsf(H.d1);
                }
                win[(slot * VC + l) * 2] = lh.x;
                win[(slot * VC + l) * 2 + 1] = lh.y;
                const int n = lh.y >= lh.x ? lh.y - lh.x + 1 : 0;
                bytes = (uint32_t)n * sizeof(B1Bin);
                // the null bin: edges 4 and 5 half-widths from the pixel,
                // beta = 0 and 1/a = 0, so conv = 0; sinogram 0
                float4* nb = srec + (st * VC + l) * kBackPlanes * WCAP + n;
                nb[0] = make_float4(0.f, 0.f, 0.f, 0.f);
                nb[WCAP] = make_float4(4.f, 5.f, 0.f, 0.f);
                nb[2 * WCAP] = make_float4(1.f, 1.f, 0.f, 0.f);
                nb[3 * WCAP] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
            if (l == 0) mbar_arrive_expect_tx(&bars[st], bytes);
            __syncwarp();
            if (l < VC && lh.y >= lh.x) {
                fence_proxy_async_smem();
                const uint32_t n = (uint32_t)(lh.y - lh.x + 1) * 16u;
                for (int q = 0; q < 4; ++q)
                    bulk_copy_g2s(srec + ((st * VC + l) * kBackPlanes + q) * WCAP,
                                  rec + ((size_t)p * 4 + q) * nu + lh.x, n, &bars[st]);
            }
        }
    };

    // sinogram values of chunk c into registers (element e = v * WCAP + k of
    // the chunk's windows, thread tid taking e = tid + s * kBackThreads; 0
    // beyond a view's window), loaded while the chunk before is evaluated
    constexpr int kSR = (VC * WCAP + kBackThreads - 1) / kBackThreads;
    auto prefetch = [&](int c, float* r) {
#pragma unroll
        for (int s2 = 0; s2 < kSR; ++s2) {
            const int e = tid + s2 * kBackThreads, v = e / WCAP, k = e - v * WCAP, p = c * VC + v;
            r[s2] = 0.f;
            if (v < VC && p < np) {
                const int2 lh = __ldg(twin + p);
                if (k <= lh.y - lh.x) r[s2] = __ldg(sino + (size_t)p * nu + lh.x + k);
            }
        }
    };
    // ... and into the .w of the staged records' last plane once chunk c's
    // copies have landed (the copies wrote that field).  Every element of
    // the slot is written: past a window's end the value is 0, which is also
    // the null bin's, and nothing reads that part of the slot.  No element
    // depends on the staged windows, which warp 0 may still be writing for
    // this chunk when the other warps get here.
    auto place = [&](int c, const float* r) {
        const int st = c & 1;
#pragma unroll
        for (int s2 = 0; s2 < kSR; ++s2) {
            const int e = tid + s2 * kBackThreads, v = e / WCAP, k = e - v * WCAP;
            if (v < VC) reinterpret_cast<float*>(srec + ((st * VC + v) * kBackPlanes + 3) * WCAP + k)[3] = r[s2];
        }
        fence_proxy_async_smem();  // before the bulk copies that will overwrite them
    };
    // wait (bounded) for chunk c's copies and place its sinogram; a wait
    // that gave up sets the device error and this thread's failed flag,
    // which the next CTA barrier ORs over the threads
    bool failed = false;
    auto land = [&](int c, const float* r) {
        if (mbar_wait_bounded(&bars[c & 1], parity(c), wait_limit)) {
            place(c, r);
        } else {
            failed = true;
            atomicExch(err, 1);
        }
    };

    // chunk f's copies never arrived: wait for them (bounded, full limit), so
    // that no bulk copy is still landing in this CTA's shared memory when it
    // moves on or exits (chunk f + 1 is staged only after f has landed)
    auto drain = [&](int f) {
        if (tid == 0) mbar_wait_bounded(&bars[f & 1], parity(f), kWaitLimit);
    };

    // One CTA barrier per chunk: chunk c + 1 is staged after the barrier that
    // ends chunk c - 1 (its slot's last reader), and its copies land while
    // chunk c is evaluated; each thread then waits for them and places its
    // share of their sinogram before the next barrier, which makes both
    // visible to chunk c + 1's evaluation.
    __syncthreads();  // the previous tile's last chunk is fully consumed
    stage(0);
    float sv[kSR];
    prefetch(0, sv);
    land(0, sv);

    const bool inA = i < nx && j < ny, hasB = iB < nx;
    double acc = 0.0, accB = 0.0;  // FP32 within a chunk (a few tens of terms), FP64 across chunks
    for (int c = 0; c < nchunks; ++c) {
        // chunk c landed, placed and its windows visible; chunk c-1 fully
        // consumed.  Every thread leaves on the same barrier's answer (a
        // flag in shared memory could be set for chunk c + 1 by a fast
        // thread before a slow one has read it for chunk c).
        if (__syncthreads_or(failed)) {
            drain(c);
            return false;
        }
        if (c + 1 < nchunks) {
            stage(c + 1);
            prefetch(c + 1, sv);  // chunk c's values are in place: sv is free
        }
        const int st = c & 1, slot = c % 3;
        if (inA) {
            float csum = 0.f, csumB = 0.f;
#pragma unroll
            for (int v = 0; v < VC; ++v) {
                const int lo = win[(slot * VC + v) * 2], hi = win[(slot * VC + v) * 2 + 1];
                if (hi < lo) continue;
                int a, b, aB, bB;
                box_bins_bound(hs + (slot * VC + v) * 8, fi, fj, nu, a, b);
                box_bins_bound(hs + (slot * VC + v) * 8, fiB, fj, nu, aB, bB);
                // window-relative ranges; top is the null bin
                const int top = hi - lo + 1;
                a = max(a, lo) - lo;
                b = min(b, hi) - lo;
                aB = max(aB, lo) - lo;
                bB = hasB ? min(bB, hi) - lo : -1;
                const float4* rb = srec + (st * VC + v) * kBackPlanes * WCAP;
                // per view, each pixel's bins in one loop: trip counts differ by
                // at most one bin between the lanes of a warp.  (A single flat
                // loop over all the chunk's (view, bin) pairs, switching views
                // per lane, measured 1.38x slower at 512^2 x 720 views: the warp
                // ran the switch on most iterations.)  The two pixels' k-th bins
                // are evaluated side by side, two independent chains; a pixel
                // whose bins ran out evaluates the null bin.
                const int n = max(b - a, bB - aB) + 1;
#pragma unroll 1
                for (int k = 0; k < n; ++k) {
                    const float4* qA = rb + (a + k <= b ? a + k : top);
                    const float4* qB = rb + (aB + k <= bB ? aB + k : top);
                    const B1Pair kA = b1_pair(B1Bin{qA[0], qA[WCAP], qA[2 * WCAP], qA[3 * WCAP]});
                    const B1Pair kB = b1_pair(B1Bin{qB[0], qB[WCAP], qB[2 * WCAP], qB[3 * WCAP]});
                    const float sA = qA[3 * WCAP].w, sB = qB[3 * WCAP].w;
                    const float convA = b1_conv_pair(b1_edges2(fi2, b1_inner2(fj2, kA), kA), kA);
                    const float convB = b1_conv_pair(b1_edges2(fiB2, b1_inner2(fj2, kB), kB), kB);
                    if (convA > kConvEps) csum = fmaf(convA, sA, csum);
                    if (convB > kConvEps) csumB = fmaf(convB, sB, csumB);
                }
            }
            acc += (double)csum;
            accB += (double)csumB;
        }
        if (c + 1 < nchunks) land(c + 1, sv);
    }
    use0 += (uint32_t)((nchunks + 1) >> 1);
    use1 += (uint32_t)(nchunks >> 1);
    if (i < nx && j < ny) img[(size_t)i * ny + j] = (float)acc * dxdy;
    if (iB < nx && j < ny) img[(size_t)iB * ny + j] = (float)accB * dxdy;
    return true;
}

}  // namespace sgd
