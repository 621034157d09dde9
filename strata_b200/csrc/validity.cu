// validity.cu - the validity of a stencil's output (internal/stencil/
// mask.go:43-161): bit (x, y) of the output is the AND of the input's bits
// over the (2r+1) x (2r+1) window at (x, y), cleared in the edge ring of
// radius r; radius 0 copies the bits.
//
// A warp owns a strip of 1024 output cells (32 a lane) and marches down a
// band of rows. Per source row a lane loads the 2-3 words holding its 32 +
// 2r source bits, erodes them horizontally (the AND of 2r+1 shifts, in
// log2(2r+1) steps) and keeps the result in a ring of the last 2r+1 rows
// in registers, whose AND is the output segment. The lanes then trade
// their segments' edges by shuffle so that each lane writes one whole
// destination word, whatever the destination's bit offset and stride;
// only the words a warp shares with its neighbours (or a row with the
// next) take atomics, which change only the warp's own bits.
#include <cuda_runtime.h>

#include "launch.h"
#include "validity.cuh"

namespace strata {
namespace {

constexpr int kStripCells = 1024;  // output cells a warp covers across a row
constexpr int kVThreads = 256;

// 32-bit word i of the source mask, 0 outside the words that hold the
// source's bits.
__device__ __forceinline__ uint32_t src_word(const ValidityParams& v, int64_t i) {
    return (i >= v.src_lo_word && i <= v.src_hi_word) ? v.src_bits[i] : 0u;
}

// Bit j (j < 32) of the result: the AND of bits j .. j + L - 1 of w.
template <int L>
__device__ __forceinline__ uint32_t erode(uint64_t w) {
    uint64_t e = w;
#pragma unroll
    for (int span = 1; span < L;) {
        const int t = span < L - span ? span : L - span;
        e &= e >> t;
        span += t;
    }
    return (uint32_t)e;
}

// Writes the 32 bits seg of lane's cells (ours: the bits that are the
// region's) at destination bit db + 32 lane, db the same for the warp.
__device__ __forceinline__ void put_bits(const ValidityParams& v, int64_t db, int lane, uint32_t seg, uint32_t ours) {
    const int64_t wb = floor_div32(db);
    const int s = (int)(db - wb * 32);
    // Every lane takes part in both shuffles; lane 0 then drops what it got.
    const uint32_t pseg = __shfl_up_sync(0xffffffffu, seg, 1);
    const uint32_t pours = __shfl_up_sync(0xffffffffu, ours, 1);
    uint32_t val = seg << s, m = ours << s;
    if (s && lane) {
        val |= pseg >> (32 - s);
        m |= pours >> (32 - s);
    }
    uint32_t* w = v.dst_bits + wb + lane;
    if (m == 0xffffffffu) {
        *w = val;
    } else if (m) {
        atomicAnd(w, ~m | val);
        atomicOr(w, val & m);
    }
    if (lane == 31 && s) {
        // The bits of lane 31 that spill into the next word.
        const uint32_t tm = ours >> (32 - s), tv = seg >> (32 - s);
        if (tm) {
            atomicAnd(w + 1, ~tm | tv);
            atomicOr(w + 1, tv & tm);
        }
    }
}

template <int R>
__global__ void __launch_bounds__(kVThreads) validity_march_kernel(const __grid_constant__ ValidityParams v, int strips,
                                                                   int band) {
    constexpr int D = 2 * R + 1;
    const int warp = (int)((blockIdx.x * (unsigned)kVThreads + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    const int strip = warp % strips, bnd = warp / strips;
    const int64_t y0 = v.out_y0 + (int64_t)bnd * band;
    if (y0 >= v.out_y1) return;  // the whole warp
    const int rows = (int)((y0 + band < v.out_y1 ? y0 + band : v.out_y1) - y0);
    const int64_t cw = v.out_x0 + (int64_t)strip * kStripCells;  // the warp's first cell
    const int64_t c0 = cw + 32 * lane;                            // the lane's first cell

    // The lane's cells inside the region, and inside the edge ring's interior.
    uint32_t ours = 0u, colin = 0u;
    {
        const int64_t n = v.out_x1 - c0;
        ours = n >= 32 ? 0xffffffffu : (n <= 0 ? 0u : ((1u << n) - 1u));
        const int64_t lo = R - c0, hi = v.width - R - c0;  // bits j with lo <= j < hi
        const uint32_t mlo = lo <= 0 ? 0xffffffffu : (lo >= 32 ? 0u : ~((1u << lo) - 1u));
        const uint32_t mhi = hi >= 32 ? 0xffffffffu : (hi <= 0 ? 0u : ((1u << hi) - 1u));
        colin = mlo & mhi;
    }
    const bool masked = v.src_bits != nullptr;
    // Source bit of cell (c0 - R) in row y0 - R, advanced a row at a time.
    int64_t sb = v.src_off + (y0 - R - v.src_y0) * v.src_stride + (c0 - R - v.src_x0);
    auto hrow = [&]() -> uint32_t {
        uint32_t h = 0xffffffffu;
        if (masked) {
            const int64_t w = floor_div32(sb);
            const int sh = (int)(sb - w * 32);
            const uint32_t a0 = src_word(v, w), a1 = src_word(v, w + 1), a2 = src_word(v, w + 2);
            const uint64_t win = (uint64_t)__funnelshift_r(a0, a1, sh) | ((uint64_t)__funnelshift_r(a1, a2, sh) << 32);
            h = erode<D>(win);
        }
        sb += v.src_stride;
        return h;
    };
    uint32_t ring[D];
#pragma unroll
    for (int k = 0; k < 2 * R; k++) ring[k] = hrow();
    // Destination bit of cell cw in row y0, advanced a row at a time.
    int64_t db = v.dst_off + (y0 - v.dst_y0) * v.dst_stride + (cw - v.dst_x0);
    int64_t y = y0;
    for (int yb = 0; yb < rows; yb += D) {
#pragma unroll
        for (int u = 0; u < D; u++) {
            if (yb + u >= rows) break;
            ring[(u + 2 * R) % D] = hrow();
            uint32_t e = 0xffffffffu;
#pragma unroll
            for (int k = 0; k < D; k++) e &= ring[k];
            const bool rowin = y >= R && y < v.height - R;
            put_bits(v, db, lane, rowin ? (e & colin) : 0u, ours);
            db += v.dst_stride;
            y++;
        }
    }
}

template <int R>
void launch_r(const ValidityParams& v, cudaStream_t s) {
    const int64_t w = v.out_x1 - v.out_x0, h = v.out_y1 - v.out_y0;
    const int64_t strips = (w + kStripCells - 1) / kStripCells;
    // About 48 warps an SM in all, in bands of at least 8 rows.
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int64_t bands = ((int64_t)sms * 48 + strips - 1) / strips;
    int64_t band = (h + bands - 1) / bands;
    if (band < 8) band = 8;
    bands = (h + band - 1) / band;
    const int64_t warps = strips * bands;
    const int64_t blocks = (warps * 32 + kVThreads - 1) / kVThreads;
    validity_march_kernel<R><<<(unsigned)blocks, kVThreads, 0, s>>>(v, (int)strips, (int)band);
}

}  // namespace

void launch_validity(const ValidityParams& v, cudaStream_t s) {
    if (v.dst_words <= 0 || v.out_x1 <= v.out_x0 || v.out_y1 <= v.out_y0) return;
    switch (v.radius) {
    case 0: launch_r<0>(v, s); break;
    case 1: launch_r<1>(v, s); break;
    case 2: launch_r<2>(v, s); break;
    case 3: launch_r<3>(v, s); break;
    case 4: launch_r<4>(v, s); break;
    case 5: launch_r<5>(v, s); break;
    case 6: launch_r<6>(v, s); break;
    case 7: launch_r<7>(v, s); break;
    case 8: launch_r<8>(v, s); break;
    }
}

}  // namespace strata
