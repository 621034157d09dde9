// validity.cuh - the word-level validity of one output row segment
// (internal/stencil/mask.go:43-161), shared by the validity kernel and the
// batch kernel.
#pragma once

#include "launch.h"

namespace strata {

__device__ __forceinline__ int64_t min64(int64_t a, int64_t b) { return a < b ? a : b; }

__device__ __forceinline__ int64_t floor_div32(int64_t b) { return b >= 0 ? b >> 5 : -((-b + 31) >> 5); }

// 64 bits of the source mask from bit b on (b may be negative), with zeros
// for words outside [lo, hi].
__device__ __forceinline__ uint64_t bits64(const ValidityParams& v, int64_t b) {
    const int64_t w = floor_div32(b);
    const int sh = (int)(b - w * 32);
    const uint32_t* m = v.src_bits;
    const uint64_t a0 = (w >= v.src_lo_word && w <= v.src_hi_word) ? m[w] : 0u;
    const uint64_t a1 = (w + 1 >= v.src_lo_word && w + 1 <= v.src_hi_word) ? m[w + 1] : 0u;
    const uint64_t a2 = (w + 2 >= v.src_lo_word && w + 2 <= v.src_hi_word) ? m[w + 2] : 0u;
    uint64_t lo = a0 | (a1 << 32);
    if (sh == 0) return lo;
    return (lo >> sh) | (a2 << (64 - sh));
}

// Output bits of global cells (x .. x+31, y), bit j for cell x + j.
__device__ __forceinline__ uint32_t segment_bits(const ValidityParams& v, int64_t x, int64_t y) {
    const int r = v.radius;
    const int64_t W = v.width, H = v.height;
    if (r > 0 && (y < r || y >= H - r)) return 0u;
    uint32_t interior = 0xffffffffu;
    if (r > 0) {
        // bits j of cells x + j with r <= x + j < W - r: j in [lo, hi)
        const int64_t lo = r - x, hi = W - r - x;
        const uint32_t mlo = lo <= 0 ? 0xffffffffu : (lo >= 32 ? 0u : ~((1u << lo) - 1u));
        const uint32_t mhi = hi >= 32 ? 0xffffffffu : (hi <= 0 ? 0u : ((1u << hi) - 1u));
        interior = mlo & mhi;
    }
    if (!v.src_bits) return interior;
    uint64_t acc = ~0ull;
    const int64_t bx = x - r - v.src_x0;
    for (int j = -r; j <= r; j++) acc &= bits64(v, v.src_off + (y + j - v.src_y0) * v.src_stride + bx);
    uint64_t e = acc;
    for (int d = 1; d <= 2 * r; d++) e &= acc >> d;
    return (uint32_t)e & interior;
}

}  // namespace strata

namespace strata {

// Word k of output row y's bits over the cells [x0, x1) (global
// coordinates): k counts the 32-bit words the row segment touches, from the
// one holding cell x0. A word wholly inside the segment holds only its
// cells and is stored; a word the segment shares with other cells (a
// neighbouring tile or row, another raster) changes only the segment's
// bits, with atomics, so concurrent writers never lose each other's bits.
__device__ __forceinline__ void row_word_validity(const ValidityParams& v, int64_t y, int64_t x0, int64_t x1,
                                                  int64_t k) {
    const int64_t rowbit = v.dst_off + (y - v.dst_y0) * v.dst_stride - v.dst_x0;  // bit of cell (0, y)
    const int64_t b0 = rowbit + x0, b1 = rowbit + x1;
    const int64_t w = (b0 >> 5) + k;
    if (w * 32 >= b1) return;
    const int64_t lo = b0 > w * 32 ? b0 : w * 32;
    const int64_t hi = b1 < w * 32 + 32 ? b1 : w * 32 + 32;
    const int len = (int)(hi - lo), sh = (int)(lo - w * 32);
    const uint32_t lenmask = len == 32 ? 0xffffffffu : ((1u << len) - 1u);
    const uint32_t bits = (segment_bits(v, lo - rowbit, y) & lenmask) << sh;
    const uint32_t m = lenmask << sh;
    if (m == 0xffffffffu) {
        v.dst_bits[w] = bits;
    } else {
        atomicAnd(&v.dst_bits[w], ~m | bits);
        atomicOr(&v.dst_bits[w], bits);
    }
}

// The validity of the output cells [x0, x1) x [y0, y1), written by the
// nthreads threads of a block, one (row, word) pair at a time.
__device__ __forceinline__ void region_validity(const ValidityParams& v, int64_t x0, int64_t y0, int64_t x1,
                                                int64_t y1, int tid, int nthreads) {
    const int wpr = (int)((x1 - x0 + 31) / 32 + 1);  // words a row of the region can touch
    const int n = (int)(y1 - y0) * wpr;
    for (int i = tid; i < n; i += nthreads) {
        const int ry = i / wpr, k = i - ry * wpr;
        row_word_validity(v, y0 + ry, x0, x1, k);
    }
}

}  // namespace strata

// ---------------------------------------------------------------------------
// The warp-marching validity (validity.cu, batch.cu): a warp owns a strip
// of 1024 output cells (32 a lane) and marches down a band of rows. Per
// source row a lane loads the 2-3 words holding its 32 + 2r source bits,
// erodes them horizontally (the AND of 2r+1 shifts, in log2(2r+1) steps)
// and keeps the result in a ring of the last 2r+1 rows in registers, whose
// AND is the output segment. The lanes then trade their segments' edges by
// shuffle so that each lane writes one whole destination word, whatever
// the destination's bit offset and stride; only the words a warp shares
// with its neighbours (or a row with the next) take atomics, which change
// only the warp's own bits.

namespace strata {
namespace {

constexpr int kStripCells = 1024;  // output cells a warp covers across a row

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

// The validity of one warp's strip: output cells [cw, cw + 1024) (clipped
// to the region) of rows [y0, y0 + rows), lane l owning cells cw + 32 l ..
// cw + 32 l + 31. Every lane of the warp takes part.
template <int R>
__device__ __forceinline__ void validity_strip(const ValidityParams& v, int64_t cw, int64_t y0, int rows) {
    constexpr int D = 2 * R + 1;
    const int lane = threadIdx.x & 31;
    const int64_t c0 = cw + 32 * lane;  // the lane's first cell

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
    // The source rows' words, loaded 2R+1 rows ahead of their use so that
    // a warp keeps that many rows of loads in flight: slot m % (2R+1) holds
    // the words of source row y0 - R + m until row m is eroded.
    struct Raw {
        uint32_t a0, a1, a2;
        int sh;
    };
    int64_t lb = v.src_off + (y0 - R - v.src_y0) * v.src_stride + (c0 - R - v.src_x0);  // next row's bit
    auto load = [&]() -> Raw {
        Raw r;
        const int64_t w = floor_div32(lb);
        r.sh = (int)(lb - w * 32);
        r.a0 = src_word(v, w);
        r.a1 = src_word(v, w + 1);
        r.a2 = src_word(v, w + 2);
        lb += v.src_stride;
        return r;
    };
    auto eroded = [&](const Raw& r) -> uint32_t {
        const uint64_t win =
            (uint64_t)__funnelshift_r(r.a0, r.a1, r.sh) | ((uint64_t)__funnelshift_r(r.a1, r.a2, r.sh) << 32);
        return erode<D>(win);
    };
    Raw pa[D];
    if (masked) {
#pragma unroll
        for (int j = 0; j < D; j++) pa[j] = load();
    }
    uint32_t ring[D];
#pragma unroll
    for (int k = 0; k < 2 * R; k++) {
        ring[k] = 0xffffffffu;
        if (masked) {
            ring[k] = eroded(pa[k]);
            pa[k] = load();
        }
    }
    // Destination bit of cell cw in row y0, advanced a row at a time.
    int64_t db = v.dst_off + (y0 - v.dst_y0) * v.dst_stride + (cw - v.dst_x0);
    int64_t y = y0;
    for (int yb = 0; yb < rows; yb += D) {
#pragma unroll
        for (int u = 0; u < D; u++) {
            if (yb + u >= rows) break;
            const int slot = (u + 2 * R) % D;
            ring[slot] = 0xffffffffu;
            if (masked) {
                ring[slot] = eroded(pa[slot]);
                pa[slot] = load();
            }
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

}  // namespace
}  // namespace strata
