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
