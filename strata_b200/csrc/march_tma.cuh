// march_tma.cuh - what the radius-1 marching kernels share: the warp's
// strip of the region, tensor copies (TMA) of source rows into a per-warp
// shared-memory ring completed on mbarriers with bounded waits, and the
// output validity a march writes beside its cells.
#pragma once

#include <cuda.h>

#include "launch.h"
#include "march.cuh"

namespace strata {
namespace {

// What every marching kernel works out first: the warp's columns, rows and
// interior tests, and where its outputs go.
struct Strip {
    int64_t xs, x, y0;
    int rows, lane;
    bool active, last;
    bool colin[4];
    int yrel, ylast;
    float* d0;
    float* d1;
};

template <int OP>
__device__ __forceinline__ bool strip_setup(const LaunchParams& P, int strip, int col_blocks, Strip& S) {
    S.lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int cb = blockIdx.x % col_blocks;
    const int sb = blockIdx.x / col_blocks;
    S.xs = P.out_x0 + (int64_t)(cb * kWarps + warp) * 128;
    if (S.xs >= P.out_x1) return false;  // warp-uniform
    S.x = S.xs + 4 * S.lane;
    S.y0 = P.out_y0 + (int64_t)sb * strip;
    S.rows = (int)min((int64_t)strip, P.out_y1 - S.y0);
    // The region's width is a multiple of 4, so a lane is wholly in or out.
    S.active = S.x < P.out_x1;
    S.last = S.active && (S.lane == 31 || S.x + 4 >= P.out_x1);
    const int64_t W = P.width;
#pragma unroll
    for (int i = 0; i < 4; i++) S.colin[i] = S.x + i >= 1 && S.x + i < W - 1;
    S.yrel = (int)(S.y0 - 1);
    S.ylast = (int)(P.height - 2);
    S.d0 = P.dst0 + (S.y0 - P.dst_y0) * P.dst0_stride + (S.x - P.dst_x0);
    S.d1 = OP == STRATA_OP_GRADIENT ? P.dst1 + (S.y0 - P.dst_y0) * P.dst1_stride + (S.x - P.dst_x0) : nullptr;
    return true;
}

template <int OP>
__device__ __forceinline__ void store_row(const LaunchParams& P, Strip& S, const float (&o0)[4],
                                          const float (&o1)[4]) {
    if (S.active) {
        *reinterpret_cast<float4*>(S.d0) = make_float4(o0[0], o0[1], o0[2], o0[3]);
        if constexpr (OP == STRATA_OP_GRADIENT)
            *reinterpret_cast<float4*>(S.d1) = make_float4(o1[0], o1[1], o1[2], o1[3]);
    }
    S.d0 += P.dst0_stride;
    if constexpr (OP == STRATA_OP_GRADIENT) S.d1 += P.dst1_stride;
}

// ---------------------------------------------------------------------------
// Output validity written by the march (VAL kernels), so that no second
// kernel walks the rows again: bit (x, y) of an output is the AND of the
// source's bits over the 3x3 window at (x, y), cleared in the edge ring
// (internal/stencil/mask.go:43-161, internal/exec/halo.go:213-229).
//
// At the start of its strip a warp copies the source words of every row
// of the strip (the 130 bits of columns xs-1 .. xs+128, six 32-bit words a
// row) into shared memory with 4-byte cp.async copies, all in flight at
// once; they land while the warp marches the strip's cells. After the
// march the warp writes the strip's validity in one short phase that holds
// none of the march's registers: each lane owns the 32 cells xs+32j ..
// xs+32j+31 (j = lane % 4) of 8 consecutive output rows, erodes each of
// the 10 source rows they read across into one word (bit i: the AND of
// columns x+i-1 .. x+i+1), and stores the AND of three of them with the
// interior and region bits per output row. A destination word wholly the
// lane's takes a plain store; words shared with other cells (another
// lane's or warp's, another row's, another raster's) take atomics that
// change only the lane's bits.

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ int64_t floor_div32_(int64_t b) { return b >= 0 ? b >> 5 : -((-b + 31) >> 5); }

constexpr int kMaxStrip = 64;             // output rows of a warp's strip (the launchers cap it)
constexpr int kVMaxRows = kMaxStrip + 2;  // source rows of a strip: its output rows and their halo rows
constexpr int kVWords = 6;                // words holding a source row's 130 bits
constexpr int kVRowsPerLane = kMaxStrip / 8;  // output rows a lane writes (8 lanes share a column word)

// Sets the bits m of word w to those of val.
__device__ __forceinline__ void put_word(uint32_t* w, uint32_t val, uint32_t m) {
    if (m == 0xffffffffu) {
        *w = val;
    } else if (m) {
        atomicAnd(w, ~m | val);
        atomicOr(w, val & m);
    }
}

// Bit of column xs - 1 of source row y0 - 1 (m = 0) of the warp's strip.
__device__ __forceinline__ int64_t vbit0(const LaunchParams& P, int64_t xs, int64_t y0) {
    return P.vf.src_off + (y0 - 1 - P.src_y0) * P.vf.src_stride + (xs - 1 - P.src_x0);
}

// Starts the copies of the source words of rows y0-1 .. y0+rows into w.
__device__ __forceinline__ void valid_prefetch(const LaunchParams& P, int64_t xs, int64_t y0, int rows, uint32_t* w,
                                               int lane) {
    if (!P.vf.src_bits) return;
    const int64_t bit0 = vbit0(P, xs, y0);
    const int row0 = (int)(y0 - 1 - P.src_y0);
    const int n = (rows + 2) * kVWords;
    for (int i = lane; i < n; i += 32) {
        const int m = i / kVWords, j = i - m * kVWords;
        const int64_t k = floor_div32_(bit0 + (int64_t)m * P.vf.src_stride) + j;
        uint32_t* d = w + i;
        if ((unsigned)(row0 + m) < (unsigned)P.src_h && k >= P.vf.src_lo_word && k <= P.vf.src_hi_word)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(d)), "l"(P.vf.src_bits + k)
                         : "memory");
        else
            *d = 0u;
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// Waits for the copies (on every path, so none outlives the block).
__device__ __forceinline__ void valid_wait(const LaunchParams& P) {
    if (!P.vf.src_bits) return;
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncwarp();
}

// Writes the 32 bits v of cells c0 .. c0+31 (ours: those of the region)
// at bit D of a destination mask.
__device__ __forceinline__ void put_bits(uint32_t* bits, int64_t D, uint32_t v, uint32_t ours) {
    const int64_t wb = D >> 5;
    const int sh = (int)(D & 31);
    if (sh == 0) {
        put_word(bits + wb, v, ours);
    } else {
        put_word(bits + wb, v << sh, ours << sh);
        put_word(bits + wb + 1, v >> (32 - sh), ours >> (32 - sh));
    }
}

// The strip's validity: output rows y0 .. y0+rows-1 of columns xs ..
// xs+127 (clipped to the region), from the words valid_prefetch copied;
// emit(y, c0, v, ours) writes the 32 bits v of cells c0 .. c0+31 of row y
// (ours: those inside the region) to every masked output.
template <class Emit>
__device__ __forceinline__ void valid_strip_emit(const LaunchParams& P, int64_t xs, int64_t y0, int rows,
                                                 const uint32_t* w, int lane, Emit emit) {
    const int j = lane & 3, k0 = (lane >> 2) * kVRowsPerLane;
    if (k0 >= rows) return;
    const int64_t c0 = xs + 32 * j;
    // cells c0 + i with 1 <= c0 + i < W - 1 (the edge ring's columns) and c0 + i < out_x1
    const int64_t lo = 1 - c0, hi = (P.width - 1 < P.out_x1 ? P.width - 1 : P.out_x1) - c0;
    const uint32_t keep = (lo <= 0 ? 0xffffffffu : (lo >= 32 ? 0u : ~((1u << lo) - 1u))) &
                          (hi >= 32 ? 0xffffffffu : (hi <= 0 ? 0u : ((1u << hi) - 1u)));
    const int64_t nreg = P.out_x1 - c0;
    const uint32_t ours = nreg >= 32 ? 0xffffffffu : (nreg <= 0 ? 0u : ((1u << nreg) - 1u));
    const int b31 = (int)(vbit0(P, xs, y0) & 31), s31 = (int)(P.vf.src_stride & 31);
    auto eroded = [&](int m) -> uint32_t {
        if (!P.vf.src_bits) return 0xffffffffu;
        const int sh = (b31 + m * s31) & 31;
        const uint32_t* r = w + m * kVWords + j;
        const uint64_t x = (uint64_t)__funnelshift_r(r[0], r[1], sh) | ((uint64_t)__funnelshift_r(r[1], r[2], sh) << 32);
        return (uint32_t)(x & (x >> 1) & (x >> 2));
    };
    uint32_t a = eroded(k0), b = eroded(k0 + 1);
    const int kend = min(k0 + kVRowsPerLane, rows);
    for (int k = k0; k < kend; k++) {
        const uint32_t c = eroded(k + 2);
        const int64_t y = y0 + k;
        const uint32_t v = (y >= 1 && y < P.height - 1) ? (a & b & c & keep) : 0u;
        a = b;
        b = c;
        emit(y, c0, v, ours);
    }
}

// The validity of a single-op launch's outputs (P.vf.dst_bits).
__device__ __forceinline__ void valid_strip(const LaunchParams& P, int64_t xs, int64_t y0, int rows,
                                            const uint32_t* w, int lane) {
    valid_strip_emit(P, xs, y0, rows, w, lane, [&](int64_t y, int64_t c0, uint32_t v, uint32_t ours) {
#pragma unroll
        for (int i = 0; i < 2; i++)
            if (P.vf.dst_bits[i])
                put_bits(P.vf.dst_bits[i], P.vf.dst_off[i] + (y - P.dst_y0) * P.vf.dst_stride[i] + (c0 - P.dst_x0), v,
                         ours);
    });
}

// ---------------------------------------------------------------------------
// Tensor copies (TMA) into a per-warp shared-memory ring.

constexpr int kBoxRows = 4;            // rows per tensor copy
constexpr int kBoxCols = 136;          // columns xs-4 .. xs+131
constexpr int kBoxes = 3;              // ring slots (boxes in flight) per warp
constexpr uint32_t kBoxBytes = kBoxRows * kBoxCols * 4;
constexpr uint32_t kSpinLimit = 1u << 20;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// The bounded wait for the phase of `parity` on bar; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = kSpinLimit) {
    for (uint32_t i = 0; !mbar_try_wait(bar, parity); i++)
        if (i >= limit) return false;
    return true;
}

// One box of the source tensor (kBoxCols x kBoxRows cells whose first cell
// is column x, row y of the source) into 128-byte aligned shared memory,
// completing on bar. Cells outside the source read as zero. No multicast:
// the destination is this CTA's own shared memory.
__device__ __forceinline__ void tma_box(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}


}  // namespace

// The source as a 2-D tensor for the box copies (march3.cu): false when the
// tensor map cannot be encoded.
bool source_map(const LaunchParams& p, CUtensorMap* map);

}  // namespace strata
