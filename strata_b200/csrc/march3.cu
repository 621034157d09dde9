// march3.cu - the radius-1 data kernels: register marching down row strips.
//
// Each warp owns 128 consecutive columns of a strip of rows, four per
// lane, and walks down the strip keeping the window's three rows in
// registers, so every input cell is read from memory once per strip plus
// two halo rows. Each lane writes its four results with one float4 store.
//
// Rows reach the registers one of two ways:
//   * march3_tma_kernel (the default): each warp has a private ring of
//     boxes in shared memory, each box four rows of its 128 columns plus
//     halo, filled by tensor copies (cp.async.bulk.tensor.2d, the TMA
//     engine, completion counted on an mbarrier; cells outside the source
//     read as zero, so no copy needs clipping). Lane 0 keeps kBoxes boxes
//     (up to 12 rows) in flight per warp, so the memory system sees many
//     rows of loads per warp without registers holding them; a lane reads
//     its four cells with one LDS.128 and takes its neighbours by warp
//     shuffle. Every wait is bounded: on a timeout the kernel records
//     STRATA_ETIMEDOUT in the status word, waits (bounded) for its own
//     copies in flight and returns.
//   * march3_kernel: aligned float4 loads straight into registers, one row
//     ahead, when the tensor map cannot be encoded.
//
// Horn ops (gradient, slope, aspect, hillshade) reuse each row's
// horizontal differences: hornDX's z3 - z1, z6 - z4 and z9 - z7
// (internal/stencil/horn.go:152-155) are one row's x+1 minus x-1 seen as
// the window's top, middle and bottom row, so each row's difference is
// computed once and used by three output rows. The operations and their
// order per cell are the reference's, so the bits are too. The other ops
// evaluate apply3 (ops3.cuh), shared with the batch kernels' march.
//
// The launcher takes these paths only when every row of the source and
// destination starts on a 16-byte boundary at the region's first column
// and the region is a multiple of 4 wide; otherwise march_any_kernel runs
// the same march with per-cell loads and stores (march.cuh march_warp).
#include <cuda.h>

#include "launch.h"
#include "march.cuh"
#include "ops3.cuh"

namespace strata {
namespace {

using namespace cell;

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

// The strip's validity: output rows y0 .. y0+rows-1 of columns xs ..
// xs+127 (clipped to the region), from the words valid_prefetch copied.
__device__ __forceinline__ void valid_strip(const LaunchParams& P, int64_t xs, int64_t y0, int rows,
                                            const uint32_t* w, int lane) {
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
#pragma unroll
        for (int i = 0; i < 2; i++) {
            if (!P.vf.dst_bits[i]) continue;
            const int64_t D = P.vf.dst_off[i] + (y - P.dst_y0) * P.vf.dst_stride[i] + (c0 - P.dst_x0);
            const int64_t wb = D >> 5;
            const int sh = (int)(D & 31);
            if (sh == 0) {
                put_word(P.vf.dst_bits[i] + wb, v, ours);
            } else {
                put_word(P.vf.dst_bits[i] + wb, v << sh, ours << sh);
                put_word(P.vf.dst_bits[i] + wb + 1, v >> (32 - sh), ours >> (32 - sh));
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Loads straight into registers.

struct Lane {
    const float* p;  // &src[row][x] of the next row to load
    int64_t stride;
    int by, src_h;  // next row, relative to the source's first row
    bool active, first, last, left_in, right_in;
};

__device__ __forceinline__ Row6 load_row(Lane& L) {
    Row6 r;
    float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
    const bool in = L.by >= 0 && L.by < L.src_h;
    if (in && L.active) q = __ldg(reinterpret_cast<const float4*>(L.p));
    float l = __shfl_up_sync(kFull, q.w, 1);
    float rr = __shfl_down_sync(kFull, q.x, 1);
    if (L.first) l = (in && L.left_in) ? __ldg(L.p - 1) : 0.f;
    if (L.last) rr = (in && L.right_in) ? __ldg(L.p + 4) : 0.f;
    r.v[0] = l;
    r.v[1] = q.x;
    r.v[2] = q.y;
    r.v[3] = q.z;
    r.v[4] = q.w;
    r.v[5] = rr;
    L.p += L.stride;
    L.by++;
    return r;
}

constexpr int kRing = 4;  // three window rows and one in flight

template <int OP, int KIND, bool EPI, bool VAL>
__global__ void __launch_bounds__(kWarps * 32, 6) march3_kernel(const __grid_constant__ LaunchParams P, int strip,
                                                                 int col_blocks) {
    constexpr bool kHorn = kIsHorn<OP>;
    EpiTables* T = EpiSmem<EPI>::get();
    if constexpr (EPI) {
        stage_epilogue(P, *T);
        __syncthreads();
    }
    Strip S;
    if (!strip_setup<OP>(P, strip, col_blocks, S)) return;
    Lane L;
    L.active = S.active;
    L.first = S.lane == 0;
    L.last = S.last;
    L.left_in = S.x - 1 >= P.src_x0;
    L.right_in = S.x + 4 < P.src_x0 + P.src_w;
    L.stride = P.src_stride;
    L.by = (int)(S.y0 - 1 - P.src_y0);
    L.src_h = (int)P.src_h;
    L.p = P.src + (int64_t)L.by * P.src_stride + (S.x - P.src_x0);
    const int rows = S.rows;

    // Ring slot m % kRing holds row y0 - 1 + m; output row y0 + k reads
    // m = k .. k + 2, and row k + 3 loads while row k computes. The
    // validity ring (VAL) has the same slots and loads four rows ahead.
    Row6 ring[kRing];
    float hr[kRing][4];
    __shared__ uint32_t vwords[VAL ? kWarps : 1][VAL ? kVMaxRows * kVWords : 1];
    if constexpr (VAL) valid_prefetch(P, S.xs, S.y0, rows, vwords[threadIdx.x >> 5], S.lane);
#pragma unroll
    for (int j = 0; j < 3; j++) {
        ring[j] = load_row(L);
        if constexpr (kHorn) hdiff(ring[j], hr[j]);
    }
    for (int k0 = 0; k0 < rows; k0 += kRing) {
#pragma unroll
        for (int u = 0; u < kRing; u++) {
            const int k = k0 + u;
            if (k >= rows) break;
            if (k + 1 < rows) {
                ring[(u + 3) % kRing] = load_row(L);
                if constexpr (kHorn) hdiff(ring[(u + 3) % kRing], hr[(u + 3) % kRing]);
            }
            S.yrel++;
            const bool rowin = S.yrel >= 1 && S.yrel <= S.ylast;
            float o0[4], o1[4];
            row_compute<OP, KIND, EPI>(P, T, ring[u % kRing], ring[(u + 1) % kRing], ring[(u + 2) % kRing],
                                       hr[u % kRing], hr[(u + 1) % kRing], hr[(u + 2) % kRing], rowin, S.colin,
                                       o0, o1);
            store_row<OP>(P, S, o0, o1);
        }
    }
    if constexpr (VAL) {
        valid_wait(P);
        valid_strip(P, S.xs, S.y0, rows, vwords[threadIdx.x >> 5], S.lane);
    }
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

template <int OP, int KIND, bool EPI, bool VAL>
__global__ void __launch_bounds__(kWarps * 32, 6)
    march3_tma_kernel(const __grid_constant__ LaunchParams P, const __grid_constant__ CUtensorMap map, int strip,
                      int col_blocks) {
    constexpr bool kHorn = kIsHorn<OP>;
    __shared__ __align__(128) float sbuf[kWarps][kBoxes][kBoxRows * kBoxCols];
    __shared__ __align__(8) uint64_t sbar[kWarps][kBoxes + 1];  // the last: the failure-path test's
    EpiTables* T = EpiSmem<EPI>::get();
    if constexpr (EPI) {
        stage_epilogue(P, *T);
        __syncthreads();
    }
    Strip S;
    if (!strip_setup<OP>(P, strip, col_blocks, S)) return;
    const int warp = threadIdx.x >> 5;
    float* boxes = &sbuf[warp][0][0];
    uint64_t* bars = sbar[warp];
    const int lane = S.lane;
    const int rows = S.rows;
    const int need = rows + 2;  // rows m = 0 .. rows + 1 (y0 - 1 .. y0 + rows)
    const int nbox = (need + kBoxRows - 1) / kBoxRows;
    // Box b holds rows m = 4b .. 4b + 3; its first cell is source column
    // xs - 4 (a multiple of 4: the copy's 16-byte rule) and source row
    // y0 - 1 + 4b.
    const int bx = (int)(S.xs - 4 - P.src_x0);
    const int by = (int)(S.y0 - 1 - P.src_y0);

    if (lane == 0) {
#pragma unroll
        for (int s = 0; s <= kBoxes; s++) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncwarp();
    // Box b into slot b % kBoxes, phase b / kBoxes of that slot's barrier.
    auto issue = [&](int b) {
        uint64_t* bar = &bars[b % kBoxes];
        mbar_arrive_expect_tx(bar, kBoxBytes);
        tma_box(boxes + (b % kBoxes) * (kBoxRows * kBoxCols), &map, bx, by + b * kBoxRows, bar);
    };
    int issued = min(nbox, kBoxes);  // boxes 0 .. issued - 1 have been issued
    int waited = 0;                  // boxes 0 .. waited - 1 have landed and been waited for
    if (lane == 0)
        for (int b = 0; b < issued; b++) issue(b);

    bool ok = true;
    // The failure-path test: a wait on a barrier that nothing arrives at
    // runs out (after 2^10 polls), as a copy that never lands would.
    if (P.test_stall) ok = __all_sync(kFull, mbar_wait(&bars[kBoxes], 0u, 1u << 10));
    // Reads row m (waiting for its box first when it is the box's first
    // row), and when m is its box's last row, gives the slot to the box
    // kBoxes later.
    auto take = [&](int m, Row6& r) {
        const int b = m / kBoxRows;
        if ((m % kBoxRows) == 0) {
            if (ok) ok = __all_sync(kFull, mbar_wait(&bars[b % kBoxes], (uint32_t)(b / kBoxes) & 1u));
            waited = b + 1;
        }
        const float* row = boxes + (b % kBoxes) * (kBoxRows * kBoxCols) + (m % kBoxRows) * kBoxCols;
        const float4 q = *reinterpret_cast<const float4*>(row + 4 + 4 * lane);
        float l = __shfl_up_sync(kFull, q.w, 1);
        float rr = __shfl_down_sync(kFull, q.x, 1);
        if (lane == 0) l = row[3];
        if (S.last) rr = row[8 + 4 * lane];
        r.v[0] = l;
        r.v[1] = q.x;
        r.v[2] = q.y;
        r.v[3] = q.z;
        r.v[4] = q.w;
        r.v[5] = rr;
        if ((m % kBoxRows) == kBoxRows - 1 && ok && b + kBoxes < nbox) {
            __syncwarp();
            if (lane == 0) {
                fence_proxy_async();  // this warp's reads of the slot before the copy overwrites it
                issue(b + kBoxes);
            }
            issued = b + kBoxes + 1;
        }
    };

    // Register slot m % 4 holds row m: output row k reads m = k .. k + 2
    // and takes row k + 2; unrolled by 4, every index is a constant. The
    // validity ring (VAL) has the same slots and loads four rows ahead.
    Row6 ring[4];
    float hr[4][4];
    __shared__ uint32_t vwords[VAL ? kWarps : 1][VAL ? kVMaxRows * kVWords : 1];
    if constexpr (VAL) valid_prefetch(P, S.xs, S.y0, rows, vwords[warp], lane);
    if (ok) {
        take(0, ring[0]);
        take(1, ring[1]);
    }
    if constexpr (kHorn) {
        hdiff(ring[0], hr[0]);
        hdiff(ring[1], hr[1]);
    }
    for (int k0 = 0; k0 < rows && ok; k0 += 4) {
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int k = k0 + u;
            if (k >= rows) break;
            take(k + 2, ring[(u + 2) % 4]);
            if constexpr (kHorn) hdiff(ring[(u + 2) % 4], hr[(u + 2) % 4]);
            S.yrel++;
            const bool rowin = S.yrel >= 1 && S.yrel <= S.ylast;
            float o0[4], o1[4];
            row_compute<OP, KIND, EPI>(P, T, ring[u % 4], ring[(u + 1) % 4], ring[(u + 2) % 4], hr[u % 4],
                                       hr[(u + 1) % 4], hr[(u + 2) % 4], rowin, S.colin, o0, o1);
            if (ok) store_row<OP>(P, S, o0, o1);
        }
    }
    if constexpr (VAL) {  // waited for on every path, so no copy outlives the block
        valid_wait(P);
        if (ok) valid_strip(P, S.xs, S.y0, rows, vwords[warp], lane);
    }
    if (!ok) {
        // A copy did not land in time: report it, then wait (bounded) for
        // the boxes this warp still has in flight before its shared memory
        // goes away.
        if (lane == 0 && P.status) atomicExch(P.status, STRATA_ETIMEDOUT);
        for (int b = waited; b < issued; b++) mbar_wait(&bars[b % kBoxes], (uint32_t)(b / kBoxes) & 1u);
    }
}

// The source as a 2-D tensor for the box copies: cuTensorMapEncodeTiled,
// reached through the runtime's driver entry point (no libcuda link).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

bool source_map(const LaunchParams& p, CUtensorMap* map) {
    EncodeTiledFn fn = encode_tiled();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)p.src_w, (cuuint64_t)p.src_h};
    const cuuint64_t strides[1] = {(cuuint64_t)p.src_stride * 4};
    const cuuint32_t box[2] = {kBoxCols, kBoxRows};
    const cuuint32_t elem[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(p.src), dims, strides, box, elem,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <int OP, int KIND, bool EPI, bool VAL>
int64_t launch_march_v(const LaunchParams& p, cudaStream_t s) {
    const int64_t w = p.out_x1 - p.out_x0, h = p.out_y1 - p.out_y0;
    const int64_t segs = (w + 127) / 128;
    const int64_t col_blocks = (segs + kWarps - 1) / kWarps;
    // Strip height: enough warps for several waves over the SMs, at least
    // 8 rows and at most 64 (the halo costs 2 rows a strip).
    int64_t strip = segs > 0 ? (h * segs) / ((int64_t)sm_count() * 48 * 4) : h;
    strip = strip < 8 ? 8 : (strip > kMaxStrip ? kMaxStrip : strip);
    const int64_t strips = (h + strip - 1) / strip;
    const int64_t blocks = col_blocks * strips;
    CUtensorMap map;
    if (source_map(p, &map))
        march3_tma_kernel<OP, KIND, EPI, VAL><<<(unsigned)blocks, kWarps * 32, 0, s>>>(p, map, (int)strip,
                                                                                      (int)col_blocks);
    else
        march3_kernel<OP, KIND, EPI, VAL><<<(unsigned)blocks, kWarps * 32, 0, s>>>(p, (int)strip,
                                                                                  (int)col_blocks);
    return blocks;
}

template <int OP, int KIND, bool EPI>
int64_t launch_march(const LaunchParams& p, cudaStream_t s) {
    return p.vf.n ? launch_march_v<OP, KIND, EPI, true>(p, s) : launch_march_v<OP, KIND, EPI, false>(p, s);
}

template <int OP, int KIND>
int64_t launch_epi(const LaunchParams& p, cudaStream_t s) {
    return p.nepi ? launch_march<OP, KIND, true>(p, s) : launch_march<OP, KIND, false>(p, s);
}

// Rasters whose rows are not 16-byte aligned where the march loads and
// stores (a window at any origin, any stride or width): the same march,
// a warp per 128 columns of a strip, with per-cell loads and stores
// (march.cuh march_warp).
template <int OP, int KIND, bool EPI>
__global__ void __launch_bounds__(kWarps * 32) march_any_kernel(const __grid_constant__ LaunchParams P, int strip,
                                                                int col_blocks) {
    EpiTables* T = EpiSmem<EPI>::get();
    if constexpr (EPI) {
        stage_epilogue(P, *T);
        __syncthreads();
    }
    const int warp = threadIdx.x >> 5;
    const int cb = blockIdx.x % col_blocks;
    const int sb = blockIdx.x / col_blocks;
    const int64_t xs = P.out_x0 + (int64_t)(cb * kWarps + warp) * 128;
    if (xs >= P.out_x1) return;  // warp-uniform
    const int64_t y0 = P.out_y0 + (int64_t)sb * strip;
    const int rows = (int)min((int64_t)strip, P.out_y1 - y0);
    march_warp<OP, KIND, EPI>(P, T, xs, y0, rows, false);
}

template <int OP, int KIND, bool EPI>
int64_t launch_any(const LaunchParams& p, cudaStream_t s) {
    const int64_t w = p.out_x1 - p.out_x0, h = p.out_y1 - p.out_y0;
    const int64_t segs = (w + 127) / 128;
    const int64_t col_blocks = (segs + kWarps - 1) / kWarps;
    int64_t strip = segs > 0 ? (h * segs) / ((int64_t)sm_count() * 48 * 4) : h;
    strip = strip < 8 ? 8 : (strip > kMaxStrip ? kMaxStrip : strip);
    const int64_t blocks = col_blocks * ((h + strip - 1) / strip);
    march_any_kernel<OP, KIND, EPI><<<(unsigned)blocks, kWarps * 32, 0, s>>>(p, (int)strip, (int)col_blocks);
    return blocks;
}

template <int OP, int KIND>
int64_t launch_any_epi(const LaunchParams& p, cudaStream_t s) {
    return p.nepi ? launch_any<OP, KIND, true>(p, s) : launch_any<OP, KIND, false>(p, s);
}

}  // namespace

bool march3_eligible(const LaunchParams& p) {
    if (p.radius != 1 && !(p.op >= STRATA_OP_GRADIENT && p.op <= STRATA_OP_CURVATURE)) return false;
    const int64_t w = p.out_x1 - p.out_x0;
    if (w <= 0 || (w & 3) || (p.src_stride & 3) || (p.dst0_stride & 3)) return false;
    if (((p.out_x0 - p.src_x0) & 3) || ((p.out_x0 - p.dst_x0) & 3)) return false;
    if (!aligned16(p.src) || !aligned16(p.dst0)) return false;
    if (p.op == STRATA_OP_GRADIENT && ((p.dst1_stride & 3) || !aligned16(p.dst1))) return false;
    // 32-bit block and row arithmetic inside the kernel.
    const int64_t col_blocks = ((w + 127) / 128 + kWarps - 1) / kWarps;
    const int64_t blocks = col_blocks * ((p.out_y1 - p.out_y0 + 7) / 8);
    return blocks < ((int64_t)1 << 31) && p.height < ((int64_t)1 << 30) && p.src_h < ((int64_t)1 << 30);
}

bool march_any_eligible(const LaunchParams& p) {
    if (p.radius > 1 || p.op < STRATA_OP_GRADIENT || p.op > STRATA_OP_MAX) return false;
    const int64_t w = p.out_x1 - p.out_x0;
    if (w <= 0) return false;
    // 32-bit block, row and column arithmetic inside the kernel.
    const int64_t col_blocks = ((w + 127) / 128 + kWarps - 1) / kWarps;
    const int64_t blocks = col_blocks * ((p.out_y1 - p.out_y0 + 7) / 8);
    return blocks < ((int64_t)1 << 31) && p.height < ((int64_t)1 << 30) && p.src_h < ((int64_t)1 << 30) &&
           p.src_w < ((int64_t)1 << 30) && p.width < ((int64_t)1 << 30);
}

int64_t launch_march_any(const LaunchParams& p, cudaStream_t s) {
    switch (p.op) {
    case STRATA_OP_GRADIENT: return launch_any<STRATA_OP_GRADIENT, 0, false>(p, s);
    case STRATA_OP_SLOPE:
        if (p.kind == kSlopeSquareClass) return launch_any<STRATA_OP_SLOPE, kSlopeSquareClass, false>(p, s);
        return p.kind ? launch_any_epi<STRATA_OP_SLOPE, 1>(p, s) : launch_any_epi<STRATA_OP_SLOPE, 0>(p, s);
    case STRATA_OP_ASPECT:
        return p.kind ? launch_any_epi<STRATA_OP_ASPECT, 1>(p, s) : launch_any_epi<STRATA_OP_ASPECT, 0>(p, s);
    case STRATA_OP_HILLSHADE: return launch_any_epi<STRATA_OP_HILLSHADE, 0>(p, s);
    case STRATA_OP_CURVATURE:
        switch (p.kind) {
        case 0: return launch_any_epi<STRATA_OP_CURVATURE, 0>(p, s);
        case 1: return launch_any_epi<STRATA_OP_CURVATURE, 1>(p, s);
        case 2: return launch_any_epi<STRATA_OP_CURVATURE, 2>(p, s);
        }
        return -1;
    case STRATA_OP_RUGGEDNESS:
        switch (p.kind) {
        case STRATA_RUG_TRI_RILEY: return launch_any_epi<STRATA_OP_RUGGEDNESS, kKindAtRun>(p, s);
        case STRATA_RUG_TRI_WILSON: return launch_any_epi<STRATA_OP_RUGGEDNESS, STRATA_RUG_TRI_WILSON>(p, s);
        case STRATA_RUG_TPI: return launch_any_epi<STRATA_OP_RUGGEDNESS, STRATA_RUG_TPI>(p, s);
        case STRATA_RUG_ROUGHNESS: return launch_any_epi<STRATA_OP_RUGGEDNESS, STRATA_RUG_ROUGHNESS>(p, s);
        }
        return -1;
    case STRATA_OP_CORRELATE: return launch_any_epi<STRATA_OP_CORRELATE, 0>(p, s);
    case STRATA_OP_SEPARABLE: return launch_any_epi<STRATA_OP_SEPARABLE, 0>(p, s);
    case STRATA_OP_MEAN: return launch_any_epi<STRATA_OP_MEAN, 0>(p, s);
    case STRATA_OP_MIN: return launch_any_epi<STRATA_OP_MIN, 0>(p, s);
    case STRATA_OP_MAX: return launch_any_epi<STRATA_OP_MAX, 0>(p, s);
    }
    return -1;
}

int64_t launch_march3(const LaunchParams& p, cudaStream_t s) {
    switch (p.op) {
    case STRATA_OP_GRADIENT: return launch_epi<STRATA_OP_GRADIENT, 0>(p, s);
    case STRATA_OP_SLOPE:
        if (p.kind == kSlopeSquareClass) return launch_march<STRATA_OP_SLOPE, kSlopeSquareClass, false>(p, s);
        return p.kind ? launch_epi<STRATA_OP_SLOPE, 1>(p, s) : launch_epi<STRATA_OP_SLOPE, 0>(p, s);
    case STRATA_OP_ASPECT:
        return p.kind ? launch_epi<STRATA_OP_ASPECT, 1>(p, s) : launch_epi<STRATA_OP_ASPECT, 0>(p, s);
    case STRATA_OP_HILLSHADE: return launch_epi<STRATA_OP_HILLSHADE, 0>(p, s);
    case STRATA_OP_CURVATURE:
        switch (p.kind) {
        case 0: return launch_epi<STRATA_OP_CURVATURE, 0>(p, s);
        case 1: return launch_epi<STRATA_OP_CURVATURE, 1>(p, s);
        case 2: return launch_epi<STRATA_OP_CURVATURE, 2>(p, s);
        }
        return -1;
    case STRATA_OP_RUGGEDNESS:
        switch (p.kind) {
        case STRATA_RUG_TRI_RILEY: return launch_epi<STRATA_OP_RUGGEDNESS, kKindAtRun>(p, s);
        case STRATA_RUG_TRI_WILSON: return launch_epi<STRATA_OP_RUGGEDNESS, STRATA_RUG_TRI_WILSON>(p, s);
        case STRATA_RUG_TPI: return launch_epi<STRATA_OP_RUGGEDNESS, STRATA_RUG_TPI>(p, s);
        case STRATA_RUG_ROUGHNESS: return launch_epi<STRATA_OP_RUGGEDNESS, STRATA_RUG_ROUGHNESS>(p, s);
        }
        return -1;
    case STRATA_OP_CORRELATE: return launch_epi<STRATA_OP_CORRELATE, 0>(p, s);
    case STRATA_OP_SEPARABLE: return launch_epi<STRATA_OP_SEPARABLE, 0>(p, s);
    case STRATA_OP_MEAN: return launch_epi<STRATA_OP_MEAN, 0>(p, s);
    case STRATA_OP_MIN: return launch_epi<STRATA_OP_MIN, 0>(p, s);
    case STRATA_OP_MAX: return launch_epi<STRATA_OP_MAX, 0>(p, s);
    }
    return -1;
}

}  // namespace strata
