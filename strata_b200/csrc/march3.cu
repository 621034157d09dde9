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
#include "march_tma.cuh"
#include "ops3.cuh"

namespace strata {
namespace {

using namespace cell;

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

}  // namespace

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

namespace {

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
    return has_tail(p) ? launch_march<OP, KIND, true>(p, s) : launch_march<OP, KIND, false>(p, s);
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
    return has_tail(p) ? launch_any<OP, KIND, true>(p, s) : launch_any<OP, KIND, false>(p, s);
}

}  // namespace

bool march3_eligible(const LaunchParams& p) {
    if (p.fit) return false;  // Wood's fit runs as separable folds and a finishing pass
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
    if (p.fit) return false;
    const bool op_ok = (p.op >= STRATA_OP_GRADIENT && p.op <= STRATA_OP_MAX) || p.op == STRATA_OP_HEATLOAD ||
                       p.op == STRATA_OP_ORIENTATION;
    if (p.radius > 1 || !op_ok) return false;
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
    case STRATA_OP_HEATLOAD: return launch_any_epi<STRATA_OP_HEATLOAD, 0>(p, s);
    case STRATA_OP_ORIENTATION: return launch_any_epi<STRATA_OP_ORIENTATION, 0>(p, s);
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
    case STRATA_OP_HEATLOAD: return launch_epi<STRATA_OP_HEATLOAD, 0>(p, s);
    case STRATA_OP_ORIENTATION: return launch_epi<STRATA_OP_ORIENTATION, 0>(p, s);
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
