// march3.cu - the radius-1 data kernel: register marching down row strips.
//
// Each warp owns 128 consecutive columns of a strip of rows, four per
// lane. A lane reads each input row once as one aligned float4 (a warp
// reads 512 contiguous bytes), takes the column to its left and right
// from its neighbours with warp shuffles (the warp's two outer columns
// with one extra load each), and keeps the rows it still needs in
// registers while it walks down the strip, so every input cell is read
// from memory once per strip plus two halo rows. Loads run kAhead rows
// ahead of the arithmetic. Each lane writes its four results with one
// float4 store.
//
// Horn ops (gradient, slope, aspect, hillshade) reuse each row's
// horizontal differences: hornDX's z3 - z1, z6 - z4 and z9 - z7
// (internal/stencil/horn.go:152-155) are one row's x+1 minus x-1 seen as
// the window's top, middle and bottom row, so each row's difference is
// computed once and used by three output rows. The operations and their
// order per cell are the reference's, so the bits are too.
//
// The per-cell arithmetic of the other ops is apply3 (ops3.cuh), shared
// with the general tile kernel. The launcher takes this path only when
// every row of the source and destination starts on a 16-byte boundary at
// the region's first column and the region is a multiple of 4 wide;
// otherwise the tile kernel runs.
#include "launch.h"
#include "ops3.cuh"

namespace strata {
namespace {

using namespace cell;

constexpr int kWarps = 4;  // warps per block, side by side: 512 columns
constexpr int kAhead = 1;  // rows loaded ahead of the arithmetic
constexpr int kRing = kAhead + 3;
constexpr unsigned kFull = 0xffffffffu;

struct Row6 {
    float v[6];  // columns x-1 .. x+4 around the lane's four
};

// Marching state for one lane: where its rows live and which are inside
// the source.
struct Lane {
    const float* p;    // &src[row][x] of the next row to load
    int64_t stride;    // source row stride
    int by, src_h;     // next row, relative to the source's first row
    bool active, first, last;
    bool left_in, right_in;  // x-1 / x+4 inside the source columns
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

// hornDX's horizontal difference of one row for the four cells.
__device__ __forceinline__ void hdiff(const Row6& r, float (&h)[4]) {
#pragma unroll
    for (int i = 0; i < 4; i++) h[i] = sub(r.v[i + 2], r.v[i]);
}

// The Horn finishers (slope, aspect, hillshade) of ops3 on gx, gy, with the
// op's kind fixed at compile time.
template <int OP, int KIND>
__device__ __forceinline__ float horn_finish(const LaunchParams& P, float gx, float gy) {
    if constexpr (OP == STRATA_OP_SLOPE) {
        return slope(gx, gy, P.k[2], KIND != 0);
    } else if constexpr (OP == STRATA_OP_ASPECT) {
        return aspect(gx, gy, P.k[2], KIND != 0);
    } else {
        return shade(gx, gy, P.k[2], P.k[3], P.k[4]);
    }
}

template <int OP, int KIND, bool EPI>
__global__ void __launch_bounds__(kWarps * 32, 8) march3_kernel(const __grid_constant__ LaunchParams P, int strip,
                                                                 int col_blocks) {
    constexpr bool kHorn = OP == STRATA_OP_GRADIENT || OP == STRATA_OP_SLOPE || OP == STRATA_OP_ASPECT ||
                           OP == STRATA_OP_HILLSHADE;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int cb = blockIdx.x % col_blocks;
    const int sb = blockIdx.x / col_blocks;
    const int64_t xs = P.out_x0 + (int64_t)(cb * kWarps + warp) * 128;
    if (xs >= P.out_x1) return;  // warp-uniform
    const int64_t x = xs + 4 * lane;
    const int64_t y0 = P.out_y0 + (int64_t)sb * strip;
    const int rows = (int)min((int64_t)strip, P.out_y1 - y0);

    Lane L;
    L.active = x < P.out_x1;
    // The region's width is a multiple of 4, so a lane is wholly in or out;
    // the last active lane fetches its right neighbour itself.
    L.first = lane == 0;
    L.last = L.active && (lane == 31 || x + 4 >= P.out_x1);
    L.left_in = x - 1 >= P.src_x0;
    L.right_in = x + 4 < P.src_x0 + P.src_w;
    L.stride = P.src_stride;
    L.by = (int)(y0 - 1 - P.src_y0);
    L.src_h = (int)P.src_h;
    L.p = P.src + (int64_t)L.by * P.src_stride + (x - P.src_x0);

    float* d0 = P.dst0 + (y0 - P.dst_y0) * P.dst0_stride + (x - P.dst_x0);
    float* d1 = OP == STRATA_OP_GRADIENT ? P.dst1 + (y0 - P.dst_y0) * P.dst1_stride + (x - P.dst_x0) : nullptr;

    // Interior: x + i in [1, W - 1) and y in [1, H - 1).
    const int64_t W = P.width;
    bool colin[4];
#pragma unroll
    for (int i = 0; i < 4; i++) colin[i] = x + i >= 1 && x + i < W - 1;
    int yrel = (int)(y0 - 1);          // y - 1 of the current output row, for the row test
    const int ylast = (int)(P.height - 2);  // last interior row
    const float nan = nanf32();

    // kRing rows live at once (three for the window, kAhead in flight),
    // kept in a ring that the unrolled loop renames instead of copying.
    Row6 ring[kRing];
    float hr[kRing][4];  // each ring row's horizontal differences (Horn ops)
    // Ring slot m % kRing holds row y0 - 1 + m: the window of output row
    // y0 + k is m = k .. k + 2, and rows m <= 1 + kAhead load up front.
#pragma unroll
    for (int j = 0; j < 2 + kAhead; j++) {
        if (j < 3 || j - 2 < rows) {
            ring[j] = load_row(L);
            if constexpr (kHorn) hdiff(ring[j], hr[j]);
        }
    }
    for (int k0 = 0; k0 < rows; k0 += kRing) {
#pragma unroll
        for (int u = 0; u < kRing; u++) {
            const int k = k0 + u;
            if (k >= rows) break;
            const Row6& a = ring[u % kRing];
            const Row6& b = ring[(u + 1) % kRing];
            const Row6& c = ring[(u + 2) % kRing];
            // Row m = k + 2 + kAhead, the bottom of output row k + kAhead's
            // window, into the slot row m = k - 1 no longer needs.
            if (k + kAhead < rows) {
                ring[(u + 3 + kAhead - 1) % kRing] = load_row(L);
                if constexpr (kHorn) hdiff(ring[(u + 3 + kAhead - 1) % kRing], hr[(u + 3 + kAhead - 1) % kRing]);
            }
            yrel++;
            const bool rowin = yrel >= 1 && yrel <= ylast;
            float o0[4], o1[4];
            if constexpr (kHorn) {
                const float(&ha)[4] = hr[u % kRing];
                const float(&hb)[4] = hr[(u + 1) % kRing];
                const float(&hc)[4] = hr[(u + 2) % kRing];
                // hornDY's vertical differences: bottom row minus top row.
                float v[6];
#pragma unroll
                for (int j = 0; j < 6; j++) v[j] = sub(c.v[j], a.v[j]);
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const float dx = add(add(ha[i], hc[i]), add(hb[i], hb[i]));
                    const float dy = add(add(v[i], v[i + 2]), add(v[i + 1], v[i + 1]));
                    const float gx = mul(dx, P.k[0]);
                    const float gy = mul(dy, P.k[1]);
                    const bool in = rowin && colin[i];
                    if constexpr (OP == STRATA_OP_GRADIENT) {
                        o0[i] = in ? gx : nan;
                        o1[i] = in ? gy : nan;
                    } else {
                        float r = horn_finish<OP, KIND>(P, gx, gy);
                        if constexpr (EPI) r = epilogue(P, r);
                        o0[i] = in ? r : nan;
                    }
                }
            } else {
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const float z[9] = {a.v[i], a.v[i + 1], a.v[i + 2], b.v[i], b.v[i + 1],
                                        b.v[i + 2], c.v[i], c.v[i + 1], c.v[i + 2]};
                    float r0 = nan, r1 = nan;
                    apply3<OP>(P, z, r0, r1);
                    if constexpr (EPI) r0 = epilogue(P, r0);
                    o0[i] = (rowin && colin[i]) ? r0 : nan;
                }
            }
            if (L.active) {
                *reinterpret_cast<float4*>(d0) = make_float4(o0[0], o0[1], o0[2], o0[3]);
                if constexpr (OP == STRATA_OP_GRADIENT)
                    *reinterpret_cast<float4*>(d1) = make_float4(o1[0], o1[1], o1[2], o1[3]);
            }
            d0 += P.dst0_stride;
            if constexpr (OP == STRATA_OP_GRADIENT) d1 += P.dst1_stride;
        }
    }
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <int OP, int KIND, bool EPI>
int64_t launch_march(const LaunchParams& p, cudaStream_t s) {
    const int64_t w = p.out_x1 - p.out_x0, h = p.out_y1 - p.out_y0;
    const int64_t segs = (w + 127) / 128;
    const int64_t col_blocks = (segs + kWarps - 1) / kWarps;
    // Strip height: enough warps for several waves over 148 SMs, at least
    // 8 rows and at most 64 (the halo costs 2 rows a strip).
    int64_t strip = segs > 0 ? (h * segs) / (148 * 48 * 4) : h;
    strip = strip < 8 ? 8 : (strip > 64 ? 64 : strip);
    const int64_t strips = (h + strip - 1) / strip;
    const int64_t blocks = col_blocks * strips;
    march3_kernel<OP, KIND, EPI><<<(unsigned)blocks, kWarps * 32, 0, s>>>(p, (int)strip, (int)col_blocks);
    return blocks;
}

template <int OP, int KIND>
int64_t launch_epi(const LaunchParams& p, cudaStream_t s) {
    return p.nepi ? launch_march<OP, KIND, true>(p, s) : launch_march<OP, KIND, false>(p, s);
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

int64_t launch_march3(const LaunchParams& p, cudaStream_t s) {
    switch (p.op) {
    case STRATA_OP_GRADIENT: return launch_epi<STRATA_OP_GRADIENT, 0>(p, s);
    case STRATA_OP_SLOPE:
        return p.kind ? launch_epi<STRATA_OP_SLOPE, 1>(p, s) : launch_epi<STRATA_OP_SLOPE, 0>(p, s);
    case STRATA_OP_ASPECT:
        return p.kind ? launch_epi<STRATA_OP_ASPECT, 1>(p, s) : launch_epi<STRATA_OP_ASPECT, 0>(p, s);
    case STRATA_OP_HILLSHADE: return launch_epi<STRATA_OP_HILLSHADE, 0>(p, s);
    case STRATA_OP_CURVATURE: return launch_epi<STRATA_OP_CURVATURE, 0>(p, s);
    case STRATA_OP_RUGGEDNESS: return launch_epi<STRATA_OP_RUGGEDNESS, 0>(p, s);
    case STRATA_OP_CORRELATE: return launch_epi<STRATA_OP_CORRELATE, 0>(p, s);
    case STRATA_OP_SEPARABLE: return launch_epi<STRATA_OP_SEPARABLE, 0>(p, s);
    case STRATA_OP_MEAN: return launch_epi<STRATA_OP_MEAN, 0>(p, s);
    case STRATA_OP_MIN: return launch_epi<STRATA_OP_MIN, 0>(p, s);
    case STRATA_OP_MAX: return launch_epi<STRATA_OP_MAX, 0>(p, s);
    }
    return -1;
}

}  // namespace strata
