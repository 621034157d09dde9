// features.cu - several radius-1 ops over one source in one march: the
// fused form of terrain.Features and terrain.Surface
// (terrain/features.go:68-117, terrain/surface.go:65-191).
//
// The reference computes each feature's cells with its own kernel and
// shares only the reading of the DEM; Surface shares the Horn gradient as
// well. Here one march (march3.cu's: a warp per 128 columns of a strip of
// rows, the rows by tensor copies into a per-warp shared-memory ring) reads
// each source row once, forms Horn's row and column differences once, and
// hands the lane's four cells of each output row to every feature in turn:
// each scales the shared differences by its own kx and ky (so its gradient
// is the bits of its own call), finishes with its own op, takes its
// Reclass epilogue if it has one, and stores its row. The outputs'
// validity is the same for every radius-1 op (the source's mask eroded by
// the 3x3 window), so the strip's validity words are computed once and
// stored into every masked output after the march.
//
// The pass takes the features whose own kernels are bound by memory rather
// than by their arithmetic (Gradient, Slope in percent or classified on its
// squared magnitude, and Wilson's TRI, TPI and roughness at radius 1): for
// them one read of the source instead of one per feature is the saving.
// The arithmetic-bound finishers (the arctangent and division chains of
// Slope in degrees, Aspect, Hillshade and the curvatures, Riley's float64
// TRI) gain nothing from sharing the read and would cost the pass its
// occupancy, so they run as their own launches. Every cell has the bits of
// the feature's own call.
#include <cuda.h>

#include "launch.h"
#include "march.cuh"
#include "march_tma.cuh"
#include "ops3.cuh"

namespace strata {
namespace {

using namespace cell;

// A lone Reclass over four cells (ops3.cuh reclass_chain4) from a slot's
// breaks and values; NaN passes through.
__device__ __forceinline__ void feature_chain(const FeatureSlot& F, float (&v)[4]) {
    float r[4];
#pragma unroll
    for (int c = 0; c < 4; c++) r[c] = F.v[0];
#pragma unroll
    for (int j = 0; j < kChainBreaks; j++) {
        if (j >= F.nb) break;
        const float t = F.t[j], y = F.v[j + 1];
#pragma unroll
        for (int c = 0; c < 4; c++) r[c] = v[c] >= t ? y : r[c];
    }
#pragma unroll
    for (int c = 0; c < 4; c++) v[c] = v[c] != v[c] ? v[c] : r[c];
}

// Masks the edge ring (NaN), takes the slot's epilogue and stores the
// lane's four cells of output k of the slot.
__device__ __forceinline__ void feature_store(const FeatureSlot& F, int k, const Strip& S, const bool (&in)[4],
                                              int64_t rowoff, int64_t coloff, float (&o)[4]) {
    const float nan = nanf32();
#pragma unroll
    for (int i = 0; i < 4; i++) o[i] = in[i] ? o[i] : nan;
    // The epilogue maps NaN to itself, so the edge ring stays NaN.
    if (F.nb > 0) feature_chain(F, o);
    if (S.active) *reinterpret_cast<float4*>(F.data[k] + rowoff * F.stride[k] + coloff) = make_float4(o[0], o[1], o[2], o[3]);
}

// Every slot's four cells of one output row (global row y) from the window
// rows a, b, c and their horizontal differences. The slots are walked in a
// fixed order with their parameters at fixed places.
__device__ __forceinline__ void features_row(const FeaturesParams& F, const Strip& S, int64_t y, const Row6& a,
                                             const Row6& b, const Row6& c, const float (&ha)[4],
                                             const float (&hb)[4], const float (&hc)[4], bool rowin) {
    const LaunchParams& P = F.g;
    bool in[4];
#pragma unroll
    for (int i = 0; i < 4; i++) in[i] = rowin && S.colin[i];
    const int64_t rowoff = y - P.dst_y0;
    const int64_t coloff = S.x - P.dst_x0;
    if (F.horn) {
        // Horn's differences, unscaled (internal/stencil/horn.go:152-160),
        // in the lane's pairs of cells (0, 1) and (2, 3), as march.cuh forms them.
        const F2 V12 = sub2(pk(c.v[1], c.v[2]), pk(a.v[1], a.v[2]));
        const F2 V34 = sub2(pk(c.v[3], c.v[4]), pk(a.v[3], a.v[4]));
        const float V0 = sub(c.v[0], a.v[0]), V5 = sub(c.v[5], a.v[5]);
        F2 DX[2], DY[2];
        DY[0] = add2(pk(add(V0, hi(V12)), add(lo(V12), lo(V34))), add2(V12, V12));
        DY[1] = add2(pk(add(hi(V12), hi(V34)), add(lo(V34), V5)), add2(V34, V34));
#pragma unroll
        for (int p = 0; p < 2; p++) {
            const F2 hb2 = pk(hb[2 * p], hb[2 * p + 1]);
            DX[p] = add2(add2(pk(ha[2 * p], ha[2 * p + 1]), pk(hc[2 * p], hc[2 * p + 1])), add2(hb2, hb2));
        }
        if (F.f[kFGradient].on) {
            const FeatureSlot& Q = F.f[kFGradient];
            float o0[4], o1[4];
#pragma unroll
            for (int p = 0; p < 2; p++) {
                const F2 gx = mul2(DX[p], splat(Q.k[0])), gy = mul2(DY[p], splat(Q.k[1]));
                o0[2 * p] = lo(gx);
                o0[2 * p + 1] = hi(gx);
                o1[2 * p] = lo(gy);
                o1[2 * p + 1] = hi(gy);
            }
            feature_store(Q, 0, S, in, rowoff, coloff, o0);
            feature_store(Q, 1, S, in, rowoff, coloff, o1);
        }
        if (F.f[kFSlopeClass].on) {
            const FeatureSlot& Q = F.f[kFSlopeClass];
            float o[4];
#pragma unroll
            for (int p = 0; p < 2; p++) {
                const F2 gx = mul2(DX[p], splat(Q.k[0])), gy = mul2(DY[p], splat(Q.k[1]));
                const F2 r = add_p(mul2(gx, gx), mul2(gy, gy));  // magnitude's radicand (horn.go:220-222)
                o[2 * p] = lo(r);
                o[2 * p + 1] = hi(r);
            }
            feature_store(Q, 0, S, in, rowoff, coloff, o);
        }
        if (F.f[kFSlopePercent].on) {
            const FeatureSlot& Q = F.f[kFSlopePercent];
            float o[4];
#pragma unroll
            for (int p = 0; p < 2; p++) {
                const F2 gx = mul2(DX[p], splat(Q.k[0])), gy = mul2(DY[p], splat(Q.k[1]));
                const F2 r = slope2(gx, gy, splat(Q.k[2]), false);  // percent: no arctangent
                o[2 * p] = lo(r);
                o[2 * p + 1] = hi(r);
            }
            feature_store(Q, 0, S, in, rowoff, coloff, o);
        }
    }
    if (F.window) {
        // The ruggedness measures at radius 1 (rugged3's float32 kinds).
        if (F.f[kFTpi].on) {
            float o[4];
#pragma unroll
            for (int i = 0; i < 4; i++)
                o[i] = rugged3(a.v[i], a.v[i + 1], a.v[i + 2], b.v[i], b.v[i + 1], b.v[i + 2], c.v[i], c.v[i + 1],
                               c.v[i + 2], STRATA_RUG_TPI);
            feature_store(F.f[kFTpi], 0, S, in, rowoff, coloff, o);
        }
        if (F.f[kFRoughness].on) {
            float o[4];
            roughness4(a.v, b.v, c.v, o);
            feature_store(F.f[kFRoughness], 0, S, in, rowoff, coloff, o);
        }
        if (F.f[kFWilson].on) {
            float o[4];
#pragma unroll
            for (int i = 0; i < 4; i++)
                o[i] = rugged3(a.v[i], a.v[i + 1], a.v[i + 2], b.v[i], b.v[i + 1], b.v[i + 2], c.v[i], c.v[i + 1],
                               c.v[i + 2], STRATA_RUG_TRI_WILSON);
            feature_store(F.f[kFWilson], 0, S, in, rowoff, coloff, o);
        }
    }
}

template <bool VAL>
__global__ void __launch_bounds__(kWarps * 32, 5)
    features_tma_kernel(const __grid_constant__ FeaturesParams F, const __grid_constant__ CUtensorMap map, int strip,
                        int col_blocks) {
    const LaunchParams& P = F.g;
    __shared__ __align__(128) float sbuf[kWarps][kBoxes][kBoxRows * kBoxCols];
    __shared__ __align__(8) uint64_t sbar[kWarps][kBoxes];
    __shared__ uint32_t vwords[VAL ? kWarps : 1][VAL ? kVMaxRows * kVWords : 1];
    Strip S;
    if (!strip_setup<STRATA_OP_SLOPE>(P, strip, col_blocks, S)) return;
    const int warp = threadIdx.x >> 5;
    float* boxes = &sbuf[warp][0][0];
    uint64_t* bars = sbar[warp];
    const int lane = S.lane;
    const int rows = S.rows;
    const int nbox = (rows + 2 + kBoxRows - 1) / kBoxRows;
    // Box b holds rows m = 4b .. 4b + 3 of the strip's source rows (y0 - 1
    // + m), from source column xs - 4 (a multiple of 4: the copy's 16-byte
    // rule), as in march3_tma_kernel.
    const int bx = (int)(S.xs - 4 - P.src_x0);
    const int by = (int)(S.y0 - 1 - P.src_y0);
    if (lane == 0) {
#pragma unroll
        for (int s = 0; s < kBoxes; s++) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncwarp();
    auto issue = [&](int b) {
        uint64_t* bar = &bars[b % kBoxes];
        mbar_arrive_expect_tx(bar, kBoxBytes);
        tma_box(boxes + (b % kBoxes) * (kBoxRows * kBoxCols), &map, bx, by + b * kBoxRows, bar);
    };
    int issued = min(nbox, kBoxes);
    int waited = 0;
    if (lane == 0)
        for (int b = 0; b < issued; b++) issue(b);
    bool ok = true;
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
    Row6 ring[4];
    float hr[4][4];
    if constexpr (VAL) valid_prefetch(P, S.xs, S.y0, rows, vwords[warp], lane);
    take(0, ring[0]);
    take(1, ring[1]);
    hdiff(ring[0], hr[0]);
    hdiff(ring[1], hr[1]);
    // A loop body of two rows, the newest two ring slots moved down after
    // each: half the code of march3_tma_kernel's four-row body, which the
    // pass (every feature's finisher inline) needs for the instruction cache
    // (1.27 -> 1.19 ms at 16384^2; the arithmetic-bound marches are faster
    // with four).
    constexpr int UB = 2;
    for (int k0 = 0; k0 < rows && ok; k0 += UB) {
#pragma unroll
        for (int u = 0; u < UB; u++) {
            const int k = k0 + u;
            if (k >= rows) break;
            take(k + 2, ring[(u + 2) % 4]);
            hdiff(ring[(u + 2) % 4], hr[(u + 2) % 4]);
            S.yrel++;
            const bool rowin = S.yrel >= 1 && S.yrel <= S.ylast;
            if (ok)
                features_row(F, S, S.y0 + k, ring[u % 4], ring[(u + 1) % 4], ring[(u + 2) % 4], hr[u % 4],
                             hr[(u + 1) % 4], hr[(u + 2) % 4], rowin);
        }
        if constexpr (UB == 2) {
            ring[0] = ring[2];
            ring[1] = ring[3];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                hr[0][i] = hr[2][i];
                hr[1][i] = hr[3][i];
            }
        }
    }
    if constexpr (VAL) {  // waited for on every path, so no copy outlives the block
        valid_wait(P);
        if (ok)
            valid_strip_emit(P, S.xs, S.y0, rows, vwords[warp], lane,
                             [&](int64_t y, int64_t c0, uint32_t v, uint32_t ours) {
#pragma unroll
                                 for (int q = 0; q < kFSlots; q++)
#pragma unroll
                                     for (int k = 0; k < 2; k++) {
                                         const FeatureSlot& Q = F.f[q];
                                         if (Q.on && Q.bits[k])
                                             put_bits(Q.bits[k],
                                                      Q.bit_off[k] + (y - P.dst_y0) * Q.bit_stride[k] + (c0 - P.dst_x0),
                                                      v, ours);
                                     }
                             });
    }
    if (!ok) {
        if (lane == 0 && P.status) atomicExch(P.status, STRATA_ETIMEDOUT);
        for (int b = waited; b < issued; b++) mbar_wait(&bars[b % kBoxes], (uint32_t)(b / kBoxes) & 1u);
    }
}

bool aligned16_(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

}  // namespace

int feature_slot(const LaunchParams& p) {
    if (p.nstep || p.nepi > 1 || (p.nepi == 1 && (p.epi[0].op != STRATA_OP_RECLASS || p.epi[0].n > kChainBreaks))) return -1;
    int q = -1;
    if (p.op == STRATA_OP_GRADIENT) q = kFGradient;
    else if (p.op == STRATA_OP_SLOPE && p.kind == kSlopeSquareClass) q = kFSlopeClass;
    else if (p.op == STRATA_OP_SLOPE && p.kind == 0) q = kFSlopePercent;
    else if (p.op == STRATA_OP_RUGGEDNESS && p.radius == 1 && p.kind == STRATA_RUG_TRI_WILSON) q = kFWilson;
    else if (p.op == STRATA_OP_RUGGEDNESS && p.radius == 1 && p.kind == STRATA_RUG_TPI) q = kFTpi;
    else if (p.op == STRATA_OP_RUGGEDNESS && p.radius == 1 && p.kind == STRATA_RUG_ROUGHNESS) q = kFRoughness;
    return q >= 0 && march3_eligible(p) ? q : -1;
}

int64_t launch_features(const FeaturesParams& f, cudaStream_t s, int64_t* window_cells) {
    const LaunchParams& p = f.g;
    const int64_t w = p.out_x1 - p.out_x0, h = p.out_y1 - p.out_y0;
    if (w <= 0 || h <= 0) {
        if (window_cells) *window_cells = 0;
        return 0;
    }
    if ((w & 3) || (p.src_stride & 3) || !aligned16_(p.src) || ((p.out_x0 - p.src_x0) & 3)) return -1;
    for (int q = 0; q < kFSlots; q++)
        for (int k = 0; k < 2 && f.f[q].on; k++)
            if (f.f[q].data[k] && ((f.f[q].stride[k] & 3) || !aligned16_(f.f[q].data[k]))) return -1;
    CUtensorMap map;
    if (!source_map(p, &map)) return -1;
    const int64_t segs = (w + 127) / 128;
    const int64_t col_blocks = (segs + kWarps - 1) / kWarps;
    int64_t strip = (h * segs) / ((int64_t)sm_count() * 40 * 4);
    strip = strip < 8 ? 8 : (strip > kMaxStrip ? kMaxStrip : strip);
    const int64_t blocks = col_blocks * ((h + strip - 1) / strip);
    if (f.masked)
        features_tma_kernel<true><<<(unsigned)blocks, kWarps * 32, 0, s>>>(f, map, (int)strip, (int)col_blocks);
    else
        features_tma_kernel<false><<<(unsigned)blocks, kWarps * 32, 0, s>>>(f, map, (int)strip, (int)col_blocks);
    if (window_cells) {
        const int64_t rows = h + 2 * (blocks / col_blocks);
        *window_cells = (w + 2 * segs) * (rows < p.height ? rows : p.height);
    }
    return blocks;
}

}  // namespace strata
