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

// A lone Reclass over four cells (ops3.cuh reclass_chain4) from a feature's
// breaks and values; NaN passes through.
__device__ __forceinline__ void feature_chain(const FeatureSpec& F, float (&v)[4]) {
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

// Every feature's four cells of one output row (global row y) from the
// window rows a, b, c and their horizontal differences.
__device__ __forceinline__ void features_row(const FeaturesParams& F, const Strip& S, int64_t y, const Row6& a,
                                             const Row6& b, const Row6& c, const float (&ha)[4],
                                             const float (&hb)[4], const float (&hc)[4], bool rowin) {
    const LaunchParams& P = F.g;
    const float nan = nanf32();
    // Horn's differences, unscaled (internal/stencil/horn.go:152-160), in
    // the lane's pairs of cells (0, 1) and (2, 3), as march.cuh forms them.
    F2 DX[2], DY[2];
    if (F.horn) {
        const F2 V12 = sub2(pk(c.v[1], c.v[2]), pk(a.v[1], a.v[2]));
        const F2 V34 = sub2(pk(c.v[3], c.v[4]), pk(a.v[3], a.v[4]));
        const float V0 = sub(c.v[0], a.v[0]), V5 = sub(c.v[5], a.v[5]);
        DY[0] = add2(pk(add(V0, hi(V12)), add(lo(V12), lo(V34))), add2(V12, V12));
        DY[1] = add2(pk(add(hi(V12), hi(V34)), add(lo(V34), V5)), add2(V34, V34));
#pragma unroll
        for (int p = 0; p < 2; p++) {
            const F2 hb2 = pk(hb[2 * p], hb[2 * p + 1]);
            DX[p] = add2(add2(pk(ha[2 * p], ha[2 * p + 1]), pk(hc[2 * p], hc[2 * p + 1])), add2(hb2, hb2));
        }
    }
    bool in[4];
#pragma unroll
    for (int i = 0; i < 4; i++) in[i] = rowin && S.colin[i];
    const int64_t rowoff = y - P.dst_y0;
    const int64_t coloff = S.x - P.dst_x0;
    for (int f = 0; f < F.nfeat; f++) {
        const FeatureSpec& s = F.f[f];
        float o0[4], o1[4] = {nan, nan, nan, nan};
        const int op = s.op;
        // One branch per op and kind, each with its own loop over the cells,
        // so that no feature evaluates another's arithmetic (selects between
        // finished values would compute every kind).
        if (op == STRATA_OP_RUGGEDNESS) {
            if (s.kind == STRATA_RUG_TPI) {
#pragma unroll
                for (int i = 0; i < 4; i++)
                    o0[i] = rugged3(a.v[i], a.v[i + 1], a.v[i + 2], b.v[i], b.v[i + 1], b.v[i + 2], c.v[i],
                                    c.v[i + 1], c.v[i + 2], STRATA_RUG_TPI);
            } else if (s.kind == STRATA_RUG_ROUGHNESS) {
#pragma unroll
                for (int i = 0; i < 4; i++)
                    o0[i] = rugged3(a.v[i], a.v[i + 1], a.v[i + 2], b.v[i], b.v[i + 1], b.v[i + 2], c.v[i],
                                    c.v[i + 1], c.v[i + 2], STRATA_RUG_ROUGHNESS);
            } else {
#pragma unroll
                for (int i = 0; i < 4; i++)
                    o0[i] = rugged3(a.v[i], a.v[i + 1], a.v[i + 2], b.v[i], b.v[i + 1], b.v[i + 2], c.v[i],
                                    c.v[i + 1], c.v[i + 2], STRATA_RUG_TRI_WILSON);
            }
        } else if (op == STRATA_OP_GRADIENT) {
#pragma unroll
            for (int p = 0; p < 2; p++) {
                const F2 gx = mul2(DX[p], splat(s.k[0])), gy = mul2(DY[p], splat(s.k[1]));
                o0[2 * p] = lo(gx);
                o0[2 * p + 1] = hi(gx);
                o1[2 * p] = lo(gy);
                o1[2 * p + 1] = hi(gy);
            }
        } else if (s.kind == kSlopeSquareClass) {
#pragma unroll
            for (int p = 0; p < 2; p++) {
                const F2 gx = mul2(DX[p], splat(s.k[0])), gy = mul2(DY[p], splat(s.k[1]));
                const F2 r = add_p(mul2(gx, gx), mul2(gy, gy));  // magnitude's radicand (horn.go:220-222)
                o0[2 * p] = lo(r);
                o0[2 * p + 1] = hi(r);
            }
        } else {
#pragma unroll
            for (int p = 0; p < 2; p++) {
                const F2 gx = mul2(DX[p], splat(s.k[0])), gy = mul2(DY[p], splat(s.k[1]));
                const F2 r = slope2(gx, gy, splat(s.k[2]), false);  // percent: no arctangent
                o0[2 * p] = lo(r);
                o0[2 * p + 1] = hi(r);
            }
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
            o0[i] = in[i] ? o0[i] : nan;
            o1[i] = in[i] ? o1[i] : nan;
        }
        // The epilogue maps NaN to itself, so the edge ring stays NaN.
        if (s.nb > 0) feature_chain(s, o0);
        if (S.active) {
            const FeatureOut& O = F.o[s.out];
            *reinterpret_cast<float4*>(O.data + rowoff * O.stride + coloff) = make_float4(o0[0], o0[1], o0[2], o0[3]);
            if (op == STRATA_OP_GRADIENT) {
                const FeatureOut& O1 = F.o[s.out + 1];
                *reinterpret_cast<float4*>(O1.data + rowoff * O1.stride + coloff) =
                    make_float4(o1[0], o1[1], o1[2], o1[3]);
            }
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
    for (int k0 = 0; k0 < rows && ok; k0 += 4) {
#pragma unroll
        for (int u = 0; u < 4; u++) {
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
    }
    if constexpr (VAL) {  // waited for on every path, so no copy outlives the block
        valid_wait(P);
        if (ok)
            valid_strip_emit(P, S.xs, S.y0, rows, vwords[warp], lane,
                             [&](int64_t y, int64_t c0, uint32_t v, uint32_t ours) {
                                 for (int i = 0; i < F.nout; i++) {
                                     const FeatureOut& O = F.o[i];
                                     if (O.bits)
                                         put_bits(O.bits, O.bit_off + (y - P.dst_y0) * O.bit_stride + (c0 - P.dst_x0),
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

bool feature_fusable(const LaunchParams& p) {
    const bool light = p.op == STRATA_OP_GRADIENT || (p.op == STRATA_OP_SLOPE && p.kind != 1) ||
                       (p.op == STRATA_OP_RUGGEDNESS && p.radius == 1 && p.kind != STRATA_RUG_TRI_RILEY);
    if (!light) return false;
    if (p.nepi > 1 || (p.nepi == 1 && (p.epi[0].op != STRATA_OP_RECLASS || p.epi[0].n > kChainBreaks))) return false;
    return march3_eligible(p);
}

int64_t launch_features(const FeaturesParams& f, cudaStream_t s, int64_t* window_cells) {
    const LaunchParams& p = f.g;
    const int64_t w = p.out_x1 - p.out_x0, h = p.out_y1 - p.out_y0;
    if (w <= 0 || h <= 0) {
        if (window_cells) *window_cells = 0;
        return 0;
    }
    if ((w & 3) || (p.src_stride & 3) || !aligned16_(p.src) || ((p.out_x0 - p.src_x0) & 3)) return -1;
    for (int i = 0; i < f.nout; i++)
        if ((f.o[i].stride & 3) || !aligned16_(f.o[i].data)) return -1;
    CUtensorMap map;
    if (!source_map(p, &map)) return -1;
    const int64_t segs = (w + 127) / 128;
    const int64_t col_blocks = (segs + kWarps - 1) / kWarps;
    int64_t strip = (h * segs) / ((int64_t)sm_count() * 40 * 4);
    strip = strip < 8 ? 8 : (strip > kMaxStrip ? kMaxStrip : strip);
    const int64_t blocks = col_blocks * ((h + strip - 1) / strip);
    bool val = false;
    for (int i = 0; i < f.nout; i++) val = val || f.o[i].bits != nullptr;
    if (val)
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
