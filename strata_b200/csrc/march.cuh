// march.cuh - the radius-1 marching row math shared by the single-raster
// kernels (march3.cu) and the batch kernels (batch.cu): a lane's four
// cells of one output row from the window's three rows in registers.
#pragma once

#include "cellops.cuh"
#include "launch.h"
#include "ops3.cuh"

namespace strata {
namespace {

using namespace cell;

constexpr int kWarps = 4;  // warps per block, side by side: 512 columns
constexpr unsigned kFull = 0xffffffffu;

struct Row6 {
    float v[6];  // columns x-1 .. x+4 around the lane's four
};

// hornDX's horizontal difference of one row for the four cells.
__device__ __forceinline__ void hdiff(const Row6& r, float (&h)[4]) {
#pragma unroll
    for (int i = 0; i < 4; i++) h[i] = sub(r.v[i + 2], r.v[i]);
}

// The shared-memory copy of the epilogue's tables, for kernels with one.
template <bool EPI>
struct EpiSmem {
    __device__ static EpiTables* get() {
        __shared__ EpiTables t;
        return &t;
    }
};
template <>
struct EpiSmem<false> {
    __device__ static EpiTables* get() { return nullptr; }
};

template <int OP>
constexpr bool kIsHorn = OP == STRATA_OP_GRADIENT || OP == STRATA_OP_SLOPE || OP == STRATA_OP_ASPECT ||
                         OP == STRATA_OP_HILLSHADE || OP == STRATA_OP_HEATLOAD || OP == STRATA_OP_ORIENTATION;

// One output row of four cells from the window rows a (top), b, c
// (bottom) and, for Horn ops, their horizontal differences.
template <int OP, int KIND, bool EPI>
__device__ __forceinline__ void row_compute(const LaunchParams& P, const EpiTables* T, const Row6& a, const Row6& b,
                                            const Row6& c,
                                            const float (&ha)[4], const float (&hb)[4], const float (&hc)[4],
                                            bool rowin, const bool (&colin)[4], float (&o0)[4], float (&o1)[4]) {
    const float nan = nanf32();
    if constexpr (OP == STRATA_OP_GRADIENT) {
        // hornDY's vertical differences: bottom row minus top row. (Two
        // outputs and no finisher: the scalar form holds fewer registers.)
        float v[6];
#pragma unroll
        for (int j = 0; j < 6; j++) v[j] = sub(c.v[j], a.v[j]);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float dx = add(add(ha[i], hc[i]), add(hb[i], hb[i]));
            const float dy = add(add(v[i], v[i + 2]), add(v[i + 1], v[i + 1]));
            const bool in = rowin && colin[i];
            o0[i] = in ? mul(dx, P.k[0]) : nan;
            o1[i] = in ? mul(dy, P.k[1]) : nan;
        }
    } else if constexpr (kIsHorn<OP>) {
        // The lane's cells in pairs (0, 1) and (2, 3), packed (cellops F2),
        // each step the scalar hornDX / hornDY / finisher step of its cell.
        // hornDY's vertical differences V_j, bottom row minus top row: the
        // centre columns 1..4 come in aligned pairs, the halo columns alone.
        const F2 V12 = sub2(pk(c.v[1], c.v[2]), pk(a.v[1], a.v[2]));
        const F2 V34 = sub2(pk(c.v[3], c.v[4]), pk(a.v[3], a.v[4]));
        const float V0 = sub(c.v[0], a.v[0]), V5 = sub(c.v[5], a.v[5]);
        // dy_i = (V_i + V_i+2) + (V_i+1 + V_i+1)
        const F2 dy[2] = {add2(pk(add(V0, hi(V12)), add(lo(V12), lo(V34))), add2(V12, V12)),
                          add2(pk(add(hi(V12), hi(V34)), add(lo(V34), V5)), add2(V34, V34))};
        // dx_i = (ha_i + hc_i) + (hb_i + hb_i)
        F2 gx[2], gy[2];
#pragma unroll
        for (int p = 0; p < 2; p++) {
            const F2 hb2 = pk(hb[2 * p], hb[2 * p + 1]);
            const F2 dx = add2(add2(pk(ha[2 * p], ha[2 * p + 1]), pk(hc[2 * p], hc[2 * p + 1])), add2(hb2, hb2));
            gx[p] = mul2(dx, splat(P.k[0]));
            gy[p] = mul2(dy[p], splat(P.k[1]));
        }
#pragma unroll
        for (int p = 0; p < 2; p++) {
            F2 r;
            if constexpr (OP == STRATA_OP_SLOPE && KIND == kSlopeSquareClass)
                r = add_p(mul2(gx[p], gx[p]), mul2(gy[p], gy[p]));  // magnitude's radicand (horn.go:220-222)
            else if constexpr (OP == STRATA_OP_SLOPE) r = slope2(gx[p], gy[p], splat(P.k[2]), KIND != 0);
            else if constexpr (OP == STRATA_OP_ASPECT) r = aspect2(gx[p], gy[p], P.k[2], KIND != 0);
            else if constexpr (OP == STRATA_OP_HEATLOAD) {
                // heatLoadKernel (terrain/heatload.go:147-160): Horn's gradient, then the equation
                double t[8];
                heat_terms(P.w, t);
                r = pk(heat_load(lo(gx[p]), lo(gy[p]), t, P.kind & 1), heat_load(hi(gx[p]), hi(gy[p]), t, P.kind & 1));
            } else if constexpr (OP == STRATA_OP_ORIENTATION) {
                // orientationKernel (terrain/orientation.go:83-95)
                const bool east = P.kind & 1, unw = (P.kind >> 1) & 1;
                r = pk(orientation(lo(gx[p]), lo(gy[p]), east, unw), orientation(hi(gx[p]), hi(gy[p]), east, unw));
            } else r = shade2(gx[p], gy[p], P.k[2], P.k[3], P.k[4]);
            o0[2 * p] = rowin && colin[2 * p] ? lo(r) : nan;
            o0[2 * p + 1] = rowin && colin[2 * p + 1] ? hi(r) : nan;
        }
        // The epilogue maps NaN to itself, so the edge ring stays NaN. A
        // Slope classified on its squared magnitude compares the radicand
        // with the thresholds the host moved its classes to.
        if constexpr (OP == STRATA_OP_SLOPE && KIND == kSlopeSquareClass) reclass_chain4(P.epi[0], o0);
        else if constexpr (EPI) epilogue4(P, *T, o0);
    } else if constexpr (OP == STRATA_OP_CURVATURE) {
        // Pairs (0, 1) and (2, 3) again: the centre column's terms come
        // packed from the rows, the terms of the shifted columns per cell.
#pragma unroll
        for (int p = 0; p < 2; p++) {
            const int i = 2 * p, j = 2 * p + 1;
            const F2 z2 = pk(a.v[i + 1], a.v[j + 1]), z5 = pk(b.v[i + 1], b.v[j + 1]);
            const F2 z8 = pk(c.v[i + 1], c.v[j + 1]);
            const F2 r = zt_curvature2(pk(sub(b.v[i + 2], b.v[i]), sub(b.v[j + 2], b.v[j])), sub2(z8, z2),
                                       add2(z5, z5), pk(add(b.v[i], b.v[i + 2]), add(b.v[j], b.v[j + 2])),
                                       add2(z2, z8), pk(add(a.v[i], c.v[i + 2]), add(a.v[j], c.v[j + 2])),
                                       pk(add(a.v[i + 2], c.v[i]), add(a.v[j + 2], c.v[j])), P.k, KIND);
            o0[i] = rowin && colin[i] ? lo(r) : nan;
            o0[j] = rowin && colin[j] ? hi(r) : nan;
        }
        if constexpr (EPI) epilogue4(P, *T, o0);
    } else if constexpr (OP == STRATA_OP_RUGGEDNESS && KIND == STRATA_RUG_ROUGHNESS) {
        // the window's column maxima and minima shared by the lane's four cells
        float r[4];
        roughness4(a.v, b.v, c.v, r);
#pragma unroll
        for (int i = 0; i < 4; i++) o0[i] = (rowin && colin[i]) ? r[i] : nan;
        if constexpr (EPI) epilogue4(P, *T, o0);
    } else {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float z[9] = {a.v[i], a.v[i + 1], a.v[i + 2], b.v[i], b.v[i + 1],
                                b.v[i + 2], c.v[i], c.v[i + 1], c.v[i + 2]};
            float r0 = nan, r1 = nan;
            apply3<OP, KIND>(P, z, r0, r1);
            o0[i] = (rowin && colin[i]) ? r0 : nan;
        }
        if constexpr (EPI) epilogue4(P, *T, o0);
    }
}

// ---------------------------------------------------------------------------
// One warp's march for rasters of any width and alignment (the batch
// kernels): output columns [xs, xs + 128) clipped to the region, rows
// [y0, y0 + rows). Every lane loads its four source cells (those inside
// the source; a float4 when vec says the rows are 16-byte aligned there),
// lanes 0 and 31 fetch the halo columns, and each lane stores its cells
// inside the region.

struct WarpRows {
    const float* p;  // source row of the next load, at column x (dereferenced only inside the source)
    int64_t stride;
    int by, h;       // next row relative to the source window, and its height
    int bx, w;       // x relative to the source window, and its width
    bool full;       // all four columns inside the source and vec
    __device__ __forceinline__ Row6 next(int lane) {
        Row6 r;
        float q[4] = {0.f, 0.f, 0.f, 0.f};
        float l = 0.f, rr = 0.f;
        const bool in = (unsigned)by < (unsigned)h;
        if (in) {
            if (full) {
                const float4 v = __ldg(reinterpret_cast<const float4*>(p));
                q[0] = v.x;
                q[1] = v.y;
                q[2] = v.z;
                q[3] = v.w;
            } else {
#pragma unroll
                for (int i = 0; i < 4; i++)
                    if ((unsigned)(bx + i) < (unsigned)w) q[i] = __ldg(p + i);
            }
            if (lane == 0 && (unsigned)(bx - 1) < (unsigned)w) l = __ldg(p - 1);
            if (lane == 31 && (unsigned)(bx + 4) < (unsigned)w) rr = __ldg(p + 4);
        }
        const float ul = __shfl_up_sync(kFull, q[3], 1);
        const float dr = __shfl_down_sync(kFull, q[0], 1);
        r.v[0] = lane == 0 ? l : ul;
        r.v[1] = q[0];
        r.v[2] = q[1];
        r.v[3] = q[2];
        r.v[4] = q[3];
        r.v[5] = lane == 31 ? rr : dr;
        p += stride;
        by++;
        return r;
    }
};

template <int OP, int KIND, bool EPI>
__device__ __forceinline__ void march_warp(const LaunchParams& P, const EpiTables* T, int64_t xs, int64_t y0, int rows,
                                           bool vec) {
    constexpr bool kHorn = kIsHorn<OP>;
    constexpr int kRing = 4;
    const int lane = threadIdx.x & 31;
    const int64_t x = xs + 4 * lane;
    const int64_t nc = P.out_x1 - x;
    const int ncols = nc >= 4 ? 4 : (nc <= 0 ? 0 : (int)nc);
    bool colin[4];
#pragma unroll
    for (int i = 0; i < 4; i++) colin[i] = x + i >= 1 && x + i < P.width - 1;
    WarpRows L;
    L.bx = (int)(x - P.src_x0);
    L.w = (int)P.src_w;
    L.by = (int)(y0 - 1 - P.src_y0);
    L.h = (int)P.src_h;
    L.stride = P.src_stride;
    L.full = vec && L.bx >= 0 && L.bx + 3 < L.w;
    L.p = P.src + (y0 - 1 - P.src_y0) * P.src_stride + (x - P.src_x0);
    float* d0 = P.dst0 + (y0 - P.dst_y0) * P.dst0_stride + (x - P.dst_x0);
    float* d1 = OP == STRATA_OP_GRADIENT ? P.dst1 + (y0 - P.dst_y0) * P.dst1_stride + (x - P.dst_x0) : nullptr;
    int yrel = (int)(y0 - 1);
    const int ylast = (int)(P.height - 2);

    // Ring slot m % kRing holds row y0 - 1 + m; output row y0 + k reads
    // m = k .. k + 2, and row k + 3 loads while row k computes.
    Row6 ring[kRing];
    float hr[kRing][4];
#pragma unroll
    for (int j = 0; j < 3; j++) {
        ring[j] = L.next(lane);
        if constexpr (kHorn) hdiff(ring[j], hr[j]);
    }
    for (int k0 = 0; k0 < rows; k0 += kRing) {
#pragma unroll
        for (int u = 0; u < kRing; u++) {
            const int k = k0 + u;
            if (k >= rows) break;
            if (k + 1 < rows) {
                ring[(u + 3) % kRing] = L.next(lane);
                if constexpr (kHorn) hdiff(ring[(u + 3) % kRing], hr[(u + 3) % kRing]);
            }
            yrel++;
            const bool rowin = yrel >= 1 && yrel <= ylast;
            float o0[4], o1[4];
            row_compute<OP, KIND, EPI>(P, T, ring[u % kRing], ring[(u + 1) % kRing], ring[(u + 2) % kRing],
                                       hr[u % kRing], hr[(u + 1) % kRing], hr[(u + 2) % kRing], rowin, colin, o0,
                                       o1);
            if (ncols == 4 && vec) {
                *reinterpret_cast<float4*>(d0) = make_float4(o0[0], o0[1], o0[2], o0[3]);
                if constexpr (OP == STRATA_OP_GRADIENT)
                    *reinterpret_cast<float4*>(d1) = make_float4(o1[0], o1[1], o1[2], o1[3]);
            } else {
#pragma unroll
                for (int i = 0; i < 4; i++)
                    if (i < ncols) {
                        d0[i] = o0[i];
                        if constexpr (OP == STRATA_OP_GRADIENT) d1[i] = o1[i];
                    }
            }
            d0 += P.dst0_stride;
            if constexpr (OP == STRATA_OP_GRADIENT) d1 += P.dst1_stride;
        }
    }
}

}  // namespace
}  // namespace strata
