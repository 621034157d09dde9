// ops3.cuh - every radius-1 op on a 3x3 window held in registers.
//
// z[0..8] is the window in row-major order (strata's z1..z9, z[4] the
// centre). The Horn, Zevenbergen-Thorne and ruggedness ops call the cell
// functions of cellops.cuh; the focal ops at radius 1 fold their terms in
// the reference's order (internal/focalrow/focalrow.go:217-315): the 2-D
// correlation from the first product in row-major order, the separable
// ops column by column (top to bottom) and then across the three column
// results (left to right).
#pragma once

#include "cellops.cuh"
#include "launch.h"

namespace strata {

// KIND: the op's kind, fixed per kernel (Curvature's type, Ruggedness's
// measure), so each kernel carries one kind's arithmetic; kKindAtRun reads
// it from the launch instead (Riley's TRI: its float64 sums over a lane's
// four cells, scheduled side by side in a kernel of its own, outgrow the
// register budget).
constexpr int kKindAtRun = -1;

template <int OP, int KIND>
__device__ __forceinline__ void apply3(const LaunchParams& P, const float (&z)[9], float& o0, float& o1) {
    using namespace cell;
    if constexpr (OP == STRATA_OP_CURVATURE) {
        o0 = zt_curvature(z[0], z[1], z[2], z[3], z[4], z[5], z[6], z[7], z[8], P.k, KIND);
    } else if constexpr (OP == STRATA_OP_RUGGEDNESS) {
        o0 = rugged3(z[0], z[1], z[2], z[3], z[4], z[5], z[6], z[7], z[8], KIND == kKindAtRun ? P.kind : KIND);
    } else if constexpr (OP == STRATA_OP_CORRELATE) {
        float acc = mul(P.w[0], z[0]);
#pragma unroll
        for (int i = 1; i < 9; i++) acc = add(acc, mul(P.w[i], z[i]));
        o0 = acc;
    } else if constexpr (OP == STRATA_OP_SEPARABLE) {
        float t[3];
#pragma unroll
        for (int c = 0; c < 3; c++)
            t[c] = add(add(mul(P.w[17], z[c]), mul(P.w[18], z[3 + c])), mul(P.w[19], z[6 + c]));
        o0 = add(add(mul(P.w[0], t[0]), mul(P.w[1], t[1])), mul(P.w[2], t[2]));
    } else if constexpr (OP == STRATA_OP_MEAN) {
        float t[3];
#pragma unroll
        for (int c = 0; c < 3; c++) t[c] = add(add(z[c], z[3 + c]), z[6 + c]);
        o0 = div(add(add(t[0], t[1]), t[2]), 9.0f);
    } else if constexpr (OP == STRATA_OP_MIN) {
        float t[3];
#pragma unroll
        for (int c = 0; c < 3; c++) t[c] = go_min(go_min(z[c], z[3 + c]), z[6 + c]);
        o0 = go_min(go_min(t[0], t[1]), t[2]);
    } else if constexpr (OP == STRATA_OP_MAX) {
        float t[3];
#pragma unroll
        for (int c = 0; c < 3; c++) t[c] = go_max(go_max(z[c], z[3 + c]), z[6 + c]);
        o0 = go_max(go_max(t[0], t[1]), t[2]);
    } else {
        float gx = mul(horn_dx(z[0], z[2], z[3], z[5], z[6], z[8]), P.k[0]);
        float gy = mul(horn_dy(z[0], z[1], z[2], z[6], z[7], z[8]), P.k[1]);
        if constexpr (OP == STRATA_OP_GRADIENT) {
            o0 = gx;
            o1 = gy;
        } else if constexpr (OP == STRATA_OP_SLOPE) {
            o0 = slope(gx, gy, P.k[2], P.kind != 0);
        } else if constexpr (OP == STRATA_OP_ASPECT) {
            o0 = aspect(gx, gy, P.k[2], P.kind != 0);
        } else {
            o0 = shade(gx, gy, P.k[2], P.k[3], P.k[4]);
        }
    }
}

// The pointwise stages fused after a stencil (exec.Pipeline's staged
// Lookup / Reclass tail, internal/exec/pipeline.go:539-574), reading their
// tables from the launch parameters.
// A tail holding chain steps (vec.Chain, internal/vec/chain.go) runs as
// its step sequence, the tables by reference; the host admits only the
// unary steps after a stencil.
__device__ __forceinline__ float table_stage(const EpiStage& e, float v) {
    return e.op == STRATA_OP_LOOKUP ? cell::lookup(v, e.a, e.b, e.n) : cell::reclass(v, e.a, e.n, e.b);
}

__device__ __forceinline__ float epilogue(const LaunchParams& P, float v) {
    if (P.nstep) {
#pragma unroll 1
        for (int i = 0; i < P.nstep; i++) {
            const ChainStep& s = P.step[i];
            v = s.op >= kStepTable ? table_stage(P.epi[s.op - kStepTable], v) : cell::vec_step(s.op, v, 0.0f, s.k0, s.k1);
        }
        return v;
    }
    for (int i = 0; i < P.nepi; i++) v = table_stage(P.epi[i], v);
    return v;
}

// The epilogue's tables staged in shared memory: each cell reads the
// knots of its own segment, and lanes reading different addresses of the
// constant bank are served one address at a time, where shared memory
// serves them together.
struct EpiTables {
    // a: the knots (breaks), padded with NaN to a power of two; b: the
    // values; p2: the padded length, the binary search's span.
    float a[kMaxEpilogue][2 * STRATA_MAX_KNOTS];
    float b[kMaxEpilogue][STRATA_MAX_KNOTS + 1];
    int p2[kMaxEpilogue];
};

// Copies the tables in with every thread of the block; the caller
// synchronises the block before reading them.
__device__ __forceinline__ void stage_epilogue(const LaunchParams& P, EpiTables& T) {
    constexpr int per = 2 * STRATA_MAX_KNOTS + STRATA_MAX_KNOTS + 1;
    const int nt = blockDim.x * blockDim.y;
    for (int i = threadIdx.x + threadIdx.y * blockDim.x; i < P.nepi * per; i += nt) {
        const int s = i / per, j = i - s * per;
        if (j < 2 * STRATA_MAX_KNOTS) T.a[s][j] = j < P.epi[s].n ? P.epi[s].a[j] : cell::nanf32();
        else T.b[s][j - 2 * STRATA_MAX_KNOTS] = P.epi[s].b[j - 2 * STRATA_MAX_KNOTS];
    }
    if (threadIdx.x + threadIdx.y * blockDim.x < P.nepi) {
        const int s = threadIdx.x + threadIdx.y * blockDim.x;
        int p2 = 1;
        while (p2 < P.epi[s].n + 1) p2 <<= 1;
        T.p2[s] = p2;
    }
}

// The number of knots at or below v (v not NaN): the reference's forward
// scan index for strictly increasing knots, found by halving the padded
// table. "t[j] <= v" holds for a prefix of the knots and never for a NaN
// pad, so each step keeps the count's invariant.
__device__ __forceinline__ int knot_count(const float* t, int p2, float v) {
    int c = 0;
    for (int step = p2 >> 1; step >= 1; step >>= 1) c += t[c + step - 1] <= v ? step : 0;
    return c;
}

// One pointwise stage (Lookup or Reclass, internal/curve/scalar.go:39-114)
// over a lane's four cells at once, so their loads and arithmetic overlap.
__device__ __forceinline__ void epi_stage4(const EpiStage& e, const float* ta, const float* tb, int p2,
                                           float (&v)[4]) {
    const int n = e.n;
    int k[4];
#pragma unroll
    for (int c = 0; c < 4; c++) k[c] = knot_count(ta, p2, v[c]);
    if (e.op == STRATA_OP_RECLASS) {
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const float r = tb[k[c]];
            v[c] = v[c] != v[c] ? v[c] : r;
        }
        return;
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int lo = k[c] == 0 ? 0 : k[c] - 1;
        const int hi = k[c] == n ? n - 1 : k[c];
        const float x0 = ta[lo], y0 = tb[lo];
        const float t = cell::div(cell::sub(v[c], x0), cell::sub(ta[hi], x0));
        float r = cell::add(y0, cell::mul(t, cell::sub(tb[hi], y0)));
        r = v[c] == x0 ? y0 : r;
        r = k[c] == n ? tb[n - 1] : r;
        r = k[c] == 0 ? tb[0] : r;
        v[c] = v[c] != v[c] ? v[c] : r;
    }
}

// A lone Reclass over four cells as a chain of selects against its breaks
// in increasing order: the last break at or below v names the class, which
// is the search's count for strictly increasing, NaN-free breaks (the host
// checks both), and a NaN cell stays NaN. A break costs a compare and a
// select per cell, with no dependent table loads; the guard on the break
// count is uniform and shared by the four cells.
__device__ __forceinline__ void reclass_chain4(const EpiStage& e, float (&v)[4]) {
    const int n = e.n;
    float r[4];
#pragma unroll
    for (int c = 0; c < 4; c++) r[c] = e.b[0];
#pragma unroll
    for (int j = 0; j < kChainBreaks; j++) {
        if (j >= n) break;
        const float t = e.a[j], y = e.b[j + 1];
#pragma unroll
        for (int c = 0; c < 4; c++) r[c] = v[c] >= t ? y : r[c];
    }
#pragma unroll
    for (int c = 0; c < 4; c++) v[c] = v[c] != v[c] ? v[c] : r[c];
}

// The epilogue over four cells, stage by stage.
__device__ __forceinline__ void epilogue4(const LaunchParams& P, const EpiTables& T, float (&v)[4]) {
    if (P.nstep) {
#pragma unroll 1
        for (int i = 0; i < P.nstep; i++) {
            const ChainStep s = P.step[i];
            if (s.op >= kStepTable) {
                const int t = s.op - kStepTable;
                epi_stage4(P.epi[t], T.a[t], T.b[t], T.p2[t], v);
            } else {
#pragma unroll
                for (int c = 0; c < 4; c++) v[c] = cell::vec_step(s.op, v[c], 0.0f, s.k0, s.k1);
            }
        }
        return;
    }
    if (P.nepi == 1 && P.epi[0].op == STRATA_OP_RECLASS && P.epi[0].n <= kChainBreaks) {
        reclass_chain4(P.epi[0], v);
        return;
    }
#pragma unroll
    for (int i = 0; i < kMaxEpilogue; i++)
        if (i < P.nepi) epi_stage4(P.epi[i], T.a[i], T.b[i], T.p2[i], v);
}

}  // namespace strata
