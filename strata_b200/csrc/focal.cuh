// focal.cuh - the bodies of the focal kernels at radius 2..8 (focal.cu),
// shared with the batch kernels (batch.cu): the separable march over one
// unit of 512 column results and a band of rows, and the windowed tile.
// Each takes its unit's place and whether its rows are 16-byte aligned
// (vector loads and stores), so the batch can run rasters of any width
// with the single-raster kernels' arithmetic, cell for cell.
#pragma once

#include <cuda_runtime.h>

#include "cellops.cuh"
#include "launch.h"
#include "ops3.cuh"

namespace strata {
namespace {

using namespace cell;

constexpr int kSepThreads = 128;
constexpr int kSepCols = 4 * kSepThreads;  // column results a block computes per row
constexpr int kStageRows = 8;              // source rows in flight per block (a power of two)

// Four source columns gx .. gx+3, read one row at a time from global row
// y on, by a running pointer and row counter (so no per-row offsets stay
// live): 0 outside the source window.
struct RowWalk {
    const float* p;  // the current row at column gx (dereferenced only inside the source)
    int64_t stride;
    int row, h;  // the current row, relative to the source window, and its height
    int bx, w;   // gx relative to the source window, and its width
    bool full;   // all four columns inside the source, on a 16-byte boundary (vec)
    __device__ __forceinline__ RowWalk(const LaunchParams& P, int64_t gx, int64_t y, bool vec) {
        bx = (int)(gx - P.src_x0);
        w = (int)P.src_w;
        row = (int)(y - P.src_y0);
        h = (int)P.src_h;
        stride = P.src_stride;
        full = vec && bx >= 0 && bx + 3 < w;
        p = P.src + (y - P.src_y0) * P.src_stride + (gx - P.src_x0);
    }
    __device__ __forceinline__ float4 next() {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if ((unsigned)row < (unsigned)h) {
            if (full) {
                v = __ldg(reinterpret_cast<const float4*>(p));
            } else {
                if ((unsigned)(bx + 0) < (unsigned)w) v.x = p[0];
                if ((unsigned)(bx + 1) < (unsigned)w) v.y = p[1];
                if ((unsigned)(bx + 2) < (unsigned)w) v.z = p[2];
                if ((unsigned)(bx + 3) < (unsigned)w) v.w = p[3];
            }
        }
        p += stride;
        row++;
        return v;
    }
};

__device__ __forceinline__ void cp_async16(float* dst, const float* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// A RowWalk fetched ahead into a ring of kStageRows shared-memory rows:
// each thread copies its own 16 bytes of a row (one 16-byte cp.async on
// aligned rows, a 4-byte one per cell otherwise, plain zero stores outside
// the source) and later reads back only those, so
// the thread's wait on its own copy groups orders them without a barrier.
// Row k goes to slot k % kStageRows; issue() starts the next row (one copy
// group a call, empty once the walk's rows are all issued) and take(k)
// returns row k once kStageRows - 1 rows have been issued ahead of it.
struct StageWalk {
    RowWalk w;
    float* mine;  // this thread's 4 floats in slot 0; slot s is s * kSepCols floats on
    int issued, limit;
    __device__ __forceinline__ StageWalk(const LaunchParams& P, int64_t gx, int64_t y, int rows, float* m, bool vec)
        : w(P, gx, y, vec), mine(m), issued(0), limit(rows) {}
    __device__ __forceinline__ void issue() {
        if (issued < limit) {
            float* d = mine + (issued & (kStageRows - 1)) * kSepCols;
            if ((unsigned)w.row < (unsigned)w.h) {
                if (w.full) {
                    cp_async16(d, w.p);
                } else {
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        if ((unsigned)(w.bx + i) < (unsigned)w.w) cp_async4(d + i, w.p + i);
                        else d[i] = 0.0f;
                    }
                }
                w.p += w.stride;
                w.row++;
            } else {
                *reinterpret_cast<float4*>(d) = w.next();
            }
        }
        cp_async_commit();
        issued++;
    }
    __device__ __forceinline__ float4 take(int k) {
        cp_async_wait<kStageRows - 2>();
        return *reinterpret_cast<const float4*>(mine + (k & (kStageRows - 1)) * kSepCols);
    }
};

// Four outputs at columns gx .. gx+3, written one row at a time from
// global row y on: NaN outside the interior (the edge ring of radius R),
// nothing past the region's right edge.
struct OutWalk {
    float* d;
    int64_t stride;
    int y, ylo, yhi;  // the current row and the interior rows [ylo, yhi)
    unsigned colin;   // bit i: column gx + i is interior
    int ncols;        // columns inside the region (4 = all)
    bool vec;         // rows on a 16-byte boundary at gx: one float4 store
    __device__ __forceinline__ OutWalk(const LaunchParams& P, int64_t gx, int64_t y0, int R, bool v) {
        vec = v;
        d = P.dst0 + (y0 - P.dst_y0) * P.dst0_stride + (gx - P.dst_x0);
        stride = P.dst0_stride;
        y = (int)y0;
        ylo = R;
        yhi = (int)P.height - R;
        colin = 0;
        for (int i = 0; i < 4; i++)
            if (gx + i >= R && gx + i < P.width - R) colin |= 1u << i;
        const int64_t n = P.out_x1 - gx;
        ncols = n >= 4 ? 4 : (int)n;
    }
    __device__ __forceinline__ void put(const LaunchParams& P, const float (&o)[4]) {
        const float nan = nanf32();
        const bool rowin = y >= ylo && y < yhi;
        float v[4];
#pragma unroll
        for (int i = 0; i < 4; i++) v[i] = (rowin && ((colin >> i) & 1u)) ? epilogue(P, o[i]) : nan;
        if (ncols == 4 && vec) {
            *reinterpret_cast<float4*>(d) = make_float4(v[0], v[1], v[2], v[3]);
        } else {
#pragma unroll
            for (int i = 0; i < 4; i++)
                if (i < ncols) d[i] = v[i];
        }
    }
    __device__ __forceinline__ void step() {
        d += stride;
        y++;
    }
};

// ---------------------------------------------------------------------------
// Separable ops.

template <int R>
constexpr int kHalo = 4 * ((R + 3) / 4);  // halo columns each side, rounded up to a float4

template <int R>
constexpr int kSepOut = kSepCols - 2 * kHalo<R>;  // output columns per block

// The fold of one column (FOLD is MEAN, MIN, MAX or SEPARABLE), top to
// bottom over ring slots (u + k) % RS, k = 0 .. 2R; u is a constant once
// the caller's row loop is unrolled, so the ring stays in registers.
template <int FOLD, int R, int RS>
__device__ __forceinline__ float col_fold(const LaunchParams& P, const float (&ring)[RS][4], int i, int u) {
    constexpr int D = 2 * R + 1;
    float a;
    if constexpr (FOLD == STRATA_OP_SEPARABLE) a = mul(P.w[17], ring[u % RS][i]);
    else a = ring[u % RS][i];
#pragma unroll
    for (int k = 1; k < D; k++) {
        const float v = ring[(u + k) % RS][i];
        if constexpr (FOLD == STRATA_OP_SEPARABLE) a = add(a, mul(P.w[17 + k], v));
        else if constexpr (FOLD == STRATA_OP_MEAN) a = add(a, v);
        else if constexpr (FOLD == STRATA_OP_MIN) a = go_min(a, v);
        else a = go_max(a, v);
    }
    return a;
}

// Rows the separable march's loop body covers: all 2R+1 (the ring slot of
// each row a constant, no moves) while that code stays small, else 4 with
// the ring's last 2R rows moved down after every 4 (the loop body would
// otherwise outgrow the instruction cache).
template <int R>
constexpr int kSepUnroll = R >= 5 ? 4 : 2 * R + 1;
template <int R>
constexpr int kSepRing = kSepUnroll<R> == 2 * R + 1 ? 2 * R + 1 : 2 * R + kSepUnroll<R>;

// Min and Max folds (Go's min/max: NaN wins, -0 below +0, as PTX min.NaN /
// max.NaN) are exactly associative and commutative, so any grouping of a
// window's terms gives the reference's bits. Their folds share work between
// neighbouring windows: the four output rows of a 4-row step share window
// rows 3 .. 2R, and a thread's four outputs share column results 3 .. 2R
// of their windows, so each such core is folded once and every window adds
// its own three edge terms (25 operations for four windows at R = 8, where
// four separate folds take 64).
template <int FOLD>
constexpr bool kMinMax = FOLD == STRATA_OP_MIN || FOLD == STRATA_OP_MAX;

template <int FOLD>
__device__ __forceinline__ float minmax(float a, float b) {
    if constexpr (FOLD == STRATA_OP_MIN) return go_min(a, b);
    else return go_max(a, b);
}

// The core of a 4-row step's column folds (ring slots 3 .. 2R, the step's
// first output row at slot 0).
template <int FOLD, int R, int RS>
__device__ __forceinline__ float col_core(const float (&ring)[RS][4], int i) {
    float a = ring[3][i];
#pragma unroll
    for (int k = 4; k <= 2 * R; k++) a = minmax<FOLD>(a, ring[k][i]);
    return a;
}

// Output row u's column fold from the core: its rows u .. 2 before the
// core and 2R+1 .. 2R+u after it.
template <int FOLD, int R, int RS>
__device__ __forceinline__ float col_from_core(const float (&ring)[RS][4], int i, int u, float core) {
    float a = core;
#pragma unroll
    for (int k = u; k <= 2; k++) a = minmax<FOLD>(a, ring[k][i]);
#pragma unroll
    for (int k = 2 * R + 1; k <= 2 * R + u; k++) a = minmax<FOLD>(a, ring[k][i]);
    return a;
}

// Term c (0 .. 2R) of a fold across column results, left to right: the
// first term starts the fold.
template <int FOLD>
__device__ __forceinline__ float fold_term(const LaunchParams& P, float a, float v, int c) {
    if constexpr (FOLD == STRATA_OP_SEPARABLE) return c == 0 ? mul(P.w[0], v) : add(a, mul(P.w[c], v));
    if (c == 0) return v;
    if constexpr (FOLD == STRATA_OP_MEAN) return add(a, v);
    else if constexpr (FOLD == STRATA_OP_MIN) return go_min(a, v);
    else return go_max(a, v);
}

// OP is SEPARABLE, MEAN, MIN, MAX, or RUGGEDNESS for roughness (the max
// fold minus the min fold). Block b covers output columns [X0, X0 +
// kSepOut) of a band of strip rows; thread t holds columns X0 - kHalo +
// 4t .. +3.
template <int OP>
constexpr int kSepFolds = OP == STRATA_OP_RUGGEDNESS ? 2 : 1;

// Rows of column results a block stores between two barriers: the whole
// 4-row step where the loop body covers 4 rows and the op has one fold
// (its four row folds then follow one barrier; roughness's two folds would
// outgrow the 48 KB of static shared memory), else one.
template <int OP, int R>
constexpr int kSepTbRows = kSepUnroll<R> == 4 && kSepFolds<OP> == 1 ? 4 : 1;

// The block's shared memory for sep_body.
template <int OP, int R>
struct SepSmem {
    float tb[2][kSepFolds<OP>][kSepTbRows<OP, R>][kSepCols];  // column results, double-buffered
    float stg[kStageRows][kSepCols];                          // source rows in flight
};

// One unit of the separable march, by a block of kSepThreads threads:
// output columns [X0, X0 + kSepOut) (clipped to the region) of rows [y0,
// y0 + rows). vec: source and destination rows start on a 16-byte boundary
// at X0 - kHalo and X0. Ends with the block's copies landed; the caller
// synchronises the block before the shared memory is used again.
template <int OP, int R>
__device__ __forceinline__ void sep_body(const LaunchParams& P, int64_t X0, int64_t y0, int rows, bool vec,
                                         SepSmem<OP, R>& sm) {
    constexpr int D = 2 * R + 1;
    constexpr int HL = kHalo<R>;
    constexpr int OW = kSepOut<R>;
    constexpr int NF = kSepFolds<OP>;
    constexpr int F0 = OP == STRATA_OP_RUGGEDNESS ? STRATA_OP_MAX : OP;
    constexpr int F1 = STRATA_OP_MIN;
    constexpr int NT = 4 + 2 * HL;  // column results a thread's four outputs span (rounded to float4s)
    auto& tb = sm.tb;
    auto& stg = sm.stg;
    const int tid = threadIdx.x;

    // The source rows y0 - R .. y0 + rows - 1 + R, kStageRows - 1 ahead of
    // the one consumed.
    StageWalk src(P, X0 - HL + 4 * tid, y0 - R, rows + 2 * R, &stg[0][4 * tid], vec);
#pragma unroll
    for (int k = 0; k < kStageRows - 1; k++) src.issue();
    constexpr int U = kSepUnroll<R>;
    constexpr int RS = kSepRing<R>;
    float ring[RS][4];
    int taken = 0;
#pragma unroll
    for (int k = 0; k < 2 * R; k++) {
        const float4 v = src.take(taken++);
        src.issue();
        ring[k][0] = v.x;
        ring[k][1] = v.y;
        ring[k][2] = v.z;
        ring[k][3] = v.w;
    }
    const bool writer = tid < OW / 4 && X0 + 4 * tid < P.out_x1;
    OutWalk dst(P, X0 + 4 * tid, y0, R, vec);
    int buf = 0;
    // Min/Max column folds through a core shared by the 4-row step (the
    // ring holds the step's 2R + 4 rows).
    constexpr bool kCoreRows = kMinMax<F0> && U == 4 && RS == 2 * R + 4;
    float core0[4], core1[4];
    (void)core0;
    (void)core1;
    // Row w of the stored column results folded across into this thread's
    // four outputs of the row, which it stores.
    auto fold_row = [&](int w) {
        if constexpr (kMinMax<F0>) {
            // Min/Max: output i's window is column results B+i ..
            // B+i+2R; results B+3 .. B+2R are common to the four, the
            // rest (B .. B+2 before, B+2R+1 .. B+2R+3 after) are kept
            // apart and added per output.
            constexpr int B = HL - R;
            float core[2], lo[2][3], hi[2][3];
#pragma unroll
            for (int q = 0; q < NT / 4; q++) {
                const float4 f0 = *reinterpret_cast<const float4*>(&tb[buf][0][w][4 * tid + 4 * q]);
                float4 f1 = f0;
                if constexpr (NF == 2) f1 = *reinterpret_cast<const float4*>(&tb[buf][NF - 1][w][4 * tid + 4 * q]);
                const float v[2][4] = {{f0.x, f0.y, f0.z, f0.w}, {f1.x, f1.y, f1.z, f1.w}};
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int t = 4 * q + e;
#pragma unroll
                    for (int f = 0; f < NF; f++) {
                        if (t < B || t > B + 2 * R + 3) continue;
                        if (t <= B + 2) lo[f][t - B] = v[f][e];
                        else if (t > B + 2 * R) hi[f][t - B - 2 * R - 1] = v[f][e];
                        else if (t == B + 3) core[f] = v[f][e];
                        else core[f] = f == 0 ? minmax<F0>(core[f], v[f][e]) : minmax<F1>(core[f], v[f][e]);
                    }
                }
            }
            float o[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                float a = core[0];
#pragma unroll
                for (int k = i; k <= 2; k++) a = minmax<F0>(a, lo[0][k]);
#pragma unroll
                for (int k = 0; k < i; k++) a = minmax<F0>(a, hi[0][k]);
                if constexpr (NF == 2) {
                    float b = core[1];
#pragma unroll
                    for (int k = i; k <= 2; k++) b = minmax<F1>(b, lo[1][k]);
#pragma unroll
                    for (int k = 0; k < i; k++) b = minmax<F1>(b, hi[1][k]);
                    a = sub(a, b);
                }
                o[i] = a;
            }
            dst.put(P, o);
        } else {
            // Stream the column results left to right; each feeds the
            // outputs whose windows hold it, so every output folds its
            // 2R+1 terms in order with only its accumulator live.
            float o[4], o1[4];
#pragma unroll
            for (int q = 0; q < NT / 4; q++) {
                const float4 f0 = *reinterpret_cast<const float4*>(&tb[buf][0][w][4 * tid + 4 * q]);
                float4 f1 = f0;
                if constexpr (NF == 2) f1 = *reinterpret_cast<const float4*>(&tb[buf][NF - 1][w][4 * tid + 4 * q]);
                const float v0[4] = {f0.x, f0.y, f0.z, f0.w};
                const float v1[4] = {f1.x, f1.y, f1.z, f1.w};
#pragma unroll
                for (int e = 0; e < 4; e++)
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        // output X0 + 4t + i folds column results from t index HL - R + i
                        const int c = 4 * q + e - (HL - R + i);
                        if (c < 0 || c > 2 * R) continue;
                        o[i] = fold_term<F0>(P, o[i], v0[e], c);
                        if constexpr (NF == 2) o1[i] = fold_term<F1>(P, o1[i], v1[e], c);
                    }
            }
#pragma unroll
            for (int i = 0; i < 4; i++) {
                if constexpr (F0 == STRATA_OP_MEAN) o[i] = div(o[i], (float)(D * D));
                if constexpr (NF == 2) o[i] = sub(o[i], o1[i]);
            }
            dst.put(P, o);
        }
    };
    for (int yb = 0; yb < rows; yb += U) {
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (yb + u >= rows) break;
            {
                const float4 v = src.take(taken++);
                src.issue();
                float* slot = ring[(u + 2 * R) % RS];
                slot[0] = v.x;
                slot[1] = v.y;
                slot[2] = v.z;
                slot[3] = v.w;
            }
            float c0[4], c1[4];
            if constexpr (kCoreRows) {
                // the core is complete once row 2R (slot 2R) has landed
                if (u == 0) {
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        core0[i] = col_core<F0, R, RS>(ring, i);
                        if constexpr (NF == 2) core1[i] = col_core<F1, R, RS>(ring, i);
                    }
                }
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    c0[i] = col_from_core<F0, R, RS>(ring, i, u, core0[i]);
                    if constexpr (NF == 2) c1[i] = col_from_core<F1, R, RS>(ring, i, u, core1[i]);
                }
            } else {
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    c0[i] = col_fold<F0, R, RS>(P, ring, i, u);
                    if constexpr (NF == 2) c1[i] = col_fold<F1, R, RS>(P, ring, i, u);
                }
            }
            constexpr int TB = kSepTbRows<OP, R>;
            const int w = TB == 1 ? 0 : u;
            *reinterpret_cast<float4*>(&tb[buf][0][w][4 * tid]) = make_float4(c0[0], c0[1], c0[2], c0[3]);
            if constexpr (NF == 2)
                *reinterpret_cast<float4*>(&tb[buf][NF - 1][w][4 * tid]) = make_float4(c1[0], c1[1], c1[2], c1[3]);
            if constexpr (TB == 1) {
                __syncthreads();
                if (writer) fold_row(0);
                dst.step();
                buf ^= 1;
            }
        }
        if constexpr (kSepTbRows<OP, R> == 4) {
            // The step's column results are all stored: one barrier, then
            // its row folds.
            const int nu = rows - yb < U ? rows - yb : U;
            __syncthreads();
#pragma unroll 1
            for (int w = 0; w < nu; w++) {
                if (writer) fold_row(w);
                dst.step();
            }
            buf ^= 1;
        }
        if constexpr (RS != D) {
            // The window's last 2R rows move down to the ring's first slots.
#pragma unroll
            for (int k = 0; k < 2 * R; k++)
#pragma unroll
                for (int i = 0; i < 4; i++) ring[k][i] = ring[k + U][i];
        }
    }
    cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// Windowed ops.

constexpr int kWinThreads = 128;  // 32 column groups x 4 row groups
constexpr int kWinTW = 128;       // output columns per tile

// Rows of outputs per thread: fewer for Riley, whose sums are doubles.
template <int OP, int KIND>
constexpr int kWinM = (OP == STRATA_OP_RUGGEDNESS && KIND == STRATA_RUG_TRI_RILEY) ? 4 : 8;

// Four source cells of global columns gx .. gx+3 in global row gy, 0 where
// outside the source window (only non-interior outputs read those).
__device__ __forceinline__ float4 load4(const LaunchParams& P, int64_t gx, int64_t gy, bool vec) {
    RowWalk w(P, gx, gy, vec);
    return w.next();
}

template <int OP, int R, int KIND>
constexpr int kWinTileFloats = (4 * kWinM<OP, KIND> + 2 * R) * (kWinTW + 2 * kHalo<R>);

// One tile of a windowed op, by a block of kWinThreads threads: outputs at
// columns [x0, x0 + 128) and rows [y0, y0 + 4M) (clipped to the region).
// OP is CORRELATE (KIND 0) or RUGGEDNESS with KIND Riley, Wilson or TPI.
// Thread (tx, ty) accumulates the outputs at columns 4 tx .. 4 tx + 3 and
// rows M ty .. M ty + M - 1 of the tile. tile: kWinTileFloats floats,
// 16-byte aligned; the caller synchronises the block before reusing it.
template <int OP, int R, int KIND>
__device__ __forceinline__ void window_body(const LaunchParams& P, int64_t x0, int64_t y0, bool vec, float* tile) {
    constexpr int D = 2 * R + 1;
    constexpr int HL = kHalo<R>;
    constexpr int M = kWinM<OP, KIND>;
    constexpr int TW = kWinTW + 2 * HL;  // staged columns
    constexpr int TH = 4 * M + 2 * R;    // staged rows
    constexpr int NT = 4 + 2 * HL;
    constexpr bool RILEY = OP == STRATA_OP_RUGGEDNESS && KIND == STRATA_RUG_TRI_RILEY;
    constexpr bool WILSON = OP == STRATA_OP_RUGGEDNESS && KIND == STRATA_RUG_TRI_WILSON;
    constexpr bool TPI = OP == STRATA_OP_RUGGEDNESS && KIND == STRATA_RUG_TPI;
    for (int i = threadIdx.x; i < TH * (TW / 4); i += kWinThreads) {
        const int r = i / (TW / 4), c = i - r * (TW / 4);
        *reinterpret_cast<float4*>(&tile[r * TW + 4 * c]) = load4(P, x0 - HL + 4 * c, y0 - R + r, vec);
    }
    __syncthreads();
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;

    // Sums start from -0 where the reference starts from its first term
    // (-0 + t == t for every t), from +0 where it starts from zero.
    float acc[M][4];
    double dacc[RILEY ? M : 1][4];
    float ctr[(RILEY || WILSON) ? M : 1][4];
#pragma unroll
    for (int m = 0; m < M; m++)
#pragma unroll
        for (int i = 0; i < 4; i++) {
            acc[m][i] = WILSON ? 0.0f : -0.0f;
            if constexpr (RILEY) dacc[m][i] = 0.0;
            if constexpr (RILEY || WILSON) ctr[m][i] = tile[(ty * M + m + R) * TW + 4 * tx + HL + i];
        }
#pragma unroll 1
    for (int j = 0; j < D; j++) {
        float w[OP == STRATA_OP_CORRELATE ? D : 1];
        if constexpr (OP == STRATA_OP_CORRELATE) {
#pragma unroll
            for (int k = 0; k < D; k++) w[k] = P.w[j * D + k];
        }
        const bool centre_row = j == R;
#pragma unroll
        for (int m = 0; m < M; m++) {
            const float* row = &tile[(ty * M + m + j) * TW + 4 * tx];
            float z[NT];
#pragma unroll
            for (int q = 0; q < NT / 4; q++) {
                const float4 a = *reinterpret_cast<const float4*>(row + 4 * q);
                z[4 * q] = a.x;
                z[4 * q + 1] = a.y;
                z[4 * q + 2] = a.z;
                z[4 * q + 3] = a.w;
            }
#pragma unroll
            for (int k = 0; k < D; k++)
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const float v = z[HL - R + i + k];
                    if constexpr (OP == STRATA_OP_CORRELATE) {
                        acc[m][i] = add(acc[m][i], mul(w[k], v));
                    } else if (k != R || !centre_row) {
                        if constexpr (RILEY) dacc[m][i] = add_sq64(dacc[m][i], sub(v, ctr[m][i]));
                        else if constexpr (WILSON) acc[m][i] = add(acc[m][i], abs32(sub(v, ctr[m][i])));
                        else acc[m][i] = add(acc[m][i], v);
                    }
                }
        }
    }
    const int64_t gx = x0 + 4 * tx;
    if (gx >= P.out_x1) return;
    constexpr float n = (float)(D * D - 1);
    OutWalk dst(P, gx, y0 + ty * M, R, vec);
#pragma unroll
    for (int m = 0; m < M; m++) {
        if (y0 + ty * M + m >= P.out_y1) break;
        float o[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            if constexpr (RILEY) o[i] = __double2float_rn(__dsqrt_rn(dacc[m][i]));
            else if constexpr (WILSON) o[i] = div(acc[m][i], n);
            else if constexpr (TPI) o[i] = sub(tile[(ty * M + m + R) * TW + 4 * tx + HL + i], div(acc[m][i], n));
            else o[i] = acc[m][i];
        }
        dst.put(P, o);
        dst.step();
    }
}

}  // namespace
}  // namespace strata
