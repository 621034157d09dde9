// focalops.cuh - the focal and windowed-ruggedness folds at radius R, on
// a window of rows s floats apart (shared by the tile and batch kernels).
#pragma once

#include "cellops.cuh"
#include "launch.h"

namespace strata {

using namespace cell;

// RuggednessWindowRow for radius R > 1 (internal/stencil/rugged.go:152-210):
// Riley, Wilson and TPI over the window in row-major order without the
// centre. c points at the centre cell.
template <int R>
__device__ __forceinline__ float rugged_window(const float* c, int s, int kind) {
    constexpr int D = 2 * R + 1;
    constexpr float n = (float)(D * D - 1);
    const float z = c[0];
    const float* q = c - R * s - R;
    if (kind == 0) {
        double a = 0.0;
#pragma unroll
        for (int j = 0; j < D; j++)
#pragma unroll
            for (int k = 0; k < D; k++)
                if (!(j == R && k == R)) a = __dadd_rn(a, sq64(sub(q[j * s + k], z)));
        return __double2float_rn(__dsqrt_rn(a));
    }
    if (kind == 1) {
        float a = 0.0f;
#pragma unroll
        for (int j = 0; j < D; j++)
#pragma unroll
            for (int k = 0; k < D; k++)
                if (!(j == R && k == R)) a = add(a, abs32(sub(q[j * s + k], z)));
        return div(a, n);
    }
    float a = q[0];  // TPI folds from the first neighbour's value
#pragma unroll
    for (int j = 0; j < D; j++)
#pragma unroll
        for (int k = 0; k < D; k++)
            if (!(j == R && k == R) && !(j == 0 && k == 0)) a = add(a, q[j * s + k]);
    return sub(z, div(a, n));
}

// CorrelateRow (internal/focalrow/focalrow.go:217-230): the first product,
// then every later product added in row-major order of the weights.
template <int R>
__device__ __forceinline__ float correlate(const LaunchParams& P, const float* c, int s) {
    constexpr int D = 2 * R + 1;
    const float* q = c - R * s - R;
    float acc = mul(P.w[0], q[0]);
#pragma unroll
    for (int j = 0; j < D; j++)
#pragma unroll
        for (int k = 0; k < D; k++)
            if (j | k) acc = add(acc, mul(P.w[j * D + k], q[j * s + k]));
    return acc;
}

// Column folds of the separable ops (focalrow.go:232-272): the 2R+1 cells
// of a column, top to bottom.
template <int OP, int R>
__device__ __forceinline__ float column_fold(const LaunchParams& P, const float* top, int s) {
    constexpr int D = 2 * R + 1;
    float a;
    if constexpr (OP == STRATA_OP_SEPARABLE) {
        a = mul(P.w[17], top[0]);
#pragma unroll
        for (int j = 1; j < D; j++) a = add(a, mul(P.w[17 + j], top[j * s]));
    } else {
        a = top[0];
#pragma unroll
        for (int j = 1; j < D; j++) {
            float v = top[j * s];
            if constexpr (OP == STRATA_OP_MEAN) a = add(a, v);
            else if constexpr (OP == STRATA_OP_MIN) a = go_min(a, v);
            else a = go_max(a, v);
        }
    }
    return a;
}

// Row folds (focalrow.go:274-315) of 2R+1 column results, left to right;
// the mean divides by (2R+1)^2 at the end (divRow, focalrow.go:406-421).
template <int OP, int R>
__device__ __forceinline__ float row_fold(const LaunchParams& P, const float* left) {
    constexpr int D = 2 * R + 1;
    float a;
    if constexpr (OP == STRATA_OP_SEPARABLE) {
        a = mul(P.w[0], left[0]);
#pragma unroll
        for (int c = 1; c < D; c++) a = add(a, mul(P.w[c], left[c]));
    } else {
        a = left[0];
#pragma unroll
        for (int c = 1; c < D; c++) {
            if constexpr (OP == STRATA_OP_MEAN) a = add(a, left[c]);
            else if constexpr (OP == STRATA_OP_MIN) a = go_min(a, left[c]);
            else a = go_max(a, left[c]);
        }
        if constexpr (OP == STRATA_OP_MEAN) a = div(a, (float)(D * D));
    }
    return a;
}

template <int OP, int R>
constexpr bool kTwoPass = OP == STRATA_OP_SEPARABLE || OP == STRATA_OP_MEAN || OP == STRATA_OP_MIN ||
                          OP == STRATA_OP_MAX;


}  // namespace strata
