// batch.cuh - what the persistent batch kernels (batch.cu, batch_focal.cu)
// share: finding the raster of a work unit and staging its descriptor.
#pragma once

#include "launch.h"

namespace strata {
namespace {

constexpr int kBatchThreads = 128;

// The item of unit u: the last whose first unit is at or before u.
__device__ __forceinline__ int batch_item_of(const BatchItem* __restrict__ items, int n, int64_t u) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].tile0 <= u) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The block copies an item's launch parameters into shared memory (the
// caller synchronises before and after).
__device__ __forceinline__ void batch_stage_params(const BatchItem& it, LaunchParams& P) {
    const int4* s = reinterpret_cast<const int4*>(&it.p);
    int4* d = reinterpret_cast<int4*>(&P);
    for (int i = threadIdx.x; i < (int)(sizeof(LaunchParams) / 16); i += blockDim.x) d[i] = s[i];
}

// The unit u's place in its item: output columns from x, rows [y0, y0 + rows).
struct BatchUnit {
    int64_t x, y0;
    int rows;
    bool vec;
};

__device__ __forceinline__ BatchUnit batch_unit(const BatchItem& it, const LaunchParams& P, int64_t u) {
    const int64_t t = u - it.tile0;
    const int64_t cy = t / it.tiles_x, cx = t - cy * it.tiles_x;
    BatchUnit b;
    b.x = P.out_x0 + cx * it.tw;
    b.y0 = P.out_y0 + cy * it.th;
    const int64_t r = P.out_y1 - b.y0;
    b.rows = r < it.th ? (int)r : it.th;
    b.vec = it.vec != 0;
    return b;
}

}  // namespace
}  // namespace strata
