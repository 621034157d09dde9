// batch_focal.cu - the batch kernels of the focal ops at radius 2..8: the
// separable march (a unit is a band of 512 column results) and the
// windowed tile (a unit is a tile of 128 columns), running the bodies of
// the single-raster kernels (focal.cuh) on each raster's units.
#include "batch.cuh"
#include "focal.cuh"
#include "launch.h"

namespace strata {
namespace {

template <int OP, int R>
__global__ void __launch_bounds__(kSepThreads, (OP == STRATA_OP_SEPARABLE || OP == STRATA_OP_RUGGEDNESS) && R >= 6 ? 3 : 4)
    batch_sep_kernel(const BatchItem* __restrict__ items, int n, int64_t total) {
    __shared__ __align__(16) LaunchParams P;
    __shared__ __align__(16) SepSmem<OP, R> sm;
    int cur = -1;
    for (int64_t u = blockIdx.x; u < total; u += gridDim.x) {
        const int it = batch_item_of(items, n, u);
        __syncthreads();  // the last unit is done with the shared memory
        if (it != cur) {
            batch_stage_params(items[it], P);
            __syncthreads();
            cur = it;
        }
        const BatchUnit b = batch_unit(items[it], P, u);
        sep_body<OP, R>(P, b.x, b.y0, b.rows, b.vec, sm);
    }
}

template <int OP, int R, int KIND>
__global__ void __launch_bounds__(kWinThreads) batch_window_kernel(const BatchItem* __restrict__ items, int n,
                                                                   int64_t total) {
    __shared__ __align__(16) LaunchParams P;
    __shared__ __align__(16) float tile[kWinTileFloats<OP, R, KIND>];
    int cur = -1;
    for (int64_t u = blockIdx.x; u < total; u += gridDim.x) {
        const int it = batch_item_of(items, n, u);
        __syncthreads();  // the last tile is done with the shared memory
        if (it != cur) {
            batch_stage_params(items[it], P);
            __syncthreads();
            cur = it;
        }
        const BatchUnit b = batch_unit(items[it], P, u);
        window_body<OP, R, KIND>(P, b.x, b.y0, b.vec, tile);
    }
}

// Blocks that fill the GPU once at the kernel's occupancy (per_sm), never
// more than the units.
int grid_for(int per_sm, int64_t total) {
    const int64_t g = (int64_t)sm_count() * per_sm;
    return (int)(total < g ? total : g);
}

template <class K>
int occupancy(K kernel, int threads) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, 0) != cudaSuccess || n < 1) n = 1;
    return n;
}

template <int OP, int R>
bool launch_sep(const BatchClass& c, const BatchItem* d, cudaStream_t s) {
    static const int per_sm = occupancy(batch_sep_kernel<OP, R>, kSepThreads);
    batch_sep_kernel<OP, R><<<grid_for(per_sm, c.total), kSepThreads, 0, s>>>(d + c.first, c.count, c.total);
    return true;
}

template <int OP, int R, int KIND>
bool launch_window(const BatchClass& c, const BatchItem* d, cudaStream_t s) {
    static const int per_sm = occupancy(batch_window_kernel<OP, R, KIND>, kWinThreads);
    batch_window_kernel<OP, R, KIND><<<grid_for(per_sm, c.total), kWinThreads, 0, s>>>(d + c.first, c.count, c.total);
    return true;
}

template <int R>
bool launch_radius(const BatchClass& c, const BatchItem* d, cudaStream_t s) {
    switch (c.op) {
    case STRATA_OP_SEPARABLE: return launch_sep<STRATA_OP_SEPARABLE, R>(c, d, s);
    case STRATA_OP_MEAN: return launch_sep<STRATA_OP_MEAN, R>(c, d, s);
    case STRATA_OP_MIN: return launch_sep<STRATA_OP_MIN, R>(c, d, s);
    case STRATA_OP_MAX: return launch_sep<STRATA_OP_MAX, R>(c, d, s);
    case STRATA_OP_CORRELATE: return launch_window<STRATA_OP_CORRELATE, R, 0>(c, d, s);
    case STRATA_OP_RUGGEDNESS:
        switch (c.kind) {
        case STRATA_RUG_TRI_RILEY: return launch_window<STRATA_OP_RUGGEDNESS, R, STRATA_RUG_TRI_RILEY>(c, d, s);
        case STRATA_RUG_TRI_WILSON: return launch_window<STRATA_OP_RUGGEDNESS, R, STRATA_RUG_TRI_WILSON>(c, d, s);
        case STRATA_RUG_TPI: return launch_window<STRATA_OP_RUGGEDNESS, R, STRATA_RUG_TPI>(c, d, s);
        default: return launch_sep<STRATA_OP_RUGGEDNESS, R>(c, d, s);
        }
    }
    return false;
}

template <int R>
void shape_r(int op, int kind, int band, int* tw, int* th) {
    if (op == STRATA_OP_CORRELATE || (op == STRATA_OP_RUGGEDNESS && kind != STRATA_RUG_ROUGHNESS)) {
        *tw = kWinTW;
        *th = 4 * ((op == STRATA_OP_RUGGEDNESS && kind == STRATA_RUG_TRI_RILEY) ? 4 : 8);
    } else {
        *tw = kSepOut<R>;
        *th = band > 0 ? band : 64;
    }
}

}  // namespace

void batch_focal_shape(int op, int radius, int kind, int band, int* tw, int* th) {
    switch (radius) {
    case 2: shape_r<2>(op, kind, band, tw, th); break;
    case 3: shape_r<3>(op, kind, band, tw, th); break;
    case 4: shape_r<4>(op, kind, band, tw, th); break;
    case 5: shape_r<5>(op, kind, band, tw, th); break;
    case 6: shape_r<6>(op, kind, band, tw, th); break;
    case 7: shape_r<7>(op, kind, band, tw, th); break;
    default: shape_r<8>(op, kind, band, tw, th); break;
    }
}

bool launch_batch_focal(const BatchClass& c, const BatchItem* d, cudaStream_t s) {
    switch (c.radius) {
    case 2: return launch_radius<2>(c, d, s);
    case 3: return launch_radius<3>(c, d, s);
    case 4: return launch_radius<4>(c, d, s);
    case 5: return launch_radius<5>(c, d, s);
    case 6: return launch_radius<6>(c, d, s);
    case 7: return launch_radius<7>(c, d, s);
    case 8: return launch_radius<8>(c, d, s);
    }
    return false;
}

}  // namespace strata
