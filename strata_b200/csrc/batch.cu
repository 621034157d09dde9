// batch.cu - many rasters of mixed sizes and ops in one CUDA-graph launch.
//
// A batch groups its rasters by op class (op and radius). Each class runs
// one persistent kernel: its blocks walk the work units of every raster of
// the class (output tiles, gridDim apart), so a class of many small
// rasters costs one launch rather than one per raster, and the classes'
// kernels sit side by side in one captured graph that replays with one
// launch. Each raster carries its own tile shape (the autotuner's choice
// for its class) and its own descriptor: the block stages the descriptor
// of the raster it works on in shared memory, loads the tile with its
// halo, computes it with the same cell functions as the single-raster
// kernels (so every cell has the same bits), and writes the tile's
// validity with word-safe updates.
#include "cellops.cuh"
#include "focalops.cuh"
#include "launch.h"
#include "ops3.cuh"
#include "validity.cuh"

namespace strata {
namespace {

constexpr int kBatchThreads = 256;

template <int OP, int R>
constexpr bool kColPass = OP == STRATA_OP_SEPARABLE || OP == STRATA_OP_MEAN || OP == STRATA_OP_MIN ||
                          OP == STRATA_OP_MAX || (OP == STRATA_OP_RUGGEDNESS && R > 1);

template <int OP, int R>
__global__ void __launch_bounds__(kBatchThreads) batch_kernel(const BatchItem* __restrict__ items, int nitems,
                                                              int64_t total) {
    extern __shared__ __align__(16) float sm[];
    __shared__ LaunchParams P;
    __shared__ ValidityParams V[2];
    const int tid = threadIdx.x;
    int cur = -1;
    int tw = 0, th = 0, nvalid = 0;
    int64_t tiles_x = 1, tile0 = 0;
    for (int64_t u = blockIdx.x; u < total; u += gridDim.x) {
        // The raster of unit u: the last whose first unit is at or before u.
        int lo = 0, hi = nitems - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (items[mid].tile0 <= u) lo = mid;
            else hi = mid - 1;
        }
        if (lo != cur) {
            __syncthreads();  // the last tile is done with the previous descriptor
            const int4* s = reinterpret_cast<const int4*>(&items[lo].p);
            int4* d = reinterpret_cast<int4*>(&P);
            for (int i = tid; i < (int)(sizeof(LaunchParams) / 16); i += kBatchThreads) d[i] = s[i];
            const int4* sv = reinterpret_cast<const int4*>(&items[lo].v[0]);
            int4* dv = reinterpret_cast<int4*>(&V[0]);
            for (int i = tid; i < (int)(2 * sizeof(ValidityParams) / 16); i += kBatchThreads) dv[i] = sv[i];
            tw = items[lo].tw;
            th = items[lo].th;
            tiles_x = items[lo].tiles_x;
            tile0 = items[lo].tile0;
            nvalid = items[lo].nvalid;
            cur = lo;
        }
        __syncthreads();
        const int64_t t = u - tile0;
        const int64_t x0 = P.out_x0 + (t % tiles_x) * tw;
        const int64_t y0 = P.out_y0 + (t / tiles_x) * th;
        const int64_t x1 = min(x0 + tw, P.out_x1), y1 = min(y0 + th, P.out_y1);
        const int SW = tw + 2 * R, SH = th + 2 * R;
        float* tile = sm;
        for (int i = tid; i < SW * SH; i += kBatchThreads) {
            const int sy = i / SW, sx = i - sy * SW;
            const int64_t bx = x0 - R + sx - P.src_x0, by = y0 - R + sy - P.src_y0;
            float v = 0.0f;
            if (bx >= 0 && bx < P.src_w && by >= 0 && by < P.src_h) v = P.src[by * P.src_stride + bx];
            tile[i] = v;
        }
        __syncthreads();
        float* colr = sm + SW * SH;     // column results: th rows of SW
        float* colr2 = colr + th * SW;  // roughness keeps the minima here
        if constexpr (kColPass<OP, R>) {
            for (int i = tid; i < th * SW; i += kBatchThreads) {
                const int oy = i / SW, sx = i - oy * SW;
                const float* top = &tile[oy * SW + sx];
                if constexpr (OP == STRATA_OP_RUGGEDNESS) {
                    colr[i] = column_fold<STRATA_OP_MAX, R>(P, top, SW);
                    colr2[i] = column_fold<STRATA_OP_MIN, R>(P, top, SW);
                } else {
                    colr[i] = column_fold<OP, R>(P, top, SW);
                }
            }
            __syncthreads();
        }
        const int64_t W = P.width, H = P.height;
        for (int i = tid; i < tw * th; i += kBatchThreads) {
            const int oy = i / tw, ox = i - oy * tw;
            const int64_t gx = x0 + ox, gy = y0 + oy;
            if (gx >= x1 || gy >= y1) continue;
            const bool interior = gx >= R && gx < W - R && gy >= R && gy < H - R;
            float o0 = cell::nanf32(), o1 = cell::nanf32();
            if (interior) {
                const float* c = &tile[(oy + R) * SW + ox + R];
                if constexpr (OP == STRATA_OP_RUGGEDNESS && R > 1) {
                    if (P.kind == STRATA_RUG_ROUGHNESS)
                        o0 = cell::sub(row_fold<STRATA_OP_MAX, R>(P, &colr[oy * SW + ox]),
                                       row_fold<STRATA_OP_MIN, R>(P, &colr2[oy * SW + ox]));
                    else
                        o0 = rugged_window<R>(c, SW, P.kind);
                } else if constexpr (kColPass<OP, R>) {
                    o0 = row_fold<OP, R>(P, &colr[oy * SW + ox]);
                } else if constexpr (OP == STRATA_OP_CORRELATE && R > 1) {
                    o0 = correlate<R>(P, c, SW);
                } else {
                    const float z[9] = {c[-SW - 1], c[-SW], c[-SW + 1], c[-1], c[0], c[1],
                                        c[SW - 1], c[SW], c[SW + 1]};
                    apply3<OP>(P, z, o0, o1);
                }
                if (P.nepi) o0 = epilogue(P, o0);
            }
            const int64_t dx = gx - P.dst_x0, dy = gy - P.dst_y0;
            P.dst0[dy * P.dst0_stride + dx] = o0;
            if constexpr (OP == STRATA_OP_GRADIENT) P.dst1[dy * P.dst1_stride + dx] = o1;
        }
        for (int k = 0; k < nvalid; k++) region_validity(V[k], x0, y0, x1, y1, tid, kBatchThreads);
    }
}

template <int OP, int R>
void launch_class(const BatchItem* items, int nitems, int64_t total, int grid, size_t smem, cudaStream_t s) {
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(batch_kernel<OP, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    batch_kernel<OP, R><<<grid, kBatchThreads, smem, s>>>(items, nitems, total);
}

using ClassLauncher = void (*)(const BatchItem*, int, int64_t, int, size_t, cudaStream_t);

template <int OP>
ClassLauncher pick(int r) {
    switch (r) {
    case 1: return launch_class<OP, 1>;
    case 2: return launch_class<OP, 2>;
    case 3: return launch_class<OP, 3>;
    case 4: return launch_class<OP, 4>;
    case 5: return launch_class<OP, 5>;
    case 6: return launch_class<OP, 6>;
    case 7: return launch_class<OP, 7>;
    case 8: return launch_class<OP, 8>;
    }
    return nullptr;
}

}  // namespace

size_t batch_smem_bytes(int op, int radius, int tw, int th) {
    const int SW = tw + 2 * radius, SH = th + 2 * radius;
    int floats = SW * SH;
    const bool colpass = op == STRATA_OP_SEPARABLE || op == STRATA_OP_MEAN || op == STRATA_OP_MIN ||
                         op == STRATA_OP_MAX || (op == STRATA_OP_RUGGEDNESS && radius > 1);
    if (colpass) floats += th * SW * (op == STRATA_OP_RUGGEDNESS ? 2 : 1);
    return (size_t)floats * 4;
}

bool launch_batch_class(int op, int radius, const BatchItem* items, int nitems, int64_t total, int grid,
                        size_t smem, cudaStream_t s) {
    ClassLauncher L = nullptr;
    switch (op) {
    case STRATA_OP_GRADIENT: L = launch_class<STRATA_OP_GRADIENT, 1>; break;
    case STRATA_OP_SLOPE: L = launch_class<STRATA_OP_SLOPE, 1>; break;
    case STRATA_OP_ASPECT: L = launch_class<STRATA_OP_ASPECT, 1>; break;
    case STRATA_OP_HILLSHADE: L = launch_class<STRATA_OP_HILLSHADE, 1>; break;
    case STRATA_OP_CURVATURE: L = launch_class<STRATA_OP_CURVATURE, 1>; break;
    case STRATA_OP_RUGGEDNESS: L = pick<STRATA_OP_RUGGEDNESS>(radius); break;
    case STRATA_OP_CORRELATE: L = pick<STRATA_OP_CORRELATE>(radius); break;
    case STRATA_OP_SEPARABLE: L = pick<STRATA_OP_SEPARABLE>(radius); break;
    case STRATA_OP_MEAN: L = pick<STRATA_OP_MEAN>(radius); break;
    case STRATA_OP_MIN: L = pick<STRATA_OP_MIN>(radius); break;
    case STRATA_OP_MAX: L = pick<STRATA_OP_MAX>(radius); break;
    }
    if (!L) return false;
    L(items, nitems, total, grid, smem, s);
    return true;
}

}  // namespace strata
