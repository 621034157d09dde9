// kernels.cu - sm_100a kernels of the raster-stencil path.
//
// Data kernels: one thread block computes a tile of output cells from a
// halo tile of the input staged in shared memory; cells within the radius
// of the raster's border get NaN (internal/exec/halo.go:61-92). Ops whose
// reference form is separable (ColumnX then RowX,
// internal/focalrow/focalrow.go:153-315) keep that two-pass order inside
// the tile, so every cell folds its terms in the reference's order. The
// validity of the outputs is written by validity.cu.
#include "cellops.cuh"
#include "focalops.cuh"
#include "launch.h"
#include "ops3.cuh"
#include "validity.cuh"

namespace strata {
namespace {

using namespace cell;

constexpr int kThreadsX = 32;
constexpr int kThreadsY = 8;
constexpr int kThreads = kThreadsX * kThreadsY;
constexpr int kCX = 2;
constexpr int kCY = 4;
constexpr int kTW = kThreadsX * kCX;  // tile width in cells
constexpr int kTH = kThreadsY * kCY;  // tile height in cells

// The general tile kernel: every op at every radius, any alignment and
// stride. Tile kTW x kTH output cells; thread (tx, ty) computes cells
// (tx + 32 i, ty + 8 j).
template <int OP, int R>
__global__ void __launch_bounds__(kThreads) tile_kernel(const __grid_constant__ LaunchParams P) {
    constexpr int SW = kTW + 2 * R;
    constexpr int SH = kTH + 2 * R;
    constexpr int SP = SW | 1;  // odd pitch: column walks stay conflict-free
    constexpr bool two_pass = kTwoPass<OP, R> || (OP == STRATA_OP_RUGGEDNESS && R > 1);
    __shared__ float tile[SH * SP];
    __shared__ float colr[two_pass ? kTH * SP : 1];
    __shared__ float colr2[(OP == STRATA_OP_RUGGEDNESS && R > 1) ? kTH * SP : 1];

    const int tid = threadIdx.y * kThreadsX + threadIdx.x;
    const int64_t W = P.width, H = P.height;
    for (int64_t t = blockIdx.x; t < P.tiles; t += gridDim.x) {
        const int64_t x0 = P.out_x0 + (t % P.tiles_x) * kTW;
        const int64_t y0 = P.out_y0 + (t / P.tiles_x) * kTH;
        __syncthreads();
        for (int i = tid; i < SW * SH; i += kThreads) {
            const int sy = i / SW, sx = i - sy * SW;
            const int64_t bx = x0 - R + sx - P.src_x0, by = y0 - R + sy - P.src_y0;
            float v = 0.0f;
            if (bx >= 0 && bx < P.src_w && by >= 0 && by < P.src_h) v = P.src[by * P.src_stride + bx];
            tile[sy * SP + sx] = v;
        }
        __syncthreads();
        if constexpr (two_pass) {
            // Column pass over the tile's output rows and every column.
            for (int i = tid; i < kTH * SW; i += kThreads) {
                const int oy = i / SW, sx = i - oy * SW;
                const float* top = &tile[oy * SP + sx];
                if constexpr (OP == STRATA_OP_RUGGEDNESS) {
                    colr[oy * SP + sx] = column_fold<STRATA_OP_MAX, R>(P, top, SP);
                    colr2[oy * SP + sx] = column_fold<STRATA_OP_MIN, R>(P, top, SP);
                } else {
                    colr[oy * SP + sx] = column_fold<OP, R>(P, top, SP);
                }
            }
            __syncthreads();
        }
#pragma unroll
        for (int j = 0; j < kCY; j++) {
#pragma unroll
            for (int i = 0; i < kCX; i++) {
                const int ox = threadIdx.x + kThreadsX * i;
                const int oy = threadIdx.y + kThreadsY * j;
                const int64_t gx = x0 + ox, gy = y0 + oy;
                if (gx >= P.out_x1 || gy >= P.out_y1) continue;
                const bool interior = gx >= R && gx < W - R && gy >= R && gy < H - R;
                float o0 = nanf32(), o1 = nanf32();
                if (interior) {
                    const float* c = &tile[(oy + R) * SP + ox + R];
                    if constexpr (OP == STRATA_OP_RUGGEDNESS && R > 1) {
                        if (P.kind == STRATA_RUG_ROUGHNESS) {
                            const float hi = row_fold<STRATA_OP_MAX, R>(P, &colr[oy * SP + ox]);
                            const float lo = row_fold<STRATA_OP_MIN, R>(P, &colr2[oy * SP + ox]);
                            o0 = sub(hi, lo);
                        } else {
                            o0 = rugged_window<R>(c, SP, P.kind);
                        }
                    } else if constexpr (two_pass) {
                        o0 = row_fold<OP, R>(P, &colr[oy * SP + ox]);
                    } else if constexpr (OP == STRATA_OP_CORRELATE) {
                        o0 = correlate<R>(P, c, SP);
                    } else {
                        const float z[9] = {c[-SP - 1], c[-SP], c[-SP + 1], c[-1], c[0], c[1],
                                            c[SP - 1], c[SP], c[SP + 1]};
                        apply3<OP>(P, z, o0, o1);
                    }
                    o0 = epilogue(P, o0);
                }
                const int64_t dx = gx - P.dst_x0, dy = gy - P.dst_y0;
                P.dst0[dy * P.dst0_stride + dx] = o0;
                if constexpr (OP == STRATA_OP_GRADIENT) P.dst1[dy * P.dst1_stride + dx] = o1;
            }
        }
    }
}

// Pointwise stages alone (radius 0): every cell through the epilogue.
__global__ void __launch_bounds__(256) pointwise_kernel(const __grid_constant__ LaunchParams P) {
    const int64_t w = P.out_x1 - P.out_x0;
    const int64_t n = w * (P.out_y1 - P.out_y0);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t y = i / w, x = i - y * w;
        const int64_t gx = P.out_x0 + x, gy = P.out_y0 + y;
        const float v = P.src[(gy - P.src_y0) * P.src_stride + (gx - P.src_x0)];
        P.dst0[(gy - P.dst_y0) * P.dst0_stride + (gx - P.dst_x0)] = epilogue(P, v);
    }
}

// ---------------------------------------------------------------------------
// Validity.


template <int OP, int R>
int64_t launch_tiles(const LaunchParams& p0, cudaStream_t s) {
    LaunchParams p = p0;
    p.tiles_x = (p.out_x1 - p.out_x0 + kTW - 1) / kTW;
    p.tiles = p.tiles_x * ((p.out_y1 - p.out_y0 + kTH - 1) / kTH);
    const int64_t grid = p.tiles < (int64_t)1 << 30 ? p.tiles : (int64_t)1 << 30;
    tile_kernel<OP, R><<<(unsigned)grid, dim3(kThreadsX, kThreadsY), 0, s>>>(p);
    return p.tiles;
}

using Launcher = int64_t (*)(const LaunchParams&, cudaStream_t);

template <int OP>
Launcher pick_radius(int r) {
    switch (r) {
    case 1: return launch_tiles<OP, 1>;
    case 2: return launch_tiles<OP, 2>;
    case 3: return launch_tiles<OP, 3>;
    case 4: return launch_tiles<OP, 4>;
    case 5: return launch_tiles<OP, 5>;
    case 6: return launch_tiles<OP, 6>;
    case 7: return launch_tiles<OP, 7>;
    case 8: return launch_tiles<OP, 8>;
    }
    return nullptr;
}

}  // namespace

void tile_shape(int op, int radius, int64_t width, int* tw, int* th) {
    (void)op;
    (void)radius;
    (void)width;
    *tw = kTW;
    *th = kTH;
}

int64_t launch_data(const LaunchParams& p, cudaStream_t s, int64_t* window_cells) {
    Launcher L = nullptr;
    switch (p.op) {
    case STRATA_OP_GRADIENT: L = launch_tiles<STRATA_OP_GRADIENT, 1>; break;
    case STRATA_OP_SLOPE: L = launch_tiles<STRATA_OP_SLOPE, 1>; break;
    case STRATA_OP_ASPECT: L = launch_tiles<STRATA_OP_ASPECT, 1>; break;
    case STRATA_OP_HILLSHADE: L = launch_tiles<STRATA_OP_HILLSHADE, 1>; break;
    case STRATA_OP_CURVATURE: L = launch_tiles<STRATA_OP_CURVATURE, 1>; break;
    case STRATA_OP_RUGGEDNESS: L = pick_radius<STRATA_OP_RUGGEDNESS>(p.radius); break;
    case STRATA_OP_CORRELATE: L = pick_radius<STRATA_OP_CORRELATE>(p.radius); break;
    case STRATA_OP_SEPARABLE: L = pick_radius<STRATA_OP_SEPARABLE>(p.radius); break;
    case STRATA_OP_MEAN: L = pick_radius<STRATA_OP_MEAN>(p.radius); break;
    case STRATA_OP_MIN: L = pick_radius<STRATA_OP_MIN>(p.radius); break;
    case STRATA_OP_MAX: L = pick_radius<STRATA_OP_MAX>(p.radius); break;
    case STRATA_OP_LOOKUP:
    case STRATA_OP_RECLASS: {
        const int64_t n = (p.out_x1 - p.out_x0) * (p.out_y1 - p.out_y0);
        int64_t blocks = (n + 255) / 256;
        if (blocks > 148 * 64) blocks = 148 * 64;
        if (blocks < 1) blocks = 1;
        pointwise_kernel<<<(unsigned)blocks, 256, 0, s>>>(p);
        if (window_cells) *window_cells = n;
        return blocks;
    }
    }
    if (!L) return -1;
    if (p.out_x1 <= p.out_x0 || p.out_y1 <= p.out_y0) {
        if (window_cells) *window_cells = 0;
        return 0;
    }
    if (march3_eligible(p)) {
        const int64_t blocks = launch_march3(p, s);
        if (window_cells) {
            // Each warp reads its 128 columns and two halo columns, over its
            // strip and one halo row above and below, clipped to the raster.
            const int64_t w = p.out_x1 - p.out_x0, segs = (w + 127) / 128;
            const int64_t rows = (p.out_y1 - p.out_y0) + 2 * (blocks / ((segs + 3) / 4));
            *window_cells = (w + 2 * segs) * (rows < p.height ? rows : p.height);
        }
        return blocks;
    }
    if (march_any_eligible(p)) {
        const int64_t blocks = launch_march_any(p, s);
        if (window_cells) {
            const int64_t w = p.out_x1 - p.out_x0, segs = (w + 127) / 128;
            const int64_t rows = (p.out_y1 - p.out_y0) + 2 * (blocks / ((segs + 3) / 4));
            *window_cells = (w + 2 * segs) * (rows < p.height ? rows : p.height);
        }
        return blocks;
    }
    if (focal_eligible(p)) return launch_focal(p, s, window_cells);
    const int64_t tiles = L(p, s);
    if (window_cells) {
        // Each tile reads its cells grown by the radius, clipped to the raster.
        const int r = p.radius;
        const int64_t tx = (p.out_x1 - p.out_x0 + kTW - 1) / kTW, ty = (p.out_y1 - p.out_y0 + kTH - 1) / kTH;
        int64_t wx = 0, wy = 0;
        for (int64_t i = 0; i < tx; i++) {
            const int64_t a = p.out_x0 + i * kTW - r, b = p.out_x0 + (i + 1) * kTW + r;
            wx += (b < p.width ? b : p.width) - (a > 0 ? a : 0);
        }
        for (int64_t i = 0; i < ty; i++) {
            const int64_t a = p.out_y0 + i * kTH - r, b = p.out_y0 + (i + 1) * kTH + r;
            wy += (b < p.height ? b : p.height) - (a > 0 ? a : 0);
        }
        *window_cells = wx * wy;
    }
    return tiles;
}


}  // namespace strata
