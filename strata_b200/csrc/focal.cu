// focal.cu - register-blocked kernels for the windowed ops at radius 2..8.
//
// Separable ops (CorrelateSeparable, Mean, Min, Max, and roughness as the
// max and min folds; internal/focalrow/focalrow.go:232-315): a block owns
// a strip of 512 column results and marches down a band of rows. Each
// thread keeps the last 2R+1 input rows of its 4 columns in registers, so
// a column fold (top to bottom) costs 2R operations and no loads; the
// block shares one row of column results through shared memory, and each
// thread folds 2R+1 of them (left to right) for 4 adjacent outputs. The
// source rows arrive through a ring of shared-memory rows filled by
// cp.async several rows ahead, so a row's load latency overlaps the folds
// of the rows before it.
//
// Windowed ops (Correlate/Convolve, focalrow.go:217-230; the Riley, Wilson
// and TPI ruggedness kinds, internal/stencil/rugged.go:152-210): a block
// stages a 128-column output tile grown by the radius in shared memory; a
// thread accumulates a 4 x M block of outputs, walking the window row by
// row and each row left to right, so every output folds its terms in the
// reference's row-major order while each staged row segment is loaded
// once per M x 4 x (2R+1) terms.
//
// Both kernels leave cells within the radius of the raster's border NaN
// (internal/exec/halo.go:61-92). They load and store whole float4s where
// the rows are 16-byte aligned at the kernel's columns, and single cells
// otherwise (the launcher decides per call).
#include <cuda_runtime.h>

#include "cellops.cuh"
#include "focal.cuh"
#include "launch.h"
#include "ops3.cuh"

namespace strata {
namespace {

template <int OP, int R>
__global__ void __launch_bounds__(kSepThreads, (OP == STRATA_OP_SEPARABLE || OP == STRATA_OP_RUGGEDNESS) && R >= 6 ? 3 : 4)
    sep_march_kernel(const __grid_constant__ LaunchParams P, int colblocks, int strip, int vec) {
    __shared__ __align__(16) SepSmem<OP, R> sm;
    const int cb = (int)(blockIdx.x % (unsigned)colblocks);
    const int sb = (int)(blockIdx.x / (unsigned)colblocks);
    const int64_t X0 = P.out_x0 + (int64_t)cb * kSepOut<R>;
    const int64_t y0 = P.out_y0 + (int64_t)sb * strip;
    const int rows = (int)((y0 + strip < P.out_y1 ? y0 + strip : P.out_y1) - y0);
    sep_body<OP, R>(P, X0, y0, rows, vec != 0, sm);
}

template <int OP, int R, int KIND>
__global__ void __launch_bounds__(kWinThreads) window_kernel(const __grid_constant__ LaunchParams P, int tiles_x,
                                                             int vec) {
    __shared__ __align__(16) float tile[kWinTileFloats<OP, R, KIND>];
    const int64_t x0 = P.out_x0 + (int64_t)(blockIdx.x % (unsigned)tiles_x) * kWinTW;
    const int64_t y0 = P.out_y0 + (int64_t)(blockIdx.x / (unsigned)tiles_x) * (4 * kWinM<OP, KIND>);
    window_body<OP, R, KIND>(P, x0, y0, vec != 0, tile);
}

// ---------------------------------------------------------------------------
// Launchers.

bool aligned16(const void* q) { return ((uintptr_t)q & 15) == 0; }

// Whether the rows of source and destination start on 16-byte boundaries
// at the columns the kernels load and store (then whole float4s).
int focal_vec(const LaunchParams& p) {
    return !(p.src_stride & 3) && !(p.dst0_stride & 3) && !((p.out_x0 - p.src_x0) & 3) &&
           !((p.out_x0 - p.dst_x0) & 3) && aligned16(p.src) && aligned16(p.dst0);
}

template <int OP, int R>
int64_t launch_sep(const LaunchParams& p, cudaStream_t s, int64_t* window_cells) {
    constexpr int OW = kSepOut<R>;
    static const int per_sm = [] {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sep_march_kernel<OP, R>, kSepThreads, 0) != cudaSuccess ||
            n < 1)
            n = 1;
        return n;
    }();
    const int64_t w = p.out_x1 - p.out_x0, h = p.out_y1 - p.out_y0;
    const int64_t colblocks = (w + OW - 1) / OW;
    // Bands of equal height, as many as fill the GPU's block slots once.
    const int64_t slots = (int64_t)sm_count() * per_sm;
    int64_t bands = slots / colblocks;
    if (bands < 1) bands = 1;
    int64_t strip = (h + bands - 1) / bands;
    if (strip < 16) strip = 16;
    bands = (h + strip - 1) / strip;
    sep_march_kernel<OP, R><<<(unsigned)(colblocks * bands), kSepThreads, 0, s>>>(p, (int)colblocks, (int)strip,
                                                                                  focal_vec(p));
    if (window_cells) {
        // each block reads its 512 columns over its band and R rows above and below, clipped to the raster
        int64_t wx = 0, wy = 0;
        for (int64_t i = 0; i < colblocks; i++) {
            const int64_t a = p.out_x0 + i * OW - kHalo<R>, b = a + kSepCols;
            wx += (b < p.width ? b : p.width) - (a > 0 ? a : 0);
        }
        for (int64_t i = 0; i < bands; i++) {
            const int64_t a = p.out_y0 + i * strip - R, e = p.out_y0 + (i + 1) * strip;
            const int64_t b = (e < p.out_y1 ? e : p.out_y1) + R;
            wy += (b < p.height ? b : p.height) - (a > 0 ? a : 0);
        }
        *window_cells = wx * wy;
    }
    return colblocks * bands;
}

template <int OP, int R, int KIND>
int64_t launch_window(const LaunchParams& p, cudaStream_t s, int64_t* window_cells) {
    constexpr int TH = 4 * kWinM<OP, KIND>;
    const int64_t w = p.out_x1 - p.out_x0, h = p.out_y1 - p.out_y0;
    const int64_t tiles_x = (w + kWinTW - 1) / kWinTW, tiles_y = (h + TH - 1) / TH;
    window_kernel<OP, R, KIND><<<(unsigned)(tiles_x * tiles_y), kWinThreads, 0, s>>>(p, (int)tiles_x, focal_vec(p));
    if (window_cells) {
        int64_t wx = 0, wy = 0;
        for (int64_t i = 0; i < tiles_x; i++) {
            const int64_t a = p.out_x0 + i * kWinTW - kHalo<R>, b = p.out_x0 + (i + 1) * kWinTW + kHalo<R>;
            wx += (b < p.width ? b : p.width) - (a > 0 ? a : 0);
        }
        for (int64_t i = 0; i < tiles_y; i++) {
            const int64_t a = p.out_y0 + i * TH - R, b = p.out_y0 + (i + 1) * TH + R;
            wy += (b < p.height ? b : p.height) - (a > 0 ? a : 0);
        }
        *window_cells = wx * wy;
    }
    return tiles_x * tiles_y;
}

template <int R>
int64_t launch_radius(const LaunchParams& p, cudaStream_t s, int64_t* wc) {
    switch (p.op) {
    case STRATA_OP_SEPARABLE: return launch_sep<STRATA_OP_SEPARABLE, R>(p, s, wc);
    case STRATA_OP_MEAN: return launch_sep<STRATA_OP_MEAN, R>(p, s, wc);
    case STRATA_OP_MIN: return launch_sep<STRATA_OP_MIN, R>(p, s, wc);
    case STRATA_OP_MAX: return launch_sep<STRATA_OP_MAX, R>(p, s, wc);
    case STRATA_OP_CORRELATE: return launch_window<STRATA_OP_CORRELATE, R, 0>(p, s, wc);
    case STRATA_OP_RUGGEDNESS:
        switch (p.kind) {
        case STRATA_RUG_TRI_RILEY: return launch_window<STRATA_OP_RUGGEDNESS, R, STRATA_RUG_TRI_RILEY>(p, s, wc);
        case STRATA_RUG_TRI_WILSON: return launch_window<STRATA_OP_RUGGEDNESS, R, STRATA_RUG_TRI_WILSON>(p, s, wc);
        case STRATA_RUG_TPI: return launch_window<STRATA_OP_RUGGEDNESS, R, STRATA_RUG_TPI>(p, s, wc);
        default: return launch_sep<STRATA_OP_RUGGEDNESS, R>(p, s, wc);
        }
    }
    return -1;
}

}  // namespace

bool focal_eligible(const LaunchParams& p) {
    if (p.radius < 2 || p.radius > STRATA_MAX_RADIUS) return false;
    switch (p.op) {
    case STRATA_OP_SEPARABLE:
    case STRATA_OP_MEAN:
    case STRATA_OP_MIN:
    case STRATA_OP_MAX:
    case STRATA_OP_CORRELATE:
    case STRATA_OP_RUGGEDNESS: break;
    default: return false;
    }
    const int64_t w = p.out_x1 - p.out_x0, h = p.out_y1 - p.out_y0;
    if (w <= 0 || h <= 0) return false;
    // 32-bit block, row and column arithmetic inside the kernels.
    const int64_t blocks = ((w + 127) / 128) * ((h + 15) / 16);
    return blocks < ((int64_t)1 << 31) && p.height < ((int64_t)1 << 30) && p.width < ((int64_t)1 << 30) &&
           p.src_h < ((int64_t)1 << 30) && p.src_w < ((int64_t)1 << 30);
}

int64_t launch_focal(const LaunchParams& p, cudaStream_t s, int64_t* window_cells) {
    switch (p.radius) {
    case 2: return launch_radius<2>(p, s, window_cells);
    case 3: return launch_radius<3>(p, s, window_cells);
    case 4: return launch_radius<4>(p, s, window_cells);
    case 5: return launch_radius<5>(p, s, window_cells);
    case 6: return launch_radius<6>(p, s, window_cells);
    case 7: return launch_radius<7>(p, s, window_cells);
    case 8: return launch_radius<8>(p, s, window_cells);
    }
    return -1;
}

}  // namespace strata
