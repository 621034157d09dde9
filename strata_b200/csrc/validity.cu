// validity.cu - the validity of a stencil's output (internal/stencil/
// mask.go:43-161): bit (x, y) of the output is the AND of the input's bits
// over the (2r+1) x (2r+1) window at (x, y), cleared in the edge ring of
// radius r; radius 0 copies the bits.
//
// The kernel launches the warp-marching body of validity.cuh, one warp a
// strip of 1024 cells and a band of rows.
#include <cuda_runtime.h>

#include "launch.h"
#include "validity.cuh"

namespace strata {
namespace {

constexpr int kVThreads = 256;

template <int R>
__global__ void __launch_bounds__(kVThreads) validity_march_kernel(const __grid_constant__ ValidityParams v, int strips,
                                                                   int band) {
    const int warp = (int)((blockIdx.x * (unsigned)kVThreads + threadIdx.x) >> 5);
    const int strip = warp % strips, bnd = warp / strips;
    const int64_t y0 = v.out_y0 + (int64_t)bnd * band;
    if (y0 >= v.out_y1) return;  // the whole warp
    const int rows = (int)((y0 + band < v.out_y1 ? y0 + band : v.out_y1) - y0);
    validity_strip<R>(v, v.out_x0 + (int64_t)strip * kStripCells, y0, rows);
}

template <int R>
void launch_r(const ValidityParams& v, cudaStream_t s) {
    const int64_t w = v.out_x1 - v.out_x0, h = v.out_y1 - v.out_y0;
    const int64_t strips = (w + kStripCells - 1) / kStripCells;
    // About 48 warps an SM in all, in bands of at least 8 rows.
    const int sms = sm_count();
    int64_t bands = ((int64_t)sms * 48 + strips - 1) / strips;
    int64_t band = (h + bands - 1) / bands;
    if (band < 8) band = 8;
    bands = (h + band - 1) / band;
    const int64_t warps = strips * bands;
    const int64_t blocks = (warps * 32 + kVThreads - 1) / kVThreads;
    validity_march_kernel<R><<<(unsigned)blocks, kVThreads, 0, s>>>(v, (int)strips, (int)band);
}

}  // namespace

void launch_validity(const ValidityParams& v, cudaStream_t s) {
    if (v.dst_words <= 0 || v.out_x1 <= v.out_x0 || v.out_y1 <= v.out_y0) return;
    switch (v.radius) {
    case 0: launch_r<0>(v, s); break;
    case 1: launch_r<1>(v, s); break;
    case 2: launch_r<2>(v, s); break;
    case 3: launch_r<3>(v, s); break;
    case 4: launch_r<4>(v, s); break;
    case 5: launch_r<5>(v, s); break;
    case 6: launch_r<6>(v, s); break;
    case 7: launch_r<7>(v, s); break;
    case 8: launch_r<8>(v, s); break;
    }
}

}  // namespace strata
