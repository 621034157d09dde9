// kernels.cu - the dispatch of a data launch to its kernel, and the
// pointwise kernel.
//
// launch_data sends a launch to the radius-1 march (march3.cu: TMA rows
// where the rows are 16-byte aligned, per-cell access otherwise), the focal
// kernels at radius 2..8 (focal.cu), or, for Lookup/Reclass alone, the
// pointwise kernel below. Every kernel leaves the cells within the radius
// of the raster's border NaN (internal/exec/halo.go:61-92); the validity of
// the outputs is written by validity.cu.
#include <cstring>

#include "cellops.cuh"
#include "launch.h"
#include "ops3.cuh"

namespace strata {
namespace {

using namespace cell;

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

}  // namespace


int64_t launch_data(const LaunchParams& p, cudaStream_t s, int64_t* window_cells) {
    if (p.op == STRATA_OP_LOOKUP || p.op == STRATA_OP_RECLASS) {
        const int64_t n = (p.out_x1 - p.out_x0) * (p.out_y1 - p.out_y0);
        int64_t blocks = (n + 255) / 256;
        if (blocks > (int64_t)sm_count() * 64) blocks = (int64_t)sm_count() * 64;
        if (blocks < 1) blocks = 1;
        pointwise_kernel<<<(unsigned)blocks, 256, 0, s>>>(p);
        if (window_cells) *window_cells = n;
        return blocks;
    }
    if (p.op < STRATA_OP_GRADIENT || p.op > STRATA_OP_MAX) return -1;
    if (p.out_x1 <= p.out_x0 || p.out_y1 <= p.out_y0) {
        if (window_cells) *window_cells = 0;
        return 0;
    }
    if (march3_eligible(p) || march_any_eligible(p)) {
        const int64_t blocks = march3_eligible(p) ? launch_march3(p, s) : launch_march_any(p, s);
        if (window_cells) {
            // Each warp reads its 128 columns and two halo columns, over its
            // strip and one halo row above and below, clipped to the raster.
            const int64_t w = p.out_x1 - p.out_x0, segs = (w + 127) / 128;
            const int64_t rows = (p.out_y1 - p.out_y0) + 2 * (blocks / ((segs + 3) / 4));
            *window_cells = (w + 2 * segs) * (rows < p.height ? rows : p.height);
        }
        return blocks;
    }
    if (focal_eligible(p)) return launch_focal(p, s, window_cells);
    return -1;  // beyond the kernels' 32-bit index limits: the caller falls back to the CPU
}

int64_t launch_stage(LaunchParams p, const ValidityParams* const v[2], cudaStream_t s, int64_t* window_cells) {
    memset(&p.vf, 0, sizeof p.vf);
    const ValidityParams* any = v[0] ? v[0] : v[1];
    bool fuse = any != nullptr && p.radius == 1 && march3_eligible(p);
    for (int i = 0; i < 2 && fuse; i++) {
        const ValidityParams* q = v[i];
        if (!q) continue;
        fuse = q->radius == 1 && q->src_bits == any->src_bits && q->src_off == any->src_off &&
               q->src_stride == any->src_stride && q->src_x0 == p.src_x0 && q->src_y0 == p.src_y0 &&
               q->dst_x0 == p.dst_x0 && q->dst_y0 == p.dst_y0 && q->out_x0 == p.out_x0 && q->out_x1 == p.out_x1 &&
               q->out_y0 == p.out_y0 && q->out_y1 == p.out_y1 && q->width == p.width && q->height == p.height;
    }
    if (fuse) {
        p.vf.src_bits = any->src_bits;
        p.vf.src_off = any->src_off;
        p.vf.src_stride = any->src_stride;
        p.vf.src_lo_word = any->src_lo_word;
        p.vf.src_hi_word = any->src_hi_word;
        for (int i = 0; i < 2; i++) {
            if (!v[i]) continue;
            p.vf.dst_bits[i] = v[i]->dst_bits;
            p.vf.dst_off[i] = v[i]->dst_off;
            p.vf.dst_stride[i] = v[i]->dst_stride;
            p.vf.n++;
        }
        return launch_data(p, s, window_cells);
    }
    const int64_t t = launch_data(p, s, window_cells);
    if (t < 0) return t;
    for (int i = 0; i < 2; i++)
        if (v[i]) launch_validity(*v[i], s);
    return t;
}


}  // namespace strata
