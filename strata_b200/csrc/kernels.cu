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
#include <memory>

#include "cellops.cuh"
#include "launch.h"
#include "ops3.cuh"

namespace strata {
namespace {

using namespace cell;

// Pointwise stages alone (radius 0): every cell through the epilogue, or,
// for a tail of chain steps, through the steps with the binary ones
// reading their input's cell (vec.Chain over its inputs, internal/vec/
// chain.go:133-155 and scalar.go:180-228: the running value starts at
// input 0 and is every step's first operand). A warp takes a run of 128
// cells of one row, 4 a lane in 4 coalesced passes; each chunk of a row
// costs one 64-bit division.
constexpr int kPointChunk = 1024;

__device__ __forceinline__ float chain_cell(const LaunchParams& P, float v, int64_t oy, int64_t ox) {
#pragma unroll 1
    for (int i = 0; i < P.nstep; i++) {
        const ChainStep& s = P.step[i];
        if (s.op >= kStepTable) {
            v = table_stage(P.epi[s.op - kStepTable], v);
        } else {
            // input 0 is the launch's own source (its window, in a tile)
            const float* in = s.src == 0 ? P.src : P.in[s.src];
            const int64_t st = s.src == 0 ? P.src_stride : P.in_stride[s.src];
            const float b = s.op <= STRATA_VEC_MAX ? in[oy * st + ox] : 0.0f;
            v = vec_step(s.op, v, b, s.k0, s.k1);
        }
    }
    return v;
}

__global__ void __launch_bounds__(256) pointwise_kernel(const __grid_constant__ LaunchParams P, int64_t chunks_x,
                                                        int64_t chunks) {
    const int64_t w = P.out_x1 - P.out_x0;
    for (int64_t c = blockIdx.x; c < chunks; c += gridDim.x) {
        const int64_t cy = c / chunks_x, cx = c - cy * chunks_x;
        const int64_t gy = P.out_y0 + cy, oy = gy - P.src_y0;
        const int64_t x0 = cx * kPointChunk;
        const float* srow = P.src + oy * P.src_stride;
        float* drow = P.dst0 + (gy - P.dst_y0) * P.dst0_stride;
#pragma unroll
        for (int k = 0; k < kPointChunk / 256; k++) {
            const int64_t x = x0 + k * 256 + threadIdx.x;
            if (x >= w) break;
            const int64_t gx = P.out_x0 + x;
            const float v = srow[gx - P.src_x0];
            drow[gx - P.dst_x0] = P.nstep ? chain_cell(P, v, oy, gx - P.src_x0) : epilogue(P, v);
        }
    }
}

// The finishing pass of Wood's fit (terrain/fit.go:121-170): the raw fit
// sums d0..d4 (p, q, and for curvature r, s, t) at each cell, each scaled
// by its factor (scaleRow), through the product's finisher: the gradient
// itself, the from-gradient finishers Surface uses (SlopeFromGradientRow
// and the rest, the same device functions as Horn's), HeatLoad and
// Orientation's equations, or ZT's curvature formulas. Cells within the
// fit's radius of the border get NaN; the epilogue maps NaN to itself.
__global__ void __launch_bounds__(256) fit_finish_kernel(const __grid_constant__ LaunchParams P,
                                                         const float* __restrict__ d0, const float* __restrict__ d1,
                                                         const float* __restrict__ d2, const float* __restrict__ d3,
                                                         const float* __restrict__ d4, int64_t ds) {
    const int64_t w = P.out_x1 - P.out_x0;
    const int64_t n = w * (P.out_y1 - P.out_y0);
    const int r = P.radius;
    const float nan = nanf32();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t y = i / w, x = i - y * w;
        const int64_t gx = P.out_x0 + x, gy = P.out_y0 + y;
        const int64_t o = (gy - P.dst_y0) * ds + (gx - P.dst_x0);
        float v0 = nan, v1 = nan;
        if (gy >= r && gy < P.height - r && gx >= r && gx < P.width - r) {
            const float p = mul(d0[o], P.k[0]), q = mul(d1[o], P.k[1]);
            switch (P.op) {
            case STRATA_OP_GRADIENT:
                v0 = p;
                v1 = q;
                break;
            case STRATA_OP_SLOPE:
                v0 = P.kind == kSlopeSquareClass ? add(mul(p, p), mul(q, q)) : slope(p, q, P.k[5], P.kind != 0);
                break;
            case STRATA_OP_ASPECT: v0 = aspect(p, q, P.k[5], P.kind != 0); break;
            case STRATA_OP_HILLSHADE: v0 = shade(p, q, P.k[5], P.k[6], P.k[7]); break;
            case STRATA_OP_HEATLOAD: {
                double t[8];
                heat_terms(P.w, t);
                v0 = heat_load(p, q, t, P.kind & 1);
                break;
            }
            case STRATA_OP_ORIENTATION: v0 = orientation(p, q, P.kind & 1, (P.kind >> 1) & 1); break;
            default:  // curvature: r, s and t scaled by kr, ks and kt
                v0 = zt_finish(p, q, mul(d2[o], P.k[2]), mul(d3[o], P.k[4]), mul(d4[o], P.k[3]), P.kind);
                break;
            }
        }
        if (has_tail(P)) v0 = epilogue(P, v0);
        P.dst0[(gy - P.dst_y0) * P.dst0_stride + (gx - P.dst_x0)] = v0;
        if (P.op == STRATA_OP_GRADIENT) P.dst1[(gy - P.dst_y0) * P.dst1_stride + (gx - P.dst_x0)] = v1;
    }
}

}  // namespace

void launch_fit_finish(const LaunchParams& p, float* const d[5], int64_t ds, cudaStream_t s) {
    const int64_t n = (p.out_x1 - p.out_x0) * (p.out_y1 - p.out_y0);
    if (n <= 0) return;
    int64_t blocks = (n + 255) / 256;
    if (blocks > (int64_t)sm_count() * 16) blocks = (int64_t)sm_count() * 16;
    fit_finish_kernel<<<(unsigned)blocks, 256, 0, s>>>(p, d[0], d[1], d[2], d[3], d[4], ds);
}

int64_t launch_data(const LaunchParams& p, cudaStream_t s, int64_t* window_cells) {
    if (p.op == STRATA_OP_LOOKUP || p.op == STRATA_OP_RECLASS || p.op == STRATA_OP_STEP) {
        const int64_t w = p.out_x1 - p.out_x0, h = p.out_y1 - p.out_y0;
        if (w <= 0 || h <= 0) {
            if (window_cells) *window_cells = 0;
            return 0;
        }
        const int64_t chunks_x = (w + kPointChunk - 1) / kPointChunk, chunks = chunks_x * h;
        int64_t blocks = chunks;
        if (blocks > (int64_t)sm_count() * 16) blocks = (int64_t)sm_count() * 16;
        pointwise_kernel<<<(unsigned)blocks, 256, 0, s>>>(p, chunks_x, chunks);
        if (window_cells) *window_cells = w * h * (p.ninputs > 1 ? p.ninputs : 1);
        return blocks;
    }
    if (p.fit || (!(p.op >= STRATA_OP_GRADIENT && p.op <= STRATA_OP_MAX) && p.op != STRATA_OP_HEATLOAD &&
                  p.op != STRATA_OP_ORIENTATION))
        return -1;
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

namespace {

// A host thread's second stream on the current device, with the two
// events that fork it from and join it back to the caller's stream; made
// on first use, released when the thread ends.
struct SideStream {
    cudaStream_t s = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    ~SideStream() {
        if (s) cudaStreamDestroy(s);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
    }
};

SideStream* side_stream() {
    thread_local std::unique_ptr<SideStream> per_device[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    auto& q = per_device[dev];
    if (!q) {
        auto n = std::make_unique<SideStream>();
        if (cudaStreamCreateWithFlags(&n->s, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&n->fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&n->join, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;  // the validity then runs on the caller's stream
        }
        q = std::move(n);
    }
    return q.get();
}

}  // namespace

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
    // The output validity reads only the source mask and writes only the
    // output masks, the data kernel only the cells: on a region large
    // enough for the overlap to outweigh the fork and join, the validity
    // runs on a second stream beside it, forked from and joined back to s.
    const int64_t cells = (p.out_x1 - p.out_x0) * (p.out_y1 - p.out_y0);
    SideStream* side = (v[0] || v[1]) && cells >= ((int64_t)1 << 22) ? side_stream() : nullptr;
    if (side) {
        cudaEventRecord(side->fork, s);
        cudaStreamWaitEvent(side->s, side->fork, 0);
        for (int i = 0; i < 2; i++)
            if (v[i]) launch_validity(*v[i], side->s);
        cudaEventRecord(side->join, side->s);
    }
    const int64_t t = launch_data(p, s, window_cells);
    if (side) cudaStreamWaitEvent(s, side->join, 0);
    else
        for (int i = 0; i < 2; i++)
            if (v[i]) launch_validity(*v[i], s);
    return t;
}


}  // namespace strata
