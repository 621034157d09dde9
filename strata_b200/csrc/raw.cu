// raw.cu - the fill value of a raw float32 file as validity, on the device
// (engine/raw.go:130-147 with vec.ValidBits, internal/vec/validity.go:
// 20-76; and fillInvalid, engine/raw.go:245-275).
//
// fill_bits: the validity of a run of cells against the file's fill value,
// a warp's 32 cells to one 32-bit word through a ballot; a cell is invalid
// when it equals the fill (by ==, so -0 matches 0), or, for a NaN fill,
// when it is any NaN. fill_invalid: the fill value stored under the
// invalid cells of a tile before it is written out.
#include <cuda_runtime.h>

#include "launch.h"

namespace strata {
namespace {

constexpr int kRawThreads = 256;

__global__ void __launch_bounds__(kRawThreads) fill_bits_kernel(const float* __restrict__ cells, int64_t n, float fill,
                                                                 uint32_t* __restrict__ bits, int64_t nwords) {
    const bool nan_fill = fill != fill;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (kRawThreads / 32);
    for (int64_t w = blockIdx.x * (int64_t)(kRawThreads / 32) + (threadIdx.x >> 5); w < nwords; w += warps) {
        const int64_t i = w * 32 + lane;
        bool valid = false;
        if (i < n) {
            const float v = cells[i];
            valid = nan_fill ? v == v : !(v == fill);
        }
        const uint32_t word = __ballot_sync(0xffffffffu, valid);
        if (lane == 0) bits[w] = word;
    }
}

__global__ void __launch_bounds__(kRawThreads) fill_invalid_kernel(float* __restrict__ data, int64_t stride, int64_t w,
                                                                    int64_t h, const uint32_t* __restrict__ bits,
                                                                    float fill) {
    const int64_t n = w * h;
    for (int64_t i = blockIdx.x * (int64_t)kRawThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kRawThreads) {
        const int64_t y = i / w, x = i - y * w;
        const int64_t c = y * stride + x;
        if (!((bits[c >> 5] >> (c & 31)) & 1u)) data[c] = fill;
    }
}

int64_t grid_for(int64_t units) {
    int64_t blocks = (units + kRawThreads - 1) / kRawThreads;
    const int64_t cap = (int64_t)sm_count() * 16;
    return blocks < 1 ? 1 : (blocks > cap ? cap : blocks);
}

}  // namespace

void launch_fill_bits(const float* cells, int64_t n, float fill, uint32_t* bits, cudaStream_t s) {
    const int64_t nwords = (n + 31) / 32;
    if (nwords <= 0) return;
    fill_bits_kernel<<<(unsigned)grid_for(nwords * 32), kRawThreads, 0, s>>>(cells, n, fill, bits, nwords);
}

void launch_fill_invalid(float* data, int64_t stride, int64_t w, int64_t h, const uint32_t* bits, float fill,
                         cudaStream_t s) {
    if (w <= 0 || h <= 0) return;
    fill_invalid_kernel<<<(unsigned)grid_for(w * h), kRawThreads, 0, s>>>(data, stride, w, h, bits, fill);
}

}  // namespace strata
