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

// n (1..32) bits of a mask from bit q on, in the low bits.
__device__ __forceinline__ uint32_t bits_at(const uint32_t* m, int64_t q, int n) {
    const int64_t w = q >> 5;
    const int sh = (int)(q & 31);
    uint32_t v = m[w] >> sh;
    if (sh && sh + n > 32) v |= m[w + 1] << (32 - sh);
    return n == 32 ? v : v & ((1u << n) - 1u);
}

// One thread a 32-bit output word: its bits walk the rows they fall on
// (a row's run, or the row padding and the cells outside [y0, y1) that
// the word keeps), each run ANDed from the inputs' words with one funnel
// shift. No two threads share a word, so the store needs no atomic.
__global__ void __launch_bounds__(256) and_validity_kernel(const __grid_constant__ AndValidityParams v, int64_t w0,
                                                           int64_t nwords) {
    const int64_t S = v.dst_stride;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nwords; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t word = w0 + i;
        const int64_t base = word * 32 - v.dst_off;  // the cell of the word's bit 0
        uint32_t keep = 0, val = 0;
        int b = 0;
        while (b < 32) {
            const int64_t c = base + b;
            int n;
            if (c < 0) {
                n = (int)(-c < 32 - b ? -c : 32 - b);
                keep |= (n == 32 ? ~0u : ((1u << n) - 1u)) << b;
            } else {
                const int64_t y = c / S, x = c - y * S;
                if (y < v.y0 || y >= v.y1 || x >= v.width) {
                    const int64_t run = S - x;
                    n = (int)(run < 32 - b ? run : 32 - b);
                    keep |= (n == 32 ? ~0u : ((1u << n) - 1u)) << b;
                } else {
                    const int64_t run = v.width - x;
                    n = (int)(run < 32 - b ? run : 32 - b);
                    uint32_t ok = n == 32 ? ~0u : ((1u << n) - 1u);
                    for (int k = 0; k < v.nsrc; k++)
                        if (v.src_bits[k]) ok &= bits_at(v.src_bits[k], v.src_off[k] + y * v.src_stride[k] + x, n);
                    val |= ok << b;
                }
            }
            b += n;
        }
        uint32_t* d = v.dst_bits + word;
        *d = keep ? (*d & keep) | val : val;
    }
}

}  // namespace

void launch_and_validity(const AndValidityParams& v, cudaStream_t s) {
    if (!v.dst_bits || v.y1 <= v.y0 || v.width <= 0) return;
    const int64_t first = v.dst_off + v.y0 * v.dst_stride;
    const int64_t last = v.dst_off + (v.y1 - 1) * v.dst_stride + v.width - 1;
    const int64_t w0 = first >> 5, nwords = (last >> 5) - w0 + 1;
    int64_t blocks = (nwords + 255) / 256;
    if (blocks > (int64_t)sm_count() * 16) blocks = (int64_t)sm_count() * 16;
    and_validity_kernel<<<(unsigned)blocks, 256, 0, s>>>(v, w0, nwords);
}

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
