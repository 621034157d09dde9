// launch.h - what the host driver (api.cu) hands the kernels (kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "strata_cuda.h"

namespace strata {

constexpr int kMaxEpilogue = 4;  // pointwise stages fused after a stencil
// Breaks of a lone Reclass epilogue that the kernels take as a chain of
// compares (ops3.cuh reclass_chain4) rather than a table search.
constexpr int kChainBreaks = 8;
// LaunchParams.kind of a Slope whose Reclass epilogue the host has moved
// onto the squared gradient magnitude (api.cu fold_slope_square): the
// kernel classifies gx*gx + gy*gy against epi[0]'s thresholds and takes no
// square root, arctangent or scale.
constexpr int kSlopeSquareClass = 2;

// The multiprocessor count of the current device, looked up once per
// device (launch shapes are sized in multiples of it).
inline int sm_count() {
    static int cache[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!cache[dev]) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 1;
        cache[dev] = n;
    }
    return cache[dev];
}
constexpr int kMaxWeights = (2 * STRATA_MAX_RADIUS + 1) * (2 * STRATA_MAX_RADIUS + 1);

// One pointwise stage fused as an epilogue: LOOKUP (a = xs, b = ys, n
// knots) or RECLASS (a = breaks, n breaks, b = values, n + 1 of them).
struct EpiStage {
    int op;
    int n;
    float a[STRATA_MAX_KNOTS];
    float b[STRATA_MAX_KNOTS + 1];
};

// One step of a pointwise tail written as a sequence (LaunchParams.nstep
// > 0): op is a STRATA_VEC_* (a vec.Chain step, internal/vec/chain.go:
// 24-38), or kStepTable + i to run table stage epi[i]; src is the input a
// binary op reads; k0, k1 the immediates.
constexpr int kStepTable = 32;
struct ChainStep {
    int op;
    int src;
    float k0, k1;
};

// The output validity a radius-1 march writes beside its cells (n > 0):
// the source mask (null: every source cell valid), whose cell (src_x0,
// src_y0) of the launch is bit src_off, and each output's mask (null: the
// output is unmasked), whose cell (dst_x0, dst_y0) is bit dst_off[i].
struct FusedValidity {
    const uint32_t* src_bits;
    int64_t src_off, src_stride;
    int64_t src_lo_word, src_hi_word;  // 32-bit words that hold the source's bits
    uint32_t* dst_bits[2];
    int64_t dst_off[2], dst_stride[2];
    int n;
    int pad_;
};

// Kernel parameters of one stage launch. Passed by value as a
// __grid_constant__ parameter, so weights and tables sit in the constant
// bank and every thread reads them through the broadcast path.
//
// Coordinates are the whole raster's: width x height decides the edge
// ring. src holds the cells [src_x0, src_x0 + src_w) x [src_y0, src_y0 +
// src_h) and dst0 / dst1 start at cell (dst_x0, dst_y0); the launch writes
// the output region [out_x0, out_x1) x [out_y0, out_y1). A plain call has
// every offset 0 and the region the whole raster; a chunked tile or a row
// strip sets them.
struct alignas(16) LaunchParams {
    const float* src;
    int64_t src_stride;
    int64_t src_x0, src_y0, src_w, src_h;
    float* dst0;
    int64_t dst0_stride;
    float* dst1;
    int64_t dst1_stride;
    int64_t dst_x0, dst_y0;
    int64_t out_x0, out_y0, out_x1, out_y1;
    int64_t width, height;
    int64_t tiles_x;  // thread-block tiles across the region (set by the launcher)
    int64_t tiles;    // thread-block tiles in the launch (set by the launcher)
    int* status;  // device word a kernel sets to a STRATA_E* code (a bounded wait that ran out)
    int op;
    int radius;
    int kind;
    int nepi;
    // Non-zero only in the failure-path test (the environment variable
    // STRATA_TEST_STALL_FIRST_WAIT=1): the TMA march's first wait is on a
    // barrier nothing arrives at, with a short bound, so it runs out.
    int test_stall;
    int fit;  // the radius of Wood's fit when the derivatives come from it (a STRATA_STAGE_FIT stage), else 0
    float k[16];
    float w[kMaxWeights];  // CORRELATE weights (rotation applied); SEPARABLE row taps w[0..], column taps w[17..];
                           // HEATLOAD the regression's eight float64 terms, bit for bit, in w[0..16)
    EpiStage epi[kMaxEpilogue];
    FusedValidity vf;  // set by launch_stage when the march writes the outputs' validity
    // The pointwise tail as a sequence, when it holds a chain step: then
    // step[0..nstep) runs in order (the table stages by reference) and
    // nepi only counts the tables; 0: the tail is epi[0..nepi) in order.
    int nstep;
    int ninputs;  // the sources a pointwise chain reads: in[0] is src
    ChainStep step[STRATA_MAX_STEPS];
    const float* in[STRATA_MAX_INPUTS];  // cell (src_x0, src_y0) of each input
    int64_t in_stride[STRATA_MAX_INPUTS];
};

// A pointwise tail to run after the stencil (tables or chain steps).
__host__ __device__ inline bool has_tail(const LaunchParams& p) { return p.nepi > 0 || p.nstep > 0; }

// The fused multi-output pass (features.cu): several radius-1 ops over one
// source in one march, terrain.Features / terrain.Surface's outputs from
// one read of the DEM and one set of Horn differences. Each kind of
// feature it takes has a slot of its own, so the kernel reads every
// parameter at a fixed place.
enum { kFGradient, kFSlopeClass, kFSlopePercent, kFWilson, kFTpi, kFRoughness, kFSlots };
struct FeatureSlot {
    int on;     // the slot holds a feature
    int nb;     // breaks of its Reclass epilogue (0: none)
    float k[5];  // the op's constants, as LaunchParams.k
    float t[kChainBreaks];      // the breaks (a squared magnitude's thresholds for the classified Slope)
    float v[kChainBreaks + 1];  // the class values
    float* data[2];       // its outputs (two for a gradient)
    int64_t stride[2];
    uint32_t* bits[2];    // null: unmasked
    int64_t bit_off[2], bit_stride[2];
};
struct alignas(16) FeaturesParams {
    LaunchParams g;  // the source, region and status word; g.vf: the source mask (op, constants unused)
    FeatureSlot f[kFSlots];
    int horn;    // some feature takes Horn's differences
    int window;  // some feature takes the 3x3 window (ruggedness)
    int masked;  // some output is masked
    int pad_;
};
// The slot of a planned stage in the fused pass, or -1 when it does not
// run there: only the features whose own kernel is bound by memory
// (Gradient, Slope in percent or classified on its squared magnitude,
// Wilson's TRI, TPI and roughness at radius 1), with at most one Reclass
// of kChainBreaks breaks after it, on rows the TMA march takes.
int feature_slot(const LaunchParams& p);
// Launches the fused pass; returns the blocks launched (-1: no kernel) and
// sets *window_cells to the cells they read.
int64_t launch_features(const FeaturesParams& p, cudaStream_t stream, int64_t* window_cells);

// Validity of one output: bits of dst for the width x height raster,
// derived from src's bits (src_valid may be null: every input cell valid)
// by erosion over the radius, with the edge ring cleared; radius 0 copies.
// Coordinates as in LaunchParams: the source mask's cell (0, 0) is global
// cell (src_x0, src_y0), the destination's is (dst_x0, dst_y0), and only
// bits of cells in the region [out_x0, out_x1) x [out_y0, out_y1) change.
struct alignas(16) ValidityParams {
    const uint32_t* src_bits;  // the source mask as 32-bit words
    int64_t src_off;           // bit offset of the source's cell (0, 0)
    int64_t src_stride;
    int64_t src_x0, src_y0;
    int64_t src_lo_word, src_hi_word;  // 32-bit words [lo, hi] that hold the source's bits
    uint32_t* dst_bits;
    int64_t dst_off;
    int64_t dst_stride;
    int64_t dst_x0, dst_y0;
    int64_t dst_lo_word;  // first 32-bit word holding a destination bit of the region
    int64_t dst_words;    // 32-bit words from dst_lo_word
    int64_t out_x0, out_y0, out_x1, out_y1;
    int64_t width, height;
    int radius;
};

// One raster of a batch (batch.cu): its launch parameters, the validity
// of its masked outputs, and its work units: tiles of tw x th output cells,
// tiles_x across, numbered from tile0 among its class's.
struct alignas(16) BatchItem {
    LaunchParams p;
    ValidityParams v[2];
    int64_t tile0;
    int64_t tiles_x;
    int tw, th;  // th: the requested band (rows a unit) before planning, 0 for the default
    int nvalid;  // masked outputs: v[0 .. nvalid)
    int vec;     // 1: the rows of src and dst start on 16-byte boundaries where units load and store
};

// One masked output of a batch raster: its units are warp strips of 1024
// cells across and band rows, numbered from unit0 among its class's.
struct alignas(16) ValidityItem {
    ValidityParams v;
    int64_t unit0;
    int64_t strips;
    int band;
    int pad;
};

// A class of batch rasters, run by one persistent kernel: the items
// [first, first + count) of the planned table, total work units.
struct BatchClass {
    int op, radius, kind, epi;  // the kernel's specialisation
    int first, count;
    int64_t total;
};

// A class of batch validity items (one radius).
struct ValidityClass {
    int radius;
    int first, count;
    int64_t total;
};

// Plans a batch in place (host): orders items[0 .. n) into classes (stable
// within a class), sets each item's unit geometry (tw, tiles_x, th from
// the requested band) and numbering, and writes the classes to cls
// (capacity n). order: n ints of scratch. Returns the number of classes,
// or -1 if an item has no batch kernel. *window_cells (if given) gets the
// input cells the units read.
int batch_plan(BatchItem* items, int n, int* order, BatchClass* cls, int64_t* window_cells);
// The validity items of planned items (at most 2n, into vitems) grouped by
// radius into vcls (capacity 9); returns the number of validity items and
// sets *nvcls.
int batch_plan_validity(const BatchItem* items, int n, ValidityItem* vitems, ValidityClass* vcls, int* nvcls);
// Launches a class's persistent kernel over its items (device memory) on
// stream; false if the class has no kernel.
bool launch_batch_class(const BatchClass& c, const BatchItem* d_items, cudaStream_t stream);
void launch_batch_validity(const ValidityClass& c, const ValidityItem* d_vitems, cudaStream_t stream);

// Launches the data kernel of stages (the first any op, the rest pointwise
// epilogues) over whole rasters. Returns the number of thread-block tiles
// launched, or -1 if the op / radius has no kernel; *window_cells gets the
// input cells the tiles read (halo included, clipped to the raster).
int64_t launch_data(const LaunchParams& p, cudaStream_t stream, int64_t* window_cells);

// The finishing pass of a Wood's-fit stage (kernels.cu): p's product
// (p.op, p.kind, p.k[5..], p.w for heat load) from the raw fit sums d[0..1]
// (p, q) and, for curvature, d[2..4] (r, s, t) over the region (rasters
// with dst0's geometry and stride ds), each scaled by its factor p.k[0..4],
// then p's pointwise epilogue; cells within p.radius of the border get NaN.
void launch_fit_finish(const LaunchParams& p, float* const d[5], int64_t ds, cudaStream_t stream);

// Launches the validity kernel for one output.
void launch_validity(const ValidityParams& v, cudaStream_t stream);

// The validity of a pointwise pipeline over several inputs
// (pointwise.BinaryValidity, and halo.go:213-229 at reach 0): bit (x, y)
// of the output, for rows [y0, y1), is the AND of every masked input's bit
// (x, y); an unmasked input counts as valid. The output's other bits are
// kept. Input i's cell (0, 0) is bit src_off[i] of src_bits[i] (null:
// unmasked).
struct AndValidityParams {
    const uint32_t* src_bits[STRATA_MAX_INPUTS];
    int64_t src_off[STRATA_MAX_INPUTS];
    int64_t src_stride[STRATA_MAX_INPUTS];
    int nsrc;
    uint32_t* dst_bits;
    int64_t dst_off, dst_stride;
    int64_t width, y0, y1;
};
void launch_and_validity(const AndValidityParams& v, cudaStream_t stream);

// A raw file's fill value as validity (raw.cu): bits[k] holds the
// validity of cells [32k, 32k + 32) of the run cells[0, n) (a cell equal
// to fill, or any NaN for a NaN fill, is invalid; bits past n are 0); and
// fill stored under the invalid cells of a w x h tile whose cell (x, y) is
// data[y * stride + x] with its bit at the same index of bits.
void launch_fill_bits(const float* cells, int64_t n, float fill, uint32_t* bits, cudaStream_t stream);
void launch_fill_invalid(float* data, int64_t stride, int64_t w, int64_t h, const uint32_t* bits, float fill,
                         cudaStream_t stream);

// Launches a stage and the validity of its masked outputs (v[i] for output
// i, null when output i is unmasked). The radius-1 march on 16-byte aligned
// rows writes the validity itself when every v[i] describes the launch's
// own region and coordinates; otherwise the validity kernel runs after the
// data kernel. Returns launch_data's count (-1: no kernel).
int64_t launch_stage(LaunchParams p, const ValidityParams* const v[2], cudaStream_t stream, int64_t* window_cells);

// The radius-1 marching kernel (march3.cu): whether it can run these
// parameters (16-byte aligned rows at the region's first column, width a
// multiple of 4), and its launcher.
bool march3_eligible(const LaunchParams& p);
int64_t launch_march3(const LaunchParams& p, cudaStream_t stream);
// The same march for any alignment and stride, with per-cell loads and
// stores (march3.cu march_any_kernel).
bool march_any_eligible(const LaunchParams& p);
int64_t launch_march_any(const LaunchParams& p, cudaStream_t stream);
// The register-blocked focal kernels (focal.cu) for the windowed ops at
// radius 2..8 (vector loads and stores where rows are 16-byte aligned,
// per-cell ones otherwise); launch_focal returns the blocks launched and
// sets *window_cells (if given) to the cells they read.
bool focal_eligible(const LaunchParams& p);
int64_t launch_focal(const LaunchParams& p, cudaStream_t stream, int64_t* window_cells);


}  // namespace strata
