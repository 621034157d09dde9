// batch.cu - many rasters of mixed sizes and ops in one CUDA-graph launch.
//
// A batch groups its rasters by op class (op, radius, and the kind and
// epilogue where the kernel is specialised on them). Each class runs one
// persistent kernel whose blocks walk the work units of every raster of
// the class, gridDim apart, so a class of many small rasters costs one
// launch rather than one per raster; the classes' kernels sit side by
// side in one captured graph that replays with one launch. A unit has the
// shape of the single-raster kernels' blocks, and the block runs the same
// body on it, so every cell has the same bits:
//   * radius-1 ops: 512 columns (a warp's march down 128 of them) by a band
//     of rows (march.cuh);
//   * separable ops and roughness at radius 2..8: a band of 512 column
//     results (focal.cuh, in batch_focal.cu);
//   * correlation and the other ruggedness kinds at radius 2..8: a tile of
//     128 columns (focal.cuh, in batch_focal.cu).
// Each raster keeps its own descriptor (the block stages it in shared
// memory when it reaches the raster's units) and its own band height (the
// autotuner's choice for its class). Radius-1 march units of at most 64
// rows write their outputs' validity themselves after their cells, from
// mask words copied to shared memory during the march (march_tma.cuh, as
// the single-raster march does); the other masked outputs' validity runs in
// persistent kernels of its own, one per radius, a warp a unit of 1024
// cells by a band of rows (validity.cuh).
#include <algorithm>
#include <cstring>

#include "batch.cuh"
#include "launch.h"
#include "march.cuh"
#include "march_tma.cuh"
#include "validity.cuh"

namespace strata {

// Launchers of the classes whose kernels batch_focal.cu holds.
bool launch_batch_focal(const BatchClass& c, const BatchItem* d_items, cudaStream_t s);
// Unit width and height of the focal families for radius r (band: the
// requested rows, 0 for the default).
void batch_focal_shape(int op, int radius, int kind, int band, int* tw, int* th);

namespace {

// Five blocks per SM: 96 registers a thread, which every class fits without
// spilling (at six, 80, the Horn and curvature classes spill).
template <int OP, int KIND, bool EPI>
__global__ void __launch_bounds__(kBatchThreads, 5) batch_march_kernel(const BatchItem* __restrict__ items, int n,
                                                                    int64_t total) {
    __shared__ __align__(16) LaunchParams P;
    __shared__ uint32_t vwords[kWarps][kVMaxRows * kVWords];
    EpiTables* T = EpiSmem<EPI>::get();
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    int cur = -1;
    for (int64_t u = blockIdx.x; u < total; u += gridDim.x) {
        const int it = batch_item_of(items, n, u);
        if (it != cur) {  // the same for the whole block
            __syncthreads();
            batch_stage_params(items[it], P);
            __syncthreads();
            if constexpr (EPI) {
                stage_epilogue(P, *T);
                __syncthreads();
            }
            cur = it;
        }
        const BatchUnit b = batch_unit(items[it], P, u);
        const int64_t xs = b.x + 128 * warp;
        if (xs < P.out_x1) {
            // Units of at most kMaxStrip rows write their outputs' validity
            // beside their cells (batch_plan sets P.vf for them), from the
            // source words copied to shared memory while the warp marches.
            const bool vfused = P.vf.n > 0;
            if (vfused) valid_prefetch(P, xs, b.y0, b.rows, vwords[warp], lane);
            march_warp<OP, KIND, EPI>(P, T, xs, b.y0, b.rows, b.vec);
            if (vfused) {
                valid_wait(P);
                valid_strip(P, xs, b.y0, b.rows, vwords[warp], lane);
                __syncwarp();  // every lane has read the words before the next unit's copies
            }
        }
    }
}

constexpr int kValidityWarps = 8;

template <int R>
__global__ void __launch_bounds__(32 * kValidityWarps) batch_validity_kernel(const ValidityItem* __restrict__ items,
                                                                             int n, int64_t total) {
    const int64_t warps = (int64_t)gridDim.x * kValidityWarps;
    for (int64_t u = (int64_t)blockIdx.x * kValidityWarps + (threadIdx.x >> 5); u < total; u += warps) {
        int lo = 0, hi = n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (items[mid].unit0 <= u) lo = mid;
            else hi = mid - 1;
        }
        const ValidityItem& I = items[lo];
        const int64_t t = u - I.unit0;
        const int64_t band = t / I.strips, strip = t - band * I.strips;
        const int64_t y0 = I.v.out_y0 + band * I.band;
        const int64_t r = I.v.out_y1 - y0;
        validity_strip<R>(I.v, I.v.out_x0 + strip * kStripCells, y0, r < I.band ? (int)r : I.band);
    }
}

// Blocks that fill the GPU once at the kernel's occupancy (per_sm, looked
// up once per kernel by its launcher), never more than the units.
int persistent_grid(int per_sm, int64_t total) {
    const int64_t g = (int64_t)sm_count() * per_sm;
    return (int)(total < g ? total : g);
}

template <class K>
int occupancy(K kernel, int threads) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, 0) != cudaSuccess || n < 1) n = 1;
    return n;
}

template <int OP, int KIND, bool EPI>
bool launch_march_class(const BatchClass& c, const BatchItem* d, cudaStream_t s) {
    static const int per_sm = occupancy(batch_march_kernel<OP, KIND, EPI>, kBatchThreads);
    batch_march_kernel<OP, KIND, EPI><<<persistent_grid(per_sm, c.total), kBatchThreads, 0, s>>>(
        d + c.first, c.count, c.total);
    return true;
}

template <int OP, int KIND>
bool launch_march_epi(const BatchClass& c, const BatchItem* d, cudaStream_t s) {
    return c.epi ? launch_march_class<OP, KIND, true>(c, d, s) : launch_march_class<OP, KIND, false>(c, d, s);
}

template <int R>
void launch_validity_class(const ValidityClass& c, const ValidityItem* d, cudaStream_t s) {
    static const int per_sm = occupancy(batch_validity_kernel<R>, 32 * kValidityWarps);
    batch_validity_kernel<R><<<persistent_grid(per_sm, (c.total + kValidityWarps - 1) / kValidityWarps),
                               32 * kValidityWarps, 0, s>>>(d + c.first, c.count, c.total);
}

// The class of an item: its family (0 march, 1 separable, 2 windowed),
// and the kind and epilogue flag its kernel is specialised on.
struct Key {
    int family, op, radius, kind, epi;
    bool operator<(const Key& o) const {
        if (family != o.family) return family < o.family;
        if (op != o.op) return op < o.op;
        if (radius != o.radius) return radius < o.radius;
        if (kind != o.kind) return kind < o.kind;
        return epi < o.epi;
    }
    bool operator==(const Key& o) const {
        return family == o.family && op == o.op && radius == o.radius && kind == o.kind && epi == o.epi;
    }
};

Key key_of(const LaunchParams& p) {
    Key k{0, p.op, p.radius, 0, 0};
    if (p.radius <= 1) {
        k.radius = 1;
        if (p.op == STRATA_OP_SLOPE || p.op == STRATA_OP_ASPECT) k.kind = p.kind;
        if (p.op == STRATA_OP_CURVATURE || p.op == STRATA_OP_RUGGEDNESS) k.kind = p.kind;
        k.epi = has_tail(p);
    } else if (p.op == STRATA_OP_CORRELATE || (p.op == STRATA_OP_RUGGEDNESS && p.kind != STRATA_RUG_ROUGHNESS)) {
        k.family = 2;
        k.kind = p.op == STRATA_OP_RUGGEDNESS ? p.kind : 0;
    } else {
        k.family = 1;
        k.kind = p.op == STRATA_OP_RUGGEDNESS ? p.kind : 0;
    }
    return k;
}

}  // namespace

int batch_plan(BatchItem* items, int n, int* order, BatchClass* cls, int64_t* window_cells) {
    // Each item's unit shape.
    int64_t window = 0;
    for (int i = 0; i < n; i++) {
        BatchItem& b = items[i];
        const LaunchParams& p = b.p;
        if (p.radius < 1 && !(p.op >= STRATA_OP_GRADIENT && p.op <= STRATA_OP_CURVATURE)) return -1;
        const Key k = key_of(p);
        if (k.family == 0) {
            b.tw = 512;
            b.th = b.th > 0 ? b.th : 32;
            // A march unit of at most kMaxStrip rows writes its outputs'
            // validity itself (the kernel's P.vf); batch_plan_validity then
            // leaves the item out.
            memset(&b.p.vf, 0, sizeof b.p.vf);
            bool fuse = b.th <= kMaxStrip && b.nvalid > 0;
            for (int v = 0; v < b.nvalid && fuse; v++)
                fuse = b.v[v].radius == 1 && b.v[v].src_x0 == p.src_x0 && b.v[v].src_y0 == p.src_y0 &&
                       b.v[v].dst_x0 == p.dst_x0 && b.v[v].dst_y0 == p.dst_y0 && b.v[v].out_x0 == p.out_x0 &&
                       b.v[v].out_x1 == p.out_x1 && b.v[v].width == p.width && b.v[v].height == p.height &&
                       b.v[v].src_bits == b.v[0].src_bits && b.v[v].src_off == b.v[0].src_off &&
                       b.v[v].src_stride == b.v[0].src_stride;
            if (fuse) {
                FusedValidity& f = b.p.vf;
                f.src_bits = b.v[0].src_bits;
                f.src_off = b.v[0].src_off;
                f.src_stride = b.v[0].src_stride;
                f.src_lo_word = b.v[0].src_lo_word;
                f.src_hi_word = b.v[0].src_hi_word;
                for (int v = 0; v < b.nvalid; v++) {
                    f.dst_bits[v] = b.v[v].dst_bits;
                    f.dst_off[v] = b.v[v].dst_off;
                    f.dst_stride[v] = b.v[v].dst_stride;
                }
                f.n = b.nvalid;
            }
        } else {
            batch_focal_shape(p.op, p.radius, p.kind, b.th, &b.tw, &b.th);
        }
        const int64_t w = p.out_x1 - p.out_x0, h = p.out_y1 - p.out_y0;
        b.tiles_x = (w + b.tw - 1) / b.tw;
        const int r = k.radius;
        window += b.tiles_x * ((h + b.th - 1) / b.th) * (int64_t)(b.tw + 2 * r) * (b.th + 2 * r);
    }
    if (window_cells) *window_cells = window;
    // Stable insertion sort of the indices by class, then the items
    // permuted into that order in place, cycle by cycle.
    for (int i = 0; i < n; i++) {
        const Key ki = key_of(items[i].p);
        int j = i;
        for (; j > 0 && ki < key_of(items[order[j - 1]].p); j--) order[j] = order[j - 1];
        order[j] = i;
    }
    for (int i = 0; i < n; i++) {
        if (order[i] < 0) continue;
        BatchItem t = items[i];
        int j = i;
        while (order[j] != i) {
            const int k = order[j];
            items[j] = items[k];
            order[j] = -1;
            j = k;
        }
        items[j] = t;
        order[j] = -1;
    }
    int nc = 0;
    for (int i = 0; i < n;) {
        const Key k = key_of(items[i].p);
        BatchClass& c = cls[nc++];
        c.op = k.op;
        c.radius = k.radius;
        c.kind = k.kind;
        c.epi = k.epi;
        c.first = i;
        c.count = 0;
        c.total = 0;
        for (; i < n && key_of(items[i].p) == k; i++) {
            BatchItem& b = items[i];
            b.tile0 = c.total;
            c.total += b.tiles_x * ((b.p.out_y1 - b.p.out_y0 + b.th - 1) / b.th);
            c.count++;
        }
    }
    return nc;
}

int batch_plan_validity(const BatchItem* items, int n, ValidityItem* vitems, ValidityClass* vcls, int* nvcls) {
    constexpr int kBand = 32;
    int nv = 0, nc = 0;
    for (int r = 0; r <= STRATA_MAX_RADIUS; r++) {
        ValidityClass c{r, nv, 0, 0};
        for (int i = 0; i < n; i++)
            for (int k = 0; k < items[i].nvalid; k++) {
                if (items[i].p.vf.n > 0) continue;  // the march units write it
                const ValidityParams& v = items[i].v[k];
                if (v.radius != r || v.dst_words <= 0 || v.out_x1 <= v.out_x0 || v.out_y1 <= v.out_y0) continue;
                ValidityItem& it = vitems[nv++];
                memset(&it, 0, sizeof it);
                it.v = v;
                it.band = kBand;
                it.strips = (v.out_x1 - v.out_x0 + kStripCells - 1) / kStripCells;
                it.unit0 = c.total;
                c.total += it.strips * ((v.out_y1 - v.out_y0 + kBand - 1) / kBand);
                c.count++;
            }
        if (c.count) vcls[nc++] = c;
    }
    *nvcls = nc;
    return nv;
}

bool launch_batch_class(const BatchClass& c, const BatchItem* d, cudaStream_t s) {
    if (c.radius > 1 || c.op == STRATA_OP_LOOKUP || c.op == STRATA_OP_RECLASS) return launch_batch_focal(c, d, s);
    switch (c.op) {
    case STRATA_OP_GRADIENT: return launch_march_class<STRATA_OP_GRADIENT, 0, false>(c, d, s);
    case STRATA_OP_SLOPE:
        if (c.kind == kSlopeSquareClass) return launch_march_class<STRATA_OP_SLOPE, kSlopeSquareClass, false>(c, d, s);
        return c.kind ? launch_march_epi<STRATA_OP_SLOPE, 1>(c, d, s) : launch_march_epi<STRATA_OP_SLOPE, 0>(c, d, s);
    case STRATA_OP_ASPECT:
        return c.kind ? launch_march_epi<STRATA_OP_ASPECT, 1>(c, d, s) : launch_march_epi<STRATA_OP_ASPECT, 0>(c, d, s);
    case STRATA_OP_HILLSHADE: return launch_march_epi<STRATA_OP_HILLSHADE, 0>(c, d, s);
    case STRATA_OP_HEATLOAD: return launch_march_epi<STRATA_OP_HEATLOAD, 0>(c, d, s);
    case STRATA_OP_ORIENTATION: return launch_march_epi<STRATA_OP_ORIENTATION, 0>(c, d, s);
    case STRATA_OP_CURVATURE:
        switch (c.kind) {
        case 0: return launch_march_epi<STRATA_OP_CURVATURE, 0>(c, d, s);
        case 1: return launch_march_epi<STRATA_OP_CURVATURE, 1>(c, d, s);
        case 2: return launch_march_epi<STRATA_OP_CURVATURE, 2>(c, d, s);
        }
        return false;
    case STRATA_OP_RUGGEDNESS:
        switch (c.kind) {
        case STRATA_RUG_TRI_RILEY: return launch_march_epi<STRATA_OP_RUGGEDNESS, kKindAtRun>(c, d, s);
        case STRATA_RUG_TRI_WILSON: return launch_march_epi<STRATA_OP_RUGGEDNESS, STRATA_RUG_TRI_WILSON>(c, d, s);
        case STRATA_RUG_TPI: return launch_march_epi<STRATA_OP_RUGGEDNESS, STRATA_RUG_TPI>(c, d, s);
        case STRATA_RUG_ROUGHNESS: return launch_march_epi<STRATA_OP_RUGGEDNESS, STRATA_RUG_ROUGHNESS>(c, d, s);
        }
        return false;
    case STRATA_OP_CORRELATE: return launch_march_epi<STRATA_OP_CORRELATE, 0>(c, d, s);
    case STRATA_OP_SEPARABLE: return launch_march_epi<STRATA_OP_SEPARABLE, 0>(c, d, s);
    case STRATA_OP_MEAN: return launch_march_epi<STRATA_OP_MEAN, 0>(c, d, s);
    case STRATA_OP_MIN: return launch_march_epi<STRATA_OP_MIN, 0>(c, d, s);
    case STRATA_OP_MAX: return launch_march_epi<STRATA_OP_MAX, 0>(c, d, s);
    }
    return false;
}

void launch_batch_validity(const ValidityClass& c, const ValidityItem* d, cudaStream_t s) {
    switch (c.radius) {
    case 0: launch_validity_class<0>(c, d, s); break;
    case 1: launch_validity_class<1>(c, d, s); break;
    case 2: launch_validity_class<2>(c, d, s); break;
    case 3: launch_validity_class<3>(c, d, s); break;
    case 4: launch_validity_class<4>(c, d, s); break;
    case 5: launch_validity_class<5>(c, d, s); break;
    case 6: launch_validity_class<6>(c, d, s); break;
    case 7: launch_validity_class<7>(c, d, s); break;
    case 8: launch_validity_class<8>(c, d, s); break;
    }
}

}  // namespace strata
