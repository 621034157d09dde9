/*
 * strata_cuda.h - C ABI of libstrata_cuda, the B200 (sm_100a) backend for
 * strata's raster-stencil path.
 *
 * Every entry point is plain C: pointers, sizes and status codes, no C++
 * types and no exceptions across the boundary. A Go cgo shim, a ctypes
 * binding or a C program binds it the same way.
 *
 * The path it replaces, in the strata sources:
 *   - internal/exec/process.go:28-35   exec.ProcessN        -> strata_process
 *   - internal/exec/chunked.go:33-40   exec.ProcessChunked  -> strata_process_chunked
 *   - internal/exec/pipeline.go:187    exec.NewPipeline (a stencil stage
 *                                      followed by pointwise stages)
 *                                      -> strata_process with nstages > 1
 *   - the kernels the terrain, focal and transfer packages build
 *     (terrain/slope.go:76-82, aspect.go, hillshade.go, gradient.go,
 *     curvature.go, ruggedness.go; focal/correlate.go:72-88,
 *     separable.go:78-89, box.go:77-80; transfer/transfer.go:184-223)
 *                                      -> the strata_stage_* builders
 *
 * Status codes: STRATA_OK (0) or a negative STRATA_E* value. The message
 * of the last failure on the calling thread is strata_last_error().
 * Argument errors that the reference reports with a panic return
 * STRATA_EINVAL with the reference's message text and prefix ("terrain:",
 * "focal:", "transfer.Lookup:", "engine:").
 */
#ifndef STRATA_CUDA_H
#define STRATA_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define STRATA_ABI_VERSION 2

/* Status codes. */
#define STRATA_OK 0
#define STRATA_EINVAL (-1)    /* an argument the reference panics on */
#define STRATA_ECUDA (-2)     /* a CUDA runtime or launch error */
#define STRATA_ENOMEM (-3)    /* device or pinned host memory exhausted */
#define STRATA_ECANCELED (-4) /* the cancel flag was set; see strata_exec_opts */
#define STRATA_ETIMEDOUT (-5) /* a bounded device-side wait ran out */
#define STRATA_EIO (-6)       /* a source or sink callback failed */
#define STRATA_ENOTSUP (-8)   /* valid for the reference, not on this backend (the caller falls back to the CPU) */

/* Ops: the kernels of the terrain, focal and transfer packages. */
enum {
    STRATA_OP_GRADIENT = 1,   /* terrain.Gradient: 2 outputs (dx, dy), radius 1 */
    STRATA_OP_SLOPE = 2,      /* terrain.Slope, radius 1 */
    STRATA_OP_ASPECT = 3,     /* terrain.Aspect, radius 1 */
    STRATA_OP_HILLSHADE = 4,  /* terrain.Hillshade, radius 1 */
    STRATA_OP_CURVATURE = 5,  /* terrain.Curvature (Zevenbergen-Thorne), radius 1 */
    STRATA_OP_RUGGEDNESS = 6, /* terrain.Ruggedness, radius 1..8 */
    STRATA_OP_CORRELATE = 7,  /* focal.Correlate / Convolve, radius 1..8 */
    STRATA_OP_SEPARABLE = 8,  /* focal.CorrelateSeparable, radius 1..8 */
    STRATA_OP_MEAN = 9,       /* focal.Mean, radius 1..8 */
    STRATA_OP_MIN = 10,       /* focal.Min, radius 1..8 */
    STRATA_OP_MAX = 11,       /* focal.Max, radius 1..8 */
    STRATA_OP_LOOKUP = 12,    /* transfer.Lookup, pointwise */
    STRATA_OP_RECLASS = 13,   /* transfer.Reclass, pointwise */
    STRATA_OP_HEATLOAD = 14,  /* terrain.HeatLoad (McCune and Keon), radius 1 */
    STRATA_OP_ORIENTATION = 15, /* terrain.Orientation (northness / eastness), radius 1 */
    STRATA_OP_STEP = 16         /* one step of a vec.Chain (Rescale, Clamp, Normalize, algebra), pointwise */
};

/*
 * strata_stage.kind for STRATA_OP_STEP: vec.Op (internal/vec/chain.go:
 * 24-38). The running value acc is the step's first operand; the binary
 * ops (ADD .. MAX) take the pipeline input named by strata_stage.input as
 * the second, the others the immediates k[0] and k[1]:
 *   ADD SUB MUL DIV: acc op src; MIN MAX: Go's min / max (NaN wins, -0 < +0)
 *   ADD_SCALAR: acc + k0; MUL_SCALAR: acc * k0; AFFINE: f32(acc * k0) + k1
 *   SUB_DIV: (acc - k0) / k1; CLAMP: min(max(acc, k0), k1)
 *   ABS: the sign bit cleared; SQRT: f32(sqrt(f64(acc)))
 */
enum {
    STRATA_VEC_ADD = 0,
    STRATA_VEC_SUB = 1,
    STRATA_VEC_MUL = 2,
    STRATA_VEC_DIV = 3,
    STRATA_VEC_MIN = 4,
    STRATA_VEC_MAX = 5,
    STRATA_VEC_ADD_SCALAR = 6,
    STRATA_VEC_MUL_SCALAR = 7,
    STRATA_VEC_AFFINE = 8,
    STRATA_VEC_SUB_DIV = 9,
    STRATA_VEC_CLAMP = 10,
    STRATA_VEC_ABS = 11,
    STRATA_VEC_SQRT = 12
};

/* vec.MaxSteps: the longest chain of pointwise stages one call takes, and
 * the most inputs a pointwise pipeline reads. */
#define STRATA_MAX_STEPS 16
#define STRATA_MAX_INPUTS 4

/* strata_stage.kind for STRATA_OP_CURVATURE (stencil.CurvatureKind). */
enum { STRATA_CURV_PROFILE = 0, STRATA_CURV_PLAN = 1, STRATA_CURV_MEAN = 2 };
/* strata_stage.kind for STRATA_OP_RUGGEDNESS (stencil.RuggednessKind). */
enum { STRATA_RUG_TRI_RILEY = 0, STRATA_RUG_TRI_WILSON = 1, STRATA_RUG_TPI = 2, STRATA_RUG_ROUGHNESS = 3 };

/* strata_stage.flags. */
#define STRATA_STAGE_ROTATE180 1 /* correlate with the weights rotated by 180 degrees (Convolve) */
#define STRATA_STAGE_FIT 2       /* the derivatives from Wood's quadratic fit over the (2 radius + 1)^2 window */

/* Largest tables a stage may carry. */
#define STRATA_MAX_RADIUS 8
#define STRATA_MAX_KNOTS 64

/*
 * A raster view: strata's raster.Float32Raster (raster/raster.go:41-54).
 * Cell (x, y) is data[y * stride + x]; its validity is bit
 * valid_offset + y * stride + x of valid (LSB first in each 64-bit word),
 * set = valid. valid == NULL means every cell is valid. on_device != 0
 * says data and valid are device pointers on the context's device;
 * otherwise they are host pointers and the call copies through device
 * memory (page-locked host memory copies fastest).
 */
typedef struct {
    float *data;
    int64_t width, height, stride;
    uint64_t *valid;
    int64_t valid_offset;
    int32_t on_device;
    int32_t reserved;
} strata_raster;

/*
 * One stage: an op and its resolved constants, as the reference's kernel
 * value holds them after its option checks.
 *   GRADIENT   k[0]=kx k[1]=ky
 *   SLOPE      k[0]=kx k[1]=ky k[2]=scale, kind=1 takes Atan32 first
 *   ASPECT     k[0]=kx k[1]=ky k[2]=flat, kind=1 trigonometric
 *   HILLSHADE  k[0]=kx k[1]=ky k[2]=c k[3]=bx k[4]=by
 *   CURVATURE  k[0..4]=kp kq kr kt ks, kind=STRATA_CURV_*
 *   RUGGEDNESS radius, kind=STRATA_RUG_*
 *   CORRELATE  radius, table[0]=(2r+1)^2 weights row-major, flags
 *   SEPARABLE  radius, table[0]=row taps, table[1]=column taps (2r+1 each)
 *   MEAN/MIN/MAX radius
 *   LOOKUP     table[0]=xs table[1]=ys (table_len[0] knots)
 *   RECLASS    table[0]=breaks (table_len[0]) table[1]=values (table_len[0]+1)
 *   HEATLOAD   k[0]=kx k[1]=ky, table[0]=the regression's eight float64
 *              terms K0 A BX BY E F CX CY as 16 floats, kind=1 takes exp
 *   ORIENTATION k[0]=kx k[1]=ky, kind bit 0 eastness, bit 1 unweighted
 *   STEP       kind=STRATA_VEC_*, k[0] k[1] the immediates, input the
 *              source a binary step reads (-1 for every other op)
 * With flags STRATA_STAGE_FIT (terrain/fit.go, FitRadius > 0) a GRADIENT,
 * SLOPE, ASPECT, HILLSHADE, HEATLOAD, ORIENTATION or CURVATURE stage takes
 * its derivatives from Wood's quadratic fit: radius is the fit's,
 * k[0..4]=kp kq kr kt ks its factors, and the product's constants follow
 * from k[5] (SLOPE scale; ASPECT flat; HILLSHADE c bx by); kind and
 * table[0] mean what they mean without the flag.
 * Tables are host memory, read during the call only.
 */
typedef struct {
    uint32_t op;
    int32_t radius;
    int32_t kind;
    int32_t flags;
    float k[16];
    const float *table[4];
    int32_t table_len[4];
    int32_t input;    /* STEP: see above; ignored by the other ops */
    int32_t reserved;
} strata_stage;

/*
 * Execution options: engine.Options (engine/engine.go:7-28) plus what a
 * device call needs. tile_width / tile_height choose the chunked tiles
 * (0 = whole raster, as the reference) and must not be negative; workers
 * is accepted for parity and must not be negative. stream is a
 * cudaStream_t (NULL = the context's stream). cancel, when not NULL, is
 * polled between row strips (plain) or tiles (chunked): a non-zero value
 * stops the call with STRATA_ECANCELED after a plan-order prefix.
 * flags: STRATA_EXEC_ASYNC returns without synchronising when every
 * operand is on the device.
 */
typedef struct {
    int64_t tile_width, tile_height;
    int32_t workers;
    int32_t flags;
    void *stream;
    const volatile int32_t *cancel;
} strata_exec_opts;

#define STRATA_EXEC_ASYNC 1

/*
 * engine.Stats (engine/stats.go:77-168), counted for the device's own
 * tiling: bands are thread-block tiles, kernel_read counts each tile's
 * window including its halo, kernel_written each output cell once.
 * A call adds to the struct it is given.
 */
typedef struct {
    int64_t cells, ideal, tiles, bands;
    int64_t source_read, sink_written, kernel_read, kernel_written;
} strata_stats;

typedef struct strata_ctx strata_ctx;

/* Library and context. */
int strata_abi_version(void);
const char *strata_last_error(void);
int strata_ctx_create(int device, strata_ctx **out);
void strata_ctx_destroy(strata_ctx *ctx);
int strata_ctx_device(const strata_ctx *ctx);
int strata_ctx_synchronize(strata_ctx *ctx);

/* Device memory owned by the context's device (for resident rasters). */
int strata_alloc(strata_ctx *ctx, size_t bytes, void **dev);
int strata_free(strata_ctx *ctx, void *dev);
int strata_upload(strata_ctx *ctx, void *dev, const void *host, size_t bytes);
int strata_download(strata_ctx *ctx, void *host, const void *dev, size_t bytes);

/*
 * exec.ProcessN (internal/exec/process.go:28) for one kernel or a
 * pipeline: stages[0] is any op, stages[1..nstages-1] pointwise ops
 * (LOOKUP / RECLASS / unary STEP) applied to its result in order, as
 * exec.Pipeline runs Slope -> Lookup -> Reclass (graph/run.go:390-486);
 * at most STRATA_MAX_STEPS pointwise stages, 4 of them LOOKUP / RECLASS.
 * src holds nsrc = 1 raster, except for a pipeline of pointwise stages
 * only (a vec.Chain, internal/exec/pipeline.go:432-490), which starts
 * from src[0] and whose binary STEPs read src[input]: 1 to
 * STRATA_MAX_INPUTS rasters of one size. dst holds 2 rasters for
 * GRADIENT, else 1. Edge cells (within the radius of the raster's border)
 * get NaN and invalid; interior validity is the AND of the inputs'
 * validity over the window (internal/exec/halo.go:21-229). stats may be
 * NULL.
 */
int strata_process(strata_ctx *ctx, const strata_stage *stages, int nstages,
                   const strata_raster *src, int nsrc, const strata_raster *dst, int ndst,
                   const strata_exec_opts *opts, strata_stats *stats);

/*
 * A row strip of a raster `height` rows tall (the multi-GPU split:
 * internal/exec/worker.go:83-181 splits a raster into bands the same way):
 * src holds input rows [src_row, src_row + src->height) and dst output rows
 * [dst_row, dst_row + dst->height). The source rows must cover every row
 * the outputs read, [dst_row - radius, dst_row + dst->height + radius)
 * clipped to the raster. The outputs are the rows strata_process writes
 * for them over the whole raster: the edge ring lies at the whole
 * raster's border only. One input; the rest as strata_process.
 */
typedef struct {
    int64_t height;
    int64_t src_row;
    int64_t dst_row;
} strata_strip;
int strata_process_strip(strata_ctx *ctx, const strata_stage *stages, int nstages, const strata_raster *src,
                         const strata_raster *dst, int ndst, const strata_strip *strip, const strata_exec_opts *opts,
                         strata_stats *stats);

/*
 * strata_process over several devices, one context each: the raster is
 * cut into nctx row strips as equal as can be, each strip with its halo
 * rows read from the host by its own device and computed there
 * (strata_process_strip) on a thread of its own, the strips' rows written
 * back in place. Host rasters, one input; no stream or cancel flag. The
 * result is strata_process's, bit for bit.
 */
int strata_process_multi(strata_ctx *const *ctxs, int nctx, const strata_stage *stages, int nstages,
                         const strata_raster *src, int nsrc, const strata_raster *dst, int ndst,
                         const strata_exec_opts *opts, strata_stats *stats);

/*
 * terrain.Features / terrain.Surface (terrain/features.go:60-92,
 * terrain/surface.go:57-98): several pipelines over one input in one call.
 * Feature f is stages[s_f .. s_f + counts[f]) (s_f the sum of the earlier
 * counts), a stencil stage with optional pointwise stages as in
 * strata_process, writing the next 1 outputs of dst (2 for GRADIENT).
 * Each output gets its own op's edge ring and validity. A host input
 * crosses to the device once, and each output's copy back overlaps the
 * next feature's kernels.
 */
int strata_process_features(strata_ctx *ctx, const strata_stage *stages, const int32_t *counts, int nfeatures,
                            const strata_raster *src, const strata_raster *dst, int ndst,
                            const strata_exec_opts *opts, strata_stats *stats);

/*
 * engine.RasterSource / RasterSink (engine/source.go:19-70) as callbacks.
 * read fills buf (a host raster of buf->width x buf->height cells, with a
 * validity mask iff masked) from the window at (x, y); write takes buf
 * for the window at (x, y). Each returns 0, or non-zero to fail the call
 * with STRATA_EIO.
 */
typedef struct {
    int64_t width, height;
    int32_t masked;
    int32_t reserved;
    void *user;
    int (*read)(void *user, const strata_raster *buf, int64_t x, int64_t y);
} strata_source;

typedef struct {
    int64_t width, height;
    int32_t masked;
    int32_t reserved;
    void *user;
    int (*write)(void *user, const strata_raster *buf, int64_t x, int64_t y);
} strata_sink;

/*
 * exec.ProcessChunked (internal/exec/chunked.go:33): reads tiles of the
 * source with their halo, computes them on the device and hands each
 * tile to the sinks, in plan order, with bounded memory (two pinned
 * buffer sets). The sinks receive the bits strata_process would write.
 */
int strata_process_chunked(strata_ctx *ctx, const strata_stage *stages, int nstages,
                           const strata_source *src, int nsrc, const strata_sink *dst, int ndst,
                           const strata_exec_opts *opts, strata_stats *stats);

/*
 * engine.RawSource / RawSink with RawOptions (engine/raw.go:15-191): a
 * raster of width x height little-endian float32 cells in row-major order
 * at byte offset `offset` of the open file fd (read with pread and written
 * with pwrite, so the descriptor's position is not used; a write past the
 * end extends the file). has_fill declares fill the file's NoData value:
 * reading marks a cell invalid when it equals fill (by ==, so -0 matches
 * 0), or, for a NaN fill, when it is any NaN; writing stores fill under
 * invalid cells. The source or sink is then Masked.
 */
typedef struct {
    int32_t fd;
    int32_t has_fill;
    float fill;
    int32_t reserved;
    int64_t width, height;
    int64_t offset;
} strata_raw_file;

/*
 * strata_process_chunked over raw files: the same tiles and results, each
 * tile read with pread straight into page-locked memory (a full-width
 * tile in one call), its validity taken from the fill value on the
 * device, the fill stored under the invalid output cells on the device,
 * and the tile written with pwrite. Read and write failures return
 * STRATA_EIO with the rows in the message, as RawSource / RawSink word
 * theirs.
 */
int strata_process_raw(strata_ctx *ctx, const strata_stage *stages, int nstages, const strata_raw_file *src,
                       int nsrc, const strata_raw_file *dst, int ndst, const strata_exec_opts *opts,
                       strata_stats *stats);

/*
 * Batches (the batched form of the path; no counterpart call in strata,
 * whose plain functions take one raster each): many device-resident
 * rasters of mixed sizes and ops, each item one pipeline (stages as in
 * strata_process) over src into dst[0] (and dst[1] for GRADIENT), with the
 * edge and validity rules of strata_process per raster. strata_batch_create
 * checks every item as strata_process would, groups the rasters by op
 * class, uploads their descriptors and captures one persistent kernel per
 * class (and one per validity radius) into a CUDA graph on parallel
 * branches; strata_batch_run replays it with one launch (synchronize != 0
 * waits for it). tile_height picks the rows of an item's work units (0 =
 * the kernel's default, at most 1024; the windowed focal ops at radius > 1
 * use fixed tiles); tile_width is not used, the kernels fix the units'
 * width. The Python autotuner chooses tile_height per class.
 * The rasters must stay allocated, and the batch be run on one stream at a
 * time, until strata_batch_destroy.
 */
typedef struct {
    const strata_stage *stages;
    int32_t nstages;
    int32_t tile_width, tile_height;
    int32_t reserved;
    strata_raster src;
    strata_raster dst[2];
} strata_batch_item;

typedef struct strata_batch strata_batch;

int strata_batch_create(strata_ctx *ctx, const strata_batch_item *items, int nitems, strata_batch **out);
int strata_batch_run(strata_batch *batch, void *stream, int synchronize);
/* Adds the batch's Stats (as one call would count them) and reports its op classes. */
int strata_batch_info(const strata_batch *batch, strata_stats *stats, int *classes);
void strata_batch_destroy(strata_batch *batch);

/*
 * A batch run that allocates nothing (no counterpart in strata, which has
 * no batched call). It does what strata_batch_create + strata_batch_run +
 * strata_batch_destroy do for the same items, with the same results, but
 * writes the descriptors into a fixed scratch area in the library's static
 * device memory (one per device, room for STRATA_NOALLOC_BATCH_MAX items;
 * more is EINVAL) and launches the class kernels directly on the stream
 * (0 = the context's), so it makes no cudaMalloc or cudaFree call and
 * builds no graph. The first call on a device looks the scratch area up
 * (and clears its status word); make that call before any stream capture.
 * The descriptors go up by copies from the library's pageable host
 * staging, which the next call rewrites, so a call on a stream that is
 * being captured returns STRATA_EINVAL. The scratch is shared by every
 * call on the device: calls on one stream follow each other in stream
 * order, but calls on different streams (or different contexts of one
 * device) that overlap on the device race on it, so a caller serialises
 * them, e.g. by keeping every call on one stream. synchronize != 0 waits
 * for the kernels and reports their status; with synchronize == 0 the
 * call returns after the launches, and a status its kernels set (a
 * bounded device wait that ran out) stays in the scratch until the next
 * call with synchronize != 0 on the device reports it and clears it. The
 * caller's current device is the same after the call as before it.
 */
#define STRATA_NOALLOC_BATCH_MAX 64
int strata_batch_run_noalloc(strata_ctx *ctx, const strata_batch_item *items, int nitems, void *stream,
                             int synchronize);

/*
 * Serving (no counterpart call in strata, which serves no requests): window
 * requests over a device-resident mosaic, run with continuous batching. A
 * scheduler thread takes queued requests whenever one of `streams` streams
 * is free, admits them in arrival order while their outputs fit in
 * budget_bytes, and launches them as one batch (up to max_batch requests);
 * batches on different streams overlap, and requests that arrive while
 * others run join the next batch. A request is one pipeline (as in
 * strata_process) over the w x h window of the mosaic at (x, y), which is
 * a raster of its own (its border is its edge ring), with the window's
 * validity bits when the mosaic has a mask. Its outputs live in device
 * memory the server allocates; strata_server_wait returns them and the
 * request's submit / start / done times (steady clock, ns), and
 * strata_server_release frees them and their budget.
 */
typedef struct {
    int64_t budget_bytes; /* 0 = 120 GiB */
    int32_t streams;      /* 0 = 4 */
    int32_t max_batch;    /* 0 = 64 */
    int32_t band;         /* rows per work unit of the radius-1 batch kernels, 1..256; 0 = 16 */
    int32_t reserved;
} strata_server_opts;

typedef struct {
    int32_t status; /* 0 done, < 0 a STRATA_E* code */
    int32_t nout;
    strata_raster out[2];
    int64_t t_submit_ns, t_start_ns, t_done_ns;
} strata_server_result;

typedef struct strata_server strata_server;

int strata_server_create(strata_ctx *ctx, const strata_raster *mosaic, const strata_server_opts *opts,
                         strata_server **out);
int strata_server_submit(strata_server *srv, const strata_stage *stages, int nstages, int64_t x, int64_t y,
                         int64_t w, int64_t h, uint64_t *ticket);
/* Waits up to timeout_ms (< 0: without limit) for a request; STRATA_ETIMEDOUT if it is not done by then. */
int strata_server_wait(strata_server *srv, uint64_t ticket, int64_t timeout_ms, strata_server_result *result);
int strata_server_release(strata_server *srv, uint64_t ticket);

/*
 * The same calls for many requests at once, for clients that hold several
 * requests together (one lock, one scheduler wake-up, one call across a
 * language boundary instead of one per request). submit_many checks every
 * request first and queues none if one is invalid; tickets[i] is request
 * i's ticket, in arrival order. wait_many waits for the tickets in order
 * (results may be NULL) and returns the first failure; release_many
 * releases in order and stops at the first failure, the earlier tickets
 * released.
 */
typedef struct {
    const strata_stage *stages;
    int32_t nstages;
    int32_t reserved;
    int64_t x, y, w, h;
} strata_server_request;

int strata_server_submit_many(strata_server *srv, const strata_server_request *reqs, int n, uint64_t *tickets);
int strata_server_wait_many(strata_server *srv, const uint64_t *tickets, int n, int64_t timeout_ms,
                            strata_server_result *results);
int strata_server_release_many(strata_server *srv, const uint64_t *tickets, int n);
int strata_server_stats(strata_server *srv, int64_t *batches, int64_t *served, int64_t *used_bytes);
void strata_server_destroy(strata_server *srv);

/* ---------------------------------------------------------------------- */
/* Stage builders: option resolution and checks of the typed entry points. */

typedef struct { double cell_size, cell_size_y, z_factor; int32_t fit_radius; int32_t reserved; } strata_gradient_options;
/* units: 0 degrees, 1 percent, 2 radians (terrain.SlopeUnits) */
typedef struct { double cell_size, cell_size_y, z_factor; int32_t fit_radius; int32_t units; } strata_slope_options;
typedef struct {
    double cell_size, cell_size_y, z_factor;
    int32_t fit_radius;
    int32_t zero_for_flat;
    int32_t trigonometric;
    int32_t reserved;
} strata_aspect_options;
typedef struct {
    double cell_size, cell_size_y, z_factor;
    int32_t fit_radius;
    int32_t reserved;
    double azimuth, altitude;
} strata_hillshade_options;
/* type: 0 profile, 1 plan, 2 mean (terrain.CurvatureType) */
typedef struct { double cell_size, cell_size_y, z_factor; int32_t fit_radius; int32_t type; } strata_curvature_options;
/* type: 0 TRI (Riley), 1 TRIWilson, 2 TPI, 3 Roughness; radius 0 means 1 */
typedef struct { int32_t type; int32_t radius; } strata_ruggedness_options;
typedef struct { int32_t radius; int32_t nweights; const float *weights; } strata_weights_options;
typedef struct { int32_t radius; int32_t nrow; const float *row; int32_t ncol; int32_t reserved; const float *col; } strata_separable_options;
typedef struct { int32_t radius; } strata_box_options;

/* equation: 0..2 (terrain.HeatLoadEquation); latitude in degrees. The
 * builder writes the regression's terms into terms, and the stage points
 * at them: the options must outlive the stage's use. */
typedef struct {
    double cell_size, cell_size_y, z_factor;
    int32_t fit_radius;
    int32_t equation;
    double latitude;
    int32_t radiation, linear;
    double terms[8];
} strata_heatload_options;
/* component: 0 northness, 1 eastness (terrain.OrientationComponent) */
typedef struct {
    double cell_size, cell_size_y, z_factor;
    int32_t fit_radius;
    int32_t component;
    int32_t unweighted;
    int32_t reserved;
} strata_orientation_options;

/* The builders of the terrain ops take fit_radius 1..8 as the reference
 * does (terrain/fit.go:187-226, newWoodFit :38-66): Wood's quadratic fit. */
/* terrain.newGradientKernel (terrain/gradient.go:70-73). */
int strata_stage_gradient(const strata_gradient_options *o, strata_stage *out);
/* terrain.newSlopeKernel / slopeScale (terrain/slope.go:76-95). */
int strata_stage_slope(const strata_slope_options *o, strata_stage *out);
/* terrain.newAspectKernel (terrain/aspect.go:90-102). */
int strata_stage_aspect(const strata_aspect_options *o, strata_stage *out);
/* terrain.newHillshadeKernel / hillshadeLight (terrain/hillshade.go:84-117). */
int strata_stage_hillshade(const strata_hillshade_options *o, strata_stage *out);
/* terrain.newCurvatureKernel (terrain/curvature.go:113-140). */
int strata_stage_curvature(const strata_curvature_options *o, strata_stage *out);
/* terrain.newRuggednessKernel (terrain/ruggedness.go:119-141). */
int strata_stage_ruggedness(const strata_ruggedness_options *o, strata_stage *out);
/* focal.newWeightsKernel (focal/correlate.go:72-88); convolve != 0 for Convolve.
 * The stage keeps the caller's weights pointer. */
int strata_stage_correlate(const strata_weights_options *o, int convolve, strata_stage *out);
/* focal.newSeparableKernel (focal/separable.go:78-89). */
int strata_stage_separable(const strata_separable_options *o, strata_stage *out);
/* focal.newBox (focal/box.go:77-80); op is STRATA_OP_MEAN, _MIN or _MAX. */
int strata_stage_box(const strata_box_options *o, uint32_t op, strata_stage *out);
/* transfer.newLookupKernel (transfer/transfer.go:197-212). */
int strata_stage_lookup(const float *xs, const float *ys, int32_t n, strata_stage *out);
/* transfer.newReclassKernel (transfer/transfer.go:187-195). */
int strata_stage_reclass(const float *breaks, int32_t nbreaks, const float *values, int32_t nvalues,
                         strata_stage *out);
/* One vec.Chain step (vec.NewChain's checks, internal/vec/chain.go:
 * 106-132): op a STRATA_VEC_*; input the source a binary op reads (0 to
 * STRATA_MAX_INPUTS - 1), -1 for the others; k0, k1 the immediates. */
int strata_stage_step(int32_t op, int32_t input, float k0, float k1, strata_stage *out);
/* transfer.Rescale's kernel (transfer/transfer.go:56-60, tiled.go:108-110):
 * an AFFINE step with a and b. */
int strata_stage_rescale(float a, float b, strata_stage *out);
/* transfer.RescaleRange (transfer/transfer.go:87-92, 236-250): the AFFINE
 * step sending [in_lo, in_hi] to [out_lo, out_hi], with its checks. */
int strata_stage_rescale_range(float in_lo, float in_hi, float out_lo, float out_hi, strata_stage *out);
/* terrain.heatLoadOp / heatLoadTerms (terrain/heatload.go:110-146). */
int strata_stage_heatload(strata_heatload_options *o, strata_stage *out);
/* terrain.orientationOp (terrain/orientation.go:55-76). */
int strata_stage_orientation(const strata_orientation_options *o, strata_stage *out);
/* focal.Gaussian (focal/separable.go:59-76): 2*radius+1 taps into taps. */
int strata_focal_gaussian(int32_t radius, double sigma, float *taps);

#ifdef __cplusplus
}
#endif

#endif
