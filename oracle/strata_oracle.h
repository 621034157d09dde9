/*
 * strata_oracle.h - TEST INFRASTRUCTURE ONLY.
 *
 * The CPU restatement of strata's scalar raster-stencil kernels, used as
 * the parity checker for the CUDA backend. Nothing in the product links,
 * loads or calls this code: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference arm of bench.py do.
 *
 * Op codes, kinds and the stage layout match include/strata_cuda.h value
 * for value; tests/test_abi.py checks that they agree.
 */
#ifndef STRATA_ORACLE_H
#define STRATA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORC_GRADIENT = 1,
    ORC_SLOPE = 2,
    ORC_ASPECT = 3,
    ORC_HILLSHADE = 4,
    ORC_CURVATURE = 5,
    ORC_RUGGEDNESS = 6,
    ORC_CORRELATE = 7,
    ORC_SEPARABLE = 8,
    ORC_MEAN = 9,
    ORC_MIN = 10,
    ORC_MAX = 11,
    ORC_LOOKUP = 12,
    ORC_RECLASS = 13,
    ORC_HEATLOAD = 14,
    ORC_ORIENTATION = 15,
    ORC_STEP = 16 /* one vec.Chain step: kind = vec.Op, k[0..1], input */
};

/* orc_stage.flags: the stage's derivatives come from Wood's quadratic fit
 * over the (2 radius + 1)^2 window (terrain/fit.go), not Horn's 3x3. */
#define ORC_STAGE_FIT 2

/* One stage of a call. k[] holds the op's float constants, table[] its
 * weights, taps or knots (see include/strata_cuda.h for the slot meaning). */
typedef struct {
    uint32_t op;
    int32_t radius;
    int32_t kind;
    int32_t flags;
    float k[16];
    const float *table[4];
    int32_t table_len[4];
    int32_t input; /* ORC_STEP: the source a binary step reads, -1 for the others */
    int32_t reserved;
} orc_stage;

typedef struct {
    float *data;
    int64_t width, height, stride;
    uint64_t *valid;
    int64_t valid_offset;
} orc_raster;

/* Per-cell building blocks, exported so tests can pin them against the
 * reference's known-answer tables. */
float orc_atan32(float x);
float orc_atan2f32(float y, float x);
float orc_go_min(float a, float b);
float orc_go_max(float a, float b);
void orc_atan32_array(const float *x, float *out, int64_t n);
int64_t orc_atan32_drops(int nthreads);
void orc_atan2f32_array(const float *y, const float *x, float *out, int64_t n);

/* Host constants, as the reference's option code derives them. */
void orc_horn_scales(double cx, double cy, double z, float *kx, float *ky);
void orc_zt_scales(double cx, double cy, double z, float out5[5]);
void orc_hillshade_light(double azimuth, double altitude, float out3[3]);
void orc_gaussian(int radius, double sigma, float *taps);

/* Runs stages[0] (any op) followed by stages[1..] (pointwise ops only)
 * over whole rasters: the semantics of strata's ProcessN for one kernel or
 * a stencil-then-pointwise Pipeline. src is one raster; dst holds one
 * raster, or two for ORC_GRADIENT. nthreads <= 1 runs on the calling
 * thread. Returns 0, or -1 for an invalid call. */
int orc_process(const orc_stage *stages, int nstages, const orc_raster *src,
                const orc_raster *dst, int ndst, int nthreads);

/* orc_process with simd != 0: the radius-1 stencils' interior rows run
 * through the restated AVX2 lanes of strata_avx2.c (the reference's
 * internal/stencil/simd_amd64.go), with the scalar kernels on each row's
 * last n % 8 cells, as the reference runs them on AVX2 hardware. The
 * results are the same bits; this is the timed CPU baseline. */
int orc_process_ex(const orc_stage *stages, int nstages, const orc_raster *src,
                   const orc_raster *dst, int ndst, int nthreads, int simd);

/* A pipeline over nsrc inputs (1 to 4): a stencil-led one takes one; a
 * pointwise one (a vec.Chain with Lookup / Reclass stages among its
 * steps) starts from src[0], its binary steps read src[input], and its
 * output is valid where every masked input is. */
int orc_process_n(const orc_stage *stages, int nstages, const orc_raster *src, int nsrc,
                  const orc_raster *dst, int ndst, int nthreads);

/* The restated AVX2 lanes of one interior row (strata_avx2.c): the first
 * multiple of eight of the n cells; returns how many it wrote. r0, r1, r2
 * point at column x0 - 1 of the rows above, at and below. */
int64_t orc_avx2_row(const orc_stage *st, float *o0, float *o1, const float *r0, const float *r1,
                     const float *r2, int64_t n);

#ifdef __cplusplus
}
#endif

#endif
