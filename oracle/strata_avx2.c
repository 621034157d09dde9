/*
 * strata_avx2.c - TEST INFRASTRUCTURE ONLY: the timed CPU baseline.
 *
 * A C restatement of the reference's AVX2 row kernels for the radius-1
 * stencils (internal/stencil/simd_amd64.go), eight lanes at a time with
 * the same operations in the same order (VMULPS / VADDPS / VSUBPS /
 * VDIVPS / VSQRTPS, blends for IfElse, no FMA), so every lane has the
 * scalar kernel's bits. The reference runs exactly these lanes on AVX2
 * hardware; this file is the "restated AVX2" baseline the benchmark times
 * beside the device, and the scalar oracle in strata_oracle.c is the
 * parity checker that pins it (tests/test_avx2_baseline.py).
 *
 * Each *_lanes function handles the first multiple of eight cells of a
 * row and returns how many it wrote; the caller runs the scalar kernel on
 * the rest, as the reference's wrappers do (simd_amd64.go:85-89 and the
 * like). r0, r1 and r2 point at column x0 - 1 of the rows above, at and
 * below the output row, and hold n + 2 cells.
 *
 * Build with -mavx2 -mno-fma -ffp-contract=off: no operation may fuse.
 */
#include <immintrin.h>
#include <stdint.h>

#include "strata_oracle.h"

/* The float32 constants of internal/stencil/horn.go:226-235 and
 * aspect.go:10-14 (the scalar oracle's), as lane vectors. */
#define K_TAN3PI8 0x1.3504f4p+1f
#define K_TANPI8 0x1.a8279ap-2f
#define K_PI2 0x1.921fb6p+0f
#define K_PI4 0x1.921fb6p-1f
#define K_C4 0x1.49e1a2p-4f
#define K_C3 0x1.1c370ap-3f
#define K_C2 0x1.9924bep-3f
#define K_C1 0x1.555454p-2f
#define K_PI 0x1.921fb6p+1f
#define K_RAD2DEG 0x1.ca5dc2p+5f

typedef __m256 v8;

static inline v8 ld(const float *p) { return _mm256_loadu_ps(p); }
static inline v8 bc(float f) { return _mm256_set1_ps(f); }
/* IfElse(mask, a, b): a where mask, else b (archsimd's a.IfElse(mask, b)). */
static inline v8 sel(v8 mask, v8 a, v8 b) { return _mm256_blendv_ps(b, a, mask); }
static inline v8 gt(v8 a, v8 b) { return _mm256_cmp_ps(a, b, _CMP_GT_OQ); }
static inline v8 ge(v8 a, v8 b) { return _mm256_cmp_ps(a, b, _CMP_GE_OQ); }
static inline v8 lt(v8 a, v8 b) { return _mm256_cmp_ps(a, b, _CMP_LT_OQ); }
static inline v8 eq(v8 a, v8 b) { return _mm256_cmp_ps(a, b, _CMP_EQ_OQ); }

/* hornDiff8 (simd_amd64.go:67-77). */
static inline void horn_diff8(const float *r0, const float *r1, const float *r2, v8 *dx, v8 *dy)
{
    const v8 z1 = ld(r0), z2 = ld(r0 + 1), z3 = ld(r0 + 2);
    const v8 z4 = ld(r1), z6 = ld(r1 + 2);
    const v8 z7 = ld(r2), z8 = ld(r2 + 1), z9 = ld(r2 + 2);
    v8 d = _mm256_sub_ps(z6, z4);
    *dx = _mm256_add_ps(_mm256_add_ps(_mm256_sub_ps(z3, z1), _mm256_sub_ps(z9, z7)), _mm256_add_ps(d, d));
    d = _mm256_sub_ps(z8, z2);
    *dy = _mm256_add_ps(_mm256_add_ps(_mm256_sub_ps(z7, z1), _mm256_sub_ps(z9, z3)), _mm256_add_ps(d, d));
}

/* magnitude8 (simd_amd64.go:121-124). */
static inline v8 magnitude8(v8 gx, v8 gy)
{
    return _mm256_sqrt_ps(_mm256_add_ps(_mm256_mul_ps(gx, gx), _mm256_mul_ps(gy, gy)));
}

/* atan8 (simd_amd64.go:183-195): both reductions computed, then selected
 * in the order of Atan32's two ifs. */
static inline v8 atan8(v8 x)
{
    const v8 mid = gt(x, bc(K_TANPI8)), big = gt(x, bc(K_TAN3PI8));
    const v8 num = sel(big, bc(-1.0f), sel(mid, _mm256_sub_ps(x, bc(1.0f)), x));
    const v8 den = sel(big, x, sel(mid, _mm256_add_ps(x, bc(1.0f)), bc(1.0f)));
    const v8 y0 = sel(big, bc(K_PI2), sel(mid, bc(K_PI4), bc(0.0f)));
    const v8 t = _mm256_div_ps(num, den);
    const v8 z = _mm256_mul_ps(t, t);
    v8 p = _mm256_sub_ps(_mm256_mul_ps(bc(K_C4), z), bc(K_C3));
    p = _mm256_add_ps(_mm256_mul_ps(p, z), bc(K_C2));
    p = _mm256_sub_ps(_mm256_mul_ps(p, z), bc(K_C1));
    return _mm256_add_ps(y0, _mm256_add_ps(_mm256_mul_ps(_mm256_mul_ps(p, z), t), t));
}

/* atan2_8 (simd_amd64.go:256-265): absolute values, sign tests and
 * copysign on the bits. */
static inline v8 atan2_8(v8 y, v8 x)
{
    const v8 sign = _mm256_castsi256_ps(_mm256_set1_epi32((int)0x80000000u));
    const v8 ay = _mm256_andnot_ps(sign, y), ax = _mm256_andnot_ps(sign, x);
    v8 a = atan8(_mm256_div_ps(ay, ax));
    a = sel(_mm256_and_ps(eq(ay, bc(0.0f)), eq(ax, bc(0.0f))), bc(0.0f), a);
    a = sel(_mm256_and_ps(eq(ay, ax), gt(ay, bc(0x1.fffffep+127f))), bc(K_PI4), a);
    const __m256i xneg = _mm256_cmpgt_epi32(_mm256_setzero_si256(), _mm256_castps_si256(x));
    a = sel(_mm256_castsi256_ps(xneg), _mm256_sub_ps(bc(K_PI), a), a);
    return _mm256_or_ps(a, _mm256_and_ps(y, sign));
}

/* shade8 (simd_amd64.go:284-291). */
static inline v8 shade8(v8 gx, v8 gy, v8 c, v8 bx, v8 by)
{
    const v8 num = _mm256_add_ps(c, _mm256_add_ps(_mm256_mul_ps(bx, gx), _mm256_mul_ps(by, gy)));
    const v8 den = _mm256_sqrt_ps(_mm256_add_ps(bc(1.0f), _mm256_add_ps(_mm256_mul_ps(gx, gx), _mm256_mul_ps(gy, gy))));
    v8 v = _mm256_div_ps(num, den);
    v = sel(lt(v, bc(0.0f)), bc(0.0f), v);
    return sel(gt(v, bc(255.0f)), bc(255.0f), v);
}

#define LANES_LOOP(...)                                                    \
    int64_t i = 0;                                                         \
    for (; i + 8 <= n; i += 8) {                                           \
        const float *a0 = r0 + i, *a1 = r1 + i, *a2 = r2 + i;              \
        __VA_ARGS__                                                        \
    }                                                                      \
    return i;

/* hornGradientLanes (simd_amd64.go:85-101). */
static int64_t gradient_lanes(float *dx, float *dy, const float *r0, const float *r1, const float *r2, int64_t n,
                              const float *k)
{
    const v8 kx = bc(k[0]), ky = bc(k[1]);
    LANES_LOOP({
        v8 gx, gy;
        horn_diff8(a0, a1, a2, &gx, &gy);
        _mm256_storeu_ps(dx + i, _mm256_mul_ps(gx, kx));
        _mm256_storeu_ps(dy + i, _mm256_mul_ps(gy, ky));
    })
}

/* hornSlopeLanes / hornSlopeAtanLanes (simd_amd64.go:126-158). */
static int64_t slope_lanes(float *dst, const float *r0, const float *r1, const float *r2, int64_t n, const float *k,
                           int take_atan)
{
    const v8 kx = bc(k[0]), ky = bc(k[1]), s = bc(k[2]);
    LANES_LOOP({
        v8 gx, gy;
        horn_diff8(a0, a1, a2, &gx, &gy);
        v8 m = magnitude8(_mm256_mul_ps(gx, kx), _mm256_mul_ps(gy, ky));
        if (take_atan) m = atan8(m);
        _mm256_storeu_ps(dst + i, _mm256_mul_ps(m, s));
    })
}

/* hornAspectLanes (simd_amd64.go:216-242). */
static int64_t aspect_lanes(float *dst, const float *r0, const float *r1, const float *r2, int64_t n, const float *k,
                            int trig)
{
    const v8 kx = bc(k[0]), ky = bc(k[1]), flat = bc(k[2]);
    LANES_LOOP({
        v8 dx, dy;
        horn_diff8(a0, a1, a2, &dx, &dy);
        const v8 gx = _mm256_mul_ps(dx, kx), gy = _mm256_mul_ps(dy, ky);
        v8 y = _mm256_sub_ps(bc(0.0f), gx), x = gy;
        if (trig) {
            y = gy;
            x = _mm256_sub_ps(bc(0.0f), gx);
        }
        v8 d = _mm256_mul_ps(atan2_8(y, x), bc(K_RAD2DEG));
        d = _mm256_add_ps(d, sel(lt(d, bc(0.0f)), bc(360.0f), bc(0.0f)));
        d = sel(ge(d, bc(360.0f)), bc(0.0f), d);
        d = sel(_mm256_and_ps(eq(y, bc(0.0f)), eq(x, bc(0.0f))), flat, d);
        _mm256_storeu_ps(dst + i, d);
    })
}

/* hornHillshadeLanes (simd_amd64.go:273-282). */
static int64_t hillshade_lanes(float *dst, const float *r0, const float *r1, const float *r2, int64_t n,
                               const float *k)
{
    const v8 kx = bc(k[0]), ky = bc(k[1]), c = bc(k[2]), bx = bc(k[3]), by = bc(k[4]);
    LANES_LOOP({
        v8 dx, dy;
        horn_diff8(a0, a1, a2, &dx, &dy);
        _mm256_storeu_ps(dst + i, shade8(_mm256_mul_ps(dx, kx), _mm256_mul_ps(dy, ky), c, bx, by));
    })
}

/* ztDerivs8 (simd_amd64.go:372-384). */
static inline void zt_derivs8(const float *r0, const float *r1, const float *r2, const v8 *kk, v8 *p, v8 *q, v8 *r,
                              v8 *s, v8 *t)
{
    const v8 z1 = ld(r0), z2 = ld(r0 + 1), z3 = ld(r0 + 2);
    const v8 z4 = ld(r1), z5 = ld(r1 + 1), z6 = ld(r1 + 2);
    const v8 z7 = ld(r2), z8 = ld(r2 + 1), z9 = ld(r2 + 2);
    *p = _mm256_mul_ps(_mm256_sub_ps(z6, z4), kk[0]);
    *q = _mm256_mul_ps(_mm256_sub_ps(z8, z2), kk[1]);
    const v8 c = _mm256_add_ps(z5, z5);
    *r = _mm256_mul_ps(_mm256_sub_ps(_mm256_add_ps(z4, z6), c), kk[2]);
    *t = _mm256_mul_ps(_mm256_sub_ps(_mm256_add_ps(z2, z8), c), kk[3]);
    *s = _mm256_mul_ps(_mm256_sub_ps(_mm256_add_ps(z1, z9), _mm256_add_ps(z3, z7)), kk[4]);
}

/* ztProfileLanes / ztPlanLanes / ztMeanLanes (simd_amd64.go:386-455). */
static int64_t curvature_lanes(float *dst, const float *r0, const float *r1, const float *r2, int64_t n,
                               const float *k, int kind)
{
    const v8 kk[5] = {bc(k[0]), bc(k[1]), bc(k[2]), bc(k[3]), bc(k[4])};
    const v8 one = bc(1.0f), zero = bc(0.0f);
    LANES_LOOP({
        v8 p, q, r, s, t;
        zt_derivs8(a0, a1, a2, kk, &p, &q, &r, &s, &t);
        const v8 p2 = _mm256_mul_ps(p, p), q2 = _mm256_mul_ps(q, q), pq = _mm256_mul_ps(p, q);
        const v8 pq2s = _mm256_mul_ps(_mm256_add_ps(pq, pq), s);
        v8 v;
        if (kind == 0) {
            const v8 g = _mm256_add_ps(p2, q2);
            const v8 w = _mm256_add_ps(one, g);
            const v8 num = _mm256_add_ps(_mm256_add_ps(_mm256_mul_ps(p2, r), pq2s), _mm256_mul_ps(q2, t));
            v = _mm256_sub_ps(zero, _mm256_div_ps(_mm256_div_ps(num, g), _mm256_mul_ps(w, _mm256_sqrt_ps(w))));
            v = sel(eq(g, zero), _mm256_add_ps(num, zero), v);
        } else if (kind == 1) {
            const v8 g = _mm256_add_ps(p2, q2);
            const v8 num = _mm256_add_ps(_mm256_sub_ps(_mm256_mul_ps(q2, r), pq2s), _mm256_mul_ps(p2, t));
            v = _mm256_sub_ps(zero, _mm256_div_ps(_mm256_div_ps(num, g), _mm256_sqrt_ps(g)));
            v = sel(eq(g, zero), _mm256_add_ps(num, zero), v);
        } else {
            const v8 w = _mm256_add_ps(one, _mm256_add_ps(p2, q2));
            const v8 num = _mm256_add_ps(_mm256_sub_ps(_mm256_mul_ps(_mm256_add_ps(one, q2), r), pq2s),
                                         _mm256_mul_ps(_mm256_add_ps(one, p2), t));
            const v8 d = _mm256_mul_ps(w, _mm256_sqrt_ps(w));
            v = _mm256_sub_ps(zero, _mm256_div_ps(num, _mm256_add_ps(d, d)));
        }
        _mm256_storeu_ps(dst + i, v);
    })
}

/* sq4x2 (simd_amd64.go:509-513): float64 squares of the low and high four
 * lanes. */
static inline void sq4x2(v8 d, __m256d *lo, __m256d *hi)
{
    const __m256d l = _mm256_cvtps_pd(_mm256_castps256_ps128(d));
    const __m256d h = _mm256_cvtps_pd(_mm256_extractf128_ps(d, 1));
    *lo = _mm256_mul_pd(l, l);
    *hi = _mm256_mul_pd(h, h);
}

static inline v8 MX(v8 a, v8 b) { return _mm256_max_ps(a, b); }
static inline v8 MN(v8 a, v8 b) { return _mm256_min_ps(a, b); }

/* rileyLanes, wilsonLanes, tpiLanes, roughnessLanes (simd_amd64.go:476-558). */
static int64_t ruggedness_lanes(float *dst, const float *r0, const float *r1, const float *r2, int64_t n, int kind)
{
    const v8 zero = bc(0.0f), eighth = bc(0.125f);
    const v8 sign = _mm256_castsi256_ps(_mm256_set1_epi32((int)0x80000000u));
    LANES_LOOP({
        const v8 z[9] = {ld(a0), ld(a0 + 1), ld(a0 + 2), ld(a1), ld(a1 + 1), ld(a1 + 2), ld(a2), ld(a2 + 1), ld(a2 + 2)};
        const v8 z5 = z[4];
        v8 out;
        if (kind == 0) {
            __m256d lo, hi, l, h;
            sq4x2(_mm256_sub_ps(z[0], z5), &lo, &hi);
            static const int order[7] = {1, 2, 3, 5, 6, 7, 8};
            for (int j = 0; j < 7; j++) {
                sq4x2(_mm256_sub_ps(z[order[j]], z5), &l, &h);
                lo = _mm256_add_pd(lo, l);
                hi = _mm256_add_pd(hi, h);
            }
            const __m128 fl = _mm256_cvtpd_ps(_mm256_sqrt_pd(lo)), fh = _mm256_cvtpd_ps(_mm256_sqrt_pd(hi));
            out = _mm256_insertf128_ps(_mm256_castps128_ps256(fl), fh, 1);
        } else if (kind == 1) {
            v8 s = _mm256_andnot_ps(sign, _mm256_sub_ps(z[0], z5));
            static const int order[7] = {1, 2, 3, 5, 6, 7, 8};
            for (int j = 0; j < 7; j++) s = _mm256_add_ps(s, _mm256_andnot_ps(sign, _mm256_sub_ps(z[order[j]], z5)));
            out = _mm256_mul_ps(s, eighth);
        } else if (kind == 2) {
            v8 s = _mm256_add_ps(z[0], z[1]);
            static const int order[6] = {2, 3, 5, 6, 7, 8};
            for (int j = 0; j < 6; j++) s = _mm256_add_ps(s, z[order[j]]);
            out = _mm256_sub_ps(z5, _mm256_mul_ps(s, eighth));
        } else {
            /* VMAXPS / VMINPS, then the NaN lanes selected and -0 turned
             * into +0 (simd_amd64.go:539-558). */
            const v8 hi = MX(MX(MX(z[0], z[1]), MX(z[2], z[3])), MX(MX(z[4], z[5]), MX(z[6], z[7])));
            const v8 lo = MN(MN(MN(z[0], z[1]), MN(z[2], z[3])), MN(MN(z[4], z[5]), MN(z[6], z[7])));
            const v8 hi9 = MX(hi, z[8]), lo9 = MN(lo, z[8]);
            v8 nan = _mm256_cmp_ps(z[0], z[0], _CMP_UNORD_Q);
            for (int j = 1; j < 9; j++) nan = _mm256_or_ps(nan, _mm256_cmp_ps(z[j], z[j], _CMP_UNORD_Q));
            const v8 v = _mm256_add_ps(_mm256_sub_ps(hi9, lo9), zero);
            out = sel(nan, bc(__builtin_nanf("")), v);
        }
        _mm256_storeu_ps(dst + i, out);
    })
}

int64_t orc_avx2_row(const orc_stage *st, float *o0, float *o1, const float *r0, const float *r1, const float *r2,
                     int64_t n)
{
    if (st->flags & ORC_STAGE_FIT) return 0; /* Wood's fit: the scalar kernels */
    switch (st->op) {
    case ORC_GRADIENT: return gradient_lanes(o0, o1, r0, r1, r2, n, st->k);
    case ORC_SLOPE: return slope_lanes(o0, r0, r1, r2, n, st->k, st->kind != 0);
    case ORC_ASPECT: return aspect_lanes(o0, r0, r1, r2, n, st->k, st->kind != 0);
    case ORC_HILLSHADE: return hillshade_lanes(o0, r0, r1, r2, n, st->k);
    case ORC_CURVATURE: return curvature_lanes(o0, r0, r1, r2, n, st->k, st->kind);
    case ORC_RUGGEDNESS: return st->radius == 1 ? ruggedness_lanes(o0, r0, r1, r2, n, st->kind) : 0;
    default: return 0;
    }
}
