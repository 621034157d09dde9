// cellops.cuh - the per-cell arithmetic of strata's raster-stencil kernels,
// as device functions.
//
// Every float operation is an explicitly rounded intrinsic (__fadd_rn,
// __fmul_rn, __fdiv_rn, ...), which the compiler never contracts into an
// FMA, so each result is the reference scalar backend's bits: strata wraps
// every product in float32(...) for the same reason
// (internal/stencil/horn.go:12-18, internal/focalrow/focalrow.go:14-33).
// The operation order of each function follows the reference function
// cited beside it.
#pragma once

#include <cstdint>

#include "strata_cuda.h"

namespace strata {
namespace cell {

__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }

// float32(math.Sqrt(float64(x))): the float64 root of a float32 rounded to
// float32 equals the correctly rounded float32 root (53 >= 2*24 + 2, so the
// double rounding is innocuous), which __fsqrt_rn computes directly.
__device__ __forceinline__ float sqrt64of32(float x) { return __fsqrt_rn(x); }

__device__ __forceinline__ float nanf32() { return __int_as_float(0x7fc00000); }
__device__ __forceinline__ float abs32(float x) { return __int_as_float(__float_as_int(x) & 0x7fffffff); }

// Go's builtin min and max for float32: NaN wins, -0 orders below +0. The
// PTX min.NaN / max.NaN instructions have exactly these rules (a NaN
// operand gives NaN, and -0 is below +0); tests/test_gpu_minmax.py pins
// them against the oracle's restatement over every ordered pair of
// special values. Any NaN matches any NaN under the reference's
// comparison rule, so the canonical NaN they return is the same result.
__device__ __forceinline__ float go_min(float a, float b) {
    float r;
    asm("min.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float go_max(float a, float b) {
    float r;
    asm("max.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}

// Atan32 constants (internal/stencil/horn.go:226-235, aspect.go:10-14),
// each the correctly rounded float32 of the reference's expression.
constexpr float kTan3Pi8 = 0x1.3504f4p+1f;
constexpr float kTanPi8 = 0x1.a8279ap-2f;
constexpr float kPi2 = 0x1.921fb6p+0f;
constexpr float kPi4 = 0x1.921fb6p-1f;
constexpr float kC4 = 0x1.49e1a2p-4f;
constexpr float kC3 = 0x1.1c370ap-3f;
constexpr float kC2 = 0x1.9924bep-3f;
constexpr float kC1 = 0x1.555454p-2f;
constexpr float kPi = 0x1.921fb6p+1f;
constexpr float kRadToDeg = 0x1.ca5dc2p+5f;

// Atan32 (internal/stencil/horn.go:249-262): the Cephes float32
// arctangent with the argument reduced around 0, pi/4 or pi/2.
__device__ __forceinline__ float atan32(float x) {
    float num = x, den = 1.0f, y0 = 0.0f;
    if (x > kTanPi8) {
        num = sub(x, 1.0f);
        den = add(x, 1.0f);
        y0 = kPi4;
    }
    if (x > kTan3Pi8) {
        num = -1.0f;
        den = x;
        y0 = kPi2;
    }
    float t = div(num, den);
    float z = mul(t, t);
    float p = sub(mul(kC4, z), kC3);
    p = add(mul(p, z), kC2);
    p = sub(mul(p, z), kC1);
    return add(y0, add(mul(mul(p, z), t), t));
}

// Atan2F32 (internal/stencil/aspect.go:33-47).
__device__ __forceinline__ float atan2f32(float y, float x) {
    float ax = abs32(x), ay = abs32(y);
    float a = atan32(div(ay, ax));
    if (ay == 0.0f && ax == 0.0f) a = 0.0f;
    if (ay == ax && ay > 0x1.fffffep+127f) a = kPi4;
    if (__float_as_uint(x) & 0x80000000u) a = sub(kPi, a);
    return __uint_as_float(__float_as_uint(a) | (__float_as_uint(y) & 0x80000000u));
}

// hornDX / hornDY (internal/stencil/horn.go:152-160).
__device__ __forceinline__ float horn_dx(float z1, float z3, float z4, float z6, float z7, float z9) {
    float d = sub(z6, z4);
    return add(add(sub(z3, z1), sub(z9, z7)), add(d, d));
}
__device__ __forceinline__ float horn_dy(float z1, float z2, float z3, float z7, float z8, float z9) {
    float d = sub(z8, z2);
    return add(add(sub(z7, z1), sub(z9, z3)), add(d, d));
}

// magnitude (internal/stencil/horn.go:220-222).
__device__ __forceinline__ float magnitude(float gx, float gy) {
    return sqrt64of32(add(mul(gx, gx), mul(gy, gy)));
}

// Slope from a gradient (horn.go:193-216, gradrow.go:44-59).
__device__ __forceinline__ float slope(float gx, float gy, float scale, bool take_atan) {
    float m = magnitude(gx, gy);
    return take_atan ? mul(atan32(m), scale) : mul(m, scale);
}

// aspectArgs + aspectDegrees (internal/stencil/aspect.go:97-121).
__device__ __forceinline__ float aspect(float gx, float gy, float flat, bool trig) {
    float y, x;
    if (trig) {
        y = gy;
        x = sub(0.0f, gx);
    } else {
        y = sub(0.0f, gx);
        x = gy;
    }
    float d = mul(atan2f32(y, x), kRadToDeg);
    float off = d < 0.0f ? 360.0f : 0.0f;
    d = add(d, off);
    if (d >= 360.0f) d = 0.0f;
    if (y == 0.0f && x == 0.0f) d = flat;
    return d;
}

// shade (internal/stencil/aspect.go:162-173).
__device__ __forceinline__ float shade(float gx, float gy, float c, float bx, float by) {
    float num = add(c, add(mul(bx, gx), mul(by, gy)));
    float den = sqrt64of32(add(1.0f, add(mul(gx, gx), mul(gy, gy))));
    float v = div(num, den);
    if (v < 0.0f) v = 0.0f;
    if (v > 255.0f) v = 255.0f;
    return v;
}

__device__ __forceinline__ float zt_finish(float P, float Q, float R, float S, float T, int kind);

// Zevenbergen-Thorne curvature (internal/stencil/curvature.go:79-129):
// ztDerivs, then the profile (0), plan (1) or mean (2) formula.
__device__ __forceinline__ float zt_curvature(float z1, float z2, float z3, float z4, float z5, float z6,
                                              float z7, float z8, float z9, const float* k, int kind) {
    float P = mul(sub(z6, z4), k[0]);
    float Q = mul(sub(z8, z2), k[1]);
    float c = add(z5, z5);
    float R = mul(sub(add(z4, z6), c), k[2]);
    float T = mul(sub(add(z2, z8), c), k[3]);
    float S = mul(sub(add(z1, z9), add(z3, z7)), k[4]);
    return zt_finish(P, Q, R, S, T, kind);
}

// CurvatureFromDerivsRow (internal/stencil/curvature.go:138-185): ZT's
// formulas from the derivatives p, q, r, s, t, however estimated (ZT's
// 3x3 window above, or Wood's fit).
__device__ __forceinline__ float zt_finish(float P, float Q, float R, float S, float T, int kind) {
    float p2 = mul(P, P), q2 = mul(Q, Q);
    float pq = mul(P, Q);
    float pq2 = add(pq, pq);
    if (kind == 0) {
        float g = add(p2, q2);
        float w = add(1.0f, g);
        float num = add(add(mul(p2, R), mul(pq2, S)), mul(q2, T));
        float v = sub(0.0f, div(div(num, g), mul(w, sqrt64of32(w))));
        if (g == 0.0f) v = add(num, 0.0f);
        return v;
    }
    if (kind == 1) {
        float g = add(p2, q2);
        float num = add(sub(mul(q2, R), mul(pq2, S)), mul(p2, T));
        float v = sub(0.0f, div(div(num, g), sqrt64of32(g)));
        if (g == 0.0f) v = add(num, 0.0f);
        return v;
    }
    float w = add(1.0f, add(p2, q2));
    float num = add(sub(mul(add(1.0f, q2), R), mul(pq2, S)), mul(add(1.0f, p2), T));
    float d = mul(w, sqrt64of32(w));
    return sub(0.0f, div(num, add(d, d)));
}

// ---------------------------------------------------------------------------
// Two cells per instruction. PTX add/sub/mul.rn.f32x2 (sm_100a) round each
// half exactly as __fadd_rn / __fsub_rn / __fmul_rn round it, subnormals
// kept (no .ftz), so a pair of cells taken through these has the scalar
// functions' bits in half the issue slots. The halves live in an aligned
// register pair: packing is free for fresh results and for neighbours
// loaded side by side, and reading a half back is free.
//
// One rule: a packed product never feeds a packed add or subtract. The
// assembler fuses that pair into one packed fused multiply-add (a single
// rounding) whatever the rounding modifiers and --fmad say, where a packed
// product summed half by half (add_p / sub_p), or scalar products summed
// packed, keep both roundings; a device check of 2^23 pairs per form
// showed the fused pair off in 5-18% of them and the split forms exact.

struct F2 {
    uint64_t r;
};
__device__ __forceinline__ F2 pk(float lo, float hi) {
    F2 p;
    asm("mov.b64 %0, {%1, %2};" : "=l"(p.r) : "f"(lo), "f"(hi));
    return p;
}
__device__ __forceinline__ F2 splat(float v) { return pk(v, v); }
__device__ __forceinline__ float lo(F2 p) { return __uint_as_float((uint32_t)p.r); }
__device__ __forceinline__ float hi(F2 p) { return __uint_as_float((uint32_t)(p.r >> 32)); }
__device__ __forceinline__ F2 add2(F2 a, F2 b) {
    F2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d.r) : "l"(a.r), "l"(b.r));
    return d;
}
__device__ __forceinline__ F2 sub2(F2 a, F2 b) {
    F2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d.r) : "l"(a.r), "l"(b.r));
    return d;
}
__device__ __forceinline__ F2 mul2(F2 a, F2 b) {
    F2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d.r) : "l"(a.r), "l"(b.r));
    return d;
}
// a + b and a - b half by half: the sums with a packed product among
// their operands.
__device__ __forceinline__ F2 add_p(F2 a, F2 b) { return pk(add(lo(a), lo(b)), add(hi(a), hi(b))); }
__device__ __forceinline__ F2 sub_p(F2 a, F2 b) { return pk(sub(lo(a), lo(b)), sub(hi(a), hi(b))); }

// atan32 over a pair: the same steps, the halves apart only for the
// argument reduction and the division. SKIP_SMALL: when no active lane of
// the warp holds an argument above tan(pi/8), every reduction is the
// identity, whose quotient x / 1 is x itself, so the warp skips the
// divisions (Slope's magnitudes on gentle terrain); the bits are the same.
template <bool SKIP_SMALL = false>
__device__ __forceinline__ F2 atan32x2(F2 x) {
    const float xs[2] = {lo(x), hi(x)};
    float t[2], y0[2];
    bool small = false;
    if constexpr (SKIP_SMALL) small = !__any_sync(__activemask(), xs[0] > kTanPi8 || xs[1] > kTanPi8);
    if (small) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            t[h] = xs[h];
            y0[h] = 0.0f;
        }
    } else {
        const F2 xm = sub2(x, splat(1.0f)), xp = add2(x, splat(1.0f));
        const float xms[2] = {lo(xm), hi(xm)}, xps[2] = {lo(xp), hi(xp)};
#pragma unroll
        for (int h = 0; h < 2; h++) {
            float num = xs[h], den = 1.0f;
            y0[h] = 0.0f;
            if (xs[h] > kTanPi8) {
                num = xms[h];
                den = xps[h];
                y0[h] = kPi4;
            }
            if (xs[h] > kTan3Pi8) {
                num = -1.0f;
                den = xs[h];
                y0[h] = kPi2;
            }
            t[h] = div(num, den);
        }
    }
    const F2 tt = pk(t[0], t[1]);
    const F2 z = mul2(tt, tt);
    F2 p = sub_p(mul2(splat(kC4), z), splat(kC3));
    p = add_p(mul2(p, z), splat(kC2));
    p = sub_p(mul2(p, z), splat(kC1));
    return add2(pk(y0[0], y0[1]), add_p(mul2(mul2(p, z), tt), tt));
}

// slope over a pair of gradients.
__device__ __forceinline__ F2 slope2(F2 gx, F2 gy, F2 scale, bool take_atan) {
    const F2 s = add_p(mul2(gx, gx), mul2(gy, gy));
    const F2 m = pk(sqrt64of32(lo(s)), sqrt64of32(hi(s)));
    return mul2(take_atan ? atan32x2<true>(m) : m, scale);
}

// aspect over a pair of gradients, atan2f32's steps inline. Its fix-up
// for two zero arguments is left out: when it applies, y and x are both
// zero and aspect's last step replaces the angle by the flat value.
__device__ __forceinline__ F2 aspect2(F2 gx, F2 gy, float flat, bool trig) {
    const F2 ngx = pk(sub(0.0f, lo(gx)), sub(0.0f, hi(gx)));
    const F2 y = trig ? gy : ngx, x = trig ? ngx : gy;
    const float ys[2] = {lo(y), hi(y)}, xs[2] = {lo(x), hi(x)};
    float ax[2], ay[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        ax[h] = abs32(xs[h]);
        ay[h] = abs32(ys[h]);
    }
    const F2 at = atan32x2(pk(div(ay[0], ax[0]), div(ay[1], ax[1])));
    const float ats[2] = {lo(at), hi(at)};
    float a[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        float v = ay[h] == ax[h] && ay[h] > 0x1.fffffep+127f ? kPi4 : ats[h];
        if (__float_as_uint(xs[h]) & 0x80000000u) v = sub(kPi, v);
        a[h] = __uint_as_float(__float_as_uint(v) | (__float_as_uint(ys[h]) & 0x80000000u));
    }
    F2 d = mul2(pk(a[0], a[1]), splat(kRadToDeg));
    const float ds[2] = {lo(d), hi(d)};
    d = add_p(d, pk(ds[0] < 0.0f ? 360.0f : 0.0f, ds[1] < 0.0f ? 360.0f : 0.0f));
    float r[2] = {lo(d), hi(d)};
#pragma unroll
    for (int h = 0; h < 2; h++) {
        if (r[h] >= 360.0f) r[h] = 0.0f;
        if (ys[h] == 0.0f && xs[h] == 0.0f) r[h] = flat;
    }
    return pk(r[0], r[1]);
}

// shade over a pair of gradients.
__device__ __forceinline__ F2 shade2(F2 gx, F2 gy, float c, float bx, float by) {
    const F2 num = add2(splat(c), add_p(mul2(splat(bx), gx), mul2(splat(by), gy)));
    const F2 s = add2(splat(1.0f), add_p(mul2(gx, gx), mul2(gy, gy)));
    float v[2] = {div(lo(num), sqrt64of32(lo(s))), div(hi(num), sqrt64of32(hi(s)))};
#pragma unroll
    for (int h = 0; h < 2; h++) {
        if (v[h] < 0.0f) v[h] = 0.0f;
        if (v[h] > 255.0f) v[h] = 255.0f;
    }
    return pk(v[0], v[1]);
}

// zt_curvature over a pair of cells, from the window sums and differences
// the caller forms: d64 = z6 - z4, d82 = z8 - z2, c = z5 + z5,
// s46 = z4 + z6, s28 = z2 + z8, s19 = z1 + z9, s37 = z3 + z7.
__device__ __forceinline__ F2 zt_curvature2(F2 d64, F2 d82, F2 c, F2 s46, F2 s28, F2 s19, F2 s37, const float* k,
                                            int kind) {
    const F2 P = mul2(d64, splat(k[0]));
    const F2 Q = mul2(d82, splat(k[1]));
    const F2 R = mul2(sub2(s46, c), splat(k[2]));
    const F2 T = mul2(sub2(s28, c), splat(k[3]));
    const F2 S = mul2(sub2(s19, s37), splat(k[4]));
    const F2 p2 = mul2(P, P), q2 = mul2(Q, Q);
    const F2 pq = mul2(P, Q);
    const F2 pq2 = add_p(pq, pq);
    const F2 one = splat(1.0f);
    float v[2];
    if (kind == 0) {
        const F2 g = add_p(p2, q2);
        const F2 w = add2(one, g);
        const F2 num = add_p(add_p(mul2(p2, R), mul2(pq2, S)), mul2(q2, T));
        const F2 den = mul2(w, pk(sqrt64of32(lo(w)), sqrt64of32(hi(w))));
        const F2 r = sub2(splat(0.0f), pk(div(div(lo(num), lo(g)), lo(den)), div(div(hi(num), hi(g)), hi(den))));
        v[0] = lo(g) == 0.0f ? add(lo(num), 0.0f) : lo(r);
        v[1] = hi(g) == 0.0f ? add(hi(num), 0.0f) : hi(r);
    } else if (kind == 1) {
        const F2 g = add_p(p2, q2);
        const F2 num = add_p(sub_p(mul2(q2, R), mul2(pq2, S)), mul2(p2, T));
        const F2 r = sub2(splat(0.0f), pk(div(div(lo(num), lo(g)), sqrt64of32(lo(g))),
                                          div(div(hi(num), hi(g)), sqrt64of32(hi(g)))));
        v[0] = lo(g) == 0.0f ? add(lo(num), 0.0f) : lo(r);
        v[1] = hi(g) == 0.0f ? add(hi(num), 0.0f) : hi(r);
    } else {
        const F2 w = add2(one, add_p(p2, q2));
        const F2 num = add_p(sub_p(mul2(add_p(one, q2), R), mul2(pq2, S)), mul2(add_p(one, p2), T));
        const F2 d = mul2(w, pk(sqrt64of32(lo(w)), sqrt64of32(hi(w))));
        const F2 dd = add_p(d, d);
        const F2 r = sub2(splat(0.0f), pk(div(lo(num), lo(dd)), div(hi(num), hi(dd))));
        v[0] = lo(r);
        v[1] = hi(r);
    }
    return pk(v[0], v[1]);
}

// heatLoad (internal/stencil/heatload.go:43-53): McCune and Keon's
// regression from the gradient, in float64 with every product rounded
// before it is added, rounded to float32 once. t: K0, A, BX, BY, E, F, CX,
// CY; with ex, exp of the sum (CUDA's exp, within one float64 ulp of
// Go's math.Exp: the float32 result differs only when the sum sits within
// that of a float32 rounding boundary).
__device__ __forceinline__ float heat_load(float gx, float gy, const double* t, bool ex) {
    const double dx = gx, dy = gy;
    const double g2 = __fma_rn(dx, dx, __dmul_rn(dy, dy));  // dx * dx exact (add_sq64)
    const double w = __ddiv_rn(1.0, __dsqrt_rn(__dadd_rn(1.0, g2)));
    const double fold = fabs(__dadd_rn(__dmul_rn(t[6], dx), __dmul_rn(t[7], dy)));
    double sum = __dadd_rn(t[1], __dmul_rn(t[2], dx));
    sum = __dadd_rn(sum, __dmul_rn(t[3], dy));
    sum = __dadd_rn(sum, __dmul_rn(t[4], __dsqrt_rn(g2)));
    sum = __dadd_rn(sum, __dmul_rn(t[5], fold));
    double v = __dadd_rn(t[0], __dmul_rn(w, sum));
    if (ex) v = exp(v);
    return __double2float_rn(v);
}

// orientation (internal/stencil/orientation.go:31-45): northness (gy) or
// eastness (-gx) over sqrt(1 + g2), or over sqrt(g2) unweighted with 0
// where flat, in float64, rounded to float32 once.
__device__ __forceinline__ float orientation(float gx, float gy, bool east, bool unweighted) {
    const double dx = gx, dy = gy;
    const double c = east ? -dx : dy;
    const double g2 = __fma_rn(dx, dx, __dmul_rn(dy, dy));  // dx * dx exact (add_sq64)
    if (!unweighted) return __double2float_rn(__ddiv_rn(c, __dsqrt_rn(__dadd_rn(1.0, g2))));
    if (g2 == 0) return 0.0f;
    return __double2float_rn(__ddiv_rn(c, __dsqrt_rn(g2)));
}

// The eight float64 terms of a heat-load launch, stored bit for bit in
// 16 float slots (low word first).
__device__ __forceinline__ void heat_terms(const float* w, double* t) {
#pragma unroll
    for (int i = 0; i < 8; i++) t[i] = __hiloint2double(__float_as_int(w[2 * i + 1]), __float_as_int(w[2 * i]));
}

__device__ __forceinline__ double sq64(float d) {
    double x = (double)d;
    return __dmul_rn(x, x);
}

// a + float64(d) * float64(d), each step rounded as the reference rounds
// it, in one fused multiply-add: the square of a float32 in float64 is
// exact (48 significant bits of 53; the float32 range squared stays within
// float64's normal range), so rounding the product first changes nothing
// and the one rounding of the sum is the reference's.
__device__ __forceinline__ double add_sq64(double a, float d) {
    const double x = (double)d;
    return __fma_rn(x, x, a);
}

// RuggednessRow at radius 1 (internal/stencil/rugged.go:70-103).
__device__ __forceinline__ float rugged3(float v1, float v2, float v3, float v4, float v5, float v6,
                                         float v7, float v8, float v9, int kind) {
    float c = v5;
    if (kind == 0) {
        double a = add_sq64(sq64(sub(v1, c)), sub(v2, c));
        a = add_sq64(a, sub(v3, c));
        a = add_sq64(a, sub(v4, c));
        a = add_sq64(a, sub(v6, c));
        a = add_sq64(a, sub(v7, c));
        a = add_sq64(a, sub(v8, c));
        a = add_sq64(a, sub(v9, c));
        return __double2float_rn(__dsqrt_rn(a));
    }
    if (kind == 1) {
        float a = add(abs32(sub(v1, c)), abs32(sub(v2, c)));
        a = add(a, abs32(sub(v3, c)));
        a = add(a, abs32(sub(v4, c)));
        a = add(a, abs32(sub(v6, c)));
        a = add(a, abs32(sub(v7, c)));
        a = add(a, abs32(sub(v8, c)));
        a = add(a, abs32(sub(v9, c)));
        return mul(a, 0.125f);
    }
    if (kind == 2) {
        float a = add(v1, v2);
        a = add(a, v3);
        a = add(a, v4);
        a = add(a, v6);
        a = add(a, v7);
        a = add(a, v8);
        a = add(a, v9);
        return sub(v5, mul(a, 0.125f));
    }
    float hi = go_max(go_max(go_max(go_max(v1, v2), go_max(v3, v4)), go_max(go_max(v5, v6), go_max(v7, v8))), v9);
    float lo = go_min(go_min(go_min(go_min(v1, v2), go_min(v3, v4)), go_min(go_min(v5, v6), go_min(v7, v8))), v9);
    return sub(hi, lo);
}

// rugged3's roughness for four adjacent cells from their window rows a, b,
// c (six columns each): the maximum and minimum of each column over the
// three rows first, then of three adjacent columns per cell. Go's min and
// max (min.NaN / max.NaN) are exactly associative and commutative, so the
// regrouping keeps rugged3's bits, in 44 operations instead of 68.
__device__ __forceinline__ void roughness4(const float (&a)[6], const float (&b)[6], const float (&c)[6],
                                           float (&o)[4]) {
    float hi[6], lo[6];
#pragma unroll
    for (int j = 0; j < 6; j++) {
        hi[j] = go_max(go_max(a[j], b[j]), c[j]);
        lo[j] = go_min(go_min(a[j], b[j]), c[j]);
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
        o[i] = sub(go_max(go_max(hi[i], hi[i + 1]), hi[i + 2]), go_min(go_min(lo[i], lo[i + 1]), lo[i + 2]));
}

// The reference's table index, k = the first j with v < xs[j] (or n):
// for strictly increasing, NaN-free knots and a non-NaN v that is the
// number of knots at or below v, which this counts without branches. The
// engine rejects tables that are not strictly increasing.
__device__ __forceinline__ int knots_at_or_below(float v, const float* xs, int n) {
    int k = 0;
    for (int j = 0; j < n; j++) k += xs[j] <= v ? 1 : 0;
    return k;
}

// scalarLookupFloat32 (internal/curve/scalar.go:84-114): NaN passes
// through, the ends clamp, a cell on a knot takes the knot's y, and
// elsewhere y0 + float32(t * (y1 - y0)) with t = (v - x0) / (x1 - x0).
__device__ __forceinline__ float lookup(float v, const float* xs, const float* ys, int n) {
    const int k = knots_at_or_below(v, xs, n);
    const int lo = k == 0 ? 0 : k - 1;
    const int hi = k == n ? n - 1 : k;
    const float x0 = xs[lo], y0 = ys[lo];
    const float t = div(sub(v, x0), sub(xs[hi], x0));
    float r = add(y0, mul(t, sub(ys[hi], y0)));
    r = v == x0 ? y0 : r;
    r = k == n ? ys[n - 1] : r;
    r = k == 0 ? ys[0] : r;
    return v != v ? v : r;
}

// scalarReclassFloat32 (internal/curve/scalar.go:39-60): values[k] for k
// the number of breaks at or below v; NaN passes through.
__device__ __forceinline__ float reclass(float v, const float* breaks, int nb, const float* values) {
    const float r = values[knots_at_or_below(v, breaks, nb)];
    return v != v ? v : r;
}

// One vec.Chain step (internal/vec/chain.go:24-38, the scalar kernels of
// internal/vec/scalar.go): acc is the running value, b the binary ops'
// second operand, k0 and k1 the immediates. Every operation is rounded
// on its own (Affine's multiply and add are two roundings, no FMA).
__device__ __forceinline__ float vec_step(int op, float acc, float b, float k0, float k1) {
    switch (op) {
    case STRATA_VEC_ADD: return add(acc, b);
    case STRATA_VEC_SUB: return sub(acc, b);
    case STRATA_VEC_MUL: return mul(acc, b);
    case STRATA_VEC_DIV: return div(acc, b);
    case STRATA_VEC_MIN: return go_min(acc, b);
    case STRATA_VEC_MAX: return go_max(acc, b);
    case STRATA_VEC_ADD_SCALAR: return add(acc, k0);
    case STRATA_VEC_MUL_SCALAR: return mul(acc, k0);
    case STRATA_VEC_AFFINE: return add(mul(acc, k0), k1);
    case STRATA_VEC_SUB_DIV: return div(sub(acc, k0), k1);
    case STRATA_VEC_CLAMP: return go_min(go_max(acc, k0), k1);
    case STRATA_VEC_ABS: return abs32(acc);
    default: return sqrt64of32(acc);  // STRATA_VEC_SQRT
    }
}

}  // namespace cell
}  // namespace strata
