/*
 * strata_oracle.c - TEST INFRASTRUCTURE ONLY: the parity oracle.
 *
 * A plain-C restatement of strata's canonical scalar backend for the
 * raster-stencil path (Horn gradient/slope/aspect/hillshade,
 * Zevenbergen-Thorne curvature, ruggedness, focal correlate / separable /
 * mean / min / max, Lookup / Reclass), and of the engine rules around it
 * (edge ring, validity erosion). Each function cites the reference file
 * and lines it restates, by path within the strata project.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline and
 * reference arm may load this code, and only as the checker or as the
 * timed CPU baseline. The CUDA product never calls it.
 *
 * Build with -ffp-contract=off and without -ffast-math: every float
 * operation below must round on its own, as the reference's explicit
 * float32(...) conversions force in Go.
 */
#include "strata_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------------- */
/* Bits and Go's builtin min / max.                                        */

static inline uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

/* Go's builtin min and max on float32 (the language spec, "Min and max"):
 * a NaN argument gives NaN, and -0 orders below +0. The reference's
 * focal and roughness folds rely on exactly this
 * (internal/focalrow/focalrow.go:22-25). */
float orc_go_min(float a, float b)
{
    if (a != a) return a;
    if (b != b) return b;
    if (a == b) return u2f(f2u(a) | f2u(b)); /* -0 if either is -0 */
    return a < b ? a : b;
}

float orc_go_max(float a, float b)
{
    if (a != a) return a;
    if (b != b) return b;
    if (a == b) return u2f(f2u(a) & f2u(b)); /* +0 if either is +0 */
    return a > b ? a : b;
}

/* ---------------------------------------------------------------------- */
/* Arctangents: internal/stencil/horn.go:224-262, aspect.go:10-47.         */

/* float32 constants of horn.go:226-235 and aspect.go:10-14, each the
 * correctly rounded float32 of the reference's constant expression. */
#define ATAN_TAN3PI8 0x1.3504f4p+1f  /* float32(2.414213562373095)  */
#define ATAN_TANPI8  0x1.a8279ap-2f  /* float32(0.4142135623730950) */
#define ATAN_PI2     0x1.921fb6p+0f  /* float32(math.Pi / 2)        */
#define ATAN_PI4     0x1.921fb6p-1f  /* float32(math.Pi / 4)        */
#define ATAN_C4      0x1.49e1a2p-4f  /* float32(8.05374449538e-2)   */
#define ATAN_C3      0x1.1c370ap-3f  /* float32(1.38776856032e-1)   */
#define ATAN_C2      0x1.9924bep-3f  /* float32(1.99777106478e-1)   */
#define ATAN_C1      0x1.555454p-2f  /* float32(3.33329491539e-1)   */
#define ATAN2_PI     0x1.921fb6p+1f  /* float32(math.Pi)            */
#define RAD_TO_DEG   0x1.ca5dc2p+5f  /* float32(180 / math.Pi)      */

/* Atan32, horn.go:249-262: Cephes atanf with the argument reduced around
 * 0, pi/4 or pi/2, in that operation order. */
float orc_atan32(float x)
{
    float num = x, den = 1.0f, y0 = 0.0f;
    if (x > ATAN_TANPI8) {
        num = x - 1.0f;
        den = x + 1.0f;
        y0 = ATAN_PI4;
    }
    if (x > ATAN_TAN3PI8) {
        num = -1.0f;
        den = x;
        y0 = ATAN_PI2;
    }
    float t = num / den;
    float z = t * t;
    float p = ATAN_C4 * z - ATAN_C3;
    p = p * z + ATAN_C2;
    p = p * z - ATAN_C1;
    return y0 + ((p * z) * t + t);
}

/* Atan2F32, aspect.go:33-47. */
float orc_atan2f32(float y, float x)
{
    float ax = u2f(f2u(x) & 0x7fffffffu);
    float ay = u2f(f2u(y) & 0x7fffffffu);
    float a = orc_atan32(ay / ax);
    if (ay == 0.0f && ax == 0.0f) a = 0.0f;
    if (ay == ax && ay > 0x1.fffffep+127f) a = ATAN_PI4;
    if (f2u(x) & 0x80000000u) a = ATAN2_PI - a;
    return u2f(f2u(a) | (f2u(y) & 0x80000000u));
}

/* The number of non-negative floats x (0 < bits(x) <= bits(+Inf)) with
 * Atan32(x) < Atan32(the float just below x): 0 when Atan32 never falls
 * as its argument grows, which the device backend relies on to classify a
 * slope by its squared gradient magnitude. nthreads threads share the
 * 2^31 arguments. */
typedef struct { uint32_t lo, hi; int64_t drops; } mono_job;

static void *mono_worker(void *arg)
{
    mono_job *j = (mono_job *)arg;
    float prev = orc_atan32(u2f(j->lo - 1));
    for (uint32_t u = j->lo;; u++) {
        const float y = orc_atan32(u2f(u));
        if (y < prev) j->drops++;
        prev = y;
        if (u == j->hi) break;
    }
    return NULL;
}

int64_t orc_atan32_drops(int nthreads)
{
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    mono_job jobs[256];
    pthread_t tid[256];
    const uint32_t first = 1, last = 0x7f800000u;
    const uint32_t per = (last - first) / (uint32_t)nthreads + 1;
    int n = 0;
    for (uint32_t lo = first; n < nthreads && lo <= last; n++, lo += per) {
        jobs[n].lo = lo;
        jobs[n].hi = (last - lo < per - 1) ? last : lo + per - 1;
        jobs[n].drops = 0;
        pthread_create(&tid[n], NULL, mono_worker, &jobs[n]);
    }
    int64_t drops = 0;
    for (int i = 0; i < n; i++) {
        pthread_join(tid[i], NULL);
        drops += jobs[i].drops;
    }
    return drops;
}

void orc_atan32_array(const float *x, float *out, int64_t n)
{
    for (int64_t i = 0; i < n; i++) out[i] = orc_atan32(x[i]);
}

void orc_atan2f32_array(const float *y, const float *x, float *out, int64_t n)
{
    for (int64_t i = 0; i < n; i++) out[i] = orc_atan2f32(y[i], x[i]);
}

/* ---------------------------------------------------------------------- */
/* Host constants.                                                         */

/* HornScales, internal/stencil/horn.go:114-116. */
void orc_horn_scales(double cx, double cy, double z, float *kx, float *ky)
{
    *kx = (float)(z / (8 * cx));
    *ky = (float)(z / (8 * cy));
}

/* ZTScales, internal/stencil/curvature.go:29-33. */
void orc_zt_scales(double cx, double cy, double z, float out5[5])
{
    out5[0] = (float)(z / (2 * cx));
    out5[1] = (float)(z / (2 * cy));
    out5[2] = (float)(z / (cx * cx));
    out5[3] = (float)(z / (cy * cy));
    out5[4] = (float)(z / (4 * cx * cy));
}

/* hillshadeLight, terrain/hillshade.go:94-117 (after its checks). */
void orc_hillshade_light(double azimuth, double altitude, float out3[3])
{
    double az = azimuth, alt = altitude;
    if (az == 0) az = 315;
    if (alt == 0) alt = 45;
    az = fmod(az, 360);
    az = az * 3.141592653589793 / 180;
    alt = alt * 3.141592653589793 / 180;
    out3[0] = (float)(255 * sin(alt));
    out3[1] = (float)(-255 * cos(alt) * sin(az));
    out3[2] = (float)(255 * cos(alt) * cos(az));
}

/* Gaussian, focal/separable.go:59-76. */
void orc_gaussian(int radius, double sigma, float *taps)
{
    int n = 2 * radius + 1;
    double g[64];
    double sum = 0;
    for (int i = 0; i < n; i++) {
        double x = (double)(i - radius);
        g[i] = exp(-x * x / (2 * sigma * sigma));
        sum += g[i];
    }
    for (int i = 0; i < n; i++) taps[i] = (float)(g[i] / sum);
}

/* ---------------------------------------------------------------------- */
/* Horn 3x3 per-cell functions.                                            */

/* hornDX / hornDY, horn.go:152-160: opposite cells first (Sterbenz). */
static inline float horn_dx(float z1, float z3, float z4, float z6, float z7, float z9)
{
    float d = z6 - z4;
    return ((z3 - z1) + (z9 - z7)) + (d + d);
}

static inline float horn_dy(float z1, float z2, float z3, float z7, float z8, float z9)
{
    float d = z8 - z2;
    return ((z7 - z1) + (z9 - z3)) + (d + d);
}

/* magnitude, horn.go:220-222: the square root in float64 of the float32
 * sum, rounded once to float32. */
static inline float magnitude(float gx, float gy)
{
    return (float)sqrt((double)(gx * gx + gy * gy));
}

/* aspectDegrees, aspect.go:107-121. */
static inline float aspect_degrees(float y, float x, float flat)
{
    float d = orc_atan2f32(y, x) * RAD_TO_DEG;
    float off = 0.0f;
    if (d < 0) off = 360.0f;
    d += off;
    if (d >= 360.0f) d = 0.0f;
    if (y == 0.0f && x == 0.0f) d = flat;
    return d;
}

/* shade, aspect.go:162-173. */
static inline float shade(float gx, float gy, float c, float bx, float by)
{
    float num = c + (bx * gx + by * gy);
    float den = (float)sqrt((double)(1.0f + (gx * gx + gy * gy)));
    float v = num / den;
    if (v < 0) v = 0;
    if (v > 255) v = 255;
    return v;
}

/* ---------------------------------------------------------------------- */
/* Per-cell kernels over a window. p points at the window's centre cell;  */
/* cell (dx, dy) of the window is p[dy * s + dx].                          */

static inline float zt_finish(float P, float Q, float R, float S, float T, int kind);

/* ZT curvature, curvature.go:79-129. */
static inline float zt_curvature(const float *p, int64_t s, const float *k, int kind)
{
    float z1 = p[-s - 1], z2 = p[-s], z3 = p[-s + 1];
    float z4 = p[-1], z5 = p[0], z6 = p[1];
    float z7 = p[s - 1], z8 = p[s], z9 = p[s + 1];
    float kp = k[0], kq = k[1], kr = k[2], kt = k[3], ks = k[4];
    /* ztDerivs, curvature.go:79-87 */
    float P = (z6 - z4) * kp;
    float Q = (z8 - z2) * kq;
    float c = z5 + z5;
    float R = ((z4 + z6) - c) * kr;
    float T = ((z2 + z8) - c) * kt;
    float S = ((z1 + z9) - (z3 + z7)) * ks;
    return zt_finish(P, Q, R, S, T, kind);
}

/* CurvatureFromDerivsRow (internal/stencil/curvature.go:138-185): ZT's
 * formulas from derivatives already computed (ZTCurvatureRow's second
 * half, so a window's ztDerivs followed by this is ZTCurvatureRow). */
static inline float zt_finish(float P, float Q, float R, float S, float T, int kind)
{
    float p2 = P * P, q2 = Q * Q;
    float pq = P * Q;
    if (kind == 0) { /* profile, curvature.go:94-106 */
        float g = p2 + q2;
        float w = 1.0f + g;
        float num = (p2 * R + (pq + pq) * S) + q2 * T;
        float v = 0.0f - num / g / (w * (float)sqrt((double)w));
        if (g == 0.0f) v = num + 0.0f;
        return v;
    }
    if (kind == 1) { /* plan, curvature.go:107-118 */
        float g = p2 + q2;
        float num = (q2 * R - (pq + pq) * S) + p2 * T;
        float v = 0.0f - num / g / (float)sqrt((double)g);
        if (g == 0.0f) v = num + 0.0f;
        return v;
    }
    /* mean, curvature.go:119-127 */
    float w = 1.0f + (p2 + q2);
    float num = ((1.0f + q2) * R - (pq + pq) * S) + (1.0f + p2) * T;
    float d = w * (float)sqrt((double)w);
    return 0.0f - num / (d + d);
}

/* heatLoad (internal/stencil/heatload.go:43-53): McCune and Keon's
 * regression from a gradient, in float64 with every product rounded
 * before it is added, rounded to float32 once. t holds K0, A, BX, BY, E,
 * F, CX, CY. */
static inline float heat_load(float gx, float gy, const double *t, int exp_)
{
    const double dx = gx, dy = gy;
    const double g2 = dx * dx + dy * dy;
    const double w = 1.0 / sqrt(1.0 + g2);
    const double fold = fabs(t[6] * dx + t[7] * dy);
    const double sum = t[1] + t[2] * dx + t[3] * dy + t[4] * sqrt(g2) + t[5] * fold;
    double v = t[0] + w * sum;
    if (exp_) v = exp(v);
    return (float)v;
}

/* orientation (internal/stencil/orientation.go:31-45): northness (gy) or
 * eastness (-gx) over sqrt(1 + g2), or over sqrt(g2) unweighted (0 when
 * flat), in float64, rounded to float32 once. */
static inline float orientation(float gx, float gy, int east, int unweighted)
{
    const double dx = gx, dy = gy;
    const double c = east ? -dx : dy;
    const double g2 = dx * dx + dy * dy;
    if (!unweighted) return (float)(c / sqrt(1.0 + g2));
    if (g2 == 0) return 0.0f;
    return (float)(c / sqrt(g2));
}

/* The 8 float64 terms of a heat load stage, from its table's raw bits. */
static inline void heat_terms(const orc_stage *st, double *t)
{
    memcpy(t, st->table[0], 8 * sizeof(double));
}

/* Wood's quadratic fit (terrain/fit.go:111-170): the derivatives of the
 * (2r+1)^2 window around p by the column folds ColumnSum and
 * ColumnCorrelate (top to bottom) and the row fold RowCorrelate (left to
 * right) with the integer taps i and 3i^2 - r(r+1), each scaled by its
 * factor (internal/focalrow/focalrow.go:214-263). want_curv also forms r,
 * s and t. */
static void wood_derivs(const float *p, int64_t s, int r, const float *k, int want_curv, float *d)
{
    float cs[2 * 8 + 1], cj[2 * 8 + 1], ct[2 * 8 + 1];
    const float q1 = (float)(r * (r + 1));
    for (int c = -r; c <= r; c++) {
        float sum = p[-r * s + c];
        float cor = (float)(-r) * p[-r * s + c];
        float co2 = (3.0f * (float)(r * r) - q1) * p[-r * s + c];
        for (int j = -r + 1; j <= r; j++) {
            const float v = p[j * s + c];
            sum = sum + v;
            cor = cor + (float)j * v;
            co2 = co2 + ((float)(3 * j * j) - q1) * v;
        }
        cs[c + r] = sum;
        cj[c + r] = cor;
        ct[c + r] = co2;
    }
    /* RowCorrelate from the first product */
    float P = (float)(-r) * cs[0], Q = 1.0f * cj[0];
    for (int c = 1; c <= 2 * r; c++) {
        P = P + (float)(c - r) * cs[c];
        Q = Q + 1.0f * cj[c];
    }
    d[0] = P * k[0];
    d[1] = Q * k[1];
    if (!want_curv) return;
    float R = (3.0f * (float)(r * r) - q1) * cs[0], T = 1.0f * ct[0], S = (float)(-r) * cj[0];
    for (int c = 1; c <= 2 * r; c++) {
        const int i = c - r;
        R = R + ((float)(3 * i * i) - q1) * cs[c];
        T = T + 1.0f * ct[c];
        S = S + (float)i * cj[c];
    }
    d[2] = R * k[2];
    d[3] = S * k[4];
    d[4] = T * k[3];
}

static inline double sq64(float d) { double x = (double)d; return x * x; }
static inline float abs32(float x) { return u2f(f2u(x) & 0x7fffffffu); }

/* RuggednessRow at r = 1, rugged.go:70-103. */
static inline float rugged3(const float *p, int64_t s, int kind)
{
    float v1 = p[-s - 1], v2 = p[-s], v3 = p[-s + 1];
    float v4 = p[-1], v5 = p[0], v6 = p[1];
    float v7 = p[s - 1], v8 = p[s], v9 = p[s + 1];
    float c = v5;
    switch (kind) {
    case 0: {
        double a = sq64(v1 - c) + sq64(v2 - c);
        a += sq64(v3 - c);
        a += sq64(v4 - c);
        a += sq64(v6 - c);
        a += sq64(v7 - c);
        a += sq64(v8 - c);
        a += sq64(v9 - c);
        return (float)sqrt(a);
    }
    case 1: {
        float a = abs32(v1 - c) + abs32(v2 - c);
        a += abs32(v3 - c);
        a += abs32(v4 - c);
        a += abs32(v6 - c);
        a += abs32(v7 - c);
        a += abs32(v8 - c);
        a += abs32(v9 - c);
        return a * 0.125f;
    }
    case 2: {
        float a = v1 + v2;
        a += v3;
        a += v4;
        a += v6;
        a += v7;
        a += v8;
        a += v9;
        return v5 - a * 0.125f;
    }
    default: {
        float hi = v1, lo = v1;
        const float v[8] = {v2, v3, v4, v5, v6, v7, v8, v9};
        for (int i = 0; i < 8; i++) {
            hi = orc_go_max(hi, v[i]);
            lo = orc_go_min(lo, v[i]);
        }
        return hi - lo;
    }
    }
}

/* RuggednessWindowRow for r > 1, rugged.go:152-210, and the separable
 * roughness of terrain/ruggedness.go:185-203 (max and min are order-free,
 * so one fold over the window gives the same bits). */
static inline float rugged_window(const float *p, int64_t s, int r, int kind)
{
    int d = 2 * r + 1;
    float n = (float)(d * d - 1);
    float c = p[0];
    if (kind == 3) {
        float hi = p[-r * s - r], lo = hi;
        for (int j = -r; j <= r; j++)
            for (int k = -r; k <= r; k++) {
                float v = p[j * s + k];
                hi = orc_go_max(hi, v);
                lo = orc_go_min(lo, v);
            }
        return hi - lo;
    }
    if (kind == 0) {
        double a = 0;
        for (int j = -r; j <= r; j++)
            for (int k = -r; k <= r; k++) {
                if (j == 0 && k == 0) continue;
                a += sq64(p[j * s + k] - c);
            }
        return (float)sqrt(a);
    }
    if (kind == 1) {
        float a = 0.0f;
        for (int j = -r; j <= r; j++)
            for (int k = -r; k <= r; k++) {
                if (j == 0 && k == 0) continue;
                a += abs32(p[j * s + k] - c);
            }
        return a / n;
    }
    /* TPI: the sum starts from the first neighbour's value. */
    float a = 0.0f;
    int first = 1;
    for (int j = -r; j <= r; j++)
        for (int k = -r; k <= r; k++) {
            if (j == 0 && k == 0) continue;
            if (first) {
                a = p[j * s + k];
                first = 0;
            } else {
                a += p[j * s + k];
            }
        }
    return c - a / n;
}

/* CorrelateRow, internal/focalrow/focalrow.go:217-230 with mulRow and
 * mulAddRow (:339-379): the first product, then each later product added
 * in row-major order of the weights, zero weights included. */
static inline float correlate(const float *p, int64_t s, int r, const float *w)
{
    int k = 2 * r + 1;
    const float *q = p - r * s - r;
    float acc = w[0] * q[0];
    for (int j = 0; j < k; j++)
        for (int c = 0; c < k; c++) {
            if (j == 0 && c == 0) continue;
            acc = acc + w[j * k + c] * q[j * s + c];
        }
    return acc;
}

/* ColumnCorrelate then RowCorrelate, focalrow.go:232-242 and :274-284:
 * the column pass folds the 2r+1 rows of each column from its first
 * product; the row pass folds 2r+1 column results the same way. */
static inline float separable(const float *p, int64_t s, int r, const float *row, const float *col)
{
    int k = 2 * r + 1;
    const float *q = p - r * s - r;
    float out = 0.0f;
    for (int c = 0; c < k; c++) {
        float tmp = col[0] * q[c];
        for (int j = 1; j < k; j++) tmp = tmp + col[j] * q[j * s + c];
        if (c == 0) out = row[0] * tmp;
        else out = out + row[c] * tmp;
    }
    return out;
}

/* ColumnSum then RowMean, focalrow.go:244-250, :286-293 and divRow
 * :406-421: sums from the first value, then a division by (2r+1)^2. */
static inline float box_mean(const float *p, int64_t s, int r)
{
    int k = 2 * r + 1;
    const float *q = p - r * s - r;
    float out = 0.0f;
    for (int c = 0; c < k; c++) {
        float tmp = q[c];
        for (int j = 1; j < k; j++) tmp += q[j * s + c];
        if (c == 0) out = tmp;
        else out += tmp;
    }
    return out / (float)(k * k);
}

/* ColumnMin/Max then RowMin/Max, focalrow.go:252-272, :295-315. */
static inline float box_minmax(const float *p, int64_t s, int r, int is_max)
{
    int k = 2 * r + 1;
    const float *q = p - r * s - r;
    float out = 0.0f;
    for (int c = 0; c < k; c++) {
        float tmp = q[c];
        for (int j = 1; j < k; j++)
            tmp = is_max ? orc_go_max(tmp, q[j * s + c]) : orc_go_min(tmp, q[j * s + c]);
        if (c == 0) out = tmp;
        else out = is_max ? orc_go_max(out, tmp) : orc_go_min(out, tmp);
    }
    return out;
}

/* scalarLookupFloat32, internal/curve/scalar.go:84-114. */
static inline float lookup(float v, const float *xs, const float *ys, int n)
{
    if (v != v) return v;
    int k = n;
    for (int j = 0; j < n; j++)
        if (v < xs[j]) {
            k = j;
            break;
        }
    if (k == 0) return ys[0];
    if (k == n) return ys[n - 1];
    float x0 = xs[k - 1], y0 = ys[k - 1];
    if (v == x0) return y0;
    float t = (v - x0) / (xs[k] - x0);
    return y0 + t * (ys[k] - y0);
}

/* scalarReclassFloat32, internal/curve/scalar.go:39-60. */
static inline float reclass(float v, const float *breaks, int nb, const float *values)
{
    if (v != v) return v;
    int k = nb;
    for (int j = 0; j < nb; j++)
        if (v < breaks[j]) {
            k = j;
            break;
        }
    return values[k];
}

/* One vec.Chain step (internal/vec/chain.go:24-38, the scalar kernels
 * of internal/vec/scalar.go:1-120): acc the running value, b the binary
 * ops' second operand. Each operation rounds on its own (no FMA). */
static inline float vec_step(int op, float acc, float b, float k0, float k1)
{
    switch (op) {
    case 0: return acc + b;
    case 1: return acc - b;
    case 2: return acc * b;
    case 3: return acc / b;
    case 4: return orc_go_min(acc, b);
    case 5: return orc_go_max(acc, b);
    case 6: return acc + k0;
    case 7: return acc * k0;
    case 8: { float t = acc * k0; return t + k1; }   /* Affine: float32(v*a) + b */
    case 9: { float t = acc - k0; return t / k1; }   /* SubDiv: (v - lo) / span */
    case 10: return orc_go_min(orc_go_max(acc, k0), k1);
    case 11: return u2f(f2u(acc) & 0x7fffffffu);      /* Abs: the sign bit cleared */
    default: return (float)sqrt((double)acc);         /* Sqrt */
    }
}

static inline int step_binary(const orc_stage *st) { return st->op == ORC_STEP && st->kind >= 0 && st->kind <= 5; }

static inline float pointwise(const orc_stage *st, float v)
{
    if (st->op == ORC_STEP) return vec_step(st->kind, v, 0.0f, st->k[0], st->k[1]);
    if (st->op == ORC_LOOKUP) return lookup(v, st->table[0], st->table[1], st->table_len[0]);
    return reclass(v, st->table[0], st->table_len[0], st->table[1]);
}

/* One stencil cell: writes out[0] (and out[1] for the gradient). */
static inline void stencil_cell(const orc_stage *st, const float *p, int64_t s, float *out)
{
    const float *k = st->k;
    if (st->flags & ORC_STAGE_FIT) {
        /* fitKernel.Process (terrain/fit.go:111-170): the fit's gradient
         * (p, q) into the from-gradient finishers, or p..t into ZT's
         * curvature formulas. Constants: k[0..4] the fit's factors, then
         * the product's (slope scale, aspect flat, hillshade c, bx, by). */
        float d[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        wood_derivs(p, s, st->radius, k, st->op == ORC_CURVATURE, d);
        const float gx = d[0], gy = d[1];
        switch (st->op) {
        case ORC_GRADIENT: out[0] = gx; out[1] = gy; return;
        case ORC_SLOPE: out[0] = (st->kind ? orc_atan32(magnitude(gx, gy)) : magnitude(gx, gy)) * k[5]; return;
        case ORC_ASPECT:
            out[0] = st->kind ? aspect_degrees(gy, 0.0f - gx, k[5]) : aspect_degrees(0.0f - gx, gy, k[5]);
            return;
        case ORC_HILLSHADE: out[0] = shade(gx, gy, k[5], k[6], k[7]); return;
        case ORC_HEATLOAD: {
            double t[8];
            heat_terms(st, t);
            out[0] = heat_load(gx, gy, t, st->kind & 1);
            return;
        }
        case ORC_ORIENTATION: out[0] = orientation(gx, gy, st->kind & 1, (st->kind >> 1) & 1); return;
        default: out[0] = zt_finish(d[0], d[1], d[2], d[3], d[4], st->kind); return;
        }
    }
    switch (st->op) {
    case ORC_HEATLOAD:
    case ORC_ORIENTATION: {
        /* heatLoadKernel / orientationKernel (terrain/heatload.go:147-160,
         * terrain/orientation.go:83-95): Horn's gradient, then the
         * from-gradient equation. */
        float z1 = p[-s - 1], z2 = p[-s], z3 = p[-s + 1];
        float z4 = p[-1], z6 = p[1];
        float z7 = p[s - 1], z8 = p[s], z9 = p[s + 1];
        float gx = horn_dx(z1, z3, z4, z6, z7, z9) * k[0];
        float gy = horn_dy(z1, z2, z3, z7, z8, z9) * k[1];
        if (st->op == ORC_HEATLOAD) {
            double t[8];
            heat_terms(st, t);
            out[0] = heat_load(gx, gy, t, st->kind & 1);
        } else {
            out[0] = orientation(gx, gy, st->kind & 1, (st->kind >> 1) & 1);
        }
        return;
    }
    case ORC_GRADIENT:
    case ORC_SLOPE:
    case ORC_ASPECT:
    case ORC_HILLSHADE: {
        float z1 = p[-s - 1], z2 = p[-s], z3 = p[-s + 1];
        float z4 = p[-1], z6 = p[1];
        float z7 = p[s - 1], z8 = p[s], z9 = p[s + 1];
        float gx = horn_dx(z1, z3, z4, z6, z7, z9) * k[0];
        float gy = horn_dy(z1, z2, z3, z7, z8, z9) * k[1];
        if (st->op == ORC_GRADIENT) { /* scalarHornGradientRow, horn.go:176-187 */
            out[0] = gx;
            out[1] = gy;
        } else if (st->op == ORC_SLOPE) { /* scalarHornSlopeRow, horn.go:193-216 */
            if (st->kind) out[0] = orc_atan32(magnitude(gx, gy)) * k[2];
            else out[0] = magnitude(gx, gy) * k[2];
        } else if (st->op == ORC_ASPECT) { /* aspectArgs + aspectDegrees, aspect.go:80-121 */
            float y, x;
            if (st->kind) {
                y = gy;
                x = 0.0f - gx;
            } else {
                y = 0.0f - gx;
                x = gy;
            }
            out[0] = aspect_degrees(y, x, k[2]);
        } else { /* scalarHornHillshadeRow, aspect.go:148-160 */
            out[0] = shade(gx, gy, k[2], k[3], k[4]);
        }
        return;
    }
    case ORC_CURVATURE:
        out[0] = zt_curvature(p, s, k, st->kind);
        return;
    case ORC_RUGGEDNESS:
        out[0] = st->radius == 1 ? rugged3(p, s, st->kind) : rugged_window(p, s, st->radius, st->kind);
        return;
    case ORC_CORRELATE:
        out[0] = correlate(p, s, st->radius, st->table[0]);
        return;
    case ORC_SEPARABLE:
        out[0] = separable(p, s, st->radius, st->table[0], st->table[1]);
        return;
    case ORC_MEAN:
        out[0] = box_mean(p, s, st->radius);
        return;
    case ORC_MIN:
        out[0] = box_minmax(p, s, st->radius, 0);
        return;
    case ORC_MAX:
        out[0] = box_minmax(p, s, st->radius, 1);
        return;
    }
}

/* ---------------------------------------------------------------------- */
/* The engine's rules: internal/exec/halo.go:21-92 (interior and edge    */
/* ring), :161-229 (validity), and pointwise validity                     */
/* (internal/pointwise UnaryValidity).                                    */

static inline int get_bit(const uint64_t *m, int64_t i) { return (int)((m[i >> 6] >> (i & 63)) & 1u); }

typedef struct {
    const orc_stage *stages;
    int nstages;
    const orc_raster *src;
    const orc_raster *srcs; /* a pointwise pipeline's inputs (src is srcs[0]) */
    int nsrc;
    const orc_raster *dst;
    int ndst;
    int r;
    int64_t band_rows;
    int64_t nbands;
    int64_t next; /* atomic band counter */
    int simd;     /* run the radius-1 stencils' rows through the restated AVX2 lanes (strata_avx2.c) */
} job_t;

/* The interior cells [x0, x1) of one row, with the op chosen once per
 * row so the cell loops stay tight for the timed CPU baseline. */
#define ROW_LOOP(expr)                                                  \
    for (int64_t x = x0; x < x1; x++) {                                 \
        const float *p = row + x;                                       \
        o0[x] = (expr);                                                 \
    }

static void stencil_row(const orc_stage *st, const float *row, int64_t s, int64_t x0, int64_t x1,
                        float *o0, float *o1)
{
    const float *k = st->k;
    int r = st->radius;
    if (st->flags & ORC_STAGE_FIT) { /* Wood's fit: cell by cell */
        for (int64_t x = x0; x < x1; x++) {
            float out[2];
            stencil_cell(st, row + x, s, out);
            o0[x] = out[0];
            if (o1) o1[x] = out[1];
        }
        return;
    }
    switch (st->op) {
    case ORC_GRADIENT:
        for (int64_t x = x0; x < x1; x++) {
            float out[2];
            stencil_cell(st, row + x, s, out);
            o0[x] = out[0];
            o1[x] = out[1];
        }
        return;
    case ORC_SLOPE:
        if (st->kind) {
            ROW_LOOP(orc_atan32(magnitude(horn_dx(p[-s - 1], p[-s + 1], p[-1], p[1], p[s - 1], p[s + 1]) * k[0],
                                          horn_dy(p[-s - 1], p[-s], p[-s + 1], p[s - 1], p[s], p[s + 1]) * k[1])) *
                     k[2]);
        } else {
            ROW_LOOP(magnitude(horn_dx(p[-s - 1], p[-s + 1], p[-1], p[1], p[s - 1], p[s + 1]) * k[0],
                               horn_dy(p[-s - 1], p[-s], p[-s + 1], p[s - 1], p[s], p[s + 1]) * k[1]) *
                     k[2]);
        }
        return;
    case ORC_CURVATURE:
        ROW_LOOP(zt_curvature(p, s, k, st->kind));
        return;
    case ORC_RUGGEDNESS:
        if (r == 1) {
            ROW_LOOP(rugged3(p, s, st->kind));
        } else {
            ROW_LOOP(rugged_window(p, s, r, st->kind));
        }
        return;
    case ORC_CORRELATE:
        ROW_LOOP(correlate(p, s, r, st->table[0]));
        return;
    case ORC_SEPARABLE:
        ROW_LOOP(separable(p, s, r, st->table[0], st->table[1]));
        return;
    case ORC_MEAN:
        ROW_LOOP(box_mean(p, s, r));
        return;
    case ORC_MIN:
        ROW_LOOP(box_minmax(p, s, r, 0));
        return;
    case ORC_MAX:
        ROW_LOOP(box_minmax(p, s, r, 1));
        return;
    default:
        for (int64_t x = x0; x < x1; x++) {
            float out[2];
            stencil_cell(st, row + x, s, out);
            o0[x] = out[0];
        }
        return;
    }
}

/* The baseline's validity of one output row at word level, as the
 * reference's engine computes it (internal/stencil/mask.go:55-82, ErodeBox
 * and shrink2Row): the AND of the 2r+1 source rows' words, shrunk by 2r
 * cells with shifted copies, the edge ring's cells cleared, and the row's
 * W bits deposited at the destination's offset (atomically only in words
 * shared with other rows). acc and out hold (W + 63) / 64 + 1 words. The
 * bits equal run_rows's cell-by-cell validity. */
static void validity_row_words(const job_t *jb, const orc_raster *D, int64_t y, uint64_t *acc, uint64_t *out)
{
    const orc_raster *src = jb->src;
    const int64_t W = src->width, H = src->height, s = src->stride;
    const int r = jb->r;
    const int64_t nw = (W + 63) >> 6;
    const int yin = y >= r && y < H - r;
    for (int64_t k = 0; k <= nw; k++) out[k] = 0;
    if (yin && W > 2 * r) {
        for (int64_t k = 0; k <= nw; k++) acc[k] = ~(uint64_t)0;
        if (src->valid)
            for (int j = -r; j <= r; j++) {
                const int64_t off = src->valid_offset + (y + j) * s;
                const int64_t last = (off + W - 1) >> 6;
                for (int64_t k = 0; k < nw; k++) {
                    const int64_t b = off + 64 * k, w = b >> 6;
                    const int sh = (int)(b & 63);
                    uint64_t v = src->valid[w] >> sh;
                    if (sh && w + 1 <= last) v |= src->valid[w + 1] << (64 - sh);
                    acc[k] &= v;
                }
            }
        if (W & 63) acc[nw - 1] &= ((uint64_t)1 << (W & 63)) - 1;
        acc[nw] = 0;
        /* e bit x: the AND of acc bits x .. x + 2r; the output cell x + r. */
        for (int64_t k = 0; k < nw; k++) {
            uint64_t e = acc[k];
            for (int d = 1; d <= 2 * r; d++) e &= (acc[k] >> d) | (acc[k + 1] << (64 - d));
            out[k] = e;
        }
        /* shift up by r into column positions, then keep columns r .. W-r-1 */
        for (int64_t k = nw; k > 0; k--) out[k] = (out[k] << r) | (out[k - 1] >> (64 - r));
        out[0] <<= r;
        for (int64_t x = 0; x < r; x++) out[x >> 6] &= ~((uint64_t)1 << (x & 63));
        for (int64_t x = W - r; x < W; x++) out[x >> 6] &= ~((uint64_t)1 << (x & 63));
    }
    /* deposit W bits at D's offset for row y */
    const int64_t base = D->valid_offset + y * D->stride;
    int64_t x = 0;
    while (x < W) {
        const int64_t b = base + x;
        const int sh = (int)(b & 63);
        int64_t take = 64 - sh;
        if (take > W - x) take = W - x;
        const int64_t k = x >> 6, o = x & 63;
        uint64_t v = out[k] >> o;
        if (o && k + 1 <= nw) v |= out[k + 1] << (64 - o);
        if (take < 64) v &= ((uint64_t)1 << take) - 1;
        const uint64_t bits = v << sh;
        const uint64_t own = take == 64 ? ~(uint64_t)0 : ((((uint64_t)1 << take) - 1) << sh);
        uint64_t *w = &D->valid[b >> 6];
        if (own == ~(uint64_t)0) {
            *w = bits;
        } else {
            __atomic_fetch_and(w, ~own | bits, __ATOMIC_RELAXED);
            __atomic_fetch_or(w, bits, __ATOMIC_RELAXED);
        }
        x += take;
    }
}

static void run_rows(const job_t *jb, int64_t y0, int64_t y1, unsigned char *colok)
{
    const orc_raster *src = jb->src;
    const orc_stage *st = &jb->stages[0];
    int64_t W = src->width, H = src->height, s = src->stride;
    int r = jb->r;
    const float nanf_ = u2f(0x7fc00000u);
    int stencil = !(st->op == ORC_LOOKUP || st->op == ORC_RECLASS || st->op == ORC_STEP);
    for (int64_t y = y0; y < y1; y++) {
        float *o0 = jb->dst[0].data + y * jb->dst[0].stride;
        float *o1 = jb->ndst > 1 ? jb->dst[1].data + y * jb->dst[1].stride : NULL;
        const float *row = src->data + y * s;
        int yin = y >= r && y < H - r;
        if (!stencil) {
            for (int64_t x = 0; x < W; x++) {
                float v = row[x];
                for (int i = 0; i < jb->nstages; i++) {
                    const orc_stage *p = &jb->stages[i];
                    if (step_binary(p)) {
                        const orc_raster *b = &jb->srcs[p->input];
                        v = vec_step(p->kind, v, b->data[y * b->stride + x], 0.0f, 0.0f);
                    } else {
                        v = pointwise(p, v);
                    }
                }
                o0[x] = v;
            }
        } else {
            /* Edge ring first, then the interior. */
            int64_t x0 = yin ? r : W, x1 = yin ? W - r : W;
            if (x1 < x0) x1 = x0;
            for (int64_t x = 0; x < W; x++) {
                if (x >= x0 && x < x1) continue;
                o0[x] = nanf_;
                if (o1) o1[x] = nanf_;
            }
            if (x0 < x1) {
                int64_t xs = x0;
                if (jb->simd && r == 1)
                    xs += orc_avx2_row(st, o0 + x0, o1 ? o1 + x0 : NULL, row - s + x0 - 1, row + x0 - 1,
                                       row + s + x0 - 1, x1 - x0);
                if (xs < x1) stencil_row(st, row, s, xs, x1, o0, o1);
                for (int i = 1; i < jb->nstages; i++)
                    for (int64_t x = x0; x < x1; x++) o0[x] = pointwise(&jb->stages[i], o0[x]);
            }
        }
        /* Validity of row y: built in vbuf, then stored a word at a time
         * (atomically only where a word is shared with another row). */
        for (int d = 0; d < jb->ndst; d++) {
            const orc_raster *D = &jb->dst[d];
            if (!D->valid) continue;
            if (jb->simd && stencil && r >= 1 && r < 64) {
                uint64_t *acc = (uint64_t *)(colok + 3 * W + 72 - ((uintptr_t)(colok + 3 * W + 64) & 7));
                validity_row_words(jb, D, y, acc, acc + ((W + 63) >> 6) + 1);
                continue;
            }
            unsigned char *vbuf = colok + W + 1;
            if (!stencil) {
                /* halo.go:213-229 at reach 0: every masked input's bit */
                for (int64_t x = 0; x < W; x++) {
                    int ok = 1;
                    for (int j = 0; j < jb->nsrc; j++) {
                        const orc_raster *in = &jb->srcs[j];
                        if (in->valid) ok &= get_bit(in->valid, in->valid_offset + y * in->stride + x);
                    }
                    vbuf[x] = (unsigned char)ok;
                }
            } else if (!yin) {
                memset(vbuf, 0, (size_t)W);
            } else {
                /* Word-level, as ErodeBox (internal/stencil/mask.go:55-82):
                 * AND the 2r+1 source rows, then AND each bit with the 2r
                 * bits above it; column x is then bit x - r. */
                int64_t nw = (W + 63) >> 6;
                uint64_t *acc = (uint64_t *)(colok + 2 * W + 2 + 8 - ((uintptr_t)(colok + 2 * W + 2) & 7));
                for (int64_t k = 0; k < nw; k++) acc[k] = ~(uint64_t)0;
                if (src->valid)
                    for (int j = -r; j <= r; j++) {
                        int64_t off = src->valid_offset + (y + j) * s;
                        int64_t last = (off + W - 1) >> 6;
                        for (int64_t k = 0; k < nw; k++) {
                            int64_t b = off + 64 * k, w = b >> 6;
                            int sh = (int)(b & 63);
                            uint64_t v = src->valid[w] >> sh;
                            if (sh && w + 1 <= last) v |= src->valid[w + 1] << (64 - sh);
                            acc[k] &= v;
                        }
                    }
                if (W & 63) acc[nw - 1] &= ((uint64_t)1 << (W & 63)) - 1;
                for (int64_t x = 0; x < W; x++) vbuf[x] = 0;
                for (int64_t x = r; x < W - r; x++) {
                    int ok = 1;
                    for (int d = 0; d <= 2 * r && ok; d++) {
                        int64_t c = x - r + d;
                        ok = (int)((acc[c >> 6] >> (c & 63)) & 1);
                    }
                    vbuf[x] = (unsigned char)ok;
                }
            }
            int64_t base = D->valid_offset + y * D->stride;
            int64_t x = 0;
            while (x < W) {
                int64_t b = base + x;
                int sh = (int)(b & 63);
                int64_t take = 64 - sh;
                if (take > W - x) take = W - x;
                uint64_t bits = 0;
                for (int64_t k = 0; k < take; k++) bits |= (uint64_t)vbuf[x + k] << (sh + k);
                uint64_t own = take == 64 ? ~(uint64_t)0 : ((((uint64_t)1 << take) - 1) << sh);
                uint64_t *w = &D->valid[b >> 6];
                if (own == ~(uint64_t)0) {
                    *w = bits;
                } else {
                    __atomic_fetch_and(w, ~own | bits, __ATOMIC_RELAXED);
                    __atomic_fetch_or(w, bits, __ATOMIC_RELAXED);
                }
                x += take;
            }
        }
    }
}

static void *worker(void *arg)
{
    job_t *jb = (job_t *)arg;
    /* bytes of the cell-by-cell validity, then the word rows of the baseline's */
    unsigned char *colok = (unsigned char *)malloc(3 * (size_t)jb->src->width + 128 +
                                                   2 * 8 * (((size_t)jb->src->width + 63) / 64 + 2));
    for (;;) {
        int64_t b = __atomic_fetch_add(&jb->next, 1, __ATOMIC_RELAXED);
        if (b >= jb->nbands) break;
        int64_t y0 = b * jb->band_rows;
        int64_t y1 = y0 + jb->band_rows;
        if (y1 > jb->src->height) y1 = jb->src->height;
        run_rows(jb, y0, y1, colok);
    }
    free(colok);
    return NULL;
}

int orc_process(const orc_stage *stages, int nstages, const orc_raster *src,
                const orc_raster *dst, int ndst, int nthreads)
{
    return orc_process_ex(stages, nstages, src, dst, ndst, nthreads, 0);
}

static int process_impl(const orc_stage *stages, int nstages, const orc_raster *srcs, int nsrc,
                        const orc_raster *dst, int ndst, int nthreads, int simd);

int orc_process_ex(const orc_stage *stages, int nstages, const orc_raster *src,
                   const orc_raster *dst, int ndst, int nthreads, int simd)
{
    return process_impl(stages, nstages, src, 1, dst, ndst, nthreads, simd);
}

int orc_process_n(const orc_stage *stages, int nstages, const orc_raster *src, int nsrc,
                  const orc_raster *dst, int ndst, int nthreads)
{
    return process_impl(stages, nstages, src, nsrc, dst, ndst, nthreads, 0);
}

static int process_impl(const orc_stage *stages, int nstages, const orc_raster *srcs, int nsrc,
                        const orc_raster *dst, int ndst, int nthreads, int simd)
{
    const orc_raster *src = srcs;
    if (nstages < 1 || !src || !dst || nsrc < 1 || nsrc > 4) return -1;
    const orc_stage *st = &stages[0];
    if (st->op < ORC_GRADIENT || st->op > ORC_STEP) return -1;
    if ((st->flags & ORC_STAGE_FIT) && (st->radius < 1 || st->radius > 8)) return -1;
    if ((st->op == ORC_HEATLOAD) && (!st->table[0] || st->table_len[0] != 16)) return -1;
    const int lead_pointwise = st->op == ORC_LOOKUP || st->op == ORC_RECLASS || st->op == ORC_STEP;
    if (!lead_pointwise && nsrc != 1) return -1;
    for (int i = 1; i < nstages; i++)
        if (stages[i].op != ORC_LOOKUP && stages[i].op != ORC_RECLASS && stages[i].op != ORC_STEP) return -1;
    /* vec.NewChain's checks (internal/vec/chain.go:106-132) */
    for (int i = 0; i < nstages; i++) {
        const orc_stage *p = &stages[i];
        if (p->op != ORC_STEP) continue;
        if (p->kind < 0 || p->kind > 12) return -1;
        if (step_binary(p) ? (p->input < 0 || p->input >= nsrc) : p->input != -1) return -1;
    }
    for (int j = 0; j < nsrc; j++) {
        if (srcs[j].width != dst[0].width || srcs[j].height != dst[0].height) return -1;
        if (srcs[j].valid)
            for (int d = 0; d < ndst; d++)
                if (!dst[d].valid) return -1;
    }
    /* Pointwise tables: Lookup's knots and values pair up (at least one);
     * Reclass has one value more than breaks (zero breaks allowed). */
    for (int i = 0; i < nstages; i++) {
        const orc_stage *p = &stages[i];
        if (p->op != ORC_LOOKUP && p->op != ORC_RECLASS) continue;
        const int n0 = p->table_len[0], n1 = p->table_len[1];
        if (p->op == ORC_LOOKUP ? (n0 < 1 || n1 != n0) : (n0 < 0 || n1 != n0 + 1)) return -1;
        if ((n0 > 0 && !p->table[0]) || !p->table[1]) return -1;
    }
    if (ndst != (st->op == ORC_GRADIENT ? 2 : 1)) return -1;
    if (src->valid)
        for (int d = 0; d < ndst; d++)
            if (!dst[d].valid) return -1;
    job_t jb;
    memset(&jb, 0, sizeof jb);
    jb.stages = stages;
    jb.nstages = nstages;
    jb.src = src;
    jb.srcs = srcs;
    jb.nsrc = nsrc;
    jb.dst = dst;
    jb.ndst = ndst;
    jb.simd = simd;
    jb.r = lead_pointwise ? 0
           : (st->flags & ORC_STAGE_FIT) ? st->radius
           : (st->op <= ORC_HILLSHADE || st->op == ORC_CURVATURE || st->op >= ORC_HEATLOAD) ? 1
           : st->radius;
    /* Bands of about 2^16 cells, whole rows, as internal/exec/tile.go:21-27. */
    int64_t rows = (int64_t)65536 / (src->width > 0 ? src->width : 1);
    jb.band_rows = rows < 1 ? 1 : rows;
    jb.nbands = (src->height + jb.band_rows - 1) / jb.band_rows;
    if (nthreads <= 1) {
        worker(&jb);
        return 0;
    }
    pthread_t tid[256];
    if (nthreads > 256) nthreads = 256;
    for (int i = 0; i < nthreads; i++) pthread_create(&tid[i], NULL, worker, &jb);
    for (int i = 0; i < nthreads; i++) pthread_join(tid[i], NULL);
    return 0;
}
