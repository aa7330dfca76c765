/*
 * agooracle.c -- plain-C restatement of the AGO HAF CPU kernels (test infrastructure
 * only; see agooracle.h).  Each function cites the reference function it follows.
 * Built with -ffp-contract=off so float expressions keep the reference's
 * multiply-then-add order (the reference's SSE code has no FMA).
 */
#include "agooracle.h"
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#define ROW(p, stride, y) ((void *)((uint8_t *)(p) + (size_t)(stride) * (size_t)(y)))

/* SIMD/tail split used by most HAF kernels: prefix = bytes to the next 16-byte boundary
 * of the destination row pointer (used as a pixel count), tail = (width - prefix) & 15. */
static void haf_split(const void *dst, int width, int *prefix, int *tail_start)
{
    int p = (int)((uintptr_t)dst & 15);
    p = p ? 16 - p : 0;
    int post = (width - p) & 15;
    *prefix = p;
    *tail_start = width - post;
}

/* x86 cvtpd2dq / cvtps2dq with the default MXCSR rounding: round half to even. */
static int rne_d(double v) { return (int)nearbyint(v); }

/* ago_haf_cpu_filter.cpp:1518 HafCpu_Gaussian_U8_U8_3x3 (SSE path, USE_AVX=0):
 * h = p[x-1] + 2p[x] + p[x+1]; out = (h[y-1] + 2h[y] + h[y+1]) >> 4 for x in [0, W). */
int oracle_Gaussian_U8_U8_3x3(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                              const uint8_t *pSrc, uint32_t srcStride)
{
    for (uint32_t y = 0; y < H; y++) {
        const uint8_t *s = (const uint8_t *)ROW(pSrc, srcStride, y);
        uint8_t *d = (uint8_t *)ROW(pDst, dstStride, y);
        for (int x = 0; x < (int)W; x++) {
            int h0 = s[x - 1 - (int)srcStride] + 2 * s[x - (int)srcStride] + s[x + 1 - (int)srcStride];
            int h1 = s[x - 1] + 2 * s[x] + s[x + 1];
            int h2 = s[x - 1 + (int)srcStride] + 2 * s[x + (int)srcStride] + s[x + 1 + (int)srcStride];
            d[x] = (uint8_t)((h0 + 2 * h1 + h2) >> 4);
        }
    }
    return 0;
}

/* ago_haf_cpu_filter.cpp:2676 (S16 3xN), :2858 (U8 3xN), :3037/:3170 (5xN), :3301/:3434 (7xN),
 * :3565/:3698 (9xN).  Rows: dstHeight rows from pDst/pSrc (the wrapper starts them rows/2
 * rows into the image, ago_kernel_api.cpp:15590).  Columns [0, W): prefix = bytes to the
 * next 16-byte boundary of the destination row, body, postfix = (W - prefix) & 15. */
static int conv_sum(const uint8_t *s, int st, int x, const int16_t *conv, int cols, int rows)
{
    int idx = cols * rows - 1, sum = 0;
    for (int i = -(rows >> 1); i <= (rows >> 1); i++)
        for (int j = -(cols >> 1); j <= (cols >> 1); j++) sum += (int)s[i * st + x + j] * (int)conv[idx--];
    return sum;
}

static int conv_clamp(int v, int lo, int hi) { return v < lo ? lo : v > hi ? hi : v; }

static int conv_rows(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, int bpp, const uint8_t *pSrc,
                     uint32_t srcStride, const int16_t *conv, uint32_t cols, uint32_t rows, int32_t shift)
{
    const int lo = bpp == 1 ? 0 : -32768, hi = bpp == 1 ? 255 : 32767;
    for (uint32_t y = 0; y < H; y++) {
        const uint8_t *s = (const uint8_t *)ROW(pSrc, srcStride, y);
        uint8_t *d = (uint8_t *)ROW(pDst, dstStride, y);
        int prefix = (int)((uintptr_t)d & 15);
        prefix = prefix ? 16 - prefix : 0;
        const int postfix = ((int)W - prefix) & 15;
        for (int x = 0; x < (int)W; x++) {
            const int sum = conv_sum(s, (int)srcStride, x, conv, (int)cols, (int)rows);
            int v;
            if (x < prefix || x >= (int)W - postfix) {
                v = conv_clamp(sum, lo, hi);                       /* scalar loops: no shift */
            } else {
                const int sh = (int)(int32_t)((uint32_t)sum >> shift);   /* _mm_srli_epi32 */
                v = conv_clamp(conv_clamp(sh, -32768, 32767), lo, hi);  /* packs_epi32 (+ packus_epi16) */
            }
            if (bpp == 1) d[x] = (uint8_t)v;
            else ((int16_t *)d)[x] = (int16_t)v;
        }
    }
    return 0;
}

int oracle_Convolve_U8_U8(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, const uint8_t *pSrc,
                          uint32_t srcStride, const int16_t *conv, uint32_t cols, uint32_t rows, int32_t shift)
{
    return conv_rows(W, H, pDst, dstStride, 1, pSrc, srcStride, conv, cols, rows, shift);
}

int oracle_Convolve_S16_U8(uint32_t W, uint32_t H, int16_t *pDst, uint32_t dstStride, const uint8_t *pSrc,
                           uint32_t srcStride, const int16_t *conv, uint32_t cols, uint32_t rows, int32_t shift)
{
    return conv_rows(W, H, (uint8_t *)pDst, dstStride, 2, pSrc, srcStride, conv, cols, rows, shift);
}

static inline void sobel3(const uint8_t *s, int st, int x, int *gx, int *gy)
{
    *gx = (s[x + 1 - st] - s[x - 1 - st]) + 2 * (s[x + 1] - s[x - 1]) + (s[x + 1 + st] - s[x - 1 + st]);
    *gy = (s[x - 1 + st] + 2 * s[x + st] + s[x + 1 + st]) - (s[x - 1 - st] + 2 * s[x - st] + s[x + 1 - st]);
}

/* ago_haf_cpu_filter.cpp:2468 HafCpu_SobelMagnitude_S16_U8_3x3: SIMD body computes
 * sqrt((double)(gx^2+gy^2)) rounded to nearest even (_mm_cvtpd_epi32) and packs with
 * unsigned saturation; the scalar prefix/tail store (int16)sqrtf(float) (truncation). */
int oracle_SobelMagnitude_S16_U8_3x3(uint32_t W, uint32_t H, int16_t *pDst, uint32_t dstStride,
                                     const uint8_t *pSrc, uint32_t srcStride)
{
    int prefix, tail;
    haf_split(pDst, (int)W, &prefix, &tail);
    for (uint32_t y = 0; y < H; y++) {
        const uint8_t *s = (const uint8_t *)ROW(pSrc, srcStride, y);
        int16_t *d = (int16_t *)ROW(pDst, dstStride, y);
        for (int x = 0; x < (int)W; x++) {
            int gx, gy;
            sobel3(s, (int)srcStride, x, &gx, &gy);
            int16_t gx16 = (int16_t)gx, gy16 = (int16_t)gy;
            if (x < prefix || x >= tail) {
                float mag = (float)(gx16 * gx16) + (float)(gy16 * gy16);
                d[x] = (int16_t)sqrtf(mag);
            } else {
                int m = rne_d(sqrt((double)(gx16 * gx16 + gy16 * gy16)));
                if (m > 65535) m = 65535;
                d[x] = (int16_t)(uint16_t)m;
            }
        }
    }
    return 0;
}

/* ago_haf_cpu_filter.cpp:2237 HafCpu_Sobel_S16S16_U8_3x3_GXY: exact integer 3x3 Sobel. */
int oracle_Sobel_S16S16_U8_3x3_GXY(uint32_t W, uint32_t H, int16_t *pGx, uint32_t gxStride,
                                   int16_t *pGy, uint32_t gyStride, const uint8_t *pSrc, uint32_t srcStride)
{
    for (uint32_t y = 0; y < H; y++) {
        const uint8_t *s = (const uint8_t *)ROW(pSrc, srcStride, y);
        int16_t *dx = (int16_t *)ROW(pGx, gxStride, y);
        int16_t *dy = (int16_t *)ROW(pGy, gyStride, y);
        for (int x = 0; x < (int)W; x++) {
            int gx, gy;
            sobel3(s, (int)srcStride, x, &gx, &gy);
            dx[x] = (int16_t)gx;
            dy[x] = (int16_t)gy;
        }
    }
    return 0;
}

/* ago_haf_cpu_arithmetic.cpp:4989 HafCpu_Magnitude_S16_S16S16: prefix (pixels to the
 * 16-byte boundary of dst) truncates sqrtf(float), the 8-wide SIMD body rounds
 * sqrt(double) to nearest even with signed 16-bit saturation (_mm_packs_epi32), and the
 * tail rounds sqrtf(float) half away from zero (round()). */
int oracle_Magnitude_S16_S16S16(uint32_t W, uint32_t H, int16_t *pMag, uint32_t magStride,
                                const int16_t *pGx, uint32_t gxStride, const int16_t *pGy, uint32_t gyStride)
{
    int prefix = (int)((uintptr_t)pMag & 15);
    prefix = prefix ? 16 - prefix : 0;
    prefix >>= 1;
    int post = ((int)W - prefix) & 7;
    int tail = (int)W - post;
    for (uint32_t y = 0; y < H; y++) {
        const int16_t *gx = (const int16_t *)ROW(pGx, gxStride, y);
        const int16_t *gy = (const int16_t *)ROW(pGy, gyStride, y);
        int16_t *d = (int16_t *)ROW(pMag, magStride, y);
        for (int x = 0; x < (int)W; x++) {
            int a = gx[x], b = gy[x];
            if (x < prefix) {
                float t = (float)(a * a) + (float)(b * b);
                d[x] = (int16_t)(int)sqrtf(t);
            } else if (x >= tail) {
                float t = (float)(a * a) + (float)(b * b);
                t = sqrtf(t);
                d[x] = (int16_t)(int)round((double)t);
            } else {
                double n = (double)(a * a) + (double)(b * b);
                int m = rne_d(sqrt(n));
                if (m > 32767) m = 32767;
                d[x] = (int16_t)m;
            }
        }
    }
    return 0;
}

/* ago_haf_cpu_arithmetic.cpp:3546 HafCpu_ColorDepth_U8_S16_Sat: clamp(v >> shift, 0, 255). */
int oracle_ColorDepth_U8_S16_Sat(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                 const int16_t *pSrc, uint32_t srcStride, int32_t shift)
{
    for (uint32_t y = 0; y < H; y++) {
        const int16_t *s = (const int16_t *)ROW(pSrc, srcStride, y);
        uint8_t *d = (uint8_t *)ROW(pDst, dstStride, y);
        for (uint32_t x = 0; x < W; x++) {
            int v = s[x] >> shift;
            d[x] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
        }
    }
    return 0;
}

/* ago_haf_cpu_arithmetic.cpp:3660 HafCpu_Threshold_U8_U8_Binary: v > thr ? 255 : 0. */
int oracle_Threshold_U8_U8_Binary(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                  const uint8_t *pSrc, uint32_t srcStride, uint8_t threshold)
{
    for (uint32_t y = 0; y < H; y++) {
        const uint8_t *s = (const uint8_t *)ROW(pSrc, srcStride, y);
        uint8_t *d = (uint8_t *)ROW(pDst, dstStride, y);
        for (uint32_t x = 0; x < W; x++) d[x] = s[x] > threshold ? 255 : 0;
    }
    return 0;
}

/* =============================== Canny ================================== */

/* ago_haf_cpu_arithmetic.cpp:9638 HafCpu_FastAtan2_Canny: direction quantised to 0..3. */
static int fast_atan2_canny(int16_t gx, int16_t gy)
{
    uint16_t ax = (uint16_t)abs(gx), ay = (uint16_t)abs(gy);
    float d1 = (float)ax * 0.4142135623730950488016887242097f;
    float d2 = (float)ax * 2.4142135623730950488016887242097f;
    int ret = (gx * gy) < 0 ? 3 : 1;
    if (ay <= d1) ret = 0;
    if (ay >= d2) ret = 2;
    return ret;
}

static uint16_t canny_pack(int16_t gx, int16_t gy)
{
    int16_t t = (int16_t)(abs(gx) + abs(gy));
    t = (int16_t)(t << 2);
    t = (int16_t)(t | (fast_atan2_canny(gx, gy) & 3));
    return (uint16_t)t;
}

/* ago_haf_cpu_canny.cpp:44 HafCpu_CannySobel_U16_U8_3x3_L1NORM, rows 1..H-2 of the full
 * image (pDst/pSrc point at row 0).  Gy is negated (canny.cpp:79).  The SIMD body keeps
 * per-row vertical sums r0 = s[y-1]+2s[y]+s[y+1] and r1 = s[y+1]-s[y-1] in a scratch
 * buffer; at x = 0 it reads r0[-1] (never written: 0) and r1[-1], which aliases
 * r0[ALIGN16(W)-1] (the column W-1 vertical sum of the current row when W%16 == 0, else
 * never written: 0).  Columns from (W - (W&15) - 1) on use the scalar formula, which reads
 * one byte past the row at x = W-1.  Assumes a 16-byte aligned destination and W >= 16. */
int oracle_CannySobel_U16_U8_3x3_L1NORM(uint32_t W, uint32_t H, uint16_t *pDst, uint32_t dstStride,
                                        const uint8_t *pSrc, uint32_t srcStride)
{
    int prefix, tail_start;
    haf_split(pDst, (int)W, &prefix, &tail_start);
    const int aligned = tail_start - prefix;
    const int A16 = ((int)W + 15) & ~15;
    const int st = (int)srcStride;
    for (int y = 1; y < (int)H - 1; y++) {
        const uint8_t *s = pSrc + (size_t)y * srcStride;
        uint16_t *d = (uint16_t *)ROW(pDst, dstStride, y);
        for (int x = 0; x < (int)W; x++) {
            int16_t gx, gy;
            if (x >= prefix && x < aligned + prefix - 1 && x <= aligned - 8 + 7) {
                /* SIMD body: gx = r0[x+1] - r0[x-1]; gy = -(r1[x-1] + 2 r1[x] + r1[x+1]) */
                int r0m, r1m;
                if (x == 0) {
                    r0m = 0;
                    r1m = (A16 - 1 < aligned) ? ((s[A16 - 1 - st] + 2 * s[A16 - 1] + s[A16 - 1 + st]) & 0xffff) : 0;
                } else {
                    r0m = s[x - 1 - st] + 2 * s[x - 1] + s[x - 1 + st];
                    r1m = s[x - 1 + st] - s[x - 1 - st];
                }
                int r0p = s[x + 1 - st] + 2 * s[x + 1] + s[x + 1 + st];
                int r1c = s[x + st] - s[x - st];
                int r1p = s[x + 1 + st] - s[x + 1 - st];
                gx = (int16_t)(r0p - r0m);
                gy = (int16_t)(0 - (int16_t)(r1m + 2 * r1c + r1p));
            } else {
                gx = (int16_t)(s[x + 1 - st] - s[x - 1 - st] + s[x + 1 + st] - s[x - 1 + st] + 2 * (s[x + 1] - s[x - 1]));
                gy = (int16_t)(s[x - 1 + st] + s[x + 1 + st] - s[x - 1 - st] - s[x + 1 - st] + 2 * (s[x + st] - s[x - st]));
                gy = (int16_t)(~gy + 1);
            }
            d[x] = canny_pack(gx, gy);
        }
    }
    return 0;
}

/* Canny gradients with 3x3 L2, 5x5 and 7x7 windows (ago_haf_cpu_canny.cpp:145 5x5 L1,
 * :272 7x7 L1, :646 3x3 L2, :756 5x5 L2, :893 7x7 L2), rows [R, H-R), R = gsize / 2.
 *
 * Each reference kernel splits a row like the 3x3 L1 one: scalar columns [0, prefix) and
 * [aligned + prefix - 1, W), SIMD columns between them computed from per-row vertical sums
 * r0 (smoothing) and r1 (difference) kept in node scratch at scratch + 16 bytes, r1 right
 * after r0 (ALIGN16(W) int16 each).  The SIMD part reads r0 / r1 up to R columns outside
 * [0, aligned), i.e. the zeroed scratch or the neighbouring row buffer; this restatement
 * keeps the same scratch layout so those reads land on the same values.  The SIMD and
 * scalar formulas differ per variant, and are restated as written:
 *   - 3x3 L2 body squares in 16-bit lanes (mullo, zero-extended), sums in float, sqrt,
 *     rounds half-even, packs with unsigned saturation; its scalar Gy is not negated.
 *   - 5x5 body is exact; L1 scalar negates Gy, L2 scalar does not and its top row term
 *     negates only the first pixel (canny.cpp:800).
 *   - 7x7 body divides both vertical sums by 4 (srai), combines with saturating adds and
 *     clamps the L1 magnitude to 0x3FFF; its scalar columns use the full-scale sums in
 *     16-bit wrapping arithmetic, Gy not negated.
 * L2 scalar columns: (int16) sqrt((double) (Gx^2 + Gy^2)), i.e. the integer square root
 * wrapped to 16 bits. */
static const int kV3[3] = { 1, 2, 1 }, kD3[3] = { -1, 0, 1 };
static const int kV5[5] = { 1, 4, 6, 4, 1 }, kD5[5] = { -1, -2, 0, 2, 1 };
static const int kV7[7] = { 1, 6, 15, 20, 15, 6, 1 }, kD7[7] = { -1, -4, -5, 0, 5, 4, 1 };

static int16_t w16(int v) { return (int16_t)v; }
static int16_t s16(int v) { return (int16_t)(v > 32767 ? 32767 : (v < -32768 ? -32768 : v)); }
static int16_t abs16(int16_t v) { return (int16_t)(v < 0 ? -(int)v : v); }

static uint16_t canny_l2_pack(int16_t gx, int16_t gy, int body3)
{
    float f;
    if (body3)
        f = (float)(uint16_t)(gx * gx) + (float)(uint16_t)(gy * gy);
    else
        f = (float)(int32_t)((uint32_t)(gx * gx) + (uint32_t)(gy * gy));
    int m = (int)nearbyintf(sqrtf(f));
    if (m < 0) m = 0;
    if (m > 65535) m = 65535;
    return (uint16_t)((uint16_t)(m << 2) | (fast_atan2_canny(gx, gy) & 3));
}

int oracle_CannySobel_U16_U8_NxN(uint32_t W, uint32_t H, uint16_t *pDst, uint32_t dstStride,
                                 const uint8_t *pSrc, uint32_t srcStride, uint32_t gsize, uint32_t l2)
{
    if (gsize != 3 && gsize != 5 && gsize != 7) return -1;
    const int R = (int)gsize / 2;
    const int *V = gsize == 3 ? kV3 : (gsize == 5 ? kV5 : kV7);
    const int *D = gsize == 3 ? kD3 : (gsize == 5 ? kD5 : kD7);
    int prefix, tail_start;
    haf_split(pDst, (int)W, &prefix, &tail_start);
    const int aligned = tail_start - prefix;
    const int L = ((int)W + 15) & ~15;
    uint8_t *scratch = (uint8_t *)calloc((size_t)L * 4 + 128, 1);
    if (!scratch) return -1;
    int16_t *r0 = (int16_t *)(scratch + 16), *r1 = r0 + L;
    const long st = (long)srcStride;
    for (int y = R; y < (int)H - R; y++) {
        const uint8_t *s = pSrc + (size_t)y * srcStride;
        uint16_t *d = (uint16_t *)ROW(pDst, dstStride, y);
        /* SIMD part: vertical sums, then the horizontal pass, 8 columns per step */
        for (int x0 = prefix; x0 <= aligned - 8; x0 += 8)
            for (int x = x0; x < x0 + 8; x++) {
                int a = 0, b = 0;
                for (int k = -R; k <= R; k++) { a += V[k + R] * s[x + k * st]; b += D[k + R] * s[x + k * st]; }
                if (gsize == 7) { a = w16(a) >> 2; b = w16(b) >> 2; }
                r0[x] = w16(a); r1[x] = w16(b);
            }
        for (int x0 = prefix; x0 <= aligned - 8; x0 += 8)
            for (int x = x0; x < x0 + 8; x++) {
                int16_t t0, t1;
                if (gsize == 3) {
                    t0 = w16(r0[x + 1] - r0[x - 1]);
                    t1 = w16(0 - w16(w16(r1[x - 1] + r1[x + 1]) + w16(r1[x] << 1)));
                } else if (gsize == 5) {
                    t0 = s16(w16(w16(r0[x + 1] - r0[x - 1]) << 1) + w16(r0[x + 2] - r0[x - 2]));
                    int16_t u = w16(w16(w16(r1[x - 1] + r1[x + 1]) << 2) + w16(r1[x - 2] + r1[x + 2]));
                    u = l2 ? s16(u + w16(r1[x] * 6)) : w16(u + w16(r1[x] * 6));
                    t1 = w16(0 - u);
                } else {
                    int16_t a = w16(s16(r0[x + 2] - r0[x - 2]) << 2);
                    int16_t b = w16(s16(r0[x + 1] - r0[x - 1]) * 5);
                    t0 = s16(s16(a + s16(r0[x + 3] - r0[x - 3])) + b);
                    int16_t u = s16(w16(w16(r1[x - 2] + r1[x + 2]) * 6) + w16(r1[x] * 20));
                    int16_t v = w16(w16(r1[x - 1] + r1[x + 1]) * 15);
                    u = s16(u + s16(r1[x - 3] + r1[x + 3]));
                    u = s16(u + v);
                    t1 = s16(0 - u);
                }
                if (l2) {
                    d[x] = canny_l2_pack(t0, t1, gsize == 3);
                } else {
                    int16_t m = w16(abs16(t0) + abs16(t1));
                    if (gsize == 7 && m > 0x3FFF) m = 0x3FFF;
                    d[x] = (uint16_t)((uint16_t)(m << 2) | (fast_atan2_canny(t0, t1) & 3));
                }
            }
        /* scalar columns */
        for (int x = 0; x < (int)W; x++) {
            if (x >= prefix && x < aligned + prefix - 1) continue;
            int gxs = 0, gys = 0;
            for (int j = -R; j <= R; j++)
                for (int i = -R; i <= R; i++) {
                    const int v = s[x + i + j * st];
                    gxs += V[j + R] * D[i + R] * v;
                    if (gsize == 5 && l2 && j == -R)   /* canny.cpp:800: only the first term negated */
                        gys += (i == -R ? -1 : 1) * V[i + R] * v;
                    else
                        gys += D[j + R] * V[i + R] * v;
                }
            int16_t gx = w16(gxs), gy = w16(gys);
            if (!l2 && gsize != 7) gy = w16(~gy + 1);
            int16_t t;
            if (l2) {
                int32_t n = (int32_t)((uint32_t)(gx * gx) + (uint32_t)(gy * gy));
                t = n < 0 ? 0 : w16((int)sqrt((double)n));
            } else {
                t = w16(abs(gx) + abs(gy));
            }
            t = w16(t << 2);
            t = w16(t | (fast_atan2_canny(gx, gy) & 3));
            d[x] = (uint16_t)t;
        }
    }
    free(scratch);
    return 0;
}

static const int kNOffset[4][2][2] = {
    { { -1, 0 }, { 1, 0 } }, { { 1, -1 }, { -1, 1 } }, { { 0, -1 }, { 0, 1 } }, { { -1, -1 }, { 1, 1 } },
};

/* ago_haf_cpu_canny.cpp:549 HafCpu_CannySuppThreshold_U8XY_U16_3x3: non-maximum
 * suppression along the quantised direction (strict > on both sides), then > upper -> 255
 * (pushed on the stack in raster order), <= lower -> 0, else 127; x,y in [1,W-1)x[1,H-1). */
int oracle_CannySuppThreshold_U8XY_U16_3x3(uint32_t capacityOfXY, oracle_coord2d_u16 *xyStack, uint32_t *pStackTop,
                                           uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                           const uint16_t *pSrc, uint32_t srcStride, uint16_t lower, uint16_t upper)
{
    (void)capacityOfXY;
    const int ss = (int)(srcStride >> 1);
    uint32_t top = 0;
    for (uint32_t y = 1; y < H - 1; y++) {
        uint8_t *out = pDst + (size_t)y * dstStride;
        const uint16_t *p = pSrc + (size_t)y * ss;
        for (uint32_t x = 1; x < W - 1; x++) {
            int mag = p[x] >> 2, ang = p[x] & 3;
            int o0 = kNOffset[ang][0][1] * ss + kNOffset[ang][0][0];
            int o1 = kNOffset[ang][1][1] * ss + kNOffset[ang][1][0];
            int edge = (mag > (p[(int)x + o0] >> 2) && mag > (p[(int)x + o1] >> 2)) ? mag : 0;
            if (edge > upper) {
                out[x] = 255;
                xyStack[top].x = (uint16_t)x; xyStack[top].y = (uint16_t)y; top++;
            } else if (edge <= lower) {
                out[x] = 0;
            } else {
                out[x] = 127;
            }
        }
    }
    *pStackTop = top;
    return 0;
}

/* ago_haf_cpu_canny.cpp:598 HafCpu_CannyEdgeTrace_U8_U8XY: grow strong pixels through
 * 8-connected 127 pixels (DFS over the stack), then 127 -> 0 over ALIGN16(W) columns. */
int oracle_CannyEdgeTrace_U8_U8XY(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                  uint32_t capacityOfXY, oracle_coord2d_u16 *xyStack, uint32_t stackTop)
{
    (void)capacityOfXY;
    static const int dx[8] = {-1, 0, 1, -1, 1, -1, 0, 1}, dy[8] = {-1, -1, -1, 0, 0, 1, 1, 1};
    uint32_t top = stackTop;
    while (top) {
        top--;
        int x = xyStack[top].x, y = xyStack[top].y;
        for (int i = 0; i < 8; i++) {
            int x1 = x + dx[i], y1 = y + dy[i];
            uint8_t *p = pDst + (size_t)y1 * dstStride + x1;
            if (*p == 127) {
                *p = 255;
                xyStack[top].x = (uint16_t)x1; xyStack[top].y = (uint16_t)y1; top++;
            }
        }
    }
    const uint32_t w16 = (W + 15) & ~15u;
    for (uint32_t y = 0; y < H; y++) {
        uint8_t *row = pDst + (size_t)y * dstStride;
        for (uint32_t x = 0; x < w16; x++) if (row[x] == 127) row[x] = 0;
    }
    return 0;
}

/* =============================== Harris ================================= */

/* ago_haf_cpu_harris.cpp:85 HafCpu_HarrisSobel_HG3_U8_3x3: rows 1..H-2 (pointers at row 0),
 * all columns (reading one pixel outside the row at x = 0 and x = W-1); products of the
 * integer 3x3 Sobel gradients in float, div_factor 1 (harris.cpp:129). */
int oracle_HarrisSobel_HG3_U8_3x3(uint32_t W, uint32_t H, float *pDstGxy, uint32_t dstStride,
                                  const uint8_t *pSrc, uint32_t srcStride)
{
    const int st = (int)srcStride;
    for (int y = 1; y < (int)H - 1; y++) {
        const uint8_t *s = pSrc + (size_t)y * srcStride;
        float *d = (float *)ROW(pDstGxy, dstStride, y);
        for (int x = 0; x < (int)W; x++) {
            int16_t hx0 = (int16_t)(s[x + 1 - st] - s[x - 1 - st]);
            int16_t hx1 = (int16_t)(s[x + 1] - s[x - 1]);
            int16_t hx2 = (int16_t)(s[x + 1 + st] - s[x - 1 + st]);
            int16_t hy0 = (int16_t)(s[x - 1 - st] + 2 * s[x - st] + s[x + 1 - st]);
            int16_t hy2 = (int16_t)(s[x - 1 + st] + 2 * s[x + st] + s[x + 1 + st]);
            int16_t gx = (int16_t)(hx2 + hx0 + 2 * hx1);
            int16_t gy = (int16_t)(hy2 - hy0);
            d[3 * x + 0] = ((float)gx * (float)gx) / 1.0f;
            d[3 * x + 1] = ((float)gx * (float)gy) / 1.0f;
            d[3 * x + 2] = ((float)gy * (float)gy) / 1.0f;
        }
    }
    return 0;
}

/* ago_haf_cpu_harris.cpp:596 HafCpu_HarrisScore_HVC_HG3_3x3: 3x3 window sums in (j, i)
 * order, Mc = (gx2*gy2 - gxy2*gxy2) - (k*trace)*trace, Mc /= norm, Mc > Tc ? Mc : 0;
 * first/last row and column are 0.  Plain float multiply-then-add (no FMA). */
int oracle_HarrisScore_HVC_HG3_3x3(uint32_t W, uint32_t H, float *pDstVc, uint32_t dstStride,
                                   const float *pSrcGxy, uint32_t srcStride, float k, float Tc, float norm)
{
    memset(pDstVc, 0, dstStride);
    for (uint32_t y = 1; y < H - 1; y++) {
        float *d = (float *)ROW(pDstVc, dstStride, y);
        const float *c = (const float *)ROW(pSrcGxy, srcStride, y);
        d[0] = 0;
        for (uint32_t x = 1; x < W - 1; x++) {
            float gx2 = 0, gy2 = 0, gxy2 = 0;
            for (int j = -1; j <= 1; j++) {
                const float *t = (const float *)((const uint8_t *)c + (ptrdiff_t)j * (ptrdiff_t)srcStride);
                for (int i = -1; i <= 1; i++) {
                    gx2 += t[3 * ((int)x + i) + 0];
                    gxy2 += t[3 * ((int)x + i) + 1];
                    gy2 += t[3 * ((int)x + i) + 2];
                }
            }
            float traceA = gx2 + gy2;
            float detA = (gx2 * gy2) - (gxy2 * gxy2);
            float Mc = detA - (k * traceA * traceA);
            Mc /= norm;
            d[x] = (Mc > Tc) ? Mc : 0;
        }
        d[W - 1] = 0;
    }
    memset(ROW(pDstVc, dstStride, H - 1), 0, dstStride);
    return 0;
}

/* Separable 5x5 / 7x7 Sobel of HafCpu_HarrisSobel_HG3_U8_{5x5,7x7}: derivative taps d and
 * smoothing taps s; gx = smoothing down the rows of the rows' horizontal derivatives, gy =
 * derivative down the rows of the rows' horizontal smoothing (exact integers). */
static const int kHarrisD5[5] = {-1, -2, 0, 2, 1}, kHarrisS5[5] = {1, 4, 6, 4, 1};
static const int kHarrisD7[7] = {-1, -4, -5, 0, 5, 4, 1}, kHarrisS7[7] = {1, 6, 15, 20, 15, 6, 1};

int oracle_HarrisSobel_HG3_U8_NxN(uint32_t W, uint32_t H, float *pDst, uint32_t dstStride, const uint8_t *pSrc,
                                  uint32_t srcStride, uint32_t gs)
{
    const int r = (int)gs / 2;
    const int *d = gs == 5 ? kHarrisD5 : kHarrisD7, *sm = gs == 5 ? kHarrisS5 : kHarrisS7;
    for (int y = r; y < (int)H - r; y++) {
        float *o = (float *)ROW(pDst, dstStride, y);
        for (int x = 0; x < (int)W; x++) {
            int gx = 0, gy = 0;
            for (int v = -r; v <= r; v++) {
                const uint8_t *row = (const uint8_t *)ROW(pSrc, srcStride, y + v);
                int hd = 0, hs = 0;
                for (int u = -r; u <= r; u++) {
                    hd += d[u + r] * (int)row[x + u];
                    hs += sm[u + r] * (int)row[x + u];
                }
                gx += sm[v + r] * hd;
                gy += d[v + r] * hs;
            }
            o[3 * x + 0] = (float)gx * (float)gx;
            o[3 * x + 1] = (float)gx * (float)gy;
            o[3 * x + 2] = (float)gy * (float)gy;
        }
    }
    return 0;
}

int oracle_HarrisScore_HVC_HG3_NxN(uint32_t W, uint32_t H, float *pDstVc, uint32_t dstStride, const float *pSrcGxy,
                                   uint32_t srcStride, float k, float Tc, float norm, uint32_t bs)
{
    const int r = (int)bs / 2;
    /* the 7x7 kernel writes its third left-border zero without advancing the output pointer
     * (ago_haf_cpu_harris.cpp:758-763): column x's score lands at x - 1, and the last column
     * of the rows it processes is never written (0 here, as in AGO's zeroed buffers) */
    const int shift = bs == 7 ? 1 : 0;
    for (int y = 0; y < (int)H; y++) {
        float *d = (float *)ROW(pDstVc, dstStride, y);
        for (int x = 0; x < (int)W; x++) d[x] = 0;
        if (y < r || y >= (int)H - r) continue;
        for (int x = r; x < (int)W - r; x++) {
            float gx2 = 0, gy2 = 0, gxy2 = 0;
            for (int j = -r; j <= r; j++) {
                const float *t = (const float *)ROW(pSrcGxy, srcStride, y + j);
                for (int i = -r; i <= r; i++) {
                    gx2 += t[3 * (x + i) + 0];
                    gxy2 += t[3 * (x + i) + 1];
                    gy2 += t[3 * (x + i) + 2];
                }
            }
            float traceA = gx2 + gy2;
            float detA = (gx2 * gy2) - (gxy2 * gxy2);
            float Mc = detA - (k * traceA * traceA);
            Mc /= norm;
            d[x - shift] = (Mc > Tc) ? Mc : 0;
        }
    }
    return 0;
}

float oracle_harris_norm_factor_block(int32_t gs, int32_t bs)
{
    float f = 255.0f * (float)(1 << (gs - 1)) * (float)bs;
    return f * f * f * f;
}

/* ============================== FAST corners ============================== */

/* The 16 pixels of the radius-3 Bresenham circle, clockwise from the pixel three rows above
 * (ago_haf_cpu_fast_corners.cpp:36 generateOffset), as (dx, dy). */
static const int kFastDx[16] = {0, 1, 2, 3, 3, 3, 2, 1, 0, -1, -2, -3, -3, -3, -2, -1};
static const int kFastDy[16] = {-3, -3, -2, -1, 0, 1, 2, 3, 3, 3, 2, 1, 0, -1, -2, -3};

/* bit i of the result: circle pixels i .. i+8 (mod 16) all set in the 16-bit mask m */
static int fast_arc9(uint32_t m)
{
    uint32_t r = m | (m << 16);
    uint32_t a = r & (r >> 1);
    a &= a >> 2;
    a &= a >> 4;
    a &= r >> 8;
    return (a & 0xFFFFu) != 0;
}

/* circle pixel i of candidate p, read by raw offset as the reference does (p[offset]) */
static void fast_circle(const uint8_t *p, int stride, int b[16])
{
    for (int i = 0; i < 16; i++) b[i] = p[kFastDy[i] * stride + kFastDx[i]];
}

/* masks of the circle pixels brighter than c + t / darker than c - t in 16-bit arithmetic
 * (:58 generateMasks_C, :297 isCorner_SSE) */
static void fast_masks(int c, const int b[16], int t, uint32_t *plus, uint32_t *minus)
{
    const int16_t hi = (int16_t)(c + t), lo = (int16_t)(c - t);
    *plus = *minus = 0;
    for (int i = 0; i < 16; i++) {
        if ((int16_t)b[i] > hi) *plus |= 1u << i;
        if ((int16_t)b[i] < lo) *minus |= 1u << i;
    }
}

/* the strength search of :216 checkForCornerAndGetStrength: a binary search between t (a
 * corner) and 255 (never one) for the largest threshold that still makes a corner */
static int fast_search(int c, const int b[16], int t, int sign)
{
    int lower = t, upper = 255;
    while (upper - lower > 1) {
        const int mid = (upper + lower) >> 1;
        uint32_t plus, minus;
        fast_masks(c, b, mid, &plus, &minus);
        if (fast_arc9(sign > 0 ? plus : minus)) lower = mid;
        else upper = mid;
    }
    return lower;
}

static int fast_strength(const uint8_t *p, int stride, int t)
{
    int b[16];
    fast_circle(p, stride, b);
    const int c = p[0];
    uint32_t plus, minus;
    fast_masks(c, b, t, &plus, &minus);
    const int sp = fast_arc9(plus) ? fast_search(c, b, t, 1) : 0;
    const int sn = fast_arc9(minus) ? fast_search(c, b, t, -1) : 0;
    return sp > sn ? sp : sn;
}

static void fast_emit(oracle_keypoint *corners, uint32_t capacity, uint32_t *n, int x, int y, float strength)
{
    if (*n < capacity) {
        oracle_keypoint *k = &corners[*n];
        k->x = x; k->y = y; k->strength = strength;
        k->scale = 0; k->orientation = 0; k->tracking_status = 1; k->error = 0;
    }
    (*n)++;
}

/* :414 HafCpu_FastCorners_XY_U8_NoSupression: rows 3 .. H-4, every column (the circle of the
 * three outer columns on each side reads across the row's end, into the neighbouring row or
 * the row padding); strength = strength_threshold. */
int oracle_FastCorners_XY_U8_NoSupression(uint32_t capacity, oracle_keypoint *corners, uint32_t *pCount, uint32_t W,
                                          uint32_t H, const uint8_t *pSrc, uint32_t srcStride, float strengthThreshold)
{
    const int t = (int16_t)floorf(strengthThreshold);
    uint32_t n = 0;
    for (int y = 3; y < (int)H - 3; y++)
        for (int x = 0; x < (int)W; x++) {
            const uint8_t *p = pSrc + (size_t)y * srcStride + x;
            int b[16];
            fast_circle(p, (int)srcStride, b);
            uint32_t plus, minus;
            fast_masks(p[0], b, t, &plus, &minus);
            if (fast_arc9(plus) || fast_arc9(minus)) fast_emit(corners, capacity, &n, x, y, strengthThreshold);
        }
    *pCount = n;
    return 0;
}

int oracle_FastCorners_strength(uint8_t *pDst, uint32_t W, uint32_t H, const uint8_t *pSrc, uint32_t srcStride,
                                float strengthThreshold)
{
    const int t = (int16_t)floorf(strengthThreshold);
    memset(pDst, 0, (size_t)W * H);
    for (int y = 3; y < (int)H - 3; y++)
        for (int x = 3; x < (int)W - 3; x++)
            pDst[(size_t)y * W + x] = (uint8_t)fast_strength(pSrc + (size_t)y * srcStride + x, (int)srcStride, t);
    return 0;
}

/* :599 HafCpu_FastCorners_XY_U8_Supression: strengths of rows 3 .. H-4 and columns 3 .. W-4
 * into a zeroed W x H map, then keep v != 0 when v >= the three neighbours above and the left
 * one, and v > the right one and the three below; strength = v. */
int oracle_FastCorners_XY_U8_Supression(uint32_t capacity, oracle_keypoint *corners, uint32_t *pCount, uint32_t W,
                                        uint32_t H, const uint8_t *pSrc, uint32_t srcStride, float strengthThreshold)
{
    uint8_t *s = (uint8_t *)malloc((size_t)W * H);
    if (!s) return -1;
    oracle_FastCorners_strength(s, W, H, pSrc, srcStride, strengthThreshold);
    uint32_t n = 0;
    for (int y = 3; y < (int)H - 3; y++)
        for (int x = 3; x < (int)W - 3; x++) {
            const uint8_t *q = s + (size_t)y * W + x;
            const uint8_t v = q[0];
            const uint8_t *u = q - W, *d = q + W;
            if (v && v >= u[-1] && v >= u[0] && v >= u[1] && v >= q[-1] && v > q[1] && v > d[-1] && v > d[0] && v > d[1])
                fast_emit(corners, capacity, &n, x, y, (float)v);
        }
    free(s);
    *pCount = n;
    return 0;
}

/* ago_haf_cpu_harris.cpp:882 HafCpu_NonMaxSupp_XY_ANY_3x3: keep v if >= the three pixels
 * above and the left one, > the right one and the three below; raster-order list. */
int oracle_NonMaxSupp_XY_ANY_3x3(uint32_t capacity, oracle_xys *list, uint32_t *pCount, uint32_t W, uint32_t H,
                                 const float *pSrc, uint32_t srcStride)
{
    uint32_t n = 0;
    for (uint32_t y = 1; y < H - 1 && n < capacity; y++) {
        const float *a = (const float *)ROW(pSrc, srcStride, y - 1);
        const float *b = (const float *)ROW(pSrc, srcStride, y);
        const float *c = (const float *)ROW(pSrc, srcStride, y + 1);
        for (uint32_t x = 1; x < W - 1; x++) {
            float v = b[x];
            if (v >= a[x - 1] && v >= a[x] && v >= a[x + 1] && v >= b[x - 1] && v > b[x + 1] &&
                v > c[x - 1] && v > c[x] && v > c[x + 1]) {
                list[n].x = (int16_t)x; list[n].y = (int16_t)y; list[n].s = v;
                if (++n >= capacity) break;
            }
        }
    }
    *pCount = n;
    return 0;
}

static int cmp_i64_desc(const void *a, const void *b)
{
    int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return x < y ? 1 : x > y ? -1 : 0;
}

/* ago_haf_cpu_harris.cpp:923 HafCpu_HarrisMergeSortAndPick_XY_XYS with the grid set up by
 * ago_kernel_api.cpp:20801-20815: the XYS records are sorted descending as raw int64
 * (strength bits, then y, then x); a point is kept when its grid cell (side
 * floor(min_distance/sqrt 2)) is empty and no kept point in the 5x5 surrounding cells is
 * closer than ceilf(min_distance^2) (strict).  min_distance <= 2 keeps everything.
 * *pCount may exceed `capacity`; only `capacity` corners are written. */
int oracle_HarrisMergeSortAndPick_XY_XYS(uint32_t capacity, oracle_keypoint *corners, uint32_t *pCount,
                                         oracle_xys *list, uint32_t n, float minDistance, uint32_t W, uint32_t H)
{
    qsort(list, n, sizeof(oracle_xys), cmp_i64_desc);
    uint32_t count = 0;
    if (minDistance > 2.0f) {
        uint32_t cell = (uint32_t)floor(minDistance / 1.41421356237309504880);
        uint32_t gw = (W + cell - 1) / cell, gh = (H + cell - 1) / cell;
        int16_t *grid = (int16_t *)malloc((size_t)gw * gh * 2 * sizeof(int16_t));
        for (size_t i = 0; i < (size_t)gw * gh * 2; i++) grid[i] = -1;
        int32_t md2 = (int32_t)ceilf(minDistance * minDistance);
        for (uint32_t i = 0; i < n; i++) {
            int x = list[i].x, y = list[i].y;
            int cx = x / (int)cell, cy = y / (int)cell;
            int16_t *cg = grid + 2 * ((size_t)cy * gw + cx);
            int found = 1;
            if (cg[0] < 0) {
                int x0 = cx - 2 > 0 ? cx - 2 : 0, x1 = cx + 2 < (int)gw - 1 ? cx + 2 : (int)gw - 1;
                int y0 = cy - 2 > 0 ? cy - 2 : 0, y1 = cy + 2 < (int)gh - 1 ? cy + 2 : (int)gh - 1;
                found = 0;
                for (int yy = y0; yy <= y1 && !found; yy++)
                    for (int xx = x0; xx <= x1; xx++) {
                        int16_t *g = grid + 2 * ((size_t)yy * gw + xx);
                        if (g[0] >= 0) {
                            int ddx = g[0] - x, ddy = g[1] - y;
                            if (ddx * ddx + ddy * ddy < md2) { found = 1; break; }
                        }
                    }
            }
            if (!found) {
                if (count < capacity) {
                    oracle_keypoint *k = &corners[count];
                    k->x = x; k->y = y; k->strength = list[i].s; k->tracking_status = 1;
                    k->error = 0; k->scale = 0; k->orientation = 0;
                }
                count++;
                cg[0] = (int16_t)x; cg[1] = (int16_t)y;
            }
        }
        free(grid);
    } else {
        count = n < capacity ? n : capacity;
        for (uint32_t i = 0; i < count; i++) {
            oracle_keypoint *k = &corners[i];
            k->x = list[i].x; k->y = list[i].y; k->strength = list[i].s; k->tracking_status = 1;
            k->error = 0; k->scale = 0; k->orientation = 0;
        }
    }
    *pCount = count;
    return 0;
}

float oracle_harris_norm_factor(int32_t gs)
{
    float f = 255.0f * (float)(1 << (gs - 1)) * 3;
    return f * f * f * f;
}
