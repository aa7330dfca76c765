/*
 * agooracle.c -- plain-C restatement of the AGO HAF CPU kernels (test infrastructure
 * only; see agooracle.h).  Each function cites the reference function it follows.
 * Built with -ffp-contract=off so float expressions keep the reference's
 * multiply-then-add order (the reference's SSE code has no FMA).
 */
#include "agooracle.h"
#include <math.h>
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
