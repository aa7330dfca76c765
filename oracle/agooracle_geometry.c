/*
 * agooracle_geometry.c -- plain-C restatement of the AGO HAF colour-conversion, scaling
 * and warp kernels (test infrastructure only; see agooracle.h).
 */
#include "agooracle.h"
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

static int rne_d(double v) { return (int)nearbyint(v); }

/* ========================= colour conversion ============================ */

/* Y/U/V of one RGB pixel in the reference's SIMD order (ago_haf_cpu_color_convert.cpp:2740-2800):
 * products then sums left to right, BT.709 weights, U/V offset by 128. */
static void rgb_yuv_f(int R, int G, int B, float *y, float *u, float *v)
{
    float r = (float)R, g = (float)G, b = (float)B;
    *y = ((r * 0.2126f) + (g * 0.7152f)) + (b * 0.0722f);
    *u = (((r * -0.1146f) + (g * -0.3854f)) + (b * 0.5f)) + 128.0f;
    *v = (((r * 0.5f) + (g * -0.4542f)) + (b * -0.0458f)) + 128.0f;
}

static int trunc_sat_u16(float f) { int i = (int)f; return i < 0 ? 0 : i > 65535 ? 65535 : i; }   /* cvttps + packus_epi32 */
static int sat_u8(int v) { return v < 0 ? 0 : v > 255 ? 255 : v; }

/* One 2x2 block at (x, y) of an RGB image: Y of the four pixels and the shared U, V.
 * SIMD body (x < W & ~3): U = ((avg(u00,u10) + avg(u01,u11)) + 1) >> 1 with the rounding
 * average of _mm_avg_epu16.  Scalar tail: the float sum of the four (u + 128) values / 4,
 * truncated, and Y computed with the double constant 0.0722 (color_convert.cpp:2866). */
static void rgb_block(const uint8_t *s0, const uint8_t *s1, int simd, uint8_t y[4], uint8_t *U, uint8_t *V)
{
    const uint8_t *px[4] = {s0, s0 + 3, s1, s1 + 3};
    if (simd) {
        int uu[4], vv[4];
        for (int i = 0; i < 4; i++) {
            float fy, fu, fv;
            rgb_yuv_f(px[i][0], px[i][1], px[i][2], &fy, &fu, &fv);
            y[i] = (uint8_t)sat_u8(trunc_sat_u16(fy));
            uu[i] = trunc_sat_u16(fu);
            vv[i] = trunc_sat_u16(fv);
        }
        int ua = (uu[0] + uu[2] + 1) >> 1, ub = (uu[1] + uu[3] + 1) >> 1;
        int va = (vv[0] + vv[2] + 1) >> 1, vb = (vv[1] + vv[3] + 1) >> 1;
        *U = (uint8_t)sat_u8(((ua + ub) + 1) >> 1);
        *V = (uint8_t)sat_u8(((va + vb) + 1) >> 1);
    } else {
        float u = 0, v = 0;
        for (int i = 0; i < 4; i++) {
            float R = (float)px[i][0], G = (float)px[i][1], B = (float)px[i][2];
            y[i] = (uint8_t)(int)((double)((R * 0.2126f) + (G * 0.7152f)) + (double)B * 0.0722);
            float uu = (R * -0.1146f) + (G * -0.3854f) + (B * 0.5f) + 128.0f;
            float vv = (R * 0.5f) + (G * -0.4542f) + (B * -0.0458f) + 128.0f;
            if (i == 0) { u = uu; v = vv; } else { u += uu; v += vv; }
        }
        u /= 4.0f; v /= 4.0f;
        *U = (uint8_t)(int)u; *V = (uint8_t)(int)v;
    }
}

/* ago_haf_cpu_color_convert.cpp:2707 HafCpu_ColorConvert_NV12_RGB */
int oracle_ColorConvert_NV12_RGB(uint32_t W, uint32_t H, uint8_t *pY, uint32_t yStride, uint8_t *pUV, uint32_t uvStride,
                                 const uint8_t *pSrc, uint32_t srcStride)
{
    const uint32_t aligned = W & ~3u;
    for (uint32_t y = 0; y < H; y += 2) {
        const uint8_t *s0 = pSrc + (size_t)y * srcStride, *s1 = s0 + srcStride;
        uint8_t *y0 = pY + (size_t)y * yStride, *y1 = y0 + yStride, *c = pUV + (size_t)(y / 2) * uvStride;
        for (uint32_t x = 0; x < W; x += 2) {
            uint8_t yy[4], U, V;
            rgb_block(s0 + 3 * x, s1 + 3 * x, x < aligned, yy, &U, &V);
            y0[x] = yy[0]; y0[x + 1] = yy[1]; y1[x] = yy[2]; y1[x + 1] = yy[3];
            c[x] = U; c[x + 1] = V;
        }
    }
    return 0;
}

/* ago_haf_cpu_color_convert.cpp:2492 HafCpu_ColorConvert_IYUV_RGB (same arithmetic) */
int oracle_ColorConvert_IYUV_RGB(uint32_t W, uint32_t H, uint8_t *pY, uint32_t yStride, uint8_t *pU, uint32_t uStride,
                                 uint8_t *pV, uint32_t vStride, const uint8_t *pSrc, uint32_t srcStride)
{
    const uint32_t aligned = W & ~3u;
    for (uint32_t y = 0; y < H; y += 2) {
        const uint8_t *s0 = pSrc + (size_t)y * srcStride, *s1 = s0 + srcStride;
        uint8_t *y0 = pY + (size_t)y * yStride, *y1 = y0 + yStride;
        for (uint32_t x = 0; x < W; x += 2) {
            uint8_t yy[4], U, V;
            rgb_block(s0 + 3 * x, s1 + 3 * x, x < aligned, yy, &U, &V);
            y0[x] = yy[0]; y0[x + 1] = yy[1]; y1[x] = yy[2]; y1[x + 1] = yy[3];
            pU[(size_t)(y / 2) * uStride + x / 2] = U;
            pV[(size_t)(y / 2) * vStride + x / 2] = V;
        }
    }
    return 0;
}

/* ============================ scaling =================================== */
/* scale matrix of the AGO wrappers (ago_kernel_api.cpp:19908-19911 bilinear, :19788-19791
 * nearest, :20272-20275 area), in float as the reference stores it */
void oracle_scale_matrix(int kind, uint32_t srcW, uint32_t srcH, uint32_t dstW, uint32_t dstH, float m[4])
{
    m[0] = (float)((double)srcW / (double)dstW);
    m[1] = (float)((double)srcH / (double)dstH);
    if (kind == 0) {        /* nearest */
        m[2] = (float)((double)srcW / (double)dstW * 0.5);
        m[3] = (float)((double)srcH / (double)dstH * 0.5);
    } else if (kind == 1) { /* bilinear */
        m[2] = (float)((double)srcW / (double)dstW * 0.5 - 0.5);
        m[3] = (float)((double)srcH / (double)dstH * 0.5 - 0.5);
    } else {                /* area */
        m[2] = -0.5f;
        m[3] = -0.5f;
    }
}

/* ago_haf_cpu_geometric.cpp:1977 HafCpu_ScaleImage_U8_U8_Bilinear: 18-bit fixed-point maps,
 * 8-bit weights ((frac + 0x200) >> 10), two rounded 8-bit stages for x < W & ~7, a single
 * (.. + 0x8000) >> 16 stage for the tail; reads x+1 even at the right edge. */
int oracle_ScaleImage_U8_U8_Bilinear(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW, uint32_t srcH,
                                     const uint8_t *pSrc, uint32_t srcStride, const float m[4])
{
    const int FPB = 18, FPM = 1 << 18;
    int yinc = (int)(FPM * m[1]), xinc = (int)(FPM * m[0]);
    int yoffs = (int)(FPM * m[3]), xoffs = (int)(FPM * m[2]);
    const uint32_t simdW = W & ~7u;
    for (int y = 0, ypos = yoffs; y < (int)H; y++, ypos += yinc) {
        int ym = ypos >> FPB, yf = ((ypos & 0x3ffff) + 0x200) >> 10, omy = 0x100 - yf;
        const uint8_t *r1, *r2;
        if (ym < 0) r1 = r2 = pSrc;
        else if (ym >= (int)srcH - 1) r1 = r2 = pSrc + (size_t)(srcH - 1) * srcStride;
        else { r1 = pSrc + (size_t)ym * srcStride; r2 = r1 + srcStride; }
        uint8_t *d = pDst + (size_t)y * dstStride;
        int xpos = xoffs;
        for (uint32_t x = 0; x < W; x++, xpos += xinc) {
            int xm = xpos >> FPB;
            if (xm < 0) xm = 0;
            int xf = ((xpos & 0x3ffff) + 0x200) >> 10, omx = 0x100 - xf;
            int p1 = r1[xm], p2 = r1[xm + 1], p3 = r2[xm], p4 = r2[xm + 1];
            if (x < simdW) {
                int t1 = (((omx * p1) & 0xffff) + ((xf * p2) & 0xffff) + 0x80) & 0xffff;
                t1 >>= 8;
                int t2 = (((omx * p3) & 0xffff) + ((xf * p4) & 0xffff) + 0x80) & 0xffff;
                t2 >>= 8;
                int o = ((((omy * t1) & 0xffff) + ((yf * t2) & 0xffff) + 0x80) & 0xffff) >> 8;
                d[x] = (uint8_t)sat_u8(o);
            } else {
                d[x] = (uint8_t)(((omx * omy * p1) + (xf * omy * p2) + (omx * yf * p3) + (xf * yf * p4) + 0x8000) >> 16);
            }
        }
    }
    return 0;
}

/* ago_haf_cpu_geometric.cpp:1874 HafCpu_ScaleImage_U8_U8_Nearest: clamped 18-bit maps. */
int oracle_ScaleImage_U8_U8_Nearest(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW, uint32_t srcH,
                                    const uint8_t *pSrc, uint32_t srcStride, const float m[4])
{
    const int FPB = 18, FPM = 1 << 18;
    int yinc = (int)(FPM * m[1]), xinc = (int)(FPM * m[0]);
    int yoffs = (int)(FPM * m[3]), xoffs = (int)(FPM * m[2]);
    for (int y = 0, ypos = yoffs; y < (int)H; y++, ypos += yinc) {
        int ym = ypos >> FPB;
        if (ym > (int)srcH - 1) ym = (int)srcH - 1;
        if (ym < 0) ym = 0;
        int xpos = xoffs;
        for (uint32_t x = 0; x < W; x++, xpos += xinc) {
            int xm = xpos >> FPB;
            if (xm > (int)srcW - 1) xm = (int)srcW - 1;
            if (xm < 0) xm = 0;
            pDst[(size_t)y * dstStride + x] = pSrc[(size_t)ym * srcStride + xm];
        }
    }
    return 0;
}

/* ago_haf_cpu_geometric.cpp:2491 HafCpu_ScaleImage_U8_U8_Area, the exact 1x and 2x paths:
 * 2x: (a+b+c+d+2) >> 2 over source rows (int)(yoffset + 2y) clamped to [0, srcH-2] and
 * columns from (int)xoffset, for the first (W & ~7) columns (the rest are not written).
 * Returns -1 for other ratios (the generic path is not restated). */
int oracle_ScaleImage_U8_U8_Area(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW, uint32_t srcH,
                                 const uint8_t *pSrc, uint32_t srcStride, const float m[4])
{
    (void)srcW;
    if (m[0] == 1.0f && m[1] == 1.0f) {
        for (uint32_t y = 0; y < H; y++) {
            long r = (long)(int)(m[3] + (float)y), c = (int)m[2];
            const uint8_t *s = pSrc + r * (long)srcStride + c;
            if (s < pSrc) s = pSrc;
            if (s > pSrc + (size_t)(H - 1) * srcStride) s = pSrc + (size_t)(H - 1) * srcStride;
            memcpy(pDst + (size_t)y * dstStride, s, W);
        }
        return 0;
    }
    if (m[0] == 2.0f && m[1] == 2.0f) {
        const uint8_t *last = pSrc + (size_t)(srcH - 2) * srcStride;
        for (uint32_t y = 0; y < H; y++) {
            const uint8_t *s0 = pSrc + (long)(int)(m[3] + (float)(y * 2)) * (long)srcStride + (int)m[2];
            if (s0 < pSrc) s0 = pSrc;
            if (s0 > last) s0 = last;
            const uint8_t *s1 = s0 + srcStride;
            for (uint32_t x = 0; x < (W & ~7u); x++)
                pDst[(size_t)y * dstStride + x] = (uint8_t)((s0[2 * x] + s0[2 * x + 1] + s1[2 * x] + s1[2 * x + 1] + 2) >> 2);
        }
        return 0;
    }
    return -1;
}

/* ============================ warp affine =============================== */
/* ago_affine_matrix_t: float matrix[3][2]; x' = m00*x + m10*y + m20, y' = m01*x + m11*y + m21
 * with m[row][col] as stored (geometric.cpp:679-684). */
static int warp_needs_border(const float *m, uint32_t dstW, uint32_t dstH, uint32_t srcW, uint32_t srcH)
{
    const float r00 = m[0], r10 = m[1], r01 = m[2], r11 = m[3], c1 = m[4], c2 = m[5];
    const float sw = (float)srcW, sh = (float)srcH;
    int b = (c1 < 0) | (c2 < 0) | (c1 >= sw) | (c2 >= sh);
    float x1 = (r00 * (float)dstW + c1), y1 = (r10 * (float)dstW + c2);
    b |= (x1 < 0) | (y1 < 0) | (x1 >= sw) | (y1 >= sh);
    x1 = (r01 * (float)dstH + c1); y1 = (r11 * (float)dstH + c2);
    b |= (x1 < 0) | (y1 < 0) | (x1 >= sw) | (y1 >= sh);
    x1 = (r00 * (float)dstW + r01 * (float)dstH + c1); y1 = (r10 * (float)dstW + r11 * (float)dstH + c2);
    b |= (x1 < 0) | (y1 < 0) | (x1 >= sw) | (y1 >= sh);
    return b;
}

/* ago_haf_cpu_geometric.cpp:658 HafCpu_WarpAffine_U8_U8_Nearest_Constant: source position
 * (m00*x) + (y*m10 + m20) in float with m00*x per column, truncated; when any mapped image
 * corner falls outside the source, pixels outside the image or the source valid rectangle
 * get the border value.  Destination width is processed in 4-pixel groups. */
int oracle_WarpAffine_U8_U8_Nearest_Constant(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW,
                                             uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride, const float *m,
                                             uint8_t border, uint32_t vsx, uint32_t vsy, uint32_t vex, uint32_t vey)
{
    const float r00 = m[0], r10 = m[1], r01 = m[2], r11 = m[3], c1 = m[4], c2 = m[5];
    const int bb = warp_needs_border(m, W, H, srcW, srcH);
    const long lim = (long)srcH * srcStride - 1;
    const uint32_t W4 = (W + 3) & ~3u;
    for (uint32_t y = 0; y < H; y++) {
        const float xd = (float)y * r01 + c1, yd = (float)y * r11 + c2;
        for (uint32_t x = 0; x < W4; x++) {
            const float xs = (r00 * (float)x) + xd, ys = (r10 * (float)x) + yd;
            long idx = (long)(int)ys * (long)srcStride + (long)(int)xs;
            uint8_t v;
            if (bb) {
                int ok = xs >= 0 && xs < (float)srcW && ys >= 0 && ys < (float)srcH && xs >= (float)vsx && xs < (float)vex &&
                         ys >= (float)vsy && ys < (float)vey;
                if (idx > lim) idx = lim;
                if (idx < 0) idx = 0;
                v = ok ? pSrc[idx] : border;
            } else {
                v = pSrc[idx];
            }
            pDst[(size_t)y * dstStride + x] = v;
        }
    }
    return 0;
}

/* ago_haf_cpu_geometric.cpp:1100 HafCpu_WarpAffine_U8_U8_Bilinear_Constant: fractions
 * from the truncated position, ((p0*(1-fx))*(1-fy) + (p1*fx)*(1-fy)) + ((p2*(1-fx))*fy +
 * (p3*fx)*fy) rounded to nearest even; the in-bounds test applies to the top-left tap. */
int oracle_WarpAffine_U8_U8_Bilinear_Constant(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW,
                                              uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride, const float *m,
                                              uint8_t border)
{
    const float r00 = m[0], r10 = m[1], r01 = m[2], r11 = m[3], c1 = m[4], c2 = m[5];
    const int bb = warp_needs_border(m, W, H, srcW, srcH);
    const long lim = (long)srcH * srcStride - 1;
    const uint32_t W4 = (W + 3) & ~3u;
    for (uint32_t y = 0; y < H; y++) {
        const float xd = (float)y * r01 + c1, yd = (float)y * r11 + c2;
        for (uint32_t x = 0; x < W4; x++) {
            const float xs = (r00 * (float)x) + xd, ys = (r10 * (float)x) + yd;
            const int xi = (int)xs, yi = (int)ys;
            const float fx = xs - (float)xi, fy = ys - (float)yi;
            const float omx = 1.0f - fx, omy = 1.0f - fy;
            long idx = (long)yi * (long)srcStride + xi;
            if (idx > lim) idx = lim;
            if (idx < 0) idx = 0;
            const uint8_t *p = pSrc + idx;
            float a = ((float)p[0] * omx) * omy, b = ((float)p[1] * fx) * omy;
            float c = ((float)p[srcStride] * omx) * fy, d = ((float)p[srcStride + 1] * fx) * fy;
            int v = rne_d((double)((a + b) + (c + d)));
            int ok = !bb || (xs >= 0 && xs < (float)srcW && ys >= 0 && ys < (float)srcH);
            v = ok ? v : border;
            pDst[(size_t)y * dstStride + x] = (uint8_t)sat_u8(v);
        }
    }
    return 0;
}

/* ---------------------------------------------------------------- WarpPerspective */
/* _mm_cvttps_epi32: truncation, 0x80000000 for NaN and values outside int32 */
static int32_t cvtt_i32(float f)
{
    return (f >= -2147483648.0f && f < 2147483648.0f) ? (int32_t)f : INT32_MIN;
}
/* _mm_packus_epi32 then _mm_packus_epi16 of one lane */
static uint8_t pack_u8(int32_t v)
{
    const int32_t u16 = v < 0 ? 0 : (v > 65535 ? 65535 : v);
    const int16_t s16 = (int16_t)(uint16_t)u16;
    return (uint8_t)(s16 < 0 ? 0 : (s16 > 255 ? 255 : s16));
}

/* ago_haf_cpu_geometric.cpp:1406 HafCpu_WarpPerspective_U8_U8_Nearest_Constant.  m is
 * ago_perspective_matrix_t (float[3][3]); per column a*x, d*x, g*x in float, per row
 * y*b + c, y*e + f, y*h + i; x' = (a*x + (y*b + c)) * (1 / (g*x + (y*h + i))).  In range
 * (0 <= x' < W, 0 <= y' < H, float compares): pixel (trunc x', trunc y'), else border.
 * The UNDEFINED-border kernel (:1372) is this with border 0. */
int oracle_WarpPerspective_U8_U8_Nearest_Constant(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                                  uint32_t srcW, uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride,
                                                  const float *m, uint8_t border)
{
    const float a = m[0], d = m[1], g = m[2], b = m[3], e = m[4], h = m[5], c = m[6], f = m[7], i = m[8];
    const int32_t srcb = (int32_t)(srcH * srcStride - 1);
    for (uint32_t y = 0; y < H; y++) {
        const float xd = (float)y * b + c, yd = (float)y * e + f, zd = (float)y * h + i;
        for (uint32_t x = 0; x < W; x++) {
            const float z = 1.0f / ((g * (float)x) + zd);
            const float xm = ((a * (float)x) + xd) * z, ym = ((d * (float)x) + yd) * z;
            const int ok = xm >= 0.f && xm < (float)srcW && ym >= 0.f && ym < (float)srcH;
            int32_t off = (int32_t)((uint32_t)cvtt_i32(ym) * srcStride + (uint32_t)cvtt_i32(xm));
            off = off > srcb ? srcb : (off < 0 ? 0 : off);
            pDst[(size_t)y * dstStride + x] = ok ? pSrc[off] : border;
        }
    }
    return 0;
}

/* ago_haf_cpu_geometric.cpp:1579 HafCpu_WarpPerspective_U8_U8_Bilinear_Constant.  Integer
 * position trunc(x') - (x' < 0); taps p0 (x, y) and p2 (x, y+1) are the border unless
 * 0 <= x < W and 0 <= y < H, taps p1 (x+1, y) and p3 (x+1, y+1) unless -1 <= x < W and
 * -1 <= y < H; the four bytes come from the flat offset y*stride + x clamped to
 * [0, H*stride - 1] (and the next row).  ((p0*(1-fx))*(1-fy) + (p1*fx)*(1-fy)) +
 * (p2*(1-fx))*fy + (p3*fx)*fy summed left to right, truncated, saturated. */
int oracle_WarpPerspective_U8_U8_Bilinear_Constant(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                                   uint32_t srcW, uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride,
                                                   const float *m, uint8_t border)
{
    const float a = m[0], d = m[1], g = m[2], b = m[3], e = m[4], h = m[5], c = m[6], f = m[7], i = m[8];
    const int32_t srcb = (int32_t)(srcH * srcStride - 1);
    for (uint32_t y = 0; y < H; y++) {
        const float xd = (float)y * b + c, yd = (float)y * e + f, zd = (float)y * h + i;
        for (uint32_t x = 0; x < W; x++) {
            const float z = 1.0f / ((g * (float)x) + zd);
            const float xm = ((a * (float)x) + xd) * z, ym = ((d * (float)x) + yd) * z;
            const int32_t xi = (int32_t)((uint32_t)cvtt_i32(xm) - (uint32_t)(xm < 0.f));
            const int32_t yi = (int32_t)((uint32_t)cvtt_i32(ym) - (uint32_t)(ym < 0.f));
            const int ok = xi >= 0 && xi < (int32_t)srcW && yi >= 0 && yi < (int32_t)srcH;
            const int ok1 = xi >= -1 && xi < (int32_t)srcW && yi >= -1 && yi < (int32_t)srcH;
            const float fx = xm - (float)xi, fy = ym - (float)yi;
            int32_t off = (int32_t)((uint32_t)yi * srcStride + (uint32_t)xi);
            off = off > srcb ? srcb : (off < 0 ? 0 : off);
            const uint8_t *p = pSrc + off;
            const float p0 = ok ? p[0] : border, p2 = ok ? p[srcStride] : border;
            const float p1 = ok1 ? p[1] : border, p3 = ok1 ? p[srcStride + 1] : border;
            const float omx = 1.0f - fx, omy = 1.0f - fy;
            const float s0 = (p0 * omx) * omy, s1 = (p1 * fx) * omy, s2 = (p2 * omx) * fy, s3 = (p3 * fx) * fy;
            pDst[(size_t)y * dstStride + x] = pack_u8(cvtt_i32(((s0 + s1) + s2) + s3));
        }
    }
    return 0;
}

/* ---------------------------------------------------------------- Remap */
/* vxSetRemapPoint (api/vx_api.cpp:7884): the table AGO's kernels read holds u16 fixed-point
 * coordinates with ago_util.cpp:2451's fractional bits (3 below 8192 pixels), rounded with
 * + 0.5f in float; a source point outside [0, W-1) x [0, H-1) stores 0xFFFF in both. */
void oracle_remap_fixed(uint32_t srcW, uint32_t srcH, const float *xy, size_t n, uint16_t *out)
{
    int bits = 3;
    if (srcW >= (1u << 15) || srcH >= (1u << 15)) bits = 0;
    else if (srcW >= (1u << 14) || srcH >= (1u << 14)) bits = 1;
    else if (srcW >= (1u << 13) || srcH >= (1u << 13)) bits = 2;
    const float s = (float)(1 << bits);
    for (size_t k = 0; k < n; k++) {
        const float sx = xy[2 * k], sy = xy[2 * k + 1];
        if (sx < 0.0f || sy < 0.0f || sx >= (float)(srcW - 1) || sy >= (float)(srcH - 1)) {
            out[2 * k] = out[2 * k + 1] = 0xFFFF;
        } else {
            out[2 * k] = (uint16_t)(uint32_t)cvtt_i32(sx * s + 0.5f);
            out[2 * k + 1] = (uint16_t)(uint32_t)cvtt_i32(sy * s + 0.5f);
        }
    }
}

/* ago_haf_cpu_geometric.cpp:372 / :249 HafCpu_Remap_U8_U8_Bilinear[_Constant]: 3 fractional
 * bits, weights (8-fx)(8-fy), fx(8-fy), (8-fx)fy, fx*fy, (sum + 32) >> 6.  A 0xFFFF x or y
 * is read as 0 (constant) or 8 (undefined); with a constant border only a 0xFFFF x gives the
 * border value (the mask is applied per 16-bit half of the 32-bit result). */
static void remap_bilinear(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, const uint8_t *pSrc,
                           uint32_t srcStride, const uint16_t *pMap, uint32_t mapStride, int constant, uint8_t border)
{
    for (uint32_t y = 0; y < H; y++) {
        const uint16_t *mr = (const uint16_t *)((const uint8_t *)pMap + (size_t)y * mapStride);
        for (uint32_t x = 0; x < W; x++) {
            uint32_t mx = mr[2 * x], my = mr[2 * x + 1];
            const int bx = mx == 0xFFFF, by = my == 0xFFFF;
            if (bx) mx = constant ? 0 : 8;
            if (by) my = constant ? 0 : 8;
            const uint32_t fx = mx & 7, fy = my & 7;
            const uint8_t *p = pSrc + (size_t)(my >> 3) * srcStride + (mx >> 3);
            const uint32_t v = (p[0] * (8 - fx) * (8 - fy) + p[1] * fx * (8 - fy) + p[srcStride] * (8 - fx) * fy +
                                p[srcStride + 1] * fx * fy + 32) >> 6;
            pDst[(size_t)y * dstStride + x] = (constant && bx) ? border : pack_u8((int32_t)v);
        }
    }
}

int oracle_Remap_U8_U8_Bilinear_Constant(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW,
                                         uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride, const uint16_t *pMap,
                                         uint32_t mapStride, uint8_t border)
{
    (void)srcW; (void)srcH;
    remap_bilinear(W, H, pDst, dstStride, pSrc, srcStride, pMap, mapStride, 1, border);
    return 0;
}

int oracle_Remap_U8_U8_Bilinear(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW, uint32_t srcH,
                                const uint8_t *pSrc, uint32_t srcStride, const uint16_t *pMap, uint32_t mapStride)
{
    (void)srcW; (void)srcH;
    remap_bilinear(W, H, pDst, dstStride, pSrc, srcStride, pMap, mapStride, 0, 0);
    return 0;
}

/* ago_haf_cpu_geometric.cpp:156 / :72 HafCpu_Remap_U8_U8_Nearest[_Constant]: position
 * (v >> 3) + (frac > 3).  The 4-pixel SIMD body (x < W & ~3) reads a 0xFFFF coordinate as 0
 * and emits the border for it (or for a flat offset past the image) with a constant border,
 * and as 7 (position 1) without one; the scalar tail (x >= W & ~3) replaces a 0xFFFF
 * coordinate by the border value (constant) or 0 (undefined) and reads that position.
 * Tail reads outside the source buffer read 0 here (the reference reads past its buffer). */
static void remap_nearest(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcH, const uint8_t *pSrc,
                          uint32_t srcStride, const uint16_t *pMap, uint32_t mapStride, int constant, uint8_t border)
{
    const int32_t srcb = (int32_t)(srcH * srcStride - 1);
    const uint32_t W4 = W & ~3u;
    for (uint32_t y = 0; y < H; y++) {
        const uint16_t *mr = (const uint16_t *)((const uint8_t *)pMap + (size_t)y * mapStride);
        uint8_t *d = pDst + (size_t)y * dstStride;
        for (uint32_t x = 0; x < W4; x++) {
            uint32_t mx = mr[2 * x], my = mr[2 * x + 1];
            const int bx = mx == 0xFFFF, by = my == 0xFFFF;
            if (bx) mx = constant ? 0 : 7;
            if (by) my = constant ? 0 : 7;
            const int32_t ix = (int32_t)(mx >> 3) + ((mx & 7) > 3), iy = (int32_t)(my >> 3) + ((my & 7) > 3);
            const int32_t off = (int32_t)((uint32_t)iy * srcStride + (uint32_t)ix);
            if (constant && (bx || by || off > srcb)) d[x] = border;
            else d[x] = pSrc[off];
        }
        for (uint32_t x = W4; x < W; x++) {
            const int16_t sx = (int16_t)mr[2 * x], sy = (int16_t)mr[2 * x + 1];
            const int xx = sx != -1 ? (sx >> 3) + ((sx & 7) >> 2) : (constant ? border : 0);
            const int yy = sy != -1 ? (sy >> 3) + ((sy & 7) >> 2) : (constant ? border : 0);
            const long off = (long)yy * srcStride + xx;
            d[x] = (off >= 0 && off <= srcb) ? pSrc[off] : 0;
        }
    }
}

int oracle_Remap_U8_U8_Nearest_Constant(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW,
                                        uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride, const uint16_t *pMap,
                                        uint32_t mapStride, uint8_t border)
{
    (void)srcW;
    remap_nearest(W, H, pDst, dstStride, srcH, pSrc, srcStride, pMap, mapStride, 1, border);
    return 0;
}

int oracle_Remap_U8_U8_Nearest(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW, uint32_t srcH,
                               const uint8_t *pSrc, uint32_t srcStride, const uint16_t *pMap, uint32_t mapStride)
{
    (void)srcW;
    remap_nearest(W, H, pDst, dstStride, srcH, pSrc, srcStride, pMap, mapStride, 0, 0);
    return 0;
}
