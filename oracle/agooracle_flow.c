/* agooracle_flow.c -- CPU restatement (test oracle) of the AGO Gaussian pyramid level and
 * pyramidal Lucas-Kanade optical flow.  Test infrastructure only: the product never calls it.
 *
 * Follows amd_openvx/openvx/ago/ago_haf_cpu_pyramid.cpp (HafCpu_ScaleGaussianHalf_U8_U8_5x5,
 * :94) and ago_haf_cpu_opticalflow.cpp (ComputeSharr :65, HafCpu_OpticalFlowPyrLK_XY_XY_Generic
 * :153).  The LK restatement reproduces the reference's floating-point evaluation order lane
 * by lane (its SSE accumulators are 4-lane float vectors summed in a fixed order), and its
 * scratch-memory layout, because values the reference reads from scratch it never wrote in
 * the current level are part of its observable output.  Compile with -ffp-contract=off.
 * Pinned against the reference build by tests/test_oracle_pin_flow.py. */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#include "agooracle.h"

/* ---------------------------------------------------------------- pyramid level */
static inline unsigned gauss5_h(const uint8_t *p)        /* [1 4 6 4 1] at p[-2..2] */
{
    return (unsigned)p[-2] + 4u * p[-1] + 6u * p[0] + 4u * p[1] + (unsigned)p[2];
}

/* HafCpu_ScaleGaussianHalf_U8_U8_5x5 (ago_haf_cpu_pyramid.cpp:94) with the same arguments:
 * pDst is destination row 1, dstHeight = (destination height - 2), pSrc is source row 2.
 * Destination pixel (j, x) is the 5x5 [1 4 6 4 1]^2 sum around source row
 * 2j + (sampleFirstRow ? 0 : 1) (relative to pSrc - 2 rows + 2) and column
 * 2x + (sampleFirstColumn ? 0 : 1), shifted right by 8.  Reads two columns outside the row
 * at both ends (the caller's buffer layout decides what they hold).  The reference misplaces
 * the row+2 samples when the destination row is not 16-byte aligned (its scalar prefix loop
 * does not advance that pointer, :184); AGO image rows are 16-byte aligned, and this follows
 * the aligned case. */
int oracle_ScaleGaussianHalf_U8_U8_5x5(uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                                       const uint8_t *pSrc, uint32_t srcStride, int sampleFirstRow,
                                       int sampleFirstColumn)
{
    const uint8_t *src = pSrc + (sampleFirstRow ? 0 : srcStride) + (sampleFirstColumn ? 0 : 1);
    for (uint32_t j = 0; j < dstHeight; j++) {
        const uint8_t *c = src + (size_t)2 * j * srcStride;   /* centre row of this output row */
        uint8_t *d = pDst + (size_t)j * dstStride;
        for (uint32_t x = 0; x < dstWidth; x++) {
            const uint8_t *p = c + 2 * x;
            unsigned v = gauss5_h(p - 2 * (ptrdiff_t)srcStride) + 4u * gauss5_h(p - (ptrdiff_t)srcStride) +
                         6u * gauss5_h(p) + 4u * gauss5_h(p + srcStride) + gauss5_h(p + 2 * (size_t)srcStride);
            d[x] = (uint8_t)(v >> 8);
        }
    }
    return 0;
}

/* ---------------------------------------------------------------- Scharr derivatives */
static inline uintptr_t up16(uintptr_t p) { return (p + 15) & ~(uintptr_t)15; }

/* ComputeSharr (ago_haf_cpu_opticalflow.cpp:65).  For rows 1..H-2 and columns
 * [0, W & ~7) writes (gx, gy) int16 pairs; the two row buffers live in `scratch` at the
 * reference's offsets and are NOT cleared: column 0 reads the word before the first buffer
 * (never written) and the word before the second one, which holds whatever an earlier level
 * or an earlier call left there.  All arithmetic is 16-bit wrap-around like the SIMD code. */
static void lk_scharr(uint32_t dstStride, uint8_t *dst, uint32_t W, uint32_t H, uint32_t srcStride,
                      const uint8_t *src, uint8_t *scratch)
{
    uint16_t *t0 = (uint16_t *)up16((uintptr_t)(scratch + 2));
    uint16_t *t1 = (uint16_t *)up16((uintptr_t)(t0 + W + 2));
    const uint32_t W8 = W & ~7u;
    for (uint32_t y = 1; y + 1 < H; y++) {
        const uint8_t *r0 = src + (size_t)(y - 1) * srcStride, *r1 = r0 + srcStride, *r2 = r1 + srcStride;
        for (uint32_t x = 0; x < W8; x++) {
            t0[x] = (uint16_t)(3u * (r0[x] + r2[x]) + 10u * r1[x]);
            t1[x] = (uint16_t)((int)r2[x] - (int)r0[x]);
        }
        int16_t *d = (int16_t *)(dst + (size_t)y * dstStride);
        for (uint32_t x = 0; x < W8; x++) {
            d[2 * x] = (int16_t)(uint16_t)(t0[(int)x + 1] - t0[(int)x - 1]);
            d[2 * x + 1] = (int16_t)(uint16_t)(3u * (uint16_t)(t1[(int)x - 1] + t1[x + 1]) + 10u * t1[x]);
        }
    }
}

/* ---------------------------------------------------------------- tracking */
enum { kWBits = 14 };
#define LK_FLT_SCALE (1.f / (1 << 20))
#define TERM_ITERATIONS 0x0000F000 /* VX_TERM_CRITERIA_ITERATIONS = VX_ENUM_BASE(KHRONOS, 0x0F) + 0 */
#define TERM_EPSILON    0x0000F001
#define TERM_BOTH       0x0000F002
/* With termination EPSILON alone the reference loop has no iteration bound (:431) and does not
 * end for a point whose steps never shrink; this restatement, like the CUDA kernel, stops such
 * a point after this many iterations. */
#define LK_EPSILON_ONLY_MAX_ITERATIONS 4096u

static inline int descale(int v, int n) { return (v + (1 << (n - 1))) >> n; }
static inline int16_t sat16(int v) { return (int16_t)(v < -32768 ? -32768 : (v > 32767 ? 32767 : v)); }

/* bilinear weights as the reference computes them: float products, +0.5 in double, truncate */
static void lk_weights(float a, float b, int w[4])
{
    w[0] = (int)((double)((1.f - a) * (1.f - b) * (float)(1 << kWBits)) + 0.5);
    w[1] = (int)((double)(a * (1.f - b) * (float)(1 << kWBits)) + 0.5);
    w[2] = (int)((double)((1.f - a) * b * (float)(1 << kWBits)) + 0.5);
    w[3] = (1 << kWBits) - w[0] - w[1] - w[2];
}

typedef struct { float x, y; } lk_pt;

/* HafCpu_OpticalFlowPyrLK_XY_XY_Generic (ago_haf_cpu_opticalflow.cpp:153), same arguments.
 * `data` is the node's scratch (zeroed when the node is initialised, then kept across
 * calls); dataStride is the level-0 width * 4. */
int oracle_OpticalFlowPyrLK_XY_XY(oracle_keypoint *newKP, float pyramidScale, uint32_t levels,
                                  const oracle_pyramid_level *oldPyr, const oracle_pyramid_level *newPyr,
                                  uint32_t count, const oracle_keypoint *oldKP,
                                  const oracle_keypoint *estKP, int32_t termination, float epsilon,
                                  uint32_t numIterations, int32_t useInitialEstimate, uint32_t dataStride,
                                  uint8_t *data, int32_t winsz)
{
    const size_t halfWin = (size_t)(winsz >> 1);
    const float fHalf = (float)halfWin;
    int16_t Imat[256], dImat[512];
    uint8_t *scharrScratch = data;
    uint8_t *deriv = data + (oldPyr[0].width + 2) * 4 + 64;
    lk_pt *nextPts = (lk_pt *)(deriv + (size_t)oldPyr[0].width * oldPyr[0].height * 4);
    const uint32_t dStride = dataStride >> 1;   /* int16 elements */
    if (winsz < 1 || winsz > 15) return -1;

    for (int level = (int)levels - 1; level >= 0; level--) {
        const uint32_t dWidth = oldPyr[level].width - 2, dHeight = oldPyr[level].height - 2;
        const uint32_t JWidth = newPyr[level].width, JHeight = newPyr[level].height;
        const uint32_t IStride = oldPyr[level].stride, JStride = newPyr[level].stride;
        const uint8_t *SrcBase = oldPyr[level].image, *JBase = newPyr[level].image;
        const int16_t *DIBase = (const int16_t *)deriv;
        lk_scharr(dataStride, deriv, oldPyr[level].width, oldPyr[level].height, oldPyr[level].stride,
                  oldPyr[level].image, scharrScratch);
        const float ptScale = (float)pow((double)pyramidScale, (double)level);

        for (uint32_t pt = 0; pt < count; pt++) {
            if (!oldKP[pt].tracking_status) {
                newKP[pt].x = oldKP[pt].x;
                newKP[pt].y = oldKP[pt].y;
                newKP[pt].strength = oldKP[pt].strength;
                newKP[pt].tracking_status = oldKP[pt].tracking_status;
                newKP[pt].scale = oldKP[pt].scale;
                newKP[pt].error = oldKP[pt].error;
                continue;
            }
            lk_pt prev, next;
            prev.x = (float)oldKP[pt].x * ptScale;
            prev.y = (float)oldKP[pt].y * ptScale;
            if (level == (int)levels - 1) {
                if (useInitialEstimate) {
                    next.x = (float)estKP[pt].x * ptScale;
                    next.y = (float)estKP[pt].y * ptScale;
                    newKP[pt].strength = estKP[pt].strength;
                    newKP[pt].tracking_status = estKP[pt].tracking_status;
                    newKP[pt].error = estKP[pt].error;
                } else {
                    next = prev;
                    newKP[pt].tracking_status = oldKP[pt].tracking_status;
                    newKP[pt].strength = oldKP[pt].strength;
                }
                nextPts[pt] = next;
            } else {
                nextPts[pt].x *= 2.0f;
                nextPts[pt].y *= 2.0f;
                next = nextPts[pt];
            }
            if (!newKP[pt].tracking_status) continue;

            prev.x = prev.x - fHalf;
            prev.y = prev.y - fHalf;
            next.x = next.x - fHalf;
            next.y = next.y - fHalf;
            const int ipx = (int)floorf(prev.x), ipy = (int)floorf(prev.y);
            int bound = (ipx >> 31) | (ipx >= (int32_t)(dWidth - winsz)) | (ipy >> 31) | (ipy >= (int32_t)(dHeight - winsz));
            if (bound) {
                if (!level) {
                    newKP[pt].x = (int32_t)next.x;
                    newKP[pt].y = (int32_t)next.y;
                    newKP[pt].tracking_status = 0;
                    newKP[pt].error = 0;
                }
                continue;
            }
            float a = prev.x - (float)ipx, b = prev.y - (float)ipy;
            float A11 = 0, A12 = 0, A22 = 0;
            if (a == 0.0f && b == 0.0f) {
                /* integer position: one running float sum per entry; 4-pixel groups enter as
                 * the int sum of the group (x < winsz-4), the rest pixel by pixel */
                for (int y = 0; y < winsz; y++) {
                    const uint8_t *src = SrcBase + (size_t)(y + ipy) * IStride + ipx;
                    const int16_t *ds = DIBase + (size_t)(y + ipy) * dStride + (size_t)ipx * 2;
                    int x = 0;
                    for (; x < winsz - 4; x += 4) {
                        int s11 = 0, s12 = 0, s22 = 0;
                        for (int k = 0; k < 4; k++) {
                            int ix = ds[2 * (x + k)], iy = ds[2 * (x + k) + 1];
                            Imat[y * winsz + x + k] = (int16_t)(src[x + k] << 5);
                            dImat[2 * (y * winsz + x + k)] = (int16_t)ix;
                            dImat[2 * (y * winsz + x + k) + 1] = (int16_t)iy;
                            s11 += ix * ix; s12 += ix * iy; s22 += iy * iy;
                        }
                        A11 += (float)s11; A22 += (float)s22; A12 += (float)s12;
                    }
                    for (; x < winsz; x++) {
                        int ix = ds[2 * x], iy = ds[2 * x + 1];
                        Imat[y * winsz + x] = (int16_t)(src[x] << 5);
                        dImat[2 * (y * winsz + x)] = (int16_t)ix;
                        dImat[2 * (y * winsz + x) + 1] = (int16_t)iy;
                        A11 += (float)(ix * ix); A12 += (float)(ix * iy); A22 += (float)(iy * iy);
                    }
                }
            } else {
                int w[4];
                lk_weights(a, b, w);
                float q11[4] = {0, 0, 0, 0}, q12[4] = {0, 0, 0, 0}, q22[4] = {0, 0, 0, 0};
                for (int y = 0; y < winsz; y++) {
                    const uint8_t *src = SrcBase + (size_t)(y + ipy) * IStride + ipx;
                    const int16_t *ds = DIBase + (size_t)(y + ipy) * dStride + (size_t)ipx * 2;
                    int x = 0;
                    for (; x <= winsz - 4; x += 4) {        /* 4-lane float accumulators, lane = x & 3 */
                        for (int k = 0; k < 4; k++) {
                            int xx = x + k;
                            int iv = descale(src[xx] * w[0] + src[xx + 1] * w[1] + src[xx + IStride] * w[2] +
                                             src[xx + IStride + 1] * w[3], kWBits - 5);
                            const int16_t *d0 = ds + 2 * xx, *d1 = d0 + dStride;
                            int ix = descale(d0[0] * w[0] + d0[2] * w[1] + d1[0] * w[2] + d1[2] * w[3], kWBits);
                            int iy = descale(d0[1] * w[0] + d0[3] * w[1] + d1[1] * w[2] + d1[3] * w[3], kWBits);
                            Imat[y * winsz + xx] = sat16(iv);
                            dImat[2 * (y * winsz + xx)] = sat16(ix);
                            dImat[2 * (y * winsz + xx) + 1] = sat16(iy);
                            float fx = (float)sat16(ix), fy = (float)sat16(iy);
                            q22[k] = q22[k] + fy * fy;
                            q12[k] = q12[k] + fx * fy;
                            q11[k] = q11[k] + fx * fx;
                        }
                    }
                    for (; x < winsz; x++) {
                        int iv = descale(src[x] * w[0] + src[x + 1] * w[1] + src[x + IStride] * w[2] +
                                         src[x + IStride + 1] * w[3], kWBits - 5);
                        const int16_t *d0 = ds + 2 * x, *d1 = d0 + dStride;
                        int ix = descale(d0[0] * w[0] + d0[2] * w[1] + d1[0] * w[2] + d1[2] * w[3], kWBits);
                        int iy = descale(d0[1] * w[0] + d0[3] * w[1] + d1[1] * w[2] + d1[3] * w[3], kWBits);
                        Imat[y * winsz + x] = (int16_t)iv;
                        dImat[2 * (y * winsz + x)] = (int16_t)ix;
                        dImat[2 * (y * winsz + x) + 1] = (int16_t)iy;
                        A11 += (float)(ix * ix); A12 += (float)(ix * iy); A22 += (float)(iy * iy);
                    }
                }
                if (winsz >= 4) {
                    A11 += ((q11[0] + q11[1]) + q11[2]) + q11[3];
                    A12 += ((q12[0] + q12[1]) + q12[2]) + q12[3];
                    A22 += ((q22[0] + q22[1]) + q22[2]) + q22[3];
                }
            }
            A11 *= LK_FLT_SCALE;
            A12 *= LK_FLT_SCALE;
            A22 *= LK_FLT_SCALE;

            float D = A11 * A22 - A12 * A12;
            float t = (A11 - A22) * (A11 - A22) + 4.f * A12 * A12;
            float minEig = (A22 + A11 - sqrtf(t)) / (float)(2 * winsz * winsz);
            if (minEig < 1.0e-04F || D < 1.0e-07F) {
                if (!level) {
                    newKP[pt].x = (int32_t)next.x;
                    newKP[pt].y = (int32_t)next.y;
                    newKP[pt].tracking_status = 0;
                    newKP[pt].error = 0;
                }
                continue;
            }
            D = 1.f / D;

            float prevDx = 0.f, prevDy = 0.f, ddx = 0.f, ddy = 0.f;
            unsigned j = 0;
            while (j < numIterations || (termination == TERM_EPSILON && j < LK_EPSILON_ONLY_MAX_ITERATIONS)) {
                const int inx = (int)floorf(next.x), iny = (int)floorf(next.y);
                bound = (inx >> 31) | (inx >= (int32_t)(JWidth - winsz)) | (iny >> 31) | (iny >= (int32_t)(JHeight - winsz));
                if (bound) {
                    if (!level) {
                        newKP[pt].tracking_status = 0;
                        newKP[pt].error = 0;
                    }
                    break;
                }
                a = next.x - (float)inx;
                b = next.y - (float)iny;
                int w[4];
                lk_weights(a, b, w);
                double ib1 = 0, ib2 = 0;
                float qb0[4] = {0, 0, 0, 0}, qb1[4] = {0, 0, 0, 0};
                for (int y = 0; y < winsz; y++) {
                    const uint8_t *J = JBase + (size_t)(y + iny) * JStride + inx;
                    const int16_t *Ip = &Imat[y * winsz];
                    const int16_t *dIp = &dImat[2 * y * winsz];
                    int x = 0;
                    for (; x <= winsz - 8; x += 8) {
                        /* per half of 4 pixels: qb0 += {Ix*It, Iy*It} of pixels 0,1; qb1 of 2,3 */
                        for (int h = 0; h < 2; h++) {
                            for (int k = 0; k < 4; k++) {
                                int xx = x + 4 * h + k;
                                int jv = descale(J[xx] * w[0] + J[xx + 1] * w[1] + J[xx + JStride] * w[2] +
                                                 J[xx + JStride + 1] * w[3], kWBits - 5);
                                int it = sat16((int)sat16(jv) - (int)Ip[xx]);
                                float px = (float)(dIp[2 * xx] * it), py = (float)(dIp[2 * xx + 1] * it);
                                float *q = (k < 2) ? qb0 : qb1;
                                int lane = 2 * (k & 1);
                                q[lane] = q[lane] + px;
                                q[lane + 1] = q[lane + 1] + py;
                            }
                        }
                    }
                    for (; x < winsz; x++) {
                        int diff = descale(J[x] * w[0] + J[x + 1] * w[1] + J[x + JStride] * w[2] +
                                           J[x + JStride + 1] * w[3], kWBits - 5);
                        diff -= Ip[x];
                        ib1 += (float)(diff * dIp[2 * x]);
                        ib2 += (float)(diff * dIp[2 * x + 1]);
                    }
                }
                if (winsz >= 8) {
                    float bb[4];
                    for (int k = 0; k < 4; k++) bb[k] = qb0[k] + qb1[k];
                    ib1 += bb[0] + bb[2];
                    ib2 += bb[1] + bb[3];
                }
                const float b1 = (float)(ib1 * LK_FLT_SCALE), b2 = (float)(ib2 * LK_FLT_SCALE);
                const float dx = (A12 * b2 - A22 * b1) * D;
                const float dy = (A12 * b1 - A11 * b2) * D;
                next.x += dx;
                next.y += dy;
                if ((dx * dx + dy * dy) <= epsilon && (termination == TERM_EPSILON || termination == TERM_BOTH)) break;
                if (j > 0 && fabsf(dx + prevDx) < 0.01 && fabsf(dy + prevDy) < 0.01) {
                    ddx = dx * 0.5f;
                    ddy = dy * 0.5f;
                    break;
                }
                prevDx = dx;
                prevDy = dy;
                j++;
            }
            if (!level) {
                newKP[pt].x = (int32_t)(next.x + fHalf - ddx + 0.5f);
                newKP[pt].y = (int32_t)(next.y + fHalf - ddy + 0.5f);
            } else {
                nextPts[pt].x = next.x + fHalf - ddx;
                nextPts[pt].y = next.y + fHalf - ddy;
            }
        }
    }
    return 0;
}

/* Bytes of node scratch the reference allocates for this node (ago_kernel_api.cpp:20636). */
size_t oracle_OpticalFlowPyrLK_scratch_size(uint32_t width0, uint32_t height0, uint32_t capacity)
{
    return ((size_t)height0 * width0 * 4 + (size_t)capacity * 8 + 256) + ((size_t)(width0 + 2) * 4 + 64);
}
