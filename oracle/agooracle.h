/*
 * agooracle.h -- CPU restatement of the AMD OpenVX (AGO) HAF CPU kernels on the
 * vision-graph hot path.  TEST INFRASTRUCTURE ONLY: used by tests/, smoke() and the
 * CPU-baseline leg of bench.py as the checker.  Nothing in the product links it.
 *
 * Every function keeps the argument order and pointer conventions of the reference
 * HafCpu_* function it restates (amd_openvx/openvx/ago/ago_haf_cpu.h): dst/src point at
 * the first processed row, strides are in bytes, stencils read one (or two) pixels
 * outside the processed area, and the SIMD-body/scalar-tail rounding quirks are kept
 * (the split is computed from the destination address exactly as the reference does).
 *
 * Parity pin: tests/test_oracle_pin.py runs each function against the reference
 * library built from source (oracle/_ref/libopenvx_ref.so) on seeded inputs.
 */
#ifndef AGOORACLE_H
#define AGOORACLE_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---- filters (ago_haf_cpu_filter.cpp) ---- */
int oracle_Gaussian_U8_U8_3x3(uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                              const uint8_t *pSrc, uint32_t srcStride);
int oracle_SobelMagnitude_S16_U8_3x3(uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                                     const uint8_t *pSrc, uint32_t srcStride);
int oracle_Sobel_S16S16_U8_3x3_GXY(uint32_t dstWidth, uint32_t dstHeight, int16_t *pGx, uint32_t gxStride,
                                   int16_t *pGy, uint32_t gyStride, const uint8_t *pSrc, uint32_t srcStride);
/* ago_haf_cpu_filter.cpp:2676-3830 HafCpu_Convolve_{S16,U8}_U8_{3,5,7,9}xN, one function for
 * every width (cols = 3, 5, 7, 9; rows odd): the kernel applied flipped, sums in int32; SIMD
 * body columns shift logically by `shift` then saturate (to int16, then to u8), the scalar
 * prefix and postfix columns saturate the sum without shifting. */
int oracle_Convolve_U8_U8(uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                          const uint8_t *pSrc, uint32_t srcStride, const int16_t *conv, uint32_t cols, uint32_t rows,
                          int32_t shift);
int oracle_Convolve_S16_U8(uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                           const uint8_t *pSrc, uint32_t srcStride, const int16_t *conv, uint32_t cols, uint32_t rows,
                           int32_t shift);
/* ---- arithmetic (ago_haf_cpu_arithmetic.cpp) ---- */
int oracle_Magnitude_S16_S16S16(uint32_t dstWidth, uint32_t dstHeight, int16_t *pMag, uint32_t magStride,
                                const int16_t *pGx, uint32_t gxStride, const int16_t *pGy, uint32_t gyStride);
int oracle_ColorDepth_U8_S16_Sat(uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                                 const int16_t *pSrc, uint32_t srcStride, int32_t shift);
int oracle_Threshold_U8_U8_Binary(uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                                  const uint8_t *pSrc, uint32_t srcStride, uint8_t threshold);


/* ---- Canny (ago_haf_cpu_canny.cpp) ---- */
typedef struct { uint16_t x, y; } oracle_coord2d_u16;   /* ago_coord2d_ushort_t */
typedef struct { int16_t x, y; float s; } oracle_xys;    /* ago_keypoint_xys_t */
typedef struct { int32_t x, y; float strength, scale, orientation; int32_t tracking_status; float error; } oracle_keypoint;

int oracle_CannySobel_U16_U8_3x3_L1NORM(uint32_t dstWidth, uint32_t dstHeight, uint16_t *pDst, uint32_t dstStride,
                                        const uint8_t *pSrc, uint32_t srcStride);
int oracle_CannySobel_U16_U8_NxN(uint32_t dstWidth, uint32_t dstHeight, uint16_t *pDst, uint32_t dstStride,
                                 const uint8_t *pSrc, uint32_t srcStride, uint32_t gsize, uint32_t l2);
int oracle_CannySuppThreshold_U8XY_U16_3x3(uint32_t capacityOfXY, oracle_coord2d_u16 *xyStack, uint32_t *pStackTop,
                                           uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                                           const uint16_t *pSrc, uint32_t srcStride, uint16_t lower, uint16_t upper);
int oracle_CannyEdgeTrace_U8_U8XY(uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                                  uint32_t capacityOfXY, oracle_coord2d_u16 *xyStack, uint32_t stackTop);
/* ---- Harris (ago_haf_cpu_harris.cpp) ---- */
int oracle_HarrisSobel_HG3_U8_3x3(uint32_t dstWidth, uint32_t dstHeight, float *pDstGxy, uint32_t dstStride,
                                  const uint8_t *pSrc, uint32_t srcStride);
int oracle_HarrisScore_HVC_HG3_3x3(uint32_t dstWidth, uint32_t dstHeight, float *pDstVc, uint32_t dstStride,
                                   const float *pSrcGxy, uint32_t srcStride, float sensitivity, float threshold,
                                   float normFactor);
/* ago_haf_cpu_harris.cpp:333 / :455 HafCpu_HarrisSobel_HG3_U8_{5x5,7x7} (gs = 5 or 7): pDst and
 * pSrc at row 0; rows [gs/2, H - gs/2) written, all columns (reading outside the row at the
 * edges). */
int oracle_HarrisSobel_HG3_U8_NxN(uint32_t dstWidth, uint32_t dstHeight, float *pDstGxy, uint32_t dstStride,
                                  const uint8_t *pSrc, uint32_t srcStride, uint32_t gs);
/* ago_haf_cpu_harris.cpp:596 / :661 / :731 HafCpu_HarrisScore_HVC_HG3_{3x3,5x5,7x7} (bs = 3, 5, 7):
 * window sums in the reference's (j, i) order, rows and columns within bs/2 of a border 0; the
 * 7x7 kernel stores column x's score at x - 1 (an output pointer it does not advance). */
int oracle_HarrisScore_HVC_HG3_NxN(uint32_t dstWidth, uint32_t dstHeight, float *pDstVc, uint32_t dstStride,
                                   const float *pSrcGxy, uint32_t srcStride, float sensitivity, float threshold,
                                   float normFactor, uint32_t bs);
/* the score normalisation of the AGO wrappers (ago_kernel_api.cpp:16941, :17012, :17083) */
float oracle_harris_norm_factor_block(int32_t gs, int32_t bs);

/* FAST-9 corners (ago_haf_cpu_fast_corners.cpp:414, :599) on an AGO-laid-out U8 buffer:
 * raster-ordered keypoints, *pCount = all corners found (items beyond capacity dropped). */
int oracle_FastCorners_XY_U8_NoSupression(uint32_t capacity, oracle_keypoint *corners, uint32_t *pCount, uint32_t W,
                                          uint32_t H, const uint8_t *pSrc, uint32_t srcStride, float strengthThreshold);
int oracle_FastCorners_XY_U8_Supression(uint32_t capacity, oracle_keypoint *corners, uint32_t *pCount, uint32_t W,
                                        uint32_t H, const uint8_t *pSrc, uint32_t srcStride, float strengthThreshold);
/* per-pixel FAST strength of the suppression variant (0 where no corner), W x H bytes */
int oracle_FastCorners_strength(uint8_t *pDst, uint32_t W, uint32_t H, const uint8_t *pSrc, uint32_t srcStride,
                                float strengthThreshold);
int oracle_NonMaxSupp_XY_ANY_3x3(uint32_t capacity, oracle_xys *list, uint32_t *pCount, uint32_t srcWidth,
                                 uint32_t srcHeight, const float *pSrc, uint32_t srcStride);
int oracle_HarrisMergeSortAndPick_XY_XYS(uint32_t capacity, oracle_keypoint *corners, uint32_t *pCount,
                                         oracle_xys *list, uint32_t listCount, float minDistance,
                                         uint32_t imageWidth, uint32_t imageHeight);
/* AGO wrapper arithmetic (ago_kernel_api.cpp:16941-16942) */
float oracle_harris_norm_factor(int32_t gradientSize);

/* ---- colour conversion (ago_haf_cpu_color_convert.cpp), agooracle_geometry.c ---- */
int oracle_ColorConvert_NV12_RGB(uint32_t W, uint32_t H, uint8_t *pY, uint32_t yStride, uint8_t *pUV, uint32_t uvStride,
                                 const uint8_t *pSrc, uint32_t srcStride);
int oracle_ColorConvert_IYUV_RGB(uint32_t W, uint32_t H, uint8_t *pY, uint32_t yStride, uint8_t *pU, uint32_t uStride,
                                 uint8_t *pV, uint32_t vStride, const uint8_t *pSrc, uint32_t srcStride);
/* ---- scaling (ago_haf_cpu_geometric.cpp); m = {xscale, yscale, xoffset, yoffset} ---- */
void oracle_scale_matrix(int kind /* 0 nearest, 1 bilinear, 2 area */, uint32_t srcW, uint32_t srcH, uint32_t dstW,
                         uint32_t dstH, float m[4]);
int oracle_ScaleImage_U8_U8_Bilinear(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW, uint32_t srcH,
                                     const uint8_t *pSrc, uint32_t srcStride, const float m[4]);
int oracle_ScaleImage_U8_U8_Nearest(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW, uint32_t srcH,
                                    const uint8_t *pSrc, uint32_t srcStride, const float m[4]);
int oracle_ScaleImage_U8_U8_Area(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW, uint32_t srcH,
                                 const uint8_t *pSrc, uint32_t srcStride, const float m[4]);
/* ---- warps; m = ago_affine_matrix_t as 6 floats {m00, m01, m10, m11, m20, m21} ---- */
int oracle_WarpAffine_U8_U8_Nearest_Constant(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW,
                                             uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride, const float *m,
                                             uint8_t border, uint32_t validStartX, uint32_t validStartY,
                                             uint32_t validEndX, uint32_t validEndY);
int oracle_WarpAffine_U8_U8_Bilinear_Constant(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW,
                                              uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride, const float *m,
                                              uint8_t border);

/* ---- WarpPerspective (m = ago_perspective_matrix_t, 9 floats) and Remap (u16 fixed-point
 *      table of (x, y) pairs, mapStride bytes per row), agooracle_geometry.c ---- */
int oracle_WarpPerspective_U8_U8_Nearest_Constant(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                                  uint32_t srcW, uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride,
                                                  const float *m, uint8_t border);
int oracle_WarpPerspective_U8_U8_Bilinear_Constant(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                                   uint32_t srcW, uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride,
                                                   const float *m, uint8_t border);
void oracle_remap_fixed(uint32_t srcW, uint32_t srcH, const float *xy, size_t n, uint16_t *out);
int oracle_Remap_U8_U8_Bilinear_Constant(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW,
                                         uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride, const uint16_t *pMap,
                                         uint32_t mapStride, uint8_t border);
int oracle_Remap_U8_U8_Bilinear(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW, uint32_t srcH,
                                const uint8_t *pSrc, uint32_t srcStride, const uint16_t *pMap, uint32_t mapStride);
int oracle_Remap_U8_U8_Nearest_Constant(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW,
                                        uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride, const uint16_t *pMap,
                                        uint32_t mapStride, uint8_t border);
int oracle_Remap_U8_U8_Nearest(uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t srcW, uint32_t srcH,
                               const uint8_t *pSrc, uint32_t srcStride, const uint16_t *pMap, uint32_t mapStride);

/* ---- pyramid level and pyramidal LK (ago_haf_cpu_pyramid.cpp, ago_haf_cpu_opticalflow.cpp),
 *      agooracle_flow.c ---- */
typedef struct {          /* ago_pyramid_u8_t (ago_haf_cpu.h:75) */
    uint32_t width, height, stride;
    uint8_t *image;
    int32_t computed;
} oracle_pyramid_level;
int oracle_ScaleGaussianHalf_U8_U8_5x5(uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                                       const uint8_t *pSrc, uint32_t srcStride, int sampleFirstRow,
                                       int sampleFirstColumn);
int oracle_OpticalFlowPyrLK_XY_XY(oracle_keypoint *newKP, float pyramidScale, uint32_t levels,
                                  const oracle_pyramid_level *oldPyr, const oracle_pyramid_level *newPyr,
                                  uint32_t count, const oracle_keypoint *oldKP,
                                  const oracle_keypoint *estKP, int32_t termination, float epsilon,
                                  uint32_t numIterations, int32_t useInitialEstimate, uint32_t dataStride,
                                  uint8_t *data, int32_t winsz);
size_t oracle_OpticalFlowPyrLK_scratch_size(uint32_t width0, uint32_t height0, uint32_t capacity);

#ifdef __cplusplus
}
#endif
#endif
