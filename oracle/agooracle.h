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
/* ---- arithmetic (ago_haf_cpu_arithmetic.cpp) ---- */
int oracle_Magnitude_S16_S16S16(uint32_t dstWidth, uint32_t dstHeight, int16_t *pMag, uint32_t magStride,
                                const int16_t *pGx, uint32_t gxStride, const int16_t *pGy, uint32_t gyStride);
int oracle_ColorDepth_U8_S16_Sat(uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                                 const int16_t *pSrc, uint32_t srcStride, int32_t shift);
int oracle_Threshold_U8_U8_Binary(uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                                  const uint8_t *pSrc, uint32_t srcStride, uint8_t threshold);

#ifdef __cplusplus
}
#endif
#endif
