/*
 * agocuda.h -- C ABI of the B200 (sm_100a) kernels behind the OpenVX/AGO vision-graph
 * target.  This is the device-launch boundary: one entry point per AGO low-level kernel,
 * mirroring the reference's HIP launch layer (amd_openvx/openvx/hipvx/hip_host_decls.h,
 * `HipExec_<Kernel>`): a stream, the destination size, device pointers with byte strides,
 * then kernel parameters; every entry returns 0 on success, -10 for invalid parameters,
 * or the positive cudaError_t of a failed launch.
 *
 * Semantics follow the reference's CPU ("HAF") kernels as called by the AGO kernel
 * wrappers (amd_openvx/openvx/ago/ago_kernel_api.cpp): destination pointers address the
 * full image (row 0), and 3x3 stencils write the interior rows [1, H-1) -- exactly the rows
 * the AGO CPU wrapper processes -- so every pixel inside the OpenVX valid region is
 * bit-identical to the reference.  Pixels outside the valid region are unspecified
 * (OpenVX border mode UNDEFINED).
 *
 * All pointers are device pointers (or pointers the device can dereference).  Streams are
 * passed as `void *` holding a cudaStream_t (NULL = legacy default stream).
 */
#ifndef AGOCUDA_H
#define AGOCUDA_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------------------ */
/* Library information                                                                   */
/* ------------------------------------------------------------------------------------ */

/* Version of this C ABI (major*10000 + minor*100 + patch). */
int agocuda_abi_version(void);
/* Number of device kernels this library has launched since load (all entry points). */
uint64_t agocuda_launch_count(void);

/* ------------------------------------------------------------------------------------ */
/* Filters (reference: hipvx/hip_host_decls.h filter_kernels)                            */
/* ------------------------------------------------------------------------------------ */

/* 3x3 Gaussian [1 2 1]^T[1 2 1] / 16.  Replaces HipExec_Gaussian_U8_U8_3x3
 * (hipvx/hip_host_decls.h:649); CPU semantics of HafCpu_Gaussian_U8_U8_3x3
 * (ago/ago_haf_cpu_filter.cpp:1518) as called at ago/ago_kernel_api.cpp:15281. */
int agocuda_Gaussian_U8_U8_3x3(void *stream, uint32_t dstWidth, uint32_t dstHeight,
                               uint8_t *pDst, uint32_t dstStride,
                               const uint8_t *pSrc, uint32_t srcStride);

/* 3x3 Sobel gradients, S16.  Replaces HipExec_Sobel_S16S16_U8_3x3_GXY
 * (hipvx/hip_host_decls.h:663); HafCpu_Sobel_S16S16_U8_3x3_GXY (ago_haf_cpu_filter.cpp:2237). */
int agocuda_Sobel_S16S16_U8_3x3_GXY(void *stream, uint32_t dstWidth, uint32_t dstHeight,
                                    int16_t *pGx, uint32_t gxStride, int16_t *pGy, uint32_t gyStride,
                                    const uint8_t *pSrc, uint32_t srcStride);

/* Sobel 3x3 + L2 magnitude (the node AGO's SOBEL+MAGNITUDE merge rule produces,
 * ago/ago_drama_remove.cpp:165).  HafCpu_SobelMagnitude_S16_U8_3x3
 * (ago_haf_cpu_filter.cpp:2468): SIMD body rounds sqrt to nearest even, the scalar
 * prefix/tail (decided from the row-1 destination address, as the reference does)
 * truncate.  The reference HIP layer has no counterpart (the merged node ran on CPU). */
int agocuda_SobelMagnitude_S16_U8_3x3(void *stream, uint32_t dstWidth, uint32_t dstHeight,
                                      int16_t *pDst, uint32_t dstStride,
                                      const uint8_t *pSrc, uint32_t srcStride);

/* ------------------------------------------------------------------------------------ */
/* Arithmetic (reference: hipvx/hip_host_decls.h arithmetic/color kernels)              */
/* ------------------------------------------------------------------------------------ */

/* Replaces HipExec_Magnitude_S16_S16S16 (hipvx/hip_host_decls.h:219);
 * HafCpu_Magnitude_S16_S16S16 (ago_haf_cpu_arithmetic.cpp:4989).  Processes all rows. */
int agocuda_Magnitude_S16_S16S16(void *stream, uint32_t dstWidth, uint32_t dstHeight,
                                 int16_t *pMag, uint32_t magStride,
                                 const int16_t *pGx, uint32_t gxStride,
                                 const int16_t *pGy, uint32_t gyStride);

/* clamp(v >> shift, 0, 255).  Replaces HipExec_ColorDepth_U8_S16_Sat
 * (hipvx/hip_host_decls.h:403); HafCpu_ColorDepth_U8_S16_Sat (ago_haf_cpu_arithmetic.cpp:3546). */
int agocuda_ColorDepth_U8_S16_Sat(void *stream, uint32_t dstWidth, uint32_t dstHeight,
                                  uint8_t *pDst, uint32_t dstStride,
                                  const int16_t *pSrc, uint32_t srcStride, int32_t shift);

/* v > threshold ? 255 : 0 (threshold as vx_uint8).  Replaces HipExec_Threshold_U8_U8_Binary
 * (hipvx/hip_host_decls.h:689); HafCpu_Threshold_U8_U8_Binary (ago_haf_cpu_arithmetic.cpp:3660).
 * Planes as for the element-wise kernels below (16-byte aligned rows). */
int agocuda_Threshold_U8_U8_Binary(void *stream, uint32_t dstWidth, uint32_t dstHeight,
                                   uint8_t *pDst, uint32_t dstStride,
                                   const uint8_t *pSrc, uint32_t srcStride, int32_t threshold);

/* ------------------------------------------------------------------------------------ */
/* Vision: Canny and Harris (reference: hipvx/hip_host_decls.h vision_kernels)           */
/*                                                                                      */
/* Border columns follow the reference CPU kernels, which read one byte outside each row */
/* (x = -1 and x = W): with AGO's buffer layout (row pitch ALIGN16(W), zero padding) that */
/* is the neighbouring row's pixel when W % 16 == 0, else 0.  Those values reach the     */
/* valid region through suppression and hysteresis, so they are reproduced.              */
/* ------------------------------------------------------------------------------------ */

/* Packed Canny gradient ((|gx|+|gy|) << 2 | direction) of rows [1, H-1); rows 0 and H-1
 * are written 0.  Replaces HipExec_CannySobel_U16_U8_3x3_L1NORM (hipvx/hip_host_decls.h:828);
 * HafCpu_CannySobel_U16_U8_3x3_L1NORM (ago_haf_cpu_canny.cpp:44). */
int agocuda_CannySobel_U16_U8_3x3_L1NORM(void *stream, uint32_t dstWidth, uint32_t dstHeight,
                                         uint16_t *pDst, uint32_t dstStride,
                                         const uint8_t *pSrc, uint32_t srcStride);

/* Packed Canny gradients of the other window sizes and norms, same layout; rows [R, H-R)
 * written (R = 1, 2, 3), the rest 0.  Each column follows the reference's own formula for
 * it (SIMD body for x < W - W % 16 - 1, scalar code after), including the body's reads of
 * its zeroed row scratch past the aligned width and the 7x7 body's quarter-scale sums.
 * Replace HipExec_CannySobel_U16_U8_{3x3_L2,5x5_L1,5x5_L2,7x7_L1,7x7_L2}NORM
 * (hipvx/hip_host_decls.h:828-851); HafCpu_CannySobel_U16_U8_3x3_L2NORM
 * (ago_haf_cpu_canny.cpp:646), _5x5_L1NORM (:145), _5x5_L2NORM (:756), _7x7_L1NORM (:272),
 * _7x7_L2NORM (:893). */
int agocuda_CannySobel_U16_U8_3x3_L2NORM(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint16_t *pDst,
                                         uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride);
int agocuda_CannySobel_U16_U8_5x5_L1NORM(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint16_t *pDst,
                                         uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride);
int agocuda_CannySobel_U16_U8_5x5_L2NORM(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint16_t *pDst,
                                         uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride);
int agocuda_CannySobel_U16_U8_7x7_L1NORM(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint16_t *pDst,
                                         uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride);
int agocuda_CannySobel_U16_U8_7x7_L2NORM(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint16_t *pDst,
                                         uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride);

/* Non-maximum suppression + double threshold (255 / 127 / 0) on [1,W-1)x[1,H-1); strong
 * pixels are appended to pStack as (y << 16 | x) (the layout of ago_coord2d_ushort_t), in no
 * particular order, *pStackCount set to their number.  Replaces
 * HipExec_CannySuppThreshold_U8XY_U16_3x3 (hipvx/hip_host_decls.h:852);
 * HafCpu_CannySuppThreshold_U8XY_U16_3x3 (ago_haf_cpu_canny.cpp:549). */
int agocuda_CannySuppThreshold_U8XY_U16_3x3(void *stream, uint32_t dstWidth, uint32_t dstHeight,
                                            uint8_t *pDst, uint32_t dstStride,
                                            const uint16_t *pSrc, uint32_t srcStride,
                                            uint32_t *pStack, uint32_t *pStackCount, uint32_t stackCapacity,
                                            uint16_t hystLower, uint16_t hystUpper);

/* Hysteresis in place: pixels 8-connected through non-zero pixels to a strong one become
 * 255, all others 0 (the whole image is written).  The stack is expected to hold every
 * strong pixel, as the suppression above leaves it.  An entry on a pixel that is not in the
 * edge map (zero, or on the image border) seeds the components of its 8 neighbours, as the
 * reference's trace grows from each entry through its neighbours; an entry outside the
 * image is ignored and sets AGOCUDA_TRACE_STATUS_BAD_ENTRY in *pStatus.  Needs `scratch`
 * device memory of agocuda_CannyEdgeTrace_scratch_size(W, H) bytes, 256-byte aligned;
 * *pStatus gets bit 0 set if a union-find walk exceeded its bound.  The reference runs this
 * on the CPU only (ago_kernel_list.cpp:486); HafCpu_CannyEdgeTrace_U8_U8XY
 * (ago_haf_cpu_canny.cpp:598). */
#define AGOCUDA_TRACE_STATUS_BAD_ENTRY 8u  /* an edge-trace stack entry lay outside the image */
size_t agocuda_CannyEdgeTrace_scratch_size(uint32_t width, uint32_t height);
int agocuda_CannyEdgeTrace_U8_U8XY(void *stream, uint32_t width, uint32_t height, uint8_t *pImg, uint32_t stride,
                                   const uint32_t *pStack, const uint32_t *pStackCount, uint32_t stackCapacity,
                                   void *scratch, size_t scratchBytes, uint32_t *pStatus);

/* The same hysteresis as agocuda_CannyEdgeTrace_U8_U8XY for callers that cannot allocate
 * device memory -- a real-time loop that must not pay cudaMalloc's implicit device
 * synchronisation, or a host application that gives this library a fixed memory budget and
 * owns every device allocation itself.  It allocates nothing: its scratch (union-find
 * labels and a root bitmap) is a fixed array of 8.25 MiB in the library's own device memory,
 * which every GPU that loads the library holds until the process exits.  Images are limited
 * to agocuda_CannyEdgeTrace_noalloc_max_pixels() = 2,097,152 pixels (W*H); larger ones return
 * -15 without launching anything.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) and should be made before any stream capture; the lookup
 * is repeated when the calling thread's current context on that device changes (after
 * cudaDeviceReset, for instance), so that call, too, belongs outside a capture.  All calls on
 * a device share that one array: the labels are rewritten and the bitmap is cleared on every
 * call, but calls whose executions overlap on the GPU (other streams, or host threads
 * without ordering) race on it.  No counterpart in the reference (its edge trace runs on the
 * CPU, ago_kernel_list.cpp:486). */
size_t agocuda_CannyEdgeTrace_noalloc_max_pixels(void);
int agocuda_CannyEdgeTrace_U8_U8XY_noalloc(void *stream, uint32_t width, uint32_t height, uint8_t *pImg, uint32_t stride,
                                           const uint32_t *pStack, const uint32_t *pStackCount, uint32_t stackCapacity,
                                           uint32_t *pStatus);

/* FAST-9 corners (vxFastCornersNode): rows 3 .. H-4 of a U8 image; without suppression every
 * column (the circle of the three outer columns reads across the row ends as AGO's layout
 * holds the image: pitch ALIGN16(W), zero padding) with strength = strengthThreshold; with
 * suppression columns 3 .. W-4, strength = the reference's binary-searched corner strength,
 * kept when >= the upper and left neighbours and > the right and lower ones.  Writes
 * vx_keypoint_t records in raster order, *pCornerCount = min(found, capacity), *pNumCorners =
 * found (either may be NULL).  `scratch` (256-byte aligned) holds
 * agocuda_FastCorners_scratch_size(W, H) bytes.  Four kernels.  HafCpu_FastCorners_XY_U8_
 * {NoSupression,Supression} (ago_haf_cpu_fast_corners.cpp:414, :599); replaces
 * HipExec_FastCorners_XY_U8_{NoSupression,Supression} (hipvx/hip_host_decls.h:858/863), which
 * append in arbitrary order. */
size_t agocuda_FastCorners_scratch_size(uint32_t width, uint32_t height);
int agocuda_FastCorners_XY_U8(void *stream, uint32_t width, uint32_t height, const uint8_t *pSrc, uint32_t srcStride,
                              float strengthThreshold, int32_t nonmaxSuppression, void *pCorners, uint32_t cornerCapacity,
                              uint32_t *pCornerCount, uint32_t *pNumCorners, void *scratch, size_t scratchBytes);

/* Convolve (vxConvolveNode): U8 source, U8 or S16 destination, cols in {3, 5, 7, 9}, rows
 * odd in [3, 9]; `conv` is a HOST pointer to the rows x cols coefficients in vx_convolution
 * order (applied flipped, as OpenVX defines convolution), `shift` = log2 of the scale.
 * Columns [simdBegin, simdEnd) take the reference SIMD body's arithmetic (sum shifted right
 * logically, then saturated), the others its scalar loops' (the unshifted sum saturated);
 * rows [rows/2, H - rows/2) are written.  HafCpu_Convolve_{U8,S16}_U8_{3,5,7,9}xN
 * (ago_haf_cpu_filter.cpp:2676-3830); replaces HipExec_Convolve_{U8,S16}_U8
 * (hipvx/hip_host_decls.h:653/658), which takes device float coefficients instead. */
int agocuda_Convolve_U8_U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                           const uint8_t *pSrc, uint32_t srcStride, const int16_t *conv, uint32_t cols, uint32_t rows,
                           int32_t shift, int32_t simdBegin, int32_t simdEnd);
int agocuda_Convolve_S16_U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                            const uint8_t *pSrc, uint32_t srcStride, const int16_t *conv, uint32_t cols, uint32_t rows,
                            int32_t shift, int32_t simdBegin, int32_t simdEnd);

/* Harris gradient products with 5x5 or 7x7 Sobel taps (gradientSize 5 or 7), every column,
 * rows [gs/2, H - gs/2) (the others written 0); the taps leaving the row read the neighbouring
 * rows' bytes as AGO lays an image out (row pitch ALIGN16(W), zero padding).  Replaces
 * HipExec_HarrisSobel_HG3_U8_{5x5,7x7} (hipvx/hip_host_decls.h:872); HafCpu_HarrisSobel_HG3_U8_5x5 /
 * _7x7 (ago_haf_cpu_harris.cpp:333 / :455). */
int agocuda_HarrisSobel_HG3_U8_NxN(void *stream, uint32_t width, uint32_t height, float *pDst, uint32_t dstStride,
                                   const uint8_t *pSrc, uint32_t srcStride, uint32_t gradientSize);
/* Harris score over a 5x5 or 7x7 block (blockSize 5 or 7) of gradient products, in the
 * reference's summation order, 0 within blockSize/2 of a border; with blockSize 7 the score of
 * column x is stored at x - 1, as the reference stores it.  normFactor: (255 * 2^(gs-1) *
 * blockSize)^4 (ago_kernel_api.cpp:17012, :17083).  Replaces HipExec_HarrisScore_HVC_HG3_{5x5,7x7}
 * (hipvx/hip_host_decls.h:886);
 * HafCpu_HarrisScore_HVC_HG3_5x5 / _7x7 (ago_haf_cpu_harris.cpp:661 / :731). */
int agocuda_HarrisScore_HVC_HG3_NxN(void *stream, uint32_t width, uint32_t height, float *pDst, uint32_t dstStride,
                                    const float *pSrc, uint32_t srcStride, float sensitivity, float strengthThreshold,
                                    float normFactor, uint32_t blockSize);

/* Harris gradient products {gx*gx, gx*gy, gy*gy} (float x3 per pixel) of rows [1, H-1);
 * rows 0 and H-1 are written 0.  Replaces HipExec_HarrisSobel_HG3_U8_3x3
 * (hipvx/hip_host_decls.h:868); HafCpu_HarrisSobel_HG3_U8_3x3 (ago_haf_cpu_harris.cpp:85). */
int agocuda_HarrisSobel_HG3_U8_3x3(void *stream, uint32_t dstWidth, uint32_t dstHeight,
                                   float *pDst, uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride);

/* Harris score over a 3x3 window; border rows/columns 0.  Replaces
 * HipExec_HarrisScore_HVC_HG3_3x3 (hipvx/hip_host_decls.h:880);
 * HafCpu_HarrisScore_HVC_HG3_3x3 (ago_haf_cpu_harris.cpp:596). */
int agocuda_HarrisScore_HVC_HG3_3x3(void *stream, uint32_t dstWidth, uint32_t dstHeight,
                                    float *pDst, uint32_t dstStride, const float *pSrc, uint32_t srcStride,
                                    float sensitivity, float strengthThreshold, float normFactor);

/* 3x3 non-maximum suppression; candidates appended as 8-byte XYS records (int16 x, int16 y,
 * float s -- ago_keypoint_xys_t) in no particular order.  Replaces
 * HipExec_NonMaxSupp_XY_ANY_3x3 (hipvx/hip_host_decls.h:898);
 * HafCpu_NonMaxSupp_XY_ANY_3x3 (ago_haf_cpu_harris.cpp:882). */
int agocuda_NonMaxSupp_XY_ANY_3x3(void *stream, uint32_t width, uint32_t height, const float *pSrc, uint32_t srcStride,
                                  uint64_t *pList, uint32_t *pListCount, uint32_t listCapacity);

/* Sort candidates (descending as int64) and keep those farther than minDistance from kept
 * ones on the reference's grid; writes vx_keypoint_t records in sorted order, *pCornerCount =
 * min(kept, capacity), *pNumCorners = kept.  Up to 8192 candidates are picked by one CTA in
 * shared memory; larger lists (the reference's holds up to W*H) by one cluster of 8 CTAs in
 * `scratch`, which must then hold agocuda_HarrisMergeSortAndPick_scratch_size(W, H,
 * listCapacity, minDistance) bytes, 256-byte aligned.  With scratch NULL a list above 8192
 * sets *pStatus |= 2 and nothing is written.  A candidate outside the WxH grid is dropped
 * and sets AGOCUDA_PICK_STATUS_BAD_ENTRY.  The reference runs this on the CPU only
 * (ago_kernel_list.cpp:483); HafCpu_HarrisMergeSortAndPick_XY_XYS (ago_haf_cpu_harris.cpp:923). */
#define AGOCUDA_PICK_STATUS_BAD_ENTRY 32u  /* a corner candidate lay outside the image */
size_t agocuda_HarrisMergeSortAndPick_scratch_size(uint32_t width, uint32_t height, uint32_t listCapacity,
                                                  float minDistance);
int agocuda_HarrisMergeSortAndPick_XY_XYS(void *stream, uint32_t width, uint32_t height, const uint64_t *pList,
                                          const uint32_t *pListCount, uint32_t listCapacity, float minDistance,
                                          void *pCorners, uint32_t cornerCapacity, uint32_t *pCornerCount,
                                          uint32_t *pNumCorners, void *scratch, size_t scratchBytes,
                                          uint32_t *pStatus);

/* ------------------------------------------------------------------------------------ */
/* Colour conversion, scaling, warps (reference: hipvx/hip_host_decls.h color/geometric)  */
/* ------------------------------------------------------------------------------------ */

/* RGB (3 B/px) -> NV12 (Y plane + interleaved UV at half resolution), BT.709 float weights,
 * truncation and the reference's chroma averaging.  W and H even.  Replaces
 * HipExec_ColorConvert_NV12_RGB (hipvx/hip_host_decls.h:555); HafCpu_ColorConvert_NV12_RGB
 * (ago_haf_cpu_color_convert.cpp:2707). */
int agocuda_ColorConvert_NV12_RGB(void *stream, uint32_t width, uint32_t height, uint8_t *pY, uint32_t yStride,
                                  uint8_t *pUV, uint32_t uvStride, const uint8_t *pSrc, uint32_t srcStride);
/* RGB -> IYUV (Y, U, V planes).  Replaces HipExec_ColorConvert_IYUV_RGB (hipvx/hip_host_decls.h:565);
 * HafCpu_ColorConvert_IYUV_RGB (ago_haf_cpu_color_convert.cpp:2492). */
int agocuda_ColorConvert_IYUV_RGB(void *stream, uint32_t width, uint32_t height, uint8_t *pY, uint32_t yStride,
                                  uint8_t *pU, uint32_t uStride, uint8_t *pV, uint32_t vStride,
                                  const uint8_t *pSrc, uint32_t srcStride);

/* ScaleImage U8 -> U8 with the AGO scale matrices (18-bit fixed-point maps).  Replace
 * HipExec_ScaleImage_U8_U8_{Nearest,Bilinear,Area} (hipvx/hip_host_decls.h:723/728/744);
 * HafCpu_ScaleImage_U8_U8_* (ago_haf_cpu_geometric.cpp:1874/1977/2491).  Area supports the
 * exact 1x and 2x ratios (returns -3, not supported, otherwise). */
int agocuda_ScaleImage_U8_U8_Nearest(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                                     uint32_t srcWidth, uint32_t srcHeight, const uint8_t *pSrc, uint32_t srcStride);
int agocuda_ScaleImage_U8_U8_Bilinear(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                                      uint32_t srcWidth, uint32_t srcHeight, const uint8_t *pSrc, uint32_t srcStride);
int agocuda_ScaleImage_U8_U8_Area(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                                  uint32_t srcWidth, uint32_t srcHeight, const uint8_t *pSrc, uint32_t srcStride);

/* WarpAffine U8 -> U8 with constant border.  affineMatrix: 6 floats in vx_matrix order
 * (3 rows x 2 columns: m00 m01 / m10 m11 / m20 m21), read on the host at launch.  The nearest
 * variant also masks by the source valid rectangle {start_x, start_y, end_x, end_y} (NULL =
 * whole image).  Widths are processed in 4-pixel groups (dstStride >= ALIGN4(width)).
 * Replace HipExec_WarpAffine_U8_U8_{Nearest,Bilinear}_Constant (hipvx/hip_host_decls.h:755/768);
 * HafCpu_WarpAffine_U8_U8_{Nearest,Bilinear}_Constant (ago_haf_cpu_geometric.cpp:658/1100). */
int agocuda_WarpAffine_U8_U8_Nearest_Constant(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                              uint32_t dstStride, uint32_t srcWidth, uint32_t srcHeight,
                                              const uint8_t *pSrc, uint32_t srcStride, const float *affineMatrix,
                                              uint8_t border, const uint32_t *srcValidRect);
int agocuda_WarpAffine_U8_U8_Bilinear_Constant(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                               uint32_t dstStride, uint32_t srcWidth, uint32_t srcHeight,
                                               const uint8_t *pSrc, uint32_t srcStride, const float *affineMatrix,
                                               uint8_t border);

/* WarpPerspective, constant border; perspectiveMatrix is a HOST pointer to
 * ago_perspective_matrix_t (float[3][3], the vx_matrix data): x' = (m00 x + m10 y + m20) /
 * (m02 x + m12 y + m22), y' likewise with m01, m11, m21.  Source taps are addressed as the
 * reference addresses them in AGO's buffer layout (row pitch ALIGN16(srcWidth)).  With an
 * UNDEFINED border the reference runs these with border 0 (geometric.cpp:1372, :1560).
 * Replace HipExec_WarpPerspective_U8_U8_{Nearest,Bilinear}[_Constant]
 * (hipvx/hip_host_decls.h:775-794); HafCpu_WarpPerspective_U8_U8_{Nearest,Bilinear}_Constant
 * (ago_haf_cpu_geometric.cpp:1406 / :1579). */
int agocuda_WarpPerspective_U8_U8_Nearest_Constant(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                                   uint32_t dstStride, uint32_t srcWidth, uint32_t srcHeight,
                                                   const uint8_t *pSrc, uint32_t srcStride,
                                                   const float *perspectiveMatrix, uint8_t border);
int agocuda_WarpPerspective_U8_U8_Bilinear_Constant(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                                    uint32_t dstStride, uint32_t srcWidth, uint32_t srcHeight,
                                                    const uint8_t *pSrc, uint32_t srcStride,
                                                    const float *perspectiveMatrix, uint8_t border);

/* Remap through AGO's fixed-point table: one uint32 per destination pixel (u16 x | u16 y
 * << 16, 3 fractional bits, 0xFFFF = outside the source: the table vxSetRemapPoint builds,
 * api/vx_api.cpp:7884), mapStride bytes per row, DEVICE memory.  The constant-border and
 * undefined-border kernels treat 0xFFFF differently, as the reference does.  Replace
 * HipExec_Remap_U8_U8_{Nearest,Nearest_Constant,Bilinear,Bilinear_Constant}
 * (hipvx/hip_host_decls.h:801-819); HafCpu_Remap_U8_U8_* (ago_haf_cpu_geometric.cpp:72 /
 * :156 / :249 / :372). */
int agocuda_Remap_U8_U8_Nearest(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                                uint32_t srcWidth, uint32_t srcHeight, const uint8_t *pSrc, uint32_t srcStride,
                                const uint32_t *pMap, uint32_t mapStride);
int agocuda_Remap_U8_U8_Nearest_Constant(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                         uint32_t dstStride, uint32_t srcWidth, uint32_t srcHeight, const uint8_t *pSrc,
                                         uint32_t srcStride, const uint32_t *pMap, uint32_t mapStride, uint8_t border);
int agocuda_Remap_U8_U8_Bilinear(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                                 uint32_t srcWidth, uint32_t srcHeight, const uint8_t *pSrc, uint32_t srcStride,
                                 const uint32_t *pMap, uint32_t mapStride);
int agocuda_Remap_U8_U8_Bilinear_Constant(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                          uint32_t dstStride, uint32_t srcWidth, uint32_t srcHeight, const uint8_t *pSrc,
                                          uint32_t srcStride, const uint32_t *pMap, uint32_t mapStride, uint8_t border);

/* ------------------------------------------------------------------------------------ */
/* Fused multi-node kernels (no reference counterpart: the HIP target launches one kernel */
/* per node, ago/ago_util_hip.cpp:686; agoGpuHipSuperNodeLaunch returns -1 at :740)      */
/* ------------------------------------------------------------------------------------ */

/* One frame descriptor of a batched launch.  Frames may have different sizes. */
typedef struct agocuda_frame {
    const uint8_t *src;    /* U8 input, row 0 */
    uint8_t *dst;          /* U8 output, row 0 */
    uint32_t width, height;
    uint32_t srcStride, dstStride;
    int32_t simdBegin, simdEnd;  /* SobelMagnitude SIMD span in columns (see above) */
} agocuda_frame;

/* Gaussian3x3 -> SobelMagnitude -> ConvertDepth(SATURATE, shift) -> Threshold(BINARY)
 * with all intermediates virtual, in one pass over HBM (1 B/px read, 1 B/px write).
 * Writes rows/cols [2, W-2) x [2, H-2) of dst, which is the valid region of the
 * unfused graph, bit-identical to it.  `frames` is a DEVICE array of `numFrames`
 * descriptors; all frames run in one launch. */
int agocuda_fused_GaussSobelMagDepthThresh(void *stream, const agocuda_frame *frames, uint32_t numFrames,
                                           uint32_t maxWidth, uint32_t maxHeight,
                                           int32_t shift, int32_t threshold);

/* The same chain with each block's source tile copied into shared memory by one TMA tensor
 * copy (cp.async.bulk.tensor.2d on an mbarrier) and the Sobel / threshold stage in exact
 * fp32; output identical to agocuda_fused_GaussSobelMagDepthThresh.  `maps` is a DEVICE array
 * of numFrames 128-byte tensor maps (64-byte aligned) that
 * agocuda_fused_GaussSobelMagDepthThresh_tensor_maps encodes on the host from the same frame
 * descriptors (each source row pointer 16-byte aligned, pitch a multiple of 16 bytes, the
 * SobelMagnitude SIMD span's bounds multiples of 8; AGOCUDA_INVALID_PARAMS otherwise).  A
 * block whose copy does not complete within a bounded wait sets
 * AGOCUDA_C1_STATUS_TMA_TIMEOUT in *pStatus (device memory).  No counterpart in the reference. */
#define AGOCUDA_C1_STATUS_TMA_TIMEOUT 512u
size_t agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_size(uint32_t numFrames);
int agocuda_fused_GaussSobelMagDepthThresh_tensor_maps(const agocuda_frame *framesHost, uint32_t numFrames,
                                                      void *mapsHost, size_t mapsBytes);
int agocuda_fused_GaussSobelMagDepthThresh_tma(void *stream, const agocuda_frame *frames, const void *maps,
                                               uint32_t numFrames, uint32_t maxWidth, uint32_t maxHeight,
                                               int32_t shift, int32_t threshold, uint32_t *pStatus);
/* The same with the tile shape chosen: warpsPerBlock warps of rowsPerWarp output rows each
 * (256 columns); rowsPerWarp in {18, 24, 36, 48}, warpsPerBlock in {1, 2, 4} but not 48 x 4
 * (AGOCUDA_INVALID_PARAMS otherwise).  The maps must come from the _shape encoder with the
 * same shape (a map's box height is the shape's).  The plain functions above use 36 x 2;
 * the autotuner (mivisionx_b200/autotune.py) picks a shape per frame size. */
int agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_shape(const agocuda_frame *framesHost, uint32_t numFrames,
                                                            uint32_t rowsPerWarp, uint32_t warpsPerBlock,
                                                            void *mapsHost, size_t mapsBytes);
int agocuda_fused_GaussSobelMagDepthThresh_tma_shape(void *stream, const agocuda_frame *frames, const void *maps,
                                                     uint32_t numFrames, uint32_t maxWidth, uint32_t maxHeight,
                                                     int32_t shift, int32_t threshold, uint32_t rowsPerWarp,
                                                     uint32_t warpsPerBlock, uint32_t *pStatus);

/* The same chain as a persistent kernel: blocksPerSM x (number of SMs) resident blocks of
 * warpsPerBlock warps take tiles -- 256 columns x warpsPerBlock * rowsPerThread rows of one
 * frame -- from one queue over every frame of the batch, whatever their sizes, so uneven
 * batches leave no idle tail per frame.  tilePrefix (device) holds numFrames + 1 entries:
 * frame i's tiles are [tilePrefix[i], tilePrefix[i+1]), each frame's count given by
 * agocuda_fused_GaussSobelMagDepthThresh_tiles.  queue (device, 8-byte aligned) is two zeroed
 * words owned by the launch site; the launch leaves them zero again.  rowsPerThread in
 * {6, 12, 18, 24}, warpsPerBlock in {2, 4, 8} (tiles returns 0 for other shapes); the
 * autotuner (mivisionx_b200/autotune.py) picks them per frame size.  No counterpart in the
 * reference (its HIP target launches one kernel per node and image). */
uint32_t agocuda_fused_GaussSobelMagDepthThresh_tiles(uint32_t width, uint32_t height, uint32_t rowsPerThread,
                                                     uint32_t warpsPerBlock);
int agocuda_fused_GaussSobelMagDepthThresh_persistent(void *stream, const agocuda_frame *frames, uint32_t numFrames,
                                                      const uint32_t *tilePrefix, uint32_t *queue, uint32_t rowsPerThread,
                                                      uint32_t warpsPerBlock, uint32_t blocksPerSM, int32_t shift,
                                                      int32_t threshold);

/* vxCannyEdgeDetectorNode (gradient 3, L1 norm) in four kernels: a front end per 64x32 tile
 * (gradient, suppression, thresholds and connected components of the edge candidates in
 * shared memory, from one read of the image) that writes the final bytes of every component
 * it sees whole or holding a strong pixel, then unions of the components that cross tile
 * borders, their strong bits, and a pass that sets the remaining runs of strong components;
 * the 0/255 edge map is bit-identical to the unfused graph inside its valid region.
 * Scratch: agocuda_fused_CannyEdgeDetector_scratch_size(W, H) bytes.  Where pSrc is 16-byte
 * aligned and srcStride a multiple of 16 the front's input tiles are copied by TMA (a tensor
 * map made by the call); a copy that does not complete within a bounded wait sets
 * AGOCUDA_CANNY_STATUS_TMA_TIMEOUT in *pStatus. */
#define AGOCUDA_CANNY_STATUS_TMA_TIMEOUT 1024u
size_t agocuda_fused_CannyEdgeDetector_scratch_size(uint32_t width, uint32_t height);
int agocuda_fused_CannyEdgeDetector_3x3_L1(void *stream, uint32_t width, uint32_t height,
                                           uint8_t *pDst, uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride,
                                           uint16_t hystLower, uint16_t hystUpper,
                                           void *scratch, size_t scratchBytes, uint32_t *pStatus);

/* RGB -> NV12 + IYUV + half-size bilinear ScaleImage + half-size area ScaleImage of Y, in
 * one pass over the RGB frame (W even, >= 16; H even).  Outputs bit-identical to the four
 * unfused AGO nodes (the scaled images read the Y plane both colour outputs share). */
int agocuda_fused_ColorScale_RGB(void *stream, uint32_t width, uint32_t height, const uint8_t *pSrc, uint32_t srcStride,
                                 uint8_t *pNV12Y, uint32_t nv12YStride, uint8_t *pNV12UV, uint32_t nv12UVStride,
                                 uint8_t *pIYUVY, uint32_t iyuvYStride, uint8_t *pU, uint32_t uStride,
                                 uint8_t *pV, uint32_t vStride, uint8_t *pHalfBilinear, uint32_t hbStride,
                                 uint8_t *pHalfArea, uint32_t haStride);

/* vxHarrisCornersNode (gradient 3, block 3) as one front-end kernel (Sobel products,
 * window sums, score and non-maximum suppression from one read of the image) plus the
 * corner pick.  The candidate list holds ceil(W/2)*ceil(H/2) entries, the most the
 * suppression can emit, so no image overflows it.  Scratch:
 * agocuda_fused_HarrisCorners_scratch_size(W, H, minDistance) bytes.  Where pSrc is 16-byte
 * aligned and srcStride a multiple of 16 the front end's source rows are copied by TMA (a
 * tensor map made by the call); a copy that does not complete within a bounded wait sets
 * AGOCUDA_HARRIS_STATUS_TMA_TIMEOUT in *pStatus. */
#define AGOCUDA_HARRIS_STATUS_TMA_TIMEOUT 2048u
size_t agocuda_fused_HarrisCorners_scratch_size(uint32_t width, uint32_t height, float minDistance);
int agocuda_fused_HarrisCorners_3x3(void *stream, uint32_t width, uint32_t height, const uint8_t *pSrc, uint32_t srcStride,
                                    float sensitivity, float strengthThreshold, float normFactor, float minDistance,
                                    void *pCorners, uint32_t cornerCapacity, uint32_t *pCornerCount,
                                    uint32_t *pNumCorners, void *scratch, size_t scratchBytes, uint32_t *pStatus);

/* ---------------------------------------------------------------- differentiable F32 warps */
/* F32 bilinear WarpAffine / Remap with a constant border and their adjoints, for batches of
 * `n` images (image i at base + i * batch elements; strides in elements; device memory).
 * No reference counterpart: the reference's warps are U8 only (ago_kernel_api.cpp:19255).
 * The coordinate convention is its U8 WarpAffine's (ago_haf_cpu_geometric.cpp:679-684):
 * xs = m00*x + m10*y + m20, ys = m01*x + m11*y + m21 with theta = (m00, m01, m10, m11, m20,
 * m21) per image (device, n x 6 floats); bilinear from floor(xs), floor(ys), each tap
 * outside the source reading `border`.  Remap samples at (x + field.x, y + field.y), field
 * an (H, W, 2) float array per image (8-byte aligned).
 * Adjoints ADD into the gradients (zero them first): pGradSrc (same layout as the source),
 * pGradTheta (double, n x 6) or pGradField.  The L2 step computes, for L_i = sum over image
 * i of (warp - target)^2, the gradients of L_i and L_i itself into pGradThetaLoss (double,
 * n x 7: six theta gradients, then L_i) from one pass over the images. */
int agocuda_WarpAffine_F32_Bilinear_Constant_batch(void *stream, int n, int width, int height, float *pDst,
                                                   long long dstBatch, int dstStride, int srcWidth, int srcHeight,
                                                   const float *pSrc, long long srcBatch, int srcStride,
                                                   const float *theta, float border);
int agocuda_WarpAffine_F32_Bilinear_Constant_adjoint_batch(void *stream, int n, int width, int height,
                                                           const float *pGradOut, long long goBatch, int goStride,
                                                           int srcWidth, int srcHeight, const float *pSrc,
                                                           long long srcBatch, int srcStride, const float *theta,
                                                           float border, float *pGradSrc, double *pGradTheta);
int agocuda_WarpAffine_F32_L2_step_batch(void *stream, int n, int width, int height, const float *pTarget,
                                         long long tBatch, int tStride, int srcWidth, int srcHeight, const float *pSrc,
                                         long long srcBatch, int srcStride, const float *theta, float border,
                                         float *pGradSrc, double *pGradThetaLoss);
/* WarpPerspective F32 bilinear with a constant border, the perspective counterpart of the
 * three entry points above: theta holds 9 floats per image, the ago_perspective_matrix_t
 * m[3][3] of the reference's U8 WarpPerspective in storage order (m00 m01 m02 / m10 m11 m12 /
 * m20 m21 m22; ago_haf_cpu_geometric.cpp:1594-1602):  z = m02*x + m12*y + m22,
 * xs = (m00*x + m10*y + m20) / z,  ys = (m01*x + m11*y + m21) / z; z == 0 samples the border.
 * The adjoint adds 9 theta gradients (double) per image; the L2 step adds 9 gradients and then
 * the loss (10 doubles per image).  No counterpart in the reference (its warps are U8 only). */
int agocuda_WarpPerspective_F32_Bilinear_Constant_batch(void *stream, int n, int width, int height, float *pDst,
                                                        long long dstBatch, int dstStride, int srcWidth, int srcHeight,
                                                        const float *pSrc, long long srcBatch, int srcStride,
                                                        const float *theta, float border);
int agocuda_WarpPerspective_F32_Bilinear_Constant_adjoint_batch(void *stream, int n, int width, int height,
                                                                const float *pGradOut, long long goBatch, int goStride,
                                                                int srcWidth, int srcHeight, const float *pSrc,
                                                                long long srcBatch, int srcStride, const float *theta,
                                                                float border, float *pGradSrc, double *pGradTheta);
int agocuda_WarpPerspective_F32_L2_step_batch(void *stream, int n, int width, int height, const float *pTarget,
                                              long long tBatch, int tStride, int srcWidth, int srcHeight, const float *pSrc,
                                              long long srcBatch, int srcStride, const float *theta, float border,
                                              float *pGradSrc, double *pGradThetaLoss);
int agocuda_Remap_F32_Bilinear_Constant_batch(void *stream, int n, int width, int height, float *pDst, long long dstBatch,
                                              int dstStride, int srcWidth, int srcHeight, const float *pSrc,
                                              long long srcBatch, int srcStride, const float *pField, long long fieldBatch,
                                              int fieldStride, float border);
int agocuda_Remap_F32_Bilinear_Constant_adjoint_batch(void *stream, int n, int width, int height, const float *pGradOut,
                                                      long long goBatch, int goStride, int srcWidth, int srcHeight,
                                                      const float *pSrc, long long srcBatch, int srcStride,
                                                      const float *pField, long long fieldBatch, int fieldStride,
                                                      float border, float *pGradSrc, float *pGradField);

/* ---------------------------------------------------------------- Gaussian pyramid */
/* One pyramid level of VX_SCALE_PYRAMID_HALF: dst (ceil(srcW/2) x ceil(srcH/2)) rows 1..H-2 are
 * the [1 4 6 4 1]^2 / 256 samples the AGO CPU kernel computes (sample parity from the source
 * size, two-pixel reads outside the row resolved with AGO's buffer layout); rows 0 and H-1
 * are written 0 (the reference never writes them).  src/dst 16-byte aligned, strides
 * multiples of 16.  Replaces HafCpu_ScaleGaussianHalf_U8_U8_5x5 (ago_haf_cpu_pyramid.cpp:94)
 * as agoKernel_ScaleGaussianHalf_U8_U8_5x5 calls it (ago_kernel_api.cpp:15420), and
 * HipExec_ScaleGaussianHalf_U8_U8_5x5 (hipvx/hip_host_decls.h:681). */
int agocuda_ScaleGaussianHalf_U8_U8_5x5(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                        uint32_t dstStride, uint32_t srcWidth, uint32_t srcHeight,
                                        const uint8_t *pSrc, uint32_t srcStride);

/* Batched levels: one launch computes one level for many images (e.g. level k of every
 * frame's pyramid).  `jobs` is a DEVICE array sorted by tileBegin; job i owns tiles
 * [tileBegin, tileBegin + agocuda_ScaleGaussianHalf_tiles(dstW, dstH)). */
typedef struct agocuda_half_job {
    const uint8_t *src;
    uint8_t *dst;
    uint32_t srcW, srcH, srcStride, dstW, dstH, dstStride, tileBegin, reserved;
} agocuda_half_job;
uint32_t agocuda_ScaleGaussianHalf_tiles(uint32_t dstWidth, uint32_t dstHeight);
int agocuda_fused_ScaleGaussianHalf_batch(void *stream, const agocuda_half_job *jobs, uint32_t numJobs,
                                          uint32_t totalTiles);
/* Persistent form of the batch: blocksPerSM x (number of SMs) resident blocks of `threads`
 * threads take tiles (8 * threads columns x rows rows of one level) from one queue over the
 * jobs; job j's tileBegin counts tiles of this shape (agocuda_ScaleGaussianHalf_tiles_shape).
 * threads in {32, 64, 128}, rows in {2, 4, 8}.  queue: two zeroed device words (8-byte
 * aligned) owned by the launch site, left zero again.  No counterpart in the reference. */
uint32_t agocuda_ScaleGaussianHalf_tiles_shape(uint32_t dstWidth, uint32_t dstHeight, uint32_t threads, uint32_t rows);
int agocuda_fused_ScaleGaussianHalf_persistent(void *stream, const agocuda_half_job *jobs, uint32_t numJobs,
                                               uint32_t totalTiles, uint32_t *queue, uint32_t threads, uint32_t rows,
                                               uint32_t blocksPerSM);
/* TMA-staged form of the batch: a block of 112 threads makes 112 x 32 outputs of one level
 * from one 256 x 68-byte source box copied by TMA onto an mbarrier (the box columns outside
 * the row then take the bytes of AGO's buffer layout), so results equal the other forms bit
 * for bit.  job j's tileBegin counts tiles of this shape (agocuda_ScaleGaussianHalf_tiles_tma);
 * `maps` is a DEVICE array of numJobs 128-byte tensor maps (64-byte aligned) filled on the
 * host by agocuda_ScaleGaussianHalf_tensor_maps from the same jobs.  A block whose copy does
 * not complete within a bounded wait sets AGOCUDA_HALF_STATUS_TMA_TIMEOUT in *pStatus.  No
 * counterpart in the reference. */
#define AGOCUDA_HALF_STATUS_TMA_TIMEOUT 256u
uint32_t agocuda_ScaleGaussianHalf_tiles_tma(uint32_t dstWidth, uint32_t dstHeight);
int agocuda_ScaleGaussianHalf_tensor_maps(const agocuda_half_job *jobsHost, uint32_t numJobs, void *mapsHost,
                                          size_t mapsBytes);
int agocuda_fused_ScaleGaussianHalf_tma(void *stream, const agocuda_half_job *jobs, const void *maps, uint32_t numJobs,
                                        uint32_t totalTiles, uint32_t *pStatus);

/* ---------------------------------------------------------------- pyramidal LK */
#define AGOCUDA_LK_MAX_LEVELS 12
#define AGOCUDA_LK_MAX_WINDOW 15      /* AGO_OPTICALFLOWPYRLK_MAX_DIM */
/* With termination VX_TERM_CRITERIA_EPSILON alone the reference loop has no iteration bound
 * (ago_haf_cpu_opticalflow.cpp:431); a point that never converges stops after this many. */
#define AGOCUDA_LK_EPSILON_ONLY_MAX_ITERATIONS 4096u
#define AGOCUDA_LK_STATUS_BAD_COUNT 16u  /* old/estimate counts differ or exceed the output capacity */

typedef struct agocuda_pyramid_level {   /* one level: device image, as ago_pyramid_u8_t */
    const uint8_t *image;
    uint32_t width, height, stride, reserved;
} agocuda_pyramid_level;

/* One OpticalFlowPyrLK node (one frame pair).  Keypoint arrays hold vx_keypoint_t records;
 * counts are device words.  scharrRows is the node's persistent Scharr row-buffer state:
 * agocuda_OpticalFlowPyrLK_scharr_rows_size(level-0 width) bytes, zeroed when the node is
 * created and kept across executions (the reference's node scratch, whose stale words
 * reach the derivatives of column 0).  count and scharrWords are written by the kernels. */
typedef struct agocuda_lk_frame {
    agocuda_pyramid_level oldPyr[AGOCUDA_LK_MAX_LEVELS], newPyr[AGOCUDA_LK_MAX_LEVELS];
    const void *oldPoints, *estPoints;
    void *newPoints;
    const uint32_t *pOldCount, *pEstCount;
    uint32_t *pNewCount;
    uint16_t *scharrRows;
    uint32_t newCapacity, levels;
    int32_t termination;
    float epsilon;
    uint32_t numIterations;
    int32_t useInitialEstimate, windowDimension;
    uint32_t count;
    uint32_t scharrWords[AGOCUDA_LK_MAX_LEVELS][2];
    /* Per node, kept between calls (zeroed before the first): level-0 Scharr (gx, gy) pairs of
     * the previous call at columns [W_l & ~7, W_l - 3] of every level l >= 1 -- derivative
     * words the reference reads at level l but only its previous call's level 0 wrote.
     * Layout [level - 1][column - (W_l & ~7)][row], AGOCUDA_LK_CARRY_COLUMNS columns of
     * carryRows rows (>= the level-1 height).  NULL: those words read as 0. */
    int32_t *carry;
    uint32_t carryRows;
} agocuda_lk_frame;
#define AGOCUDA_LK_CARRY_COLUMNS 5
size_t agocuda_OpticalFlowPyrLK_scharr_rows_size(uint32_t width0);
/* Bytes of the carry buffer for a pyramid of `levels` levels whose level 1 is height1 rows. */
size_t agocuda_OpticalFlowPyrLK_carry_size(uint32_t levels, uint32_t height1);

/* Pyramidal LK for many frame pairs in three launches (row-buffer replay, one warp per
 * keypoint, carry of the level-0 derivative columns for the next call).  `frames` is a DEVICE
 * array; maxPoints bounds every frame's count.  Results are identical to
 * HafCpu_OpticalFlowPyrLK_XY_XY_Generic (ago_haf_cpu_opticalflow.cpp:153; CPU only in the
 * reference, ago_kernel_api.cpp:20587) for HALF pyramids whose level widths are all >= 8,
 * over consecutive calls too: on a level above 0 whose width % 8 >= 3 the reference's window
 * can reach derivative columns [W & ~7, W - 3], which it never writes at that level -- they
 * hold 0 on a node's first call and the previous call's level-0 derivatives afterwards; the
 * frame's `carry` buffer provides exactly those (without one they read as 0). */
int agocuda_OpticalFlowPyrLK_batch(void *stream, agocuda_lk_frame *frames, uint32_t numFrames, uint32_t maxPoints,
                                   uint32_t *pStatus);

/* Single node with the reference's argument meaning.  oldPyramid/newPyramid are HOST arrays
 * of `levels` descriptors (device images); counts are device words.  scratch (device,
 * zeroed before the node's first call and kept between calls) holds the frame descriptor and
 * the Scharr row-buffer state: agocuda_OpticalFlowPyrLK_scratch_size(width0) bytes, or
 * agocuda_OpticalFlowPyrLK_scratch_size_carry(width0, height0, levels) bytes to also carry the
 * level-0 derivative columns between calls (see agocuda_OpticalFlowPyrLK_batch). */
size_t agocuda_OpticalFlowPyrLK_scratch_size(uint32_t width0);
size_t agocuda_OpticalFlowPyrLK_scratch_size_carry(uint32_t width0, uint32_t height0, uint32_t levels);
int agocuda_OpticalFlowPyrLK_XY_XY(void *stream, void *newKeyPoint, uint32_t newCapacity, uint32_t *pNewCount,
                                   float pyramidScale, uint32_t levels, const agocuda_pyramid_level *oldPyramid,
                                   const agocuda_pyramid_level *newPyramid, const uint32_t *pKeyPointCount,
                                   const void *oldKeyPoint, const uint32_t *pEstimateCount,
                                   const void *newKeyPointEstimate, int32_t termination, float epsilon,
                                   uint32_t numIterations, int32_t useInitialEstimate, int32_t windowDimension,
                                   void *scratch, size_t scratchBytes, uint32_t *pStatus);

/* ------------------------------------------------------------------------------------ */
/* Array transfers inside a captured CUDA graph (engine internals; no HIP counterpart: the */
/* reference copies an array's count word, then its items, with blocking copies in        */
/* agoGpuHipDataInputSync / agoGpuHipDataOutputSync, ago_util_hip.cpp:321-608).          */
/* hostItemsMapped and countSlotMapped are DEVICE aliases of page-locked host memory     */
/* (cudaHostRegister/cudaHostAlloc with the mapped flag).                                */
/* ------------------------------------------------------------------------------------ */
#define AGOCUDA_ARRAY_SKIP 0xFFFFFFFFu   /* upload count slot: leave the device array as it is */

/* devItems[0 .. n) = hostItems[0 .. n), *devCount = n, n = min(*countSlot, capacity);
 * nothing when *countSlot == AGOCUDA_ARRAY_SKIP. */
int agocuda_array_upload(void *stream, void *devItems, uint32_t *devCount, const void *hostItemsMapped,
                         const uint32_t *countSlotMapped, uint32_t itemSize, uint32_t capacity);
/* agocuda_array_upload for `count` arrays in one launch; `xfers` is a DEVICE array. */
typedef struct agocuda_array_xfer {
    void *devItems;
    uint32_t *devCount;
    const void *hostItemsMapped;
    const uint32_t *countSlotMapped;
    uint32_t itemSize, capacity;
} agocuda_array_xfer;
int agocuda_array_upload_batch(void *stream, const agocuda_array_xfer *xfers, uint32_t count);
/* hostItems[0 .. n) = devItems[0 .. n), *countSlot = n, n = min(*devCount, capacity). */
int agocuda_array_download(void *stream, void *hostItemsMapped, uint32_t *countSlotMapped, const void *devItems,
                           const uint32_t *devCount, uint32_t itemSize, uint32_t capacity);

/* ------------------------------------------------------------------------------------ */
/* Element-wise kernels (reference: hipvx/hip_host_decls.h arithmetic/logical kernels;   */
/* CPU semantics ago/ago_haf_cpu_arithmetic.cpp, ago/ago_haf_cpu_logical.cpp)            */
/* Every pixel of [0,W)x[0,H).  Planes: row base 16-byte aligned and the stride a         */
/* multiple of 16.  _Wrap keeps the low bits of the exact result, _Sat clamps it to the    */
/* output type; S16 results of two U8 inputs are exact.                                   */
/* ------------------------------------------------------------------------------------ */

/* dst = src1 + src2.  Replace HipExec_Add_U8_U8U8_Wrap / _Sat (hip_host_decls.h:43, :48),
 * HipExec_Add_S16_U8U8 (:53), HipExec_Add_S16_S16U8_Wrap / _Sat (:58, :63) and
 * HipExec_Add_S16_S16S16_Wrap / _Sat (:68, :73). */
int agocuda_Add_U8_U8U8_Wrap(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                             const uint8_t *pSrc1, uint32_t src1Stride, const uint8_t *pSrc2, uint32_t src2Stride);
int agocuda_Add_U8_U8U8_Sat(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                            const uint8_t *pSrc1, uint32_t src1Stride, const uint8_t *pSrc2, uint32_t src2Stride);
int agocuda_Add_S16_U8U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                         const uint8_t *pSrc1, uint32_t src1Stride, const uint8_t *pSrc2, uint32_t src2Stride);
int agocuda_Add_S16_S16U8_Wrap(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                               const int16_t *pSrc1, uint32_t src1Stride, const uint8_t *pSrc2, uint32_t src2Stride);
int agocuda_Add_S16_S16U8_Sat(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                              const int16_t *pSrc1, uint32_t src1Stride, const uint8_t *pSrc2, uint32_t src2Stride);
int agocuda_Add_S16_S16S16_Wrap(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                                const int16_t *pSrc1, uint32_t src1Stride, const int16_t *pSrc2, uint32_t src2Stride);
int agocuda_Add_S16_S16S16_Sat(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                               const int16_t *pSrc1, uint32_t src1Stride, const int16_t *pSrc2, uint32_t src2Stride);

/* dst = src1 - src2.  Replace HipExec_Sub_U8_U8U8_Wrap / _Sat (hip_host_decls.h:78, :83),
 * HipExec_Sub_S16_U8U8 (:88), HipExec_Sub_S16_S16U8_Wrap / _Sat (:93, :98),
 * HipExec_Sub_S16_U8S16_Wrap / _Sat (:103, :108), HipExec_Sub_S16_S16S16_Wrap / _Sat (:113, :118). */
int agocuda_Sub_U8_U8U8_Wrap(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                             const uint8_t *pSrc1, uint32_t src1Stride, const uint8_t *pSrc2, uint32_t src2Stride);
int agocuda_Sub_U8_U8U8_Sat(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                            const uint8_t *pSrc1, uint32_t src1Stride, const uint8_t *pSrc2, uint32_t src2Stride);
int agocuda_Sub_S16_U8U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                         const uint8_t *pSrc1, uint32_t src1Stride, const uint8_t *pSrc2, uint32_t src2Stride);
int agocuda_Sub_S16_S16U8_Wrap(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                               const int16_t *pSrc1, uint32_t src1Stride, const uint8_t *pSrc2, uint32_t src2Stride);
int agocuda_Sub_S16_S16U8_Sat(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                              const int16_t *pSrc1, uint32_t src1Stride, const uint8_t *pSrc2, uint32_t src2Stride);
int agocuda_Sub_S16_U8S16_Wrap(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                               const uint8_t *pSrc1, uint32_t src1Stride, const int16_t *pSrc2, uint32_t src2Stride);
int agocuda_Sub_S16_U8S16_Sat(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                              const uint8_t *pSrc1, uint32_t src1Stride, const int16_t *pSrc2, uint32_t src2Stride);
int agocuda_Sub_S16_S16S16_Wrap(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                                const int16_t *pSrc1, uint32_t src1Stride, const int16_t *pSrc2, uint32_t src2Stride);
int agocuda_Sub_S16_S16S16_Sat(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                               const int16_t *pSrc1, uint32_t src1Stride, const int16_t *pSrc2, uint32_t src2Stride);

/* dst = |src1 - src2| (S16: clamped to 32767).  Replace HipExec_AbsDiff_U8_U8U8
 * (hip_host_decls.h:33) and HipExec_AbsDiff_S16_S16S16_Sat (:38). */
int agocuda_AbsDiff_U8_U8U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                            const uint8_t *pSrc1, uint32_t src1Stride, const uint8_t *pSrc2, uint32_t src2Stride);
int agocuda_AbsDiff_S16_S16S16_Sat(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                                   const int16_t *pSrc1, uint32_t src1Stride, const int16_t *pSrc2, uint32_t src2Stride);

/* Bitwise and / or / xor / not.  Replace HipExec_And_U8_U8U8 (hip_host_decls.h:238),
 * HipExec_Or_U8_U8U8 (:278), HipExec_Xor_U8_U8U8 (:318), HipExec_Not_U8_U8 (:358). */
int agocuda_And_U8_U8U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                        const uint8_t *pSrc1, uint32_t src1Stride, const uint8_t *pSrc2, uint32_t src2Stride);
int agocuda_Or_U8_U8U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                       const uint8_t *pSrc1, uint32_t src1Stride, const uint8_t *pSrc2, uint32_t src2Stride);
int agocuda_Xor_U8_U8U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                        const uint8_t *pSrc1, uint32_t src1Stride, const uint8_t *pSrc2, uint32_t src2Stride);
int agocuda_Not_U8_U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                      const uint8_t *pSrc, uint32_t srcStride);

/* ConvertDepth WRAP: low byte of (v >> shift) (arithmetic shift); and U8 -> S16: v << shift
 * kept to 16 bits.  Replace HipExec_ColorDepth_U8_S16_Wrap (hip_host_decls.h:398) and
 * HipExec_ColorDepth_S16_U8 (:408); ago_haf_cpu_arithmetic.cpp:3488, :3604.  shift 0..15. */
int agocuda_ColorDepth_U8_S16_Wrap(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                   uint32_t dstStride, const int16_t *pSrc, uint32_t srcStride, int32_t shift);
int agocuda_ColorDepth_S16_U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                              const uint8_t *pSrc, uint32_t srcStride, int32_t shift);

/* 255 where lower <= v <= upper, else 0 (bounds taken as vx_uint8).  Replaces
 * HipExec_Threshold_U8_U8_Range (hip_host_decls.h:694); HafCpu_Threshold_U8_U8_Range
 * (ago_haf_cpu_arithmetic.cpp:3742). */
int agocuda_Threshold_U8_U8_Range(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                  uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride, int32_t thresholdLower,
                                  int32_t thresholdUpper);

/* ------------------------------------------------------------------------------------ */
/* 3x3 neighbourhood filters on U8 (reference: hipvx/hip_host_decls.h filter_kernels;    */
/* CPU semantics ago/ago_haf_cpu_filter.cpp).  Rows [1, H-1) are written, every column;  */
/* pixels of columns 0 and W-1 are unspecified (outside the valid region).  Row bases   */
/* 4-byte aligned, strides multiples of 4.                                                */
/* ------------------------------------------------------------------------------------ */

/* floor(sum of the 3x3 window / 9).  Replaces HipExec_Box_U8_U8_3x3 (hip_host_decls.h:633);
 * HafCpu_Box_U8_U8_3x3 (ago_haf_cpu_filter.cpp:34). */
int agocuda_Box_U8_U8_3x3(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                          const uint8_t *pSrc, uint32_t srcStride);
/* Maximum / minimum of the 3x3 window.  Replace HipExec_Dilate_U8_U8_3x3 (hip_host_decls.h:637)
 * and HipExec_Erode_U8_U8_3x3 (:641); ago_haf_cpu_filter.cpp:221, :298. */
int agocuda_Dilate_U8_U8_3x3(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                             const uint8_t *pSrc, uint32_t srcStride);
int agocuda_Erode_U8_U8_3x3(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                            const uint8_t *pSrc, uint32_t srcStride);
/* Median of the 3x3 window.  Replaces HipExec_Median_U8_U8_3x3 (hip_host_decls.h:645);
 * HafCpu_Median_U8_U8_3x3 (ago_haf_cpu_filter.cpp:3842). */
int agocuda_Median_U8_U8_3x3(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                             const uint8_t *pSrc, uint32_t srcStride);

/* dst = lut[src] for U8 (pLut: 256 device bytes); dst = lut[clamp(src + offset, 0, count-1)]
 * for S16 (pLut: count device int16, offset = count / 2 for OpenVX LUTs).  Planes 16-byte
 * aligned.  Replace HipExec_Lut_U8_U8 (hip_host_decls.h:377) and the CPU-only
 * HafCpu_Lut_S16_S16 (ago_haf_cpu_arithmetic.cpp:4916). */
int agocuda_Lut_U8_U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                      const uint8_t *pSrc, uint32_t srcStride, const uint8_t *pLut);
int agocuda_Lut_S16_S16(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                        const int16_t *pSrc, uint32_t srcStride, const int16_t *pLut, uint32_t count, uint32_t offset);

/* Integral image: dst(x, y) = sum of src over [0, x] x [0, y], modulo 2^32.  Needs `scratch`
 * device memory of agocuda_IntegralImage_scratch_size(W, H) bytes; three launches.  Replaces
 * HafCpu_IntegralImage_U32_U8 (ago_haf_cpu_arithmetic.cpp:7057; CPU only in the reference). */
size_t agocuda_IntegralImage_scratch_size(uint32_t width, uint32_t height);
int agocuda_IntegralImage_U32_U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint32_t *pDst, uint32_t dstStride,
                                 const uint8_t *pSrc, uint32_t srcStride, void *scratch, size_t scratchBytes);

/* Histogram into pHist[numBins] (device; cleared first): pixels v with offset <= v <
 * offset + range count into bin (v - offset) * numBins / range.  Source rows 16-byte
 * aligned.  The reference computes it on the CPU only (HafCpu_HistogramFixedBins_DATA_U8,
 * ago_haf_cpu_histogram.cpp:519). */
int agocuda_Histogram_DATA_U8(void *stream, uint32_t *pHist, uint32_t srcWidth, uint32_t srcHeight, const uint8_t *pSrc,
                              uint32_t srcStride, uint32_t numBins, int32_t offset, uint32_t range);

/* ------------------------------------------------------------------------------------ */
/* Channel extract / combine (reference: hipvx/hip_host_decls.h:413-492; CPU semantics    */
/* ago/ago_haf_cpu_ch_extract_combine.cpp).  Row bases 4-byte aligned, strides multiples  */
/* of 4.                                                                                   */
/* ------------------------------------------------------------------------------------ */

/* dst[x] = src[x * n + k] for the n-byte units of an interleaved plane (U16: NV12/NV21 UV
 * plane, YUYV/UYVY luma; U24: RGB; U32: RGBX, or YUYV/UYVY chroma over pixel pairs);
 * dstWidth counts output pixels.  Replace HipExec_ChannelExtract_U8_U16_Pos0 .. _U8_U32_Pos3
 * (hip_host_decls.h:413-448). */
int agocuda_ChannelExtract_U8_U16_Pos0(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                       uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride);
int agocuda_ChannelExtract_U8_U16_Pos1(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                       uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride);
int agocuda_ChannelExtract_U8_U24_Pos0(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                       uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride);
int agocuda_ChannelExtract_U8_U24_Pos1(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                       uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride);
int agocuda_ChannelExtract_U8_U24_Pos2(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                       uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride);
int agocuda_ChannelExtract_U8_U32_Pos0(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                       uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride);
int agocuda_ChannelExtract_U8_U32_Pos1(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                       uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride);
int agocuda_ChannelExtract_U8_U32_Pos2(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                       uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride);
int agocuda_ChannelExtract_U8_U32_Pos3(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                       uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride);
/* Interleave U8 planes: UV (NV12 chroma), RGB, RGBX, and UYVY / YUYV from Y (full width) +
 * U, V (half width), dstWidth in pixels.  Replace HipExec_ChannelCombine_U16_U8U8 (:465),
 * _U24_U8U8U8_RGB (:470), _U32_U8U8U8_UYVY (:476), _U32_U8U8U8_YUYV (:482),
 * _U32_U8U8U8U8_RGBX (:488). */
int agocuda_ChannelCombine_U16_U8U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                    uint32_t dstStride, const uint8_t *pSrc1, uint32_t src1Stride, const uint8_t *pSrc2,
                                    uint32_t src2Stride);
int agocuda_ChannelCombine_U24_U8U8U8_RGB(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                          uint32_t dstStride, const uint8_t *pSrc1, uint32_t src1Stride,
                                          const uint8_t *pSrc2, uint32_t src2Stride, const uint8_t *pSrc3,
                                          uint32_t src3Stride);
int agocuda_ChannelCombine_U32_U8U8U8_UYVY(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                           uint32_t dstStride, const uint8_t *pSrc1, uint32_t src1Stride,
                                           const uint8_t *pSrc2, uint32_t src2Stride, const uint8_t *pSrc3,
                                           uint32_t src3Stride);
int agocuda_ChannelCombine_U32_U8U8U8_YUYV(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                           uint32_t dstStride, const uint8_t *pSrc1, uint32_t src1Stride,
                                           const uint8_t *pSrc2, uint32_t src2Stride, const uint8_t *pSrc3,
                                           uint32_t src3Stride);
int agocuda_ChannelCombine_U32_U8U8U8U8_RGBX(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                             uint32_t dstStride, const uint8_t *pSrc1, uint32_t src1Stride,
                                             const uint8_t *pSrc2, uint32_t src2Stride, const uint8_t *pSrc3,
                                             uint32_t src3Stride, const uint8_t *pSrc4, uint32_t src4Stride);

/* ------------------------------------------------------------------------------------ */
/* Fused U8 pixel chains: element-wise and 3x3 kernels through on-chip intermediates.    */
/* The device counterpart of AGO's GPU supernodes (ago/ago_drama_alloc.cpp:484), which   */
/* merge element-wise and fixed-neighbourhood kernels into one generated kernel; the     */
/* HIP target has no equivalent.  Each op applies to the chain's current value; binary   */
/* ops take their other operand from the frame's side image `side`.                     */
/* ------------------------------------------------------------------------------------ */
enum agocuda_pixel_opcode {
    AGOCUDA_PX_NOT = 1,                /* Not_U8_U8                                         */
    AGOCUDA_PX_AND, AGOCUDA_PX_OR, AGOCUDA_PX_XOR, AGOCUDA_PX_ABSDIFF,
    AGOCUDA_PX_ADD_WRAP, AGOCUDA_PX_ADD_SAT, AGOCUDA_PX_SUB_WRAP, AGOCUDA_PX_SUB_SAT,
    AGOCUDA_PX_THRESHOLD_BINARY,       /* p0: threshold (v > p0 -> 255)                     */
    AGOCUDA_PX_THRESHOLD_RANGE,        /* p0, p1: lower, upper                              */
    AGOCUDA_PX_BOX3x3, AGOCUDA_PX_MEDIAN3x3, AGOCUDA_PX_DILATE3x3, AGOCUDA_PX_ERODE3x3,
    AGOCUDA_PX_GAUSSIAN3x3
};
#define AGOCUDA_PX_MAX_OPS 16
#define AGOCUDA_PX_MAX_SIDES 3
#define AGOCUDA_PX_MAX_STENCILS 4      /* 3x3 ops per chain */
typedef struct agocuda_pixel_op {
    int32_t code;                      /* agocuda_pixel_opcode */
    int32_t side;                      /* binary ops: index into agocuda_pixel_frame.side */
    int32_t sideFirst;                 /* SUB: 1 when the side image is the minuend */
    int32_t p0, p1;                    /* threshold parameters (as vx_uint8) */
} agocuda_pixel_op;
typedef struct agocuda_pixel_program {
    int32_t numOps;
    agocuda_pixel_op ops[AGOCUDA_PX_MAX_OPS];
} agocuda_pixel_program;
/* src / side planes: row bases 16-byte aligned, strides multiples of 16; dst: 4-byte aligned
 * base and stride; every stride at least the width. */
typedef struct agocuda_pixel_frame {
    const uint8_t *src;
    uint8_t *dst;
    const uint8_t *side[AGOCUDA_PX_MAX_SIDES];
    uint32_t width, height, srcStride, dstStride, sideStride[AGOCUDA_PX_MAX_SIDES];
} agocuda_pixel_frame;
/* Runs `program` over every frame (`frames` is a DEVICE array) in one launch.  Inside the
 * valid rectangle of the chain's last output (every 3x3 op trims one pixel per side) the
 * result equals the ops run one by one; other pixels are unspecified. */
int agocuda_fused_PixelChain_U8(void *stream, const agocuda_pixel_program *program,
                                const agocuda_pixel_frame *frames, uint32_t numFrames, uint32_t maxWidth,
                                uint32_t maxHeight);

/* The same chain with each block's input tiles staged by TMA: one 2D tensor copy per plane
 * (box 160 x (64 + 2 x stencils) bytes) completing on a shared-memory mbarrier, instead of
 * ~700 16-byte cp.async copies per plane.  `maps` is a DEVICE array of
 * agocuda_PixelChain_tensor_maps_size(numFrames) bytes (64-byte aligned) filled on the host
 * by agocuda_PixelChain_tensor_maps for the same program and frames (source and side planes
 * need 16-byte aligned bases and strides).  Results are identical to
 * agocuda_fused_PixelChain_U8 inside the chain's valid rectangle.  A block whose copies do not
 * complete within a bounded wait sets AGOCUDA_PX_STATUS_TMA_TIMEOUT in *pStatus.  No
 * counterpart in the reference (its OpenCL supernodes, ago_drama_alloc.cpp:484, load per
 * work-item). */
#define AGOCUDA_PX_STATUS_TMA_TIMEOUT 128u
size_t agocuda_PixelChain_tensor_maps_size(uint32_t numFrames);
int agocuda_PixelChain_tensor_maps(const agocuda_pixel_program *program, const agocuda_pixel_frame *framesHost,
                                   uint32_t numFrames, void *mapsHost, size_t mapsBytes);
int agocuda_fused_PixelChain_U8_tma(void *stream, const agocuda_pixel_program *program,
                                    const agocuda_pixel_frame *frames, const void *maps, uint32_t numFrames,
                                    uint32_t maxWidth, uint32_t maxHeight, uint32_t *pStatus);

#ifdef __cplusplus
}
#endif
#endif /* AGOCUDA_H */
