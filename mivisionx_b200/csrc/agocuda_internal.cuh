// agocuda_internal.cuh -- helpers shared by the sm_100a kernels behind include/agocuda.h.
#pragma once
#include <cuda.h>          // CUtensorMap and its enums (the encoder comes through the runtime)
#include <cuda_runtime.h>
#include <stdint.h>
#include "agocuda.h"

#define AGOCUDA_INVALID_PARAMS (-10)   // same value as VX_ERROR_INVALID_PARAMETERS
#define AGOCUDA_NO_MEMORY      (-8)    // same value as VX_ERROR_NO_MEMORY
#define AGOCUDA_TOO_LARGE      (-15)   // same value as VX_ERROR_INVALID_DIMENSION

// Map the launch status to the C-ABI return convention: 0 on success, else the
// cudaError_t (positive) of the failed launch.
static inline int agocuda_launch_status()
{
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}

static inline cudaStream_t as_stream(void *s) { return (cudaStream_t)s; }

static inline unsigned div_up(unsigned a, unsigned b) { return (a + b - 1) / b; }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link); null
// when the driver does not provide it.
using agocuda_encode_tiled_fn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                             const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                             CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                             CUtensorMapFloatOOBfill);
static inline agocuda_encode_tiled_fn agocuda_encode_tiled()
{
    static agocuda_encode_tiled_fn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (agocuda_encode_tiled_fn) nullptr;
        return (agocuda_encode_tiled_fn)p;
    }();
    return fn;
}

// A 2D U8 tensor map of a pitched plane with a boxW x boxH box; zero fill outside the plane.
static inline bool agocuda_u8_tensor_map(CUtensorMap *m, const void *base, uint32_t width, uint32_t height,
                                         uint32_t stride, uint32_t boxW, uint32_t boxH)
{
    agocuda_encode_tiled_fn enc = agocuda_encode_tiled();
    if (!enc || !base || ((uintptr_t)base & 15) || (stride & 15) || stride < width || !width || !height) return false;
    const cuuint64_t dims[2] = {width, height}, strides[1] = {stride};
    const cuuint32_t box[2] = {boxW, boxH}, estr[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void *)base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// A 2D tensor map of a pitched U8 plane seen as rows of 32-bit elements (widthBytes rounded
// up to whole elements, which must lie inside the row pitch), so that one box can span up to
// 1024 bytes of a row; zero fill outside the plane.
static inline bool agocuda_u8_as_u32_tensor_map(CUtensorMap *m, const void *base, uint32_t widthBytes, uint32_t height,
                                                uint32_t stride, uint32_t boxWords, uint32_t boxH)
{
    agocuda_encode_tiled_fn enc = agocuda_encode_tiled();
    const uint32_t words = (widthBytes + 3) / 4;
    if (!enc || !base || ((uintptr_t)base & 15) || (stride & 15) || stride < 4 * words || !widthBytes || !height)
        return false;
    const cuuint64_t dims[2] = {words, height}, strides[1] = {stride};
    const cuuint32_t box[2] = {boxWords, boxH}, estr[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, (void *)base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

__device__ __forceinline__ uint32_t smem_addr_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbarrier_try_wait_parity(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}

// Multiprocessors of the current device (persistent kernels size their grid by it).
static inline int agocuda_sm_count()
{
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 148;
    return n > 0 ? n : 148;
}

// The reference HAF kernels split each row into a scalar prefix (bytes up to the next
// 16-byte boundary of the destination row pointer, used as a pixel count), a 16-wide SIMD
// body and a scalar tail of (width - prefix) & 15 pixels, and some of them round
// differently in the scalar parts.  This returns the column range [simd_begin, simd_end)
// that the reference handles in its SIMD body for a destination row starting at `row`.
struct SimdSpan { int begin, end; };
static inline SimdSpan haf_simd_span(const void *row, int width, int lanes_mask = 15)
{
    int p = (int)((uintptr_t)row & 15);
    p = p ? 16 - p : 0;
    int post = (width - p) & lanes_mask;
    return SimdSpan{p, width - post};
}

__device__ __forceinline__ uint32_t ldg_u32(const uint8_t *p) { return __ldg((const unsigned int *)p); }
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Load the 32-bit word that holds columns [c, c+4) of a U8 row, with c clamped into
// [0, stride-4]; rows are clamped by the caller.  Values read through a clamp only feed
// pixels outside the valid region, which OpenVX leaves undefined for these kernels.
__device__ __forceinline__ uint32_t load_word_clamped(const uint8_t *row, int c, int stride)
{
    c = clampi(c, 0, stride - 4);
    return ldg_u32(row + c);
}

// layout of vx_keypoint_t (OpenVX vx_types.h)
struct vx_keypoint_like {
    int32_t x, y;
    float strength, scale, orientation;
    int32_t tracking_status;
    float error;
};

__device__ __forceinline__ int byte_of(uint32_t w, int i) { return (w >> (8 * i)) & 0xff; }

// Byte (r, c) of a U8 image stored as AGO stores it: row pitch ALIGN16(W), rows contiguous,
// zeros before the first and after the last row and between W and the pitch.  Reading
// column -1 therefore gives the previous row's padding (0) or, when W % 16 == 0, its last
// pixel; column W gives padding or the next row's first pixel.  The reference's stencils
// make such reads at the image edges.
__device__ __forceinline__ uint32_t ago_byte(const uint8_t *img, size_t stride, int W, int H, int r, int c)
{
    if (c >= 0 && c < W && r >= 0 && r < H) return img[(size_t)r * stride + c];
    const long long S = (W + 15) & ~15;
    const long long f = (long long)r * S + c;
    if (f < 0 || f >= (long long)H * S) return 0;
    const int rr = (int)(f / S), cc = (int)(f - rr * S);
    return cc < W ? img[(size_t)rr * stride + cc] : 0;
}
