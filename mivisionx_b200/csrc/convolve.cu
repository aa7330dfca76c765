// convolve.cu -- vxConvolveNode (org.khronos.openvx.custom_convolution) on sm_100a: U8 input,
// U8 or S16 output, odd kernels of 3, 5, 7 or 9 columns and 3..9 rows.
//
// Reference arithmetic (HafCpu_Convolve_{U8,S16}_U8_{3,5,7,9}xN, ago_haf_cpu_filter.cpp:2676-
// 3830): the coefficients are applied flipped in both directions (a true convolution) with
// exact int32 sums.  In the SIMD body the sum is shifted right LOGICALLY by the
// convolution's scale shift and saturated to int16 (and then to u8); in the scalar prefix and
// postfix columns the unshifted sum is saturated directly.  Callers give the body's column
// range (the split depends on the destination row address in the reference; AGO rows are
// 16-byte aligned, so the body is [0, W - W % 16)).  Rows [rows/2, H - rows/2) are written.
//
// A block of 32 x 8 threads computes a 128 x 16 tile (4 columns x 2 rows per thread) from a
// shared-memory copy of the source tile with a 4-pixel halo on every side, loaded as words.
#include "agocuda_internal.cuh"

uint64_t agocuda_count_launch(unsigned n);

namespace {

constexpr int kCvTX = 128, kCvTY = 16, kCvHalo = 4;
constexpr int kCvSW = kCvTX + 2 * kCvHalo, kCvSH = kCvTY + 2 * kCvHalo;   // 136 x 24 bytes

struct ConvArgs {
    int16_t k[81];                 // flipped: k[i * cols + j] multiplies src(y - rows/2 + i, x - cols/2 + j)
    int rows, shift, simdBegin, simdEnd;
};

template <int COLS, bool S16>
__global__ void __launch_bounds__(256) k_convolve(int W, int H, uint8_t *dst, int dstStride, const uint8_t *src, int srcStride,
                                                  ConvArgs A)
{
    __shared__ __align__(16) uint8_t t[kCvSH][kCvSW];
    const int x0 = blockIdx.x * kCvTX, y0 = blockIdx.y * kCvTY;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    // the tile's rows [y0 - 4, y0 + 20) and columns [x0 - 4, x0 + 132) as 34 words per row;
    // rows clamp into the image, columns into the row's allocation (values read there only
    // reach columns outside the valid region)
    for (int i = tid; i < kCvSH * (kCvSW / 4); i += 256) {
        const int r = i / (kCvSW / 4), w = i - r * (kCvSW / 4);
        const int y = clampi(y0 - kCvHalo + r, 0, H - 1);
        *(uint32_t *)&t[r][4 * w] = load_word_clamped(src + (size_t)y * srcStride, x0 - kCvHalo + 4 * w, srcStride);
    }
    __syncthreads();
    const int hy = A.rows >> 1, lx = 4 * threadIdx.x, ly = 2 * threadIdx.y;
    const int x = x0 + lx;
    int acc[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
    for (int i = 0; i < A.rows; i++) {
        const uint8_t *row0 = &t[kCvHalo - hy + ly + i][kCvHalo - COLS / 2 + lx];
        const uint8_t *row1 = row0 + kCvSW;
#pragma unroll
        for (int j = 0; j < COLS; j++) {
            const int c = A.k[i * COLS + j];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                acc[0][q] += c * (int)row0[j + q];
                acc[1][q] += c * (int)row1[j + q];
            }
        }
    }
    const int lo = S16 ? -32768 : 0, hi = S16 ? 32767 : 255;
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const int y = y0 + ly + r;
        if (y < hy || y >= H - hy || x >= W) continue;
        int v[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int s = acc[r][q];
            const bool body = x + q >= A.simdBegin && x + q < A.simdEnd;
            const int sh = (int)((uint32_t)s >> A.shift);
            v[q] = body ? clampi(clampi(sh, -32768, 32767), lo, hi) : clampi(s, lo, hi);
        }
        uint8_t *d = dst + (size_t)y * dstStride + (size_t)x * (S16 ? 2 : 1);
        if (x + 4 <= W) {
            if (S16) *(uint2 *)d = make_uint2((uint32_t)(uint16_t)v[0] | ((uint32_t)(uint16_t)v[1] << 16),
                                              (uint32_t)(uint16_t)v[2] | ((uint32_t)(uint16_t)v[3] << 16));
            else *(uint32_t *)d = (uint32_t)v[0] | ((uint32_t)v[1] << 8) | ((uint32_t)v[2] << 16) | ((uint32_t)v[3] << 24);
        } else {
            for (int q = 0; q < W - x; q++) {
                if (S16) ((int16_t *)d)[q] = (int16_t)v[q];
                else d[q] = (uint8_t)v[q];
            }
        }
    }
}

template <bool S16>
int convolve(void *stream, uint32_t W, uint32_t H, void *pDst, uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride,
             const int16_t *conv, uint32_t cols, uint32_t rows, int32_t shift, int32_t simdBegin, int32_t simdEnd)
{
    const unsigned bpp = S16 ? 2 : 1;
    if (!pDst || !pSrc || !conv || !(cols == 3 || cols == 5 || cols == 7 || cols == 9) || !(rows & 1) || rows < 3 ||
        rows > 9 || W < cols || H < rows || shift < 0 || shift > 31 || ((uintptr_t)pDst & (4 * bpp - 1)) ||
        (dstStride % (4 * bpp)) || dstStride < W * bpp || ((uintptr_t)pSrc & 3) || (srcStride & 3) || srcStride < W)
        return AGOCUDA_INVALID_PARAMS;
    ConvArgs A{};
    const int n = (int)(cols * rows);
    for (int k = 0; k < n; k++) A.k[k] = conv[n - 1 - k];
    A.rows = (int)rows;
    A.shift = shift;
    A.simdBegin = simdBegin;
    A.simdEnd = simdEnd;
    const dim3 grd(div_up(W, kCvTX), div_up(H, kCvTY)), blk(32, 8);
    cudaStream_t s = as_stream(stream);
    uint8_t *d = (uint8_t *)pDst;
    switch (cols) {
    case 3: k_convolve<3, S16><<<grd, blk, 0, s>>>((int)W, (int)H, d, (int)dstStride, pSrc, (int)srcStride, A); break;
    case 5: k_convolve<5, S16><<<grd, blk, 0, s>>>((int)W, (int)H, d, (int)dstStride, pSrc, (int)srcStride, A); break;
    case 7: k_convolve<7, S16><<<grd, blk, 0, s>>>((int)W, (int)H, d, (int)dstStride, pSrc, (int)srcStride, A); break;
    default: k_convolve<9, S16><<<grd, blk, 0, s>>>((int)W, (int)H, d, (int)dstStride, pSrc, (int)srcStride, A); break;
    }
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

}  // namespace

extern "C" int agocuda_Convolve_U8_U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                                      const uint8_t *pSrc, uint32_t srcStride, const int16_t *conv, uint32_t cols,
                                      uint32_t rows, int32_t shift, int32_t simdBegin, int32_t simdEnd)
{
    return convolve<false>(stream, dstWidth, dstHeight, pDst, dstStride, pSrc, srcStride, conv, cols, rows, shift, simdBegin,
                           simdEnd);
}

extern "C" int agocuda_Convolve_S16_U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                                       const uint8_t *pSrc, uint32_t srcStride, const int16_t *conv, uint32_t cols,
                                       uint32_t rows, int32_t shift, int32_t simdBegin, int32_t simdEnd)
{
    return convolve<true>(stream, dstWidth, dstHeight, pDst, dstStride, pSrc, srcStride, conv, cols, rows, shift, simdBegin,
                          simdEnd);
}
