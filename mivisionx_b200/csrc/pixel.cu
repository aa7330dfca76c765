// pixel.cu -- the AGO kernels on either side of the vision graphs, for sm_100a:
// element-wise arithmetic / logical / range-threshold kernels and the 3x3 Box, Median,
// Dilate and Erode filters.
//
// Element-wise kernels are HBM-bound: a thread owns 8 pixels of a row (one 8- or 16-byte
// vector per plane), a warp 256 contiguous pixels, and rows are spread over blockIdx.y.
// The 3x3 filters use the stencil decomposition of filters.cu (one 32-bit word of 4 pixels
// per thread, rows walked downwards with the previous rows' partial results in registers);
// Dilate, Erode and Median run on all 4 pixels at once with byte-lane min/max.
#include "agocuda_internal.cuh"

uint64_t agocuda_count_launch(unsigned n);

namespace {

// ---------------------------------------------------------------------------------
// Element-wise kernels (ago_haf_cpu_arithmetic.cpp, ago_haf_cpu_logical.cpp)
// ---------------------------------------------------------------------------------
enum EwOp : int {
    EW_ADD_WRAP_U8, EW_ADD_SAT_U8, EW_SUB_WRAP_U8, EW_SUB_SAT_U8,
    EW_ADD_S16, EW_SUB_S16,                      // U8 x U8 -> S16, exact
    EW_ADD_WRAP_S16, EW_ADD_SAT_S16, EW_SUB_WRAP_S16, EW_SUB_SAT_S16,
    EW_ABSDIFF_U8, EW_ABSDIFF_SAT_S16,
    EW_AND, EW_OR, EW_XOR, EW_NOT,
    EW_RANGE,                                    // 255 inside [lower, upper], else 0
};

__device__ __forceinline__ int sat_s16(int v) { return v < -32768 ? -32768 : (v > 32767 ? 32767 : v); }

template <int OP>
__device__ __forceinline__ int ew_apply(int a, int b, int p0, int p1)
{
    switch (OP) {
    case EW_ADD_WRAP_U8: return (a + b) & 0xff;                        // :26
    case EW_ADD_SAT_U8: return min(a + b, 255);                        // :186
    case EW_SUB_WRAP_U8: return (a - b) & 0xff;                        // :352
    case EW_SUB_SAT_U8: return max(a - b, 0);                          // :512
    case EW_ADD_S16: return a + b;                                     // :672
    case EW_SUB_S16: return a - b;                                     // :863
    case EW_ADD_WRAP_S16: return (int)(int16_t)(a + b);                // :1050, :2158
    case EW_ADD_SAT_S16: return sat_s16(a + b);                        // :1232, :2346
    case EW_SUB_WRAP_S16: return (int)(int16_t)(a - b);                // :1418, :1790, :2534
    case EW_SUB_SAT_S16: return sat_s16(a - b);                        // :1604, :1972, :2722
    case EW_ABSDIFF_U8: return abs(a - b);                             // :2910
    case EW_ABSDIFF_SAT_S16: return min(abs(a - b), 32767);            // :3114
    case EW_AND: return a & b;
    case EW_OR: return a | b;
    case EW_XOR: return a ^ b;
    case EW_NOT: return ~a & 0xff;
    case EW_RANGE: return (a > p1 || a < p0) ? 0 : 255;                // :3742
    }
    return 0;
}

template <typename T> struct Vec8;
template <> struct Vec8<uint8_t> { using V = uint2; };
template <> struct Vec8<int16_t> { using V = uint4; };

template <typename T>
__device__ __forceinline__ void load8(const T *p, int *v)
{
    const typename Vec8<T>::V w = __ldg((const typename Vec8<T>::V *)p);
    const T *e = (const T *)&w;
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = (int)e[i];
}

template <typename T>
__device__ __forceinline__ void store8(T *p, const int *v)
{
    typename Vec8<T>::V w;
    T *e = (T *)&w;
#pragma unroll
    for (int i = 0; i < 8; i++) e[i] = (T)v[i];
    *(typename Vec8<T>::V *)p = w;
}

constexpr int kEwBX = 32, kEwBY = 8;

// one thread: pixels [x, x+8) of row y; the last group of a row that W cuts goes pixel by pixel
template <int OP, typename TO, typename TA, typename TB>
__global__ void __launch_bounds__(kEwBX * kEwBY)
k_elementwise(int W, int H, TO *dst, int dstStride, const TA *a, int aStride, const TB *b, int bStride, int p0, int p1)
{
    const int x = (blockIdx.x * kEwBX + threadIdx.x) * 8;
    const int y = blockIdx.y * kEwBY + threadIdx.y;
    if (x >= W || y >= H) return;
    TO *d = (TO *)((uint8_t *)dst + (size_t)y * dstStride) + x;
    const TA *pa = (const TA *)((const uint8_t *)a + (size_t)y * aStride) + x;
    const TB *pb = b ? (const TB *)((const uint8_t *)b + (size_t)y * bStride) + x : nullptr;
    if (x + 8 <= W) {
        int va[8], vb[8] = {0, 0, 0, 0, 0, 0, 0, 0}, r[8];
        load8(pa, va);
        if (pb) load8(pb, vb);
#pragma unroll
        for (int i = 0; i < 8; i++) r[i] = ew_apply<OP>(va[i], vb[i], p0, p1);
        store8(d, r);
    } else {
        for (int i = 0; i < W - x; i++) d[i] = (TO)ew_apply<OP>((int)pa[i], pb ? (int)pb[i] : 0, p0, p1);
    }
}

template <typename T> bool ew_plane_ok(const T *p, uint32_t stride, uint32_t W)
{
    constexpr unsigned vec = 8 * sizeof(T);      // bytes of an 8-pixel vector
    return p && ((uintptr_t)p % vec) == 0 && (stride % vec) == 0 && stride >= W * sizeof(T);
}

template <int OP, typename TO, typename TA, typename TB>
int ew_launch(void *stream, uint32_t W, uint32_t H, TO *dst, uint32_t dstStride, const TA *a, uint32_t aStride,
              const TB *b, uint32_t bStride, int p0 = 0, int p1 = 0)
{
    const bool unary = OP == EW_NOT || OP == EW_RANGE;
    if (!W || !H || !ew_plane_ok(dst, dstStride, W) || !ew_plane_ok(a, aStride, W) ||
        (!unary && !ew_plane_ok(b, bStride, W)))
        return AGOCUDA_INVALID_PARAMS;
    dim3 grd(div_up(W, kEwBX * 8), div_up(H, kEwBY));
    k_elementwise<OP, TO, TA, TB><<<grd, dim3(kEwBX, kEwBY), 0, as_stream(stream)>>>(
        (int)W, (int)H, dst, (int)dstStride, a, (int)aStride, unary ? nullptr : b, (int)bStride, p0, p1);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

// ---------------------------------------------------------------------------------
// 3x3 filters on U8 (ago_haf_cpu_filter.cpp): interior rows [1, H-1), every column
// ---------------------------------------------------------------------------------
enum FOp : int { F_BOX, F_DILATE, F_ERODE, F_MEDIAN };   // F_BOX runs k_box3x3
constexpr int kFBX = 32, kFBY = 4, kFRows = 8;

// one row around the word at x: columns x-1..x+2 (l), x..x+3 (c), x+1..x+4 (r)
struct Row3 { uint32_t l, c, r; };
__device__ __forceinline__ Row3 row3(const uint8_t *row, int x, int stride)
{
    const uint32_t L = load_word_clamped(row, x - 4, stride), C = load_word_clamped(row, x, stride),
                   R = load_word_clamped(row, x + 4, stride);
    return Row3{__funnelshift_r(L, C, 24), C, __funnelshift_r(C, R, 8)};
}

// per-byte sort of three words
__device__ __forceinline__ void sort3(uint32_t a, uint32_t b, uint32_t c, uint32_t &lo, uint32_t &mid, uint32_t &hi)
{
    const uint32_t l1 = __vminu4(a, b), h1 = __vmaxu4(a, b);
    lo = __vminu4(l1, c);
    const uint32_t t = __vmaxu4(l1, c);
    mid = __vminu4(h1, t);
    hi = __vmaxu4(h1, t);
}

__device__ __forceinline__ uint32_t med3(uint32_t a, uint32_t b, uint32_t c)
{
    return __vmaxu4(__vminu4(a, b), __vminu4(__vmaxu4(a, b), c));
}

// Row sums of three neighbours in 16-bit lanes: E = columns (x, x+2), O = (x+1, x+3)
struct Sum3 { uint32_t E, O; };
__device__ __forceinline__ Sum3 sum3(const Row3 &r)
{
    return Sum3{__byte_perm(r.l, 0, 0x4240) + __byte_perm(r.c, 0, 0x4240) + __byte_perm(r.r, 0, 0x4240),
                __byte_perm(r.l, 0, 0x4341) + __byte_perm(r.c, 0, 0x4341) + __byte_perm(r.r, 0, 0x4341)};
}

// Box: floor(sum / 9) -- the reference's SIMD body computes (sum * 7282) >> 16 and its
// scalar parts (int)((float)sum / 9.0f); both equal floor(sum / 9) for every sum of nine
// bytes (<= 2295), and so does (sum * 7282) >> 16 here.
__device__ __forceinline__ uint32_t box_word(const Sum3 &a, const Sum3 &b, const Sum3 &c)
{
    const uint32_t e = a.E + b.E + c.E, o = a.O + b.O + c.O;
    const uint32_t q0 = ((e & 0xffff) * 7282u) >> 16, q2 = ((e >> 16) * 7282u) >> 16;
    const uint32_t q1 = ((o & 0xffff) * 7282u) >> 16, q3 = ((o >> 16) * 7282u) >> 16;
    return q0 | (q1 << 8) | (q2 << 16) | (q3 << 24);
}

__global__ void __launch_bounds__(kFBX * kFBY)
k_box3x3(int W, int H, uint8_t *dst, int dstStride, const uint8_t *src, int srcStride)
{
    const int x = (blockIdx.x * kFBX + threadIdx.x) * 4;
    const int y0 = 1 + (blockIdx.y * kFBY + threadIdx.y) * kFRows;
    if (x >= W || y0 >= H - 1) return;
    const int y1 = min(y0 + kFRows, H - 1);
    Sum3 a = sum3(row3(src + (size_t)(y0 - 1) * srcStride, x, srcStride));
    Sum3 b = sum3(row3(src + (size_t)y0 * srcStride, x, srcStride));
    for (int y = y0; y < y1; y++) {
        const Sum3 c = sum3(row3(src + (size_t)(y + 1) * srcStride, x, srcStride));
        const uint32_t o = box_word(a, b, c);
        uint8_t *d = dst + (size_t)y * dstStride + x;
        if (x + 4 <= W) {
            *(uint32_t *)d = o;
        } else {
            for (int i = 0; i < W - x; i++) d[i] = (uint8_t)(o >> (8 * i));
        }
        a = b;
        b = c;
    }
}

template <int OP>
__global__ void __launch_bounds__(kFBX * kFBY)
k_filter3x3(int W, int H, uint8_t *dst, int dstStride, const uint8_t *src, int srcStride)
{
    const int x = (blockIdx.x * kFBX + threadIdx.x) * 4;
    const int y0 = 1 + (blockIdx.y * kFBY + threadIdx.y) * kFRows;
    if (x >= W || y0 >= H - 1) return;
    const int y1 = min(y0 + kFRows, H - 1);
    Row3 a = row3(src + (size_t)(y0 - 1) * srcStride, x, srcStride);
    Row3 b = row3(src + (size_t)y0 * srcStride, x, srcStride);
    for (int y = y0; y < y1; y++) {
        const Row3 c = row3(src + (size_t)(y + 1) * srcStride, x, srcStride);
        uint32_t o;
        if (OP == F_DILATE) {
            o = __vmaxu4(__vmaxu4(__vmaxu4(a.l, a.c), __vmaxu4(a.r, b.l)),
                         __vmaxu4(__vmaxu4(b.c, b.r), __vmaxu4(__vmaxu4(c.l, c.c), c.r)));
        } else if (OP == F_ERODE) {
            o = __vminu4(__vminu4(__vminu4(a.l, a.c), __vminu4(a.r, b.l)),
                         __vminu4(__vminu4(b.c, b.r), __vminu4(__vminu4(c.l, c.c), c.r)));
        } else {
            // median of 9 = med3(max of the column minima, med3 of the column medians,
            // min of the column maxima) once each column is sorted
            uint32_t lL, mL, hL, lC, mC, hC, lR, mR, hR;
            sort3(a.l, b.l, c.l, lL, mL, hL);
            sort3(a.c, b.c, c.c, lC, mC, hC);
            sort3(a.r, b.r, c.r, lR, mR, hR);
            o = med3(__vmaxu4(__vmaxu4(lL, lC), lR), med3(mL, mC, mR), __vminu4(__vminu4(hL, hC), hR));
        }
        uint8_t *d = dst + (size_t)y * dstStride + x;
        if (x + 4 <= W) {
            *(uint32_t *)d = o;
        } else {
            for (int i = 0; i < W - x; i++) d[i] = (uint8_t)(o >> (8 * i));
        }
        a = b;
        b = c;
    }
}

template <int OP>
int filter_launch(void *stream, uint32_t W, uint32_t H, uint8_t *dst, uint32_t dstStride, const uint8_t *src,
                  uint32_t srcStride)
{
    auto ok = [&](const uint8_t *p, uint32_t s) { return p && ((uintptr_t)p & 3) == 0 && (s & 3) == 0 && s >= W; };
    if (W < 3 || H < 3 || !ok(dst, dstStride) || !ok(src, srcStride)) return AGOCUDA_INVALID_PARAMS;
    dim3 grd(div_up(W, kFBX * 4), div_up(H - 2, kFBY * kFRows));
    if (OP == F_BOX)
        k_box3x3<<<grd, dim3(kFBX, kFBY), 0, as_stream(stream)>>>((int)W, (int)H, dst, (int)dstStride, src, (int)srcStride);
    else
        k_filter3x3<OP><<<grd, dim3(kFBX, kFBY), 0, as_stream(stream)>>>((int)W, (int)H, dst, (int)dstStride, src, (int)srcStride);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

}  // namespace

// ---------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------
#define EW_BINARY(NAME, OP, TO, TA, TB)                                                                         \
    extern "C" int agocuda_##NAME(void *stream, uint32_t dstWidth, uint32_t dstHeight, TO *pDst, uint32_t dstStride, \
                                  const TA *pSrc1, uint32_t src1Stride, const TB *pSrc2, uint32_t src2Stride)     \
    {                                                                                                          \
        return ew_launch<OP>(stream, dstWidth, dstHeight, pDst, dstStride, pSrc1, src1Stride, pSrc2, src2Stride); \
    }

EW_BINARY(Add_U8_U8U8_Wrap, EW_ADD_WRAP_U8, uint8_t, uint8_t, uint8_t)
EW_BINARY(Add_U8_U8U8_Sat, EW_ADD_SAT_U8, uint8_t, uint8_t, uint8_t)
EW_BINARY(Sub_U8_U8U8_Wrap, EW_SUB_WRAP_U8, uint8_t, uint8_t, uint8_t)
EW_BINARY(Sub_U8_U8U8_Sat, EW_SUB_SAT_U8, uint8_t, uint8_t, uint8_t)
EW_BINARY(Add_S16_U8U8, EW_ADD_S16, int16_t, uint8_t, uint8_t)
EW_BINARY(Sub_S16_U8U8, EW_SUB_S16, int16_t, uint8_t, uint8_t)
EW_BINARY(Add_S16_S16U8_Wrap, EW_ADD_WRAP_S16, int16_t, int16_t, uint8_t)
EW_BINARY(Add_S16_S16U8_Sat, EW_ADD_SAT_S16, int16_t, int16_t, uint8_t)
EW_BINARY(Sub_S16_S16U8_Wrap, EW_SUB_WRAP_S16, int16_t, int16_t, uint8_t)
EW_BINARY(Sub_S16_S16U8_Sat, EW_SUB_SAT_S16, int16_t, int16_t, uint8_t)
EW_BINARY(Sub_S16_U8S16_Wrap, EW_SUB_WRAP_S16, int16_t, uint8_t, int16_t)
EW_BINARY(Sub_S16_U8S16_Sat, EW_SUB_SAT_S16, int16_t, uint8_t, int16_t)
EW_BINARY(Add_S16_S16S16_Wrap, EW_ADD_WRAP_S16, int16_t, int16_t, int16_t)
EW_BINARY(Add_S16_S16S16_Sat, EW_ADD_SAT_S16, int16_t, int16_t, int16_t)
EW_BINARY(Sub_S16_S16S16_Wrap, EW_SUB_WRAP_S16, int16_t, int16_t, int16_t)
EW_BINARY(Sub_S16_S16S16_Sat, EW_SUB_SAT_S16, int16_t, int16_t, int16_t)
EW_BINARY(AbsDiff_U8_U8U8, EW_ABSDIFF_U8, uint8_t, uint8_t, uint8_t)
EW_BINARY(AbsDiff_S16_S16S16_Sat, EW_ABSDIFF_SAT_S16, int16_t, int16_t, int16_t)
EW_BINARY(And_U8_U8U8, EW_AND, uint8_t, uint8_t, uint8_t)
EW_BINARY(Or_U8_U8U8, EW_OR, uint8_t, uint8_t, uint8_t)
EW_BINARY(Xor_U8_U8U8, EW_XOR, uint8_t, uint8_t, uint8_t)
#undef EW_BINARY

extern "C" int agocuda_Not_U8_U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                                 const uint8_t *pSrc, uint32_t srcStride)
{
    return ew_launch<EW_NOT>(stream, dstWidth, dstHeight, pDst, dstStride, pSrc, srcStride, (const uint8_t *)nullptr, 0);
}

extern "C" int agocuda_Threshold_U8_U8_Range(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                             uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride,
                                             int32_t thresholdLower, int32_t thresholdUpper)
{
    // the reference passes both bounds as vx_uint8 (HafCpu_Threshold_U8_U8_Range)
    return ew_launch<EW_RANGE>(stream, dstWidth, dstHeight, pDst, dstStride, pSrc, srcStride, (const uint8_t *)nullptr, 0,
                               (int)(uint8_t)thresholdLower, (int)(uint8_t)thresholdUpper);
}

#define FILTER(NAME, OP)                                                                                          \
    extern "C" int agocuda_##NAME(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride, \
                                  const uint8_t *pSrc, uint32_t srcStride)                                        \
    {                                                                                                          \
        return filter_launch<OP>(stream, dstWidth, dstHeight, pDst, dstStride, pSrc, srcStride);                \
    }
FILTER(Box_U8_U8_3x3, F_BOX)
FILTER(Dilate_U8_U8_3x3, F_DILATE)
FILTER(Erode_U8_U8_3x3, F_ERODE)
FILTER(Median_U8_U8_3x3, F_MEDIAN)
#undef FILTER

// ---------------------------------------------------------------------------------
// Fused U8 pixel chains: a sequence of element-wise and 3x3 neighbourhood kernels whose
// intermediates are private virtual images runs as one kernel; the intermediates live in
// shared memory.  This is the device-side counterpart of AGO's GPU "supernodes", which group
// element-wise (AGO_KERNEL_OP_TYPE_ELEMENT_WISE) and fixed-neighbourhood kernels
// (AGO_KERNEL_OP_TYPE_FIXED_NEIGHBORS, ago_internal.h:96-97) into one generated kernel
// (ago_drama_alloc.cpp:484).
//
// A block owns a 128x32 output tile.  It loads the input (and each side input of a binary
// op) over the tile plus 4 columns and K rows on every side, K = number of 3x3 stages, as
// 32-bit words into shared memory; each 3x3 stage shrinks the rows it produces by one on
// each side (the columns keep their 4-pixel margin, enough for K <= 4), element-wise
// stages update in place.  Pixels inside the chain's valid rectangle read only image
// pixels, so they equal the per-node kernels' results; pixels outside it are unspecified.
// ---------------------------------------------------------------------------------
namespace {

constexpr int kPxTW = 128, kPxTH = 32, kPxWords = (kPxTW + 8) / 4;   // 34 words: 4-column margins
constexpr int kPxMaxBH = kPxTH + 2 * AGOCUDA_PX_MAX_STENCILS;
constexpr int kPxThreads = 256, kPxGroups = kPxThreads / kPxWords;    // 7 row groups of 34 word columns

__device__ __forceinline__ bool px_stencil(int code)
{
    return code == AGOCUDA_PX_BOX3x3 || code == AGOCUDA_PX_MEDIAN3x3 || code == AGOCUDA_PX_DILATE3x3 ||
           code == AGOCUDA_PX_ERODE3x3 || code == AGOCUDA_PX_GAUSSIAN3x3;
}

__device__ __forceinline__ Row3 srow3(const uint32_t (*b)[kPxWords], int r, int w)
{
    const uint32_t L = b[r][w > 0 ? w - 1 : 0], C = b[r][w], R = b[r][w + 1 < kPxWords ? w + 1 : w];
    return Row3{__funnelshift_r(L, C, 24), C, __funnelshift_r(C, R, 8)};
}

// Gaussian 3x3 ([1 2 1]^T [1 2 1]) >> 4 (HafCpu_Gaussian_U8_U8_3x3, ago_haf_cpu_filter.cpp:1518)
__device__ __forceinline__ Sum3 gsum(const Row3 &r)
{
    return Sum3{__byte_perm(r.l, 0, 0x4240) + 2 * __byte_perm(r.c, 0, 0x4240) + __byte_perm(r.r, 0, 0x4240),
                __byte_perm(r.l, 0, 0x4341) + 2 * __byte_perm(r.c, 0, 0x4341) + __byte_perm(r.r, 0, 0x4341)};
}

__device__ __forceinline__ uint32_t gauss_word(const Row3 &a, const Row3 &b, const Row3 &c)
{
    const Sum3 A = gsum(a), B = gsum(b), C = gsum(c);
    const uint32_t e = ((A.E + 2 * B.E + C.E) >> 4) & 0x00ff00ffu, o = ((A.O + 2 * B.O + C.O) >> 4) & 0x00ff00ffu;
    return e | (o << 8);
}

__device__ __forceinline__ uint32_t stencil_word(int code, const Row3 &a, const Row3 &b, const Row3 &c)
{
    switch (code) {
    case AGOCUDA_PX_BOX3x3: return box_word(sum3(a), sum3(b), sum3(c));
    case AGOCUDA_PX_GAUSSIAN3x3: return gauss_word(a, b, c);
    case AGOCUDA_PX_DILATE3x3:
        return __vmaxu4(__vmaxu4(__vmaxu4(a.l, a.c), __vmaxu4(a.r, b.l)),
                        __vmaxu4(__vmaxu4(b.c, b.r), __vmaxu4(__vmaxu4(c.l, c.c), c.r)));
    case AGOCUDA_PX_ERODE3x3:
        return __vminu4(__vminu4(__vminu4(a.l, a.c), __vminu4(a.r, b.l)),
                        __vminu4(__vminu4(b.c, b.r), __vminu4(__vminu4(c.l, c.c), c.r)));
    default: {   // median
        uint32_t lL, mL, hL, lC, mC, hC, lR, mR, hR;
        sort3(a.l, b.l, c.l, lL, mL, hL);
        sort3(a.c, b.c, c.c, lC, mC, hC);
        sort3(a.r, b.r, c.r, lR, mR, hR);
        return med3(__vmaxu4(__vmaxu4(lL, lC), lR), med3(mL, mC, mR), __vminu4(__vminu4(hL, hC), hR));
    }
    }
}

// element-wise op on 4 pixels: v = the chain's value, o = the side operand
__device__ __forceinline__ uint32_t ew_word(const agocuda_pixel_op &op, uint32_t v, uint32_t o)
{
    const uint32_t a = op.sideFirst ? o : v, b = op.sideFirst ? v : o;
    switch (op.code) {
    case AGOCUDA_PX_NOT: return ~v;
    case AGOCUDA_PX_AND: return v & o;
    case AGOCUDA_PX_OR: return v | o;
    case AGOCUDA_PX_XOR: return v ^ o;
    case AGOCUDA_PX_ABSDIFF: return __vabsdiffu4(v, o);
    case AGOCUDA_PX_ADD_WRAP: return __vadd4(v, o);
    case AGOCUDA_PX_ADD_SAT: return __vaddus4(v, o);
    case AGOCUDA_PX_SUB_WRAP: return __vsub4(a, b);
    case AGOCUDA_PX_SUB_SAT: return __vsubus4(a, b);
    case AGOCUDA_PX_THRESHOLD_BINARY: return __vcmpgtu4(v, (uint32_t)(op.p0 & 0xff) * 0x01010101u);
    case AGOCUDA_PX_THRESHOLD_RANGE:
        return ~(__vcmpgtu4(v, (uint32_t)(op.p1 & 0xff) * 0x01010101u) | __vcmpltu4(v, (uint32_t)(op.p0 & 0xff) * 0x01010101u));
    }
    return v;
}

__global__ void __launch_bounds__(kPxThreads)
k_pixel_chain(const agocuda_pixel_program prog, const agocuda_pixel_frame *__restrict__ frames, int K, int nSides)
{
    __shared__ uint32_t buf[2][kPxMaxBH][kPxWords];
    __shared__ uint32_t side[AGOCUDA_PX_MAX_SIDES][kPxMaxBH][kPxWords];
    const agocuda_pixel_frame f = frames[blockIdx.z];
    const int W = (int)f.width, H = (int)f.height;
    const int x0 = blockIdx.x * kPxTW, y0 = blockIdx.y * kPxTH, tid = threadIdx.x;
    if (x0 >= W || y0 >= H) return;
    const int BH = kPxTH + 2 * K;
    for (int i = tid; i < BH * kPxWords; i += kPxThreads) {
        const int r = i / kPxWords, w = i - r * kPxWords;
        const int y = clampi(y0 - K + r, 0, H - 1), x = x0 - 4 + 4 * w;
        buf[0][r][w] = load_word_clamped(f.src + (size_t)y * f.srcStride, x, (int)f.srcStride);
        for (int s = 0; s < nSides; s++)
            side[s][r][w] = load_word_clamped(f.side[s] + (size_t)y * f.sideStride[s], x, (int)f.sideStride[s]);
    }
    __syncthreads();
    int cur = 0, st = 0;
    for (int k = 0; k < prog.numOps; k++) {
        const agocuda_pixel_op op = prog.ops[k];
        if (px_stencil(op.code)) {
            st++;
            // rows [st, BH - st) from rows [st - 1, BH - st + 1): a word column per thread,
            // its rows split over the row groups, the three rows of the window in registers
            const int rows = BH - 2 * st, per = (rows + kPxGroups - 1) / kPxGroups;
            const int w = tid % kPxWords, grp = tid / kPxWords;
            const int r0 = st + grp * per, r1 = min(r0 + per, BH - st);
            if (grp < kPxGroups && r0 < r1) {
                Row3 a = srow3(buf[cur], r0 - 1, w), b = srow3(buf[cur], r0, w);
                for (int r = r0; r < r1; r++) {
                    const Row3 c = srow3(buf[cur], r + 1, w);
                    buf[cur ^ 1][r][w] = stencil_word(op.code, a, b, c);
                    a = b;
                    b = c;
                }
            }
            cur ^= 1;
        } else {
            const int rows = BH - 2 * st;
            for (int i = tid; i < rows * kPxWords; i += kPxThreads) {
                const int r = st + i / kPxWords, w = i % kPxWords;
                const uint32_t o = op.side >= 0 ? side[op.side][r][w] : 0u;
                buf[cur][r][w] = ew_word(op, buf[cur][r][w], o);
            }
        }
        __syncthreads();
    }
    // tile rows [K, K + 32) of the buffer, words 1..32 (columns x0 .. x0 + 127)
    for (int i = tid; i < kPxTH * (kPxTW / 4); i += kPxThreads) {
        const int r = i / (kPxTW / 4), w = i % (kPxTW / 4);
        const int y = y0 + r, x = x0 + 4 * w;
        if (y >= H || x >= W) continue;
        const uint32_t v = buf[cur][K + r][w + 1];
        uint8_t *d = f.dst + (size_t)y * f.dstStride + x;
        if (x + 4 <= W) {
            *(uint32_t *)d = v;
        } else {
            for (int j = 0; j < W - x; j++) d[j] = (uint8_t)(v >> (8 * j));
        }
    }
}

}  // namespace

extern "C" int agocuda_fused_PixelChain_U8(void *stream, const agocuda_pixel_program *program,
                                           const agocuda_pixel_frame *frames, uint32_t numFrames, uint32_t maxWidth,
                                           uint32_t maxHeight)
{
    if (!program || !frames || !numFrames || numFrames > 65535 || !maxWidth || !maxHeight || program->numOps < 1 ||
        program->numOps > AGOCUDA_PX_MAX_OPS)
        return AGOCUDA_INVALID_PARAMS;
    int K = 0, nSides = 0;
    for (int k = 0; k < program->numOps; k++) {
        const agocuda_pixel_op &op = program->ops[k];
        if (op.code < AGOCUDA_PX_NOT || op.code > AGOCUDA_PX_GAUSSIAN3x3) return AGOCUDA_INVALID_PARAMS;
        const bool stencil = op.code >= AGOCUDA_PX_BOX3x3;
        const bool binary = op.code >= AGOCUDA_PX_AND && op.code <= AGOCUDA_PX_SUB_SAT;
        if (stencil) K++;
        if (binary) {
            if (op.side < 0 || op.side >= AGOCUDA_PX_MAX_SIDES) return AGOCUDA_INVALID_PARAMS;
            nSides = op.side + 1 > nSides ? op.side + 1 : nSides;
        } else if (op.side >= AGOCUDA_PX_MAX_SIDES) {
            return AGOCUDA_INVALID_PARAMS;
        }
    }
    if (K > AGOCUDA_PX_MAX_STENCILS) return AGOCUDA_INVALID_PARAMS;
    agocuda_pixel_program p = *program;
    for (int k = 0; k < p.numOps; k++) {   // unary ops read no side operand
        const int c = p.ops[k].code;
        if (!(c >= AGOCUDA_PX_AND && c <= AGOCUDA_PX_SUB_SAT)) p.ops[k].side = -1;
    }
    dim3 grd(div_up(maxWidth, kPxTW), div_up(maxHeight, kPxTH), numFrames);
    k_pixel_chain<<<grd, kPxThreads, 0, as_stream(stream)>>>(p, frames, K, nSides);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}
