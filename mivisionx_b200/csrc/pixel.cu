// pixel.cu -- the AGO kernels on either side of the vision graphs, for sm_100a:
// element-wise arithmetic / logical / range-threshold kernels and the 3x3 Box, Median,
// Dilate and Erode filters.
//
// Element-wise kernels are HBM-bound: a thread owns 16 pixels of a row (16-byte vectors),
// a warp 512 contiguous pixels, and rows are spread over blockIdx.y.
// The 3x3 filters give a thread 8 pixels of a row and walk it down the rows with the window's
// rows in registers, two pixels per 32-bit register: 16-bit integer lanes for Box and
// Gaussian, and for Dilate, Erode and Median half-float lanes holding 1024 + v, which
// f16x2 min / max order exactly like the bytes.
#include "agocuda_internal.cuh"

#include <mutex>

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
    EW_BINARY,                                   // 255 above the threshold, else 0
    EW_DEPTH_DOWN_WRAP,                          // S16 -> U8: low byte of v >> shift
    EW_DEPTH_UP,                                 // U8 -> S16: v << shift in 16 bits
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
    case EW_BINARY: return a > p0 ? 255 : 0;                           // :3660
    case EW_DEPTH_DOWN_WRAP: return (a >> p0) & 0xff;                  // :3488
    case EW_DEPTH_UP: return (int)(int16_t)(a << p0);                  // :3604
    }
    return 0;
}

constexpr int kEwPx = 16;                        // pixels per thread: 16 B of a U8 plane, 32 B of S16

template <typename T>
__device__ __forceinline__ void load16(const T *p, int *v)
{
#pragma unroll
    for (int h = 0; h < (int)sizeof(T); h++) {
        const uint4 w = __ldg((const uint4 *)p + h);
        const T *e = (const T *)&w;
#pragma unroll
        for (int i = 0; i < 16 / (int)sizeof(T); i++) v[h * (16 / sizeof(T)) + i] = (int)e[i];
    }
}

template <typename T>
__device__ __forceinline__ void store16(T *p, const int *v)
{
#pragma unroll
    for (int h = 0; h < (int)sizeof(T); h++) {
        uint4 w;
        T *e = (T *)&w;
#pragma unroll
        for (int i = 0; i < 16 / (int)sizeof(T); i++) e[i] = (T)v[h * (16 / sizeof(T)) + i];
        *((uint4 *)p + h) = w;
    }
}

constexpr int kEwBX = 32, kEwBY = 8;

// one thread: pixels [x, x+16) of row y; the last group of a row that W cuts goes pixel by pixel
template <int OP, typename TO, typename TA, typename TB>
__global__ void __launch_bounds__(kEwBX * kEwBY)
k_elementwise(int W, int H, TO *dst, int dstStride, const TA *a, int aStride, const TB *b, int bStride, int p0, int p1)
{
    const int x = (blockIdx.x * kEwBX + threadIdx.x) * kEwPx;
    const int y = blockIdx.y * kEwBY + threadIdx.y;
    if (x >= W || y >= H) return;
    TO *d = (TO *)((uint8_t *)dst + (size_t)y * dstStride) + x;
    const TA *pa = (const TA *)((const uint8_t *)a + (size_t)y * aStride) + x;
    const TB *pb = b ? (const TB *)((const uint8_t *)b + (size_t)y * bStride) + x : nullptr;
    if (x + kEwPx <= W) {
        int va[kEwPx], vb[kEwPx], r[kEwPx];
        load16(pa, va);
        if (pb) load16(pb, vb);
#pragma unroll
        for (int i = 0; i < kEwPx; i++) r[i] = ew_apply<OP>(va[i], pb ? vb[i] : 0, p0, p1);
        store16(d, r);
    } else {
        for (int i = 0; i < W - x; i++) d[i] = (TO)ew_apply<OP>((int)pa[i], pb ? (int)pb[i] : 0, p0, p1);
    }
}

template <typename T> bool ew_plane_ok(const T *p, uint32_t stride, uint32_t W)
{
    return p && ((uintptr_t)p % 16) == 0 && (stride % 16) == 0 && stride >= W * sizeof(T);
}

template <int OP, typename TO, typename TA, typename TB>
int ew_launch(void *stream, uint32_t W, uint32_t H, TO *dst, uint32_t dstStride, const TA *a, uint32_t aStride,
              const TB *b, uint32_t bStride, int p0 = 0, int p1 = 0)
{
    const bool unary = OP == EW_NOT || OP == EW_RANGE || OP == EW_BINARY || OP == EW_DEPTH_DOWN_WRAP || OP == EW_DEPTH_UP;
    if (!W || !H || !ew_plane_ok(dst, dstStride, W) || !ew_plane_ok(a, aStride, W) ||
        (!unary && !ew_plane_ok(b, bStride, W)))
        return AGOCUDA_INVALID_PARAMS;
    dim3 grd(div_up(W, kEwBX * kEwPx), div_up(H, kEwBY));
    k_elementwise<OP, TO, TA, TB><<<grd, dim3(kEwBX, kEwBY), 0, as_stream(stream)>>>(
        (int)W, (int)H, dst, (int)dstStride, a, (int)aStride, unary ? nullptr : b, (int)bStride, p0, p1);
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

extern "C" int agocuda_Threshold_U8_U8_Binary(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                              uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride, int32_t threshold)
{
    // the reference passes the threshold as vx_uint8 (threshold_value.U1, ago_kernel_api.cpp:3442)
    return ew_launch<EW_BINARY>(stream, dstWidth, dstHeight, pDst, dstStride, pSrc, srcStride, (const uint8_t *)nullptr, 0,
                                (int)(uint8_t)threshold);
}

extern "C" int agocuda_ColorDepth_U8_S16_Wrap(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                              uint32_t dstStride, const int16_t *pSrc, uint32_t srcStride, int32_t shift)
{
    if (shift < 0 || shift > 15) return AGOCUDA_INVALID_PARAMS;
    return ew_launch<EW_DEPTH_DOWN_WRAP>(stream, dstWidth, dstHeight, pDst, dstStride, pSrc, srcStride,
                                         (const uint8_t *)nullptr, 0, shift);
}

extern "C" int agocuda_ColorDepth_S16_U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst,
                                         uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride, int32_t shift)
{
    if (shift < 0 || shift > 15) return AGOCUDA_INVALID_PARAMS;
    return ew_launch<EW_DEPTH_UP>(stream, dstWidth, dstHeight, pDst, dstStride, pSrc, srcStride, (const uint8_t *)nullptr,
                                  0, shift);
}

extern "C" int agocuda_Threshold_U8_U8_Range(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                             uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride,
                                             int32_t thresholdLower, int32_t thresholdUpper)
{
    // the reference passes both bounds as vx_uint8 (HafCpu_Threshold_U8_U8_Range)
    return ew_launch<EW_RANGE>(stream, dstWidth, dstHeight, pDst, dstStride, pSrc, srcStride, (const uint8_t *)nullptr, 0,
                               (int)(uint8_t)thresholdLower, (int)(uint8_t)thresholdUpper);
}


// ---------------------------------------------------------------------------------
// Fused U8 pixel chains: a sequence of element-wise and 3x3 neighbourhood kernels whose
// intermediates are private virtual images runs as one kernel; the intermediates live in
// shared memory.  This is the device-side counterpart of AGO's GPU "supernodes", which group
// element-wise (AGO_KERNEL_OP_TYPE_ELEMENT_WISE) and fixed-neighbourhood kernels
// (AGO_KERNEL_OP_TYPE_FIXED_NEIGHBORS, ago_internal.h:96-97) into one generated kernel
// (ago_drama_alloc.cpp:484).
//
// A block owns a 128x64 output tile.  It copies the input (and each side input of a binary
// op) over the tile plus 16 columns and K rows on every side, K = number of 3x3 stages, into
// shared memory: with one TMA tensor copy per plane (cp.async.bulk.tensor.2d, box 160 x
// (64 + 2K) bytes, completion counted on an mbarrier; rows and columns outside the image come
// back as zeros), or in the other form with 16-byte cp.async copies; each 3x3 stage shrinks
// the rows it produces by one on each side (the columns keep a margin of at least 4, enough
// for K <= 4) and runs on 16-bit lanes of 8 pixels per thread; element-wise stages update in
// place.  Pixels inside the chain's valid rectangle read only image pixels, so they equal
// the per-node kernels' results; pixels outside it are unspecified.
// ---------------------------------------------------------------------------------
namespace {

constexpr int kPxTW = 128, kPxTH = 64;                  // output tile
constexpr int kPxWords = (kPxTW + 32) / 4;              // 40 words per buffer row: columns x0-16 .. x0+143
constexpr int kPxChunks = kPxWords / 4;                 // 16-byte chunks per row
constexpr int kPxPairs = 18;                            // 3x3 stages compute words 2..37 (columns x0-8 .. x0+135),
constexpr int kPxThreads = 256, kPxGroups = kPxThreads / kPxPairs;   // 8 pixels per thread; 14 row groups

// 16-bit lane pairs of the 10 columns x-1 .. x+8 around words C0 (x..x+3) and C1 (x+4..x+7):
// e0 = (x, x+2), o0 = (x+1, x+3), e1 = (x+4, x+6), o1 = (x+5, x+7), b = (x-1, x+8).  The high
// byte of every lane is `hi`: 0 for integer sums, 0x64 for min / max as half floats (the half
// with bits 0x64vv is 1024 + vv, exact and ordered like vv).
struct Lanes8 { uint32_t e0, o0, e1, o1, b; };
__device__ __forceinline__ Lanes8 lanes8(uint32_t L, uint32_t C0, uint32_t C1, uint32_t R, uint32_t hi)
{
    Lanes8 v;
    v.e0 = __byte_perm(C0, hi, 0x4240);
    v.o0 = __byte_perm(C0, hi, 0x4341);
    v.e1 = __byte_perm(C1, hi, 0x4240);
    v.o1 = __byte_perm(C1, hi, 0x4341);
    v.b = __byte_perm(__byte_perm(L, R, 0x0043), hi, 0x4140);
    return v;
}

// the neighbour lane pairs of the four outputs: left of e0 = (x-1, x+1), right of o0 =
// (x+2, x+4), left of e1 = (x+3, x+5), right of o1 = (x+6, x+8)
__device__ __forceinline__ uint32_t lft_e0(const Lanes8 &v) { return __byte_perm(v.b, v.o0, 0x5410); }
__device__ __forceinline__ uint32_t rgt_o0(const Lanes8 &v) { return __byte_perm(v.e0, v.e1, 0x5432); }
__device__ __forceinline__ uint32_t lft_e1(const Lanes8 &v) { return __byte_perm(v.o0, v.o1, 0x5432); }
__device__ __forceinline__ uint32_t rgt_o1(const Lanes8 &v) { return __byte_perm(v.e1, v.b, 0x7632); }

// low bytes of the four output lane pairs -> words x..x+3, x+4..x+7
__device__ __forceinline__ uint2 pack8(uint32_t e0, uint32_t o0, uint32_t e1, uint32_t o1)
{
    return make_uint2(__byte_perm(e0, o0, 0x6240), __byte_perm(e1, o1, 0x6240));
}

// lane-wise max / min of two f16x2 registers (no NaNs occur: every lane is 1024 + a byte)
__device__ __forceinline__ uint32_t hmx(uint32_t a, uint32_t b)
{
    uint32_t d;
    asm("max.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t hmn(uint32_t a, uint32_t b)
{
    uint32_t d;
    asm("min.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t hmed3(uint32_t a, uint32_t b, uint32_t c) { return hmx(hmn(a, b), hmn(hmx(a, b), c)); }

// Row sources / sinks of the 3x3 stages: 8 pixels (word pair p) of a shared-memory tile
// row, or of an image row in global memory
struct SmemRows {
    const uint32_t *buf;
    int p;
    __device__ __forceinline__ Lanes8 row(int r, uint32_t hi) const
    {
        const uint32_t *w = buf + r * kPxWords + 2 * p;   // words 2 .. 37: the neighbour words exist
        return lanes8(w[-1], w[0], w[1], w[2], hi);
    }
};
struct SmemOut {
    uint32_t *buf;
    int p;
    __device__ __forceinline__ void put(int r, uint2 v) const { *reinterpret_cast<uint2 *>(buf + r * kPxWords + 2 * p) = v; }
};
struct GlobalRows {
    const uint8_t *src;
    int stride, x;
    __device__ __forceinline__ Lanes8 row(int r, uint32_t hi) const
    {
        const uint8_t *q = src + (size_t)r * stride;
        return lanes8(load_word_clamped(q, x - 4, stride), load_word_clamped(q, x, stride),
                      load_word_clamped(q, x + 4, stride), load_word_clamped(q, x + 8, stride), hi);
    }
};
struct GlobalOut {
    uint8_t *dst;
    int stride, x, W;
    __device__ __forceinline__ void put(int r, uint2 v) const
    {
        uint8_t *d = dst + (size_t)r * stride + x;
        if (x + 8 <= W) {
            *reinterpret_cast<uint32_t *>(d) = v.x;
            *reinterpret_cast<uint32_t *>(d + 4) = v.y;
        } else {
            for (int j = 0; j < W - x; j++) d[j] = (uint8_t)((j < 4 ? v.x : v.y) >> (8 * (j & 3)));
        }
    }
};

// Dilate (max) / Erode (min) over rows [r0, r1): column extreme of three rows, then across
template <bool MAX, class In, class Out>
__device__ __forceinline__ void stage_minmax(const In &in, const Out &out, int r0, int r1)
{
    auto f = [](uint32_t a, uint32_t b) { return MAX ? hmx(a, b) : hmn(a, b); };
    const uint32_t hi = 0x64646464u;
    Lanes8 a = in.row(r0 - 1, hi), b = in.row(r0, hi);
    Lanes8 pr{f(a.e0, b.e0), f(a.o0, b.o0), f(a.e1, b.e1), f(a.o1, b.o1), f(a.b, b.b)};   // rows r-1, r
    for (int r = r0; r < r1; r++) {
        const Lanes8 c = in.row(r + 1, hi);
        const Lanes8 v{f(pr.e0, c.e0), f(pr.o0, c.o0), f(pr.e1, c.e1), f(pr.o1, c.o1), f(pr.b, c.b)};
        out.put(r, pack8(f(f(lft_e0(v), v.e0), v.o0), f(f(v.e0, v.o0), rgt_o0(v)),
                                f(f(lft_e1(v), v.e1), v.o1), f(f(v.e1, v.o1), rgt_o1(v))));
        pr = Lanes8{f(b.e0, c.e0), f(b.o0, c.o0), f(b.e1, c.e1), f(b.o1, c.o1), f(b.b, c.b)};
        b = c;
    }
}

// Median: sort each column of the three rows, then med3(max of minima, med3 of medians,
// min of maxima) over the three columns of each output
template <class In, class Out>
__device__ __forceinline__ void stage_median(const In &in, const Out &out, int r0, int r1)
{
    const uint32_t hi = 0x64646464u;
    Lanes8 a = in.row(r0 - 1, hi), b = in.row(r0, hi);
    for (int r = r0; r < r1; r++) {
        const Lanes8 c = in.row(r + 1, hi);
        Lanes8 lo, md, hg;
        auto sort = [](uint32_t x, uint32_t y, uint32_t z, uint32_t &l, uint32_t &m, uint32_t &h) {
            const uint32_t l1 = hmn(x, y), h1 = hmx(x, y), t = hmx(l1, z);
            l = hmn(l1, z);
            m = hmn(h1, t);
            h = hmx(h1, t);
        };
        sort(a.e0, b.e0, c.e0, lo.e0, md.e0, hg.e0);
        sort(a.o0, b.o0, c.o0, lo.o0, md.o0, hg.o0);
        sort(a.e1, b.e1, c.e1, lo.e1, md.e1, hg.e1);
        sort(a.o1, b.o1, c.o1, lo.o1, md.o1, hg.o1);
        sort(a.b, b.b, c.b, lo.b, md.b, hg.b);
        auto med9 = [&](uint32_t l0, uint32_t l1, uint32_t l2, uint32_t m0, uint32_t m1, uint32_t m2, uint32_t h0,
                        uint32_t h1, uint32_t h2) {
            return hmed3(hmx(hmx(l0, l1), l2), hmed3(m0, m1, m2), hmn(hmn(h0, h1), h2));
        };
        const uint32_t oe0 = med9(lft_e0(lo), lo.e0, lo.o0, lft_e0(md), md.e0, md.o0, lft_e0(hg), hg.e0, hg.o0);
        const uint32_t oo0 = med9(lo.e0, lo.o0, rgt_o0(lo), md.e0, md.o0, rgt_o0(md), hg.e0, hg.o0, rgt_o0(hg));
        const uint32_t oe1 = med9(lft_e1(lo), lo.e1, lo.o1, lft_e1(md), md.e1, md.o1, lft_e1(hg), hg.e1, hg.o1);
        const uint32_t oo1 = med9(lo.e1, lo.o1, rgt_o1(lo), md.e1, md.o1, rgt_o1(md), hg.e1, hg.o1, rgt_o1(hg));
        out.put(r, pack8(oe0, oo0, oe1, oo1));
        a = b;
        b = c;
    }
}

// Box and Gaussian ([1 2 1]^T [1 2 1] >> 4) in integer lanes: row sums of three columns,
// rolled down the rows.  Box is floor(sum / 9): the reference's SIMD body computes
// (sum * 7282) >> 16 and its scalar parts (int)((float)sum / 9.0f) (HafCpu_Box_U8_U8_3x3,
// ago_haf_cpu_filter.cpp:34); both equal floor(sum / 9) for every sum of nine bytes (<= 2295),
// and so does (sum * 7282) >> 16 here.
template <bool GAUSS, class In, class Out>
__device__ __forceinline__ void stage_linear(const In &in, const Out &out, int r0, int r1)
{
    auto hsum = [](const Lanes8 &v) {
        const uint32_t k = GAUSS ? 2u : 1u;
        return Lanes8{lft_e0(v) + k * v.e0 + v.o0, v.e0 + k * v.o0 + rgt_o0(v), lft_e1(v) + k * v.e1 + v.o1,
                      v.e1 + k * v.o1 + rgt_o1(v), 0u};
    };
    Lanes8 ha = hsum(in.row(r0 - 1, 0u)), hb = hsum(in.row(r0, 0u));
    for (int r = r0; r < r1; r++) {
        const Lanes8 hc = hsum(in.row(r + 1, 0u));
        uint32_t q[4];
        const uint32_t s[4] = {ha.e0 + (GAUSS ? 2u : 1u) * hb.e0 + hc.e0, ha.o0 + (GAUSS ? 2u : 1u) * hb.o0 + hc.o0,
                               ha.e1 + (GAUSS ? 2u : 1u) * hb.e1 + hc.e1, ha.o1 + (GAUSS ? 2u : 1u) * hb.o1 + hc.o1};
#pragma unroll
        for (int i = 0; i < 4; i++)
            q[i] = GAUSS ? (s[i] >> 4) & 0x00ff00ffu
                         : ((((s[i] & 0xffffu) * 7282u) >> 16) | ((((s[i] >> 16) * 7282u) >> 16) << 16));
        out.put(r, pack8(q[0], q[1], q[2], q[3]));
        ha = hb;
        hb = hc;
    }
}

// element-wise op on 4 pixels: v = the chain's value, o = the side operand
__device__ __forceinline__ uint32_t ew_word(int code, int sideFirst, int p0, int p1, uint32_t v, uint32_t o)
{
    const uint32_t a = sideFirst ? o : v, b = sideFirst ? v : o;
    switch (code) {
    case AGOCUDA_PX_NOT: return ~v;
    case AGOCUDA_PX_AND: return v & o;
    case AGOCUDA_PX_OR: return v | o;
    case AGOCUDA_PX_XOR: return v ^ o;
    case AGOCUDA_PX_ABSDIFF: return __vabsdiffu4(v, o);
    case AGOCUDA_PX_ADD_WRAP: return __vadd4(v, o);
    case AGOCUDA_PX_ADD_SAT: return __vaddus4(v, o);
    case AGOCUDA_PX_SUB_WRAP: return __vsub4(a, b);
    case AGOCUDA_PX_SUB_SAT: return __vsubus4(a, b);
    case AGOCUDA_PX_THRESHOLD_BINARY: return __vcmpgtu4(v, (uint32_t)(p0 & 0xff) * 0x01010101u);
    case AGOCUDA_PX_THRESHOLD_RANGE:
        return ~(__vcmpgtu4(v, (uint32_t)(p1 & 0xff) * 0x01010101u) | __vcmpltu4(v, (uint32_t)(p0 & 0xff) * 0x01010101u));
    }
    return v;
}

constexpr int kPxMapsPerFrame = 1 + AGOCUDA_PX_MAX_SIDES;   // tensor maps: source, then the side planes
constexpr int kTmaWaitLimit = 1 << 20;                       // bounded mbarrier waits

// words of one shared-memory plane; TMA destinations start on 128-byte boundaries
__host__ __device__ constexpr int px_plane_words(int BH, bool tma)
{
    return tma ? ((BH * kPxWords + 31) & ~31) : BH * kPxWords;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return smem_addr_u32(p); }
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) { return mbarrier_try_wait_parity(bar, parity); }

// dynamic shared memory: two buffers of BH x 40 words, then one per side input
template <bool TMA>
__global__ void __launch_bounds__(kPxThreads)
k_pixel_chain(const agocuda_pixel_program prog, const agocuda_pixel_frame *__restrict__ frames,
              const CUtensorMap *__restrict__ maps, int K, int nSides, uint32_t *status)
{
    extern __shared__ __align__(128) uint32_t smem[];
    __shared__ int4 sop[AGOCUDA_PX_MAX_OPS];            // code, side, sideFirst, p0 | p1 << 16
    __shared__ __align__(8) uint64_t bar;
    const agocuda_pixel_frame f = frames[blockIdx.z];
    const int W = (int)f.width, H = (int)f.height;
    const int x0 = blockIdx.x * kPxTW, y0 = blockIdx.y * kPxTH, tid = threadIdx.x;
    if (x0 >= W || y0 >= H) return;
    const int BH = kPxTH + 2 * K, plane = px_plane_words(BH, TMA);
    uint32_t *const buf0 = smem, *const buf1 = smem + plane;
    uint32_t *const side = smem + 2 * plane;
    if (tid < prog.numOps) {
        const agocuda_pixel_op &o = prog.ops[tid];
        sop[tid] = make_int4(o.code, o.side, o.sideFirst, (o.p0 & 0xffff) | (o.p1 << 16));
    }
    if constexpr (TMA) {
        // one thread arms the barrier with the bytes of every plane and issues one tensor copy
        // per plane, its box at columns x0-16 .. x0+143 and rows y0-K .. y0+63+K of this
        // frame's plane (each plane has its own map); the block waits on the barrier
        const uint32_t b = smem_u32(&bar);
        if (tid == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        if (tid == 0) {
            const uint32_t bytes = (uint32_t)((1 + nSides) * BH * kPxWords * 4);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
            const CUtensorMap *m = maps + (size_t)blockIdx.z * kPxMapsPerFrame;
            for (int s = -1; s < nSides; s++) {
                const uint32_t d = smem_u32(s < 0 ? buf0 : side + s * plane);
                asm volatile(
                    "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                    ::"r"(d), "l"((uint64_t)(m + 1 + s)), "r"(x0 - 16), "r"(y0 - K), "r"(b) : "memory");
            }
        }
        bool done = false;
        for (int i = 0; i < kTmaWaitLimit && !done; i++) done = mbar_try_wait(b, 0);
        if (!done) {
            // the copies did not complete: report it, give them one more bounded wait, leave
            if (tid == 0) atomicOr(status, AGOCUDA_PX_STATUS_TMA_TIMEOUT);
            for (int i = 0; i < kTmaWaitLimit && !done; i++) done = mbar_try_wait(b, 0);
            return;
        }
    } else {
        // every 16-byte chunk of every plane in flight at once (cp.async, global -> shared); a
        // chunk outside the row is read from inside it instead (its columns are outside the image)
        for (int s = -1; s < nSides; s++) {
            const agocuda_pixel_frame *fp = frames + blockIdx.z;   // side[s]: indexed in global memory
            const uint8_t *base = s < 0 ? f.src : fp->side[s];
            const int stride = (int)(s < 0 ? f.srcStride : fp->sideStride[s]);
            uint32_t *dst = s < 0 ? buf0 : side + s * plane;
            for (int i = tid; i < BH * kPxChunks; i += kPxThreads) {
                const int r = i / kPxChunks, c = i - r * kPxChunks;
                const int y = clampi(y0 - K + r, 0, H - 1), x = clampi(x0 - 16 + 16 * c, 0, stride - 16);
                const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst + r * kPxWords + 4 * c);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(base + (size_t)y * stride + x) : "memory");
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    }
    __syncthreads();
    int cur = 0, st = 0;
    const int pp = 1 + tid % kPxPairs, grp = tid / kPxPairs;
    for (int k = 0; k < prog.numOps; k++) {
        const int4 op = sop[k];
        const int code = op.x;
        if (code >= AGOCUDA_PX_BOX3x3) {
            st++;
            // rows [st, BH - st) from rows [st - 1, BH - st + 1): 8 pixels of a row per thread,
            // the rows split over the row groups
            const int rows = BH - 2 * st, per = (rows + kPxGroups - 1) / kPxGroups;
            const int r0 = st + grp * per, r1 = min(r0 + per, BH - st);
            if (grp < kPxGroups && r0 < r1) {
                const SmemRows in{cur ? buf1 : buf0, pp};
                const SmemOut out{cur ? buf0 : buf1, pp};
                switch (code) {
                case AGOCUDA_PX_DILATE3x3: stage_minmax<true>(in, out, r0, r1); break;
                case AGOCUDA_PX_ERODE3x3: stage_minmax<false>(in, out, r0, r1); break;
                case AGOCUDA_PX_MEDIAN3x3: stage_median(in, out, r0, r1); break;
                case AGOCUDA_PX_GAUSSIAN3x3: stage_linear<true>(in, out, r0, r1); break;
                default: stage_linear<false>(in, out, r0, r1); break;
                }
            }
            cur ^= 1;
        } else {
            const int sd = op.y, sf = op.z, p0 = op.w & 0xffff, p1 = op.w >> 16;
            const int rows = BH - 2 * st;
            uint32_t *b = (cur ? buf1 : buf0) + st * kPxWords;
            const uint32_t *o = sd >= 0 ? side + sd * plane + st * kPxWords : nullptr;
            for (int i = tid; i < rows * kPxWords; i += kPxThreads) b[i] = ew_word(code, sf, p0, p1, b[i], o ? o[i] : 0u);
        }
        __syncthreads();
    }
    // tile rows [K, K + 64) of the buffer, words 4..35 (columns x0 .. x0 + 127)
    const uint32_t *res = cur ? buf1 : buf0;
    for (int i = tid; i < kPxTH * (kPxTW / 4); i += kPxThreads) {
        const int r = i / (kPxTW / 4), w = i % (kPxTW / 4);
        const int y = y0 + r, x = x0 + 4 * w;
        if (y >= H || x >= W) continue;
        const uint32_t v = res[(K + r) * kPxWords + w + 4];
        uint8_t *d = f.dst + (size_t)y * f.dstStride + x;
        if (x + 4 <= W) {
            *(uint32_t *)d = v;
        } else {
            for (int j = 0; j < W - x; j++) d[j] = (uint8_t)(v >> (8 * j));
        }
    }
}

// stencil count and side-plane count of a program; false when it is not a valid chain
static bool chain_shape(const agocuda_pixel_program *program, int &K, int &nSides)
{
    K = 0;
    nSides = 0;
    if (!program || program->numOps < 1 || program->numOps > AGOCUDA_PX_MAX_OPS) return false;
    for (int k = 0; k < program->numOps; k++) {
        const agocuda_pixel_op &op = program->ops[k];
        if (op.code < AGOCUDA_PX_NOT || op.code > AGOCUDA_PX_GAUSSIAN3x3) return false;
        const bool stencil = op.code >= AGOCUDA_PX_BOX3x3;
        const bool binary = op.code >= AGOCUDA_PX_AND && op.code <= AGOCUDA_PX_SUB_SAT;
        if (stencil) K++;
        if (binary) {
            if (op.side < 0 || op.side >= AGOCUDA_PX_MAX_SIDES) return false;
            nSides = op.side + 1 > nSides ? op.side + 1 : nSides;
        } else if (op.side >= AGOCUDA_PX_MAX_SIDES) {
            return false;
        }
    }
    return K <= AGOCUDA_PX_MAX_STENCILS;
}

template <bool TMA>
static int launch_chain(void *stream, const agocuda_pixel_program *program, const agocuda_pixel_frame *frames,
                        const CUtensorMap *maps, uint32_t numFrames, uint32_t maxWidth, uint32_t maxHeight,
                        uint32_t *pStatus)
{
    int K, nSides;
    if (!chain_shape(program, K, nSides) || !frames || !numFrames || numFrames > 65535 || !maxWidth || !maxHeight)
        return AGOCUDA_INVALID_PARAMS;
    agocuda_pixel_program p = *program;
    for (int k = 0; k < p.numOps; k++) {   // unary ops read no side operand
        const int c = p.ops[k].code;
        if (!(c >= AGOCUDA_PX_AND && c <= AGOCUDA_PX_SUB_SAT)) p.ops[k].side = -1;
    }
    dim3 grd(div_up(maxWidth, kPxTW), div_up(maxHeight, kPxTH), numFrames);
    const size_t smem = (size_t)(2 + nSides) * px_plane_words(kPxTH + 2 * K, TMA) * sizeof(uint32_t);
    static std::once_flag once;
    std::call_once(once, [] {   // up to 5 planes of 72 x 40 words: above the 48 KB default
        cudaFuncSetAttribute(k_pixel_chain<TMA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (2 + AGOCUDA_PX_MAX_SIDES) * px_plane_words(kPxTH + 2 * AGOCUDA_PX_MAX_STENCILS, TMA) * 4);
    });
    k_pixel_chain<TMA><<<grd, kPxThreads, smem, as_stream(stream)>>>(p, frames, maps, K, nSides, pStatus);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

}  // namespace

extern "C" int agocuda_fused_PixelChain_U8(void *stream, const agocuda_pixel_program *program,
                                           const agocuda_pixel_frame *frames, uint32_t numFrames, uint32_t maxWidth,
                                           uint32_t maxHeight)
{
    return launch_chain<false>(stream, program, frames, nullptr, numFrames, maxWidth, maxHeight, nullptr);
}

extern "C" size_t agocuda_PixelChain_tensor_maps_size(uint32_t numFrames)
{
    return (size_t)numFrames * kPxMapsPerFrame * sizeof(CUtensorMap);
}

extern "C" int agocuda_PixelChain_tensor_maps(const agocuda_pixel_program *program, const agocuda_pixel_frame *framesHost,
                                              uint32_t numFrames, void *mapsHost, size_t mapsBytes)
{
    int K, nSides;
    if (!chain_shape(program, K, nSides) || !framesHost || !numFrames || !mapsHost ||
        ((uintptr_t)mapsHost & 63) || mapsBytes < agocuda_PixelChain_tensor_maps_size(numFrames))
        return AGOCUDA_INVALID_PARAMS;
    CUtensorMap *maps = (CUtensorMap *)mapsHost;
    memset(maps, 0, agocuda_PixelChain_tensor_maps_size(numFrames));
    for (uint32_t i = 0; i < numFrames; i++) {
        const agocuda_pixel_frame &f = framesHost[i];
        for (int s = -1; s < nSides; s++) {
            const uint8_t *base = s < 0 ? f.src : f.side[s];
            const uint32_t stride = s < 0 ? f.srcStride : f.sideStride[s];
            if (!agocuda_u8_tensor_map(&maps[i * kPxMapsPerFrame + 1 + s], base, f.width, f.height, stride, kPxWords * 4,
                                       kPxTH + 2 * K))
                return AGOCUDA_INVALID_PARAMS;
        }
    }
    return 0;
}

extern "C" int agocuda_fused_PixelChain_U8_tma(void *stream, const agocuda_pixel_program *program,
                                               const agocuda_pixel_frame *frames, const void *maps, uint32_t numFrames,
                                               uint32_t maxWidth, uint32_t maxHeight, uint32_t *pStatus)
{
    if (!maps || ((uintptr_t)maps & 63) || !pStatus) return AGOCUDA_INVALID_PARAMS;
    return launch_chain<true>(stream, program, frames, (const CUtensorMap *)maps, numFrames, maxWidth, maxHeight, pStatus);
}

// ---------------------------------------------------------------------------------
// 3x3 filters on U8 (ago_haf_cpu_filter.cpp) as per-node kernels: the pixel-chain stages on
// image rows in global memory; interior rows [1, H-1), every column.
// ---------------------------------------------------------------------------------
namespace {

constexpr int kFBX = 32, kFBY = 4, kFRows = 16;   // 8 pixels x 16 rows per thread

template <int OP>
__global__ void __launch_bounds__(kFBX * kFBY)
k_filter3x3(int W, int H, uint8_t *dst, int dstStride, const uint8_t *src, int srcStride)
{
    const int x = (blockIdx.x * kFBX + threadIdx.x) * 8;
    const int y0 = 1 + (blockIdx.y * kFBY + threadIdx.y) * kFRows;
    if (x >= W || y0 >= H - 1) return;
    const int y1 = min(y0 + kFRows, H - 1);
    const GlobalRows in{src, srcStride, x};
    const GlobalOut out{dst, dstStride, x, W};
    switch (OP) {
    case AGOCUDA_PX_DILATE3x3: stage_minmax<true>(in, out, y0, y1); break;
    case AGOCUDA_PX_ERODE3x3: stage_minmax<false>(in, out, y0, y1); break;
    case AGOCUDA_PX_MEDIAN3x3: stage_median(in, out, y0, y1); break;
    case AGOCUDA_PX_GAUSSIAN3x3: stage_linear<true>(in, out, y0, y1); break;
    default: stage_linear<false>(in, out, y0, y1); break;   // box
    }
}

template <int OP>
int filter_launch(void *stream, uint32_t W, uint32_t H, uint8_t *dst, uint32_t dstStride, const uint8_t *src,
                  uint32_t srcStride)
{
    auto ok = [&](const uint8_t *p, uint32_t s) { return p && ((uintptr_t)p & 3) == 0 && (s & 3) == 0 && s >= W; };
    if (W < 3 || H < 3 || !ok(dst, dstStride) || !ok(src, srcStride)) return AGOCUDA_INVALID_PARAMS;
    dim3 grd(div_up(W, kFBX * 8), div_up(H - 2, kFBY * kFRows));
    k_filter3x3<OP><<<grd, dim3(kFBX, kFBY), 0, as_stream(stream)>>>((int)W, (int)H, dst, (int)dstStride, src, (int)srcStride);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

}  // namespace

#define FILTER(NAME, OP)                                                                                          \
    extern "C" int agocuda_##NAME(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride, \
                                  const uint8_t *pSrc, uint32_t srcStride)                                        \
    {                                                                                                          \
        return filter_launch<OP>(stream, dstWidth, dstHeight, pDst, dstStride, pSrc, srcStride);                \
    }
FILTER(Gaussian_U8_U8_3x3, AGOCUDA_PX_GAUSSIAN3x3)   // HafCpu_Gaussian_U8_U8_3x3 (ago_haf_cpu_filter.cpp:1518)
FILTER(Box_U8_U8_3x3, AGOCUDA_PX_BOX3x3)
FILTER(Dilate_U8_U8_3x3, AGOCUDA_PX_DILATE3x3)
FILTER(Erode_U8_U8_3x3, AGOCUDA_PX_ERODE3x3)
FILTER(Median_U8_U8_3x3, AGOCUDA_PX_MEDIAN3x3)
#undef FILTER

// ---------------------------------------------------------------------------------
// Channel extract / combine between U8 planes and interleaved formats
// (ago_haf_cpu_ch_extract_combine.cpp).  A thread owns 4 output units: their bytes are
// gathered with 32-bit loads and byte permutes and written as whole words; the units a row's
// width cuts go byte by byte.
// ---------------------------------------------------------------------------------
namespace {

constexpr int kChBX = 64, kChBY = 4;

// dst[x] = src[x * UNIT + POS]
template <int UNIT, int POS>
__global__ void __launch_bounds__(kChBX * kChBY)
k_channel_extract(int W, int H, uint8_t *dst, int dstStride, const uint8_t *src, int srcStride)
{
    const int x = (blockIdx.x * kChBX + threadIdx.x) * 4;
    const int y = blockIdx.y * kChBY + threadIdx.y;
    if (x >= W || y >= H) return;
    const uint8_t *s = src + (size_t)y * srcStride + (size_t)x * UNIT;
    uint8_t *d = dst + (size_t)y * dstStride + x;
    if (x + 4 <= W) {
        uint32_t w[UNIT];
#pragma unroll
        for (int i = 0; i < UNIT; i++) w[i] = __ldg((const uint32_t *)s + i);
        auto byte = [&](int k) { return (w[k >> 2] >> (8 * (k & 3))) & 0xffu; };
        *(uint32_t *)d = byte(POS) | (byte(UNIT + POS) << 8) | (byte(2 * UNIT + POS) << 16) | (byte(3 * UNIT + POS) << 24);
    } else {
        for (int i = 0; i < W - x; i++) d[i] = s[i * UNIT + POS];
    }
}

enum ChCombine { CH_UV, CH_RGB, CH_RGBX, CH_UYVY, CH_YUYV };

// one output unit: UV = (u, v); RGB = (r, g, b); RGBX = (r, g, b, x); UYVY = (u, y0, v, y1) and
// YUYV = (y0, u, y1, v) for a pair of pixels (y at 2x, 2x+1; u, v at x)
template <int MODE>
__global__ void __launch_bounds__(kChBX * kChBY)
k_channel_combine(int W, int H, uint8_t *dst, int dstStride, const uint8_t *a, int aStride, const uint8_t *b,
                  int bStride, const uint8_t *c, int cStride, const uint8_t *e, int eStride)
{
    constexpr int UNIT = MODE == CH_UV ? 2 : MODE == CH_RGB ? 3 : 4;
    const int x = (blockIdx.x * kChBX + threadIdx.x) * 4;   // first output unit
    const int y = blockIdx.y * kChBY + threadIdx.y;
    if (x >= W || y >= H) return;
    const uint8_t *pa = a + (size_t)y * aStride, *pb = b + (size_t)y * bStride;
    const uint8_t *pc = c ? c + (size_t)y * cStride : nullptr, *pe = e ? e + (size_t)y * eStride : nullptr;
    uint8_t *d = dst + (size_t)y * dstStride + (size_t)x * UNIT;
    auto unit_byte = [&](int u, int k) -> uint32_t {   // byte k of output unit u
        switch (MODE) {
        case CH_UV: return k == 0 ? pa[u] : pb[u];
        case CH_RGB: return k == 0 ? pa[u] : k == 1 ? pb[u] : pc[u];
        case CH_RGBX: return k == 0 ? pa[u] : k == 1 ? pb[u] : k == 2 ? pc[u] : pe[u];
        case CH_UYVY: return k == 0 ? pb[u] : k == 1 ? pa[2 * u] : k == 2 ? pc[u] : pa[2 * u + 1];
        default: return k == 0 ? pa[2 * u] : k == 1 ? pb[u] : k == 2 ? pa[2 * u + 1] : pc[u];
        }
    };
    if (x + 4 <= W) {
        uint32_t out[UNIT] = {};
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int k = 0; k < UNIT; k++) {
                const int o = u * UNIT + k;
                out[o >> 2] |= unit_byte(x + u, k) << (8 * (o & 3));
            }
#pragma unroll
        for (int i = 0; i < UNIT; i++) ((uint32_t *)d)[i] = out[i];
    } else {
        for (int u = 0; u < W - x; u++)
            for (int k = 0; k < UNIT; k++) d[u * UNIT + k] = (uint8_t)unit_byte(x + u, k);
    }
}

bool ch_plane_ok(const uint8_t *p, uint32_t stride) { return p && ((uintptr_t)p & 3) == 0 && (stride & 3) == 0; }

template <int UNIT, int POS>
int extract_launch(void *stream, uint32_t W, uint32_t H, uint8_t *dst, uint32_t dstStride, const uint8_t *src,
                   uint32_t srcStride)
{
    if (!W || !H || !ch_plane_ok(dst, dstStride) || !ch_plane_ok(src, srcStride) || dstStride < W || srcStride < W * UNIT)
        return AGOCUDA_INVALID_PARAMS;
    dim3 grd(div_up(W, kChBX * 4), div_up(H, kChBY));
    k_channel_extract<UNIT, POS><<<grd, dim3(kChBX, kChBY), 0, as_stream(stream)>>>((int)W, (int)H, dst, (int)dstStride,
                                                                                    src, (int)srcStride);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

template <int MODE>
int combine_launch(void *stream, uint32_t W, uint32_t H, uint8_t *dst, uint32_t dstStride, const uint8_t *a,
                   uint32_t aStride, const uint8_t *b, uint32_t bStride, const uint8_t *c, uint32_t cStride,
                   const uint8_t *e, uint32_t eStride)
{
    constexpr int UNIT = MODE == CH_UV ? 2 : MODE == CH_RGB ? 3 : 4;
    const int planes = MODE == CH_UV ? 2 : MODE == CH_RGBX ? 4 : 3;
    const bool pairs = MODE == CH_UYVY || MODE == CH_YUYV;   // W counts pixels: one unit per pair
    const uint32_t units = pairs ? W / 2 : W;
    if (!units || !H || (pairs && (W & 1)) || !ch_plane_ok(dst, dstStride) || dstStride < units * UNIT || !a || !b ||
        (planes > 2 && !c) || (planes > 3 && !e))
        return AGOCUDA_INVALID_PARAMS;
    dim3 grd(div_up(units, kChBX * 4), div_up(H, kChBY));
    k_channel_combine<MODE><<<grd, dim3(kChBX, kChBY), 0, as_stream(stream)>>>(
        (int)units, (int)H, dst, (int)dstStride, a, (int)aStride, b, (int)bStride, planes > 2 ? c : nullptr, (int)cStride,
        planes > 3 ? e : nullptr, (int)eStride);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

}  // namespace

#define EXTRACT(NAME, UNIT, POS)                                                                                  \
    extern "C" int agocuda_##NAME(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride, \
                                  const uint8_t *pSrc, uint32_t srcStride)                                        \
    {                                                                                                          \
        return extract_launch<UNIT, POS>(stream, dstWidth, dstHeight, pDst, dstStride, pSrc, srcStride);        \
    }
EXTRACT(ChannelExtract_U8_U16_Pos0, 2, 0)
EXTRACT(ChannelExtract_U8_U16_Pos1, 2, 1)
EXTRACT(ChannelExtract_U8_U24_Pos0, 3, 0)
EXTRACT(ChannelExtract_U8_U24_Pos1, 3, 1)
EXTRACT(ChannelExtract_U8_U24_Pos2, 3, 2)
EXTRACT(ChannelExtract_U8_U32_Pos0, 4, 0)
EXTRACT(ChannelExtract_U8_U32_Pos1, 4, 1)
EXTRACT(ChannelExtract_U8_U32_Pos2, 4, 2)
EXTRACT(ChannelExtract_U8_U32_Pos3, 4, 3)
#undef EXTRACT

extern "C" int agocuda_ChannelCombine_U16_U8U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                               uint32_t dstStride, const uint8_t *pSrc1, uint32_t src1Stride,
                                               const uint8_t *pSrc2, uint32_t src2Stride)
{
    return combine_launch<CH_UV>(stream, dstWidth, dstHeight, pDst, dstStride, pSrc1, src1Stride, pSrc2, src2Stride,
                                 nullptr, 0, nullptr, 0);
}

#define COMBINE3(NAME, MODE)                                                                                      \
    extern "C" int agocuda_##NAME(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride, \
                                  const uint8_t *pSrc1, uint32_t src1Stride, const uint8_t *pSrc2, uint32_t src2Stride, \
                                  const uint8_t *pSrc3, uint32_t src3Stride)                                      \
    {                                                                                                          \
        return combine_launch<MODE>(stream, dstWidth, dstHeight, pDst, dstStride, pSrc1, src1Stride, pSrc2, src2Stride, \
                                    pSrc3, src3Stride, nullptr, 0);                                            \
    }
COMBINE3(ChannelCombine_U24_U8U8U8_RGB, CH_RGB)
COMBINE3(ChannelCombine_U32_U8U8U8_UYVY, CH_UYVY)
COMBINE3(ChannelCombine_U32_U8U8U8_YUYV, CH_YUYV)
#undef COMBINE3

extern "C" int agocuda_ChannelCombine_U32_U8U8U8U8_RGBX(void *stream, uint32_t dstWidth, uint32_t dstHeight,
                                                       uint8_t *pDst, uint32_t dstStride, const uint8_t *pSrc1,
                                                       uint32_t src1Stride, const uint8_t *pSrc2, uint32_t src2Stride,
                                                       const uint8_t *pSrc3, uint32_t src3Stride, const uint8_t *pSrc4,
                                                       uint32_t src4Stride)
{
    return combine_launch<CH_RGBX>(stream, dstWidth, dstHeight, pDst, dstStride, pSrc1, src1Stride, pSrc2, src2Stride,
                                   pSrc3, src3Stride, pSrc4, src4Stride);
}

// ---------------------------------------------------------------------------------
// Table lookup (HafCpu_Lut_U8_U8, ago_haf_cpu_arithmetic.cpp; HafCpu_Lut_S16_S16 :4916)
// ---------------------------------------------------------------------------------
namespace {

// U8: the 256-entry table in shared memory, 16 pixels (one 16-byte vector) per thread
__global__ void __launch_bounds__(kEwBX * kEwBY)
k_lut_u8(int W, int H, uint8_t *dst, int dstStride, const uint8_t *src, int srcStride, const uint8_t *__restrict__ lut)
{
    __shared__ uint8_t tab[256];
    const int tid = threadIdx.y * kEwBX + threadIdx.x;
    if (tid < 256) tab[tid] = lut[tid];
    __syncthreads();
    const int x = (blockIdx.x * kEwBX + threadIdx.x) * 16;
    const int y = blockIdx.y * kEwBY + threadIdx.y;
    if (x >= W || y >= H) return;
    const uint8_t *s = src + (size_t)y * srcStride + x;
    uint8_t *d = dst + (size_t)y * dstStride + x;
    if (x + 16 <= W) {
        const uint4 v = __ldg((const uint4 *)s);
        const uint32_t in[4] = {v.x, v.y, v.z, v.w};
        uint32_t out[4];
#pragma unroll
        for (int k = 0; k < 4; k++)
            out[k] = (uint32_t)tab[in[k] & 0xff] | ((uint32_t)tab[(in[k] >> 8) & 0xff] << 8) |
                     ((uint32_t)tab[(in[k] >> 16) & 0xff] << 16) | ((uint32_t)tab[in[k] >> 24] << 24);
        *(uint4 *)d = make_uint4(out[0], out[1], out[2], out[3]);
    } else {
        for (int i = 0; i < W - x; i++) d[i] = tab[s[i]];
    }
}

// S16: table in global memory (cached), index v + offset clamped into the table
__global__ void __launch_bounds__(kEwBX * kEwBY)
k_lut_s16(int W, int H, int16_t *dst, int dstStride, const int16_t *src, int srcStride, const int16_t *__restrict__ lut,
          int count, int offset)
{
    const int x = (blockIdx.x * kEwBX + threadIdx.x) * 8;
    const int y = blockIdx.y * kEwBY + threadIdx.y;
    if (x >= W || y >= H) return;
    const int16_t *s = (const int16_t *)((const uint8_t *)src + (size_t)y * srcStride) + x;
    int16_t *d = (int16_t *)((uint8_t *)dst + (size_t)y * dstStride) + x;
    auto look = [&](int v) { return __ldg(lut + clampi(v + offset, 0, count - 1)); };
    if (x + 8 <= W) {
        const uint4 v = __ldg((const uint4 *)s);
        const int16_t *e = (const int16_t *)&v;
        uint4 o;
        int16_t *oe = (int16_t *)&o;
#pragma unroll
        for (int i = 0; i < 8; i++) oe[i] = look(e[i]);
        *(uint4 *)d = o;
    } else {
        for (int i = 0; i < W - x; i++) d[i] = look(s[i]);
    }
}

}  // namespace

extern "C" int agocuda_Lut_U8_U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst, uint32_t dstStride,
                                 const uint8_t *pSrc, uint32_t srcStride, const uint8_t *pLut)
{
    if (!dstWidth || !dstHeight || !pLut || !ew_plane_ok(pDst, dstStride, dstWidth) || !ew_plane_ok(pSrc, srcStride, dstWidth))
        return AGOCUDA_INVALID_PARAMS;
    dim3 grd(div_up(dstWidth, kEwBX * 16), div_up(dstHeight, kEwBY));
    k_lut_u8<<<grd, dim3(kEwBX, kEwBY), 0, as_stream(stream)>>>((int)dstWidth, (int)dstHeight, pDst, (int)dstStride, pSrc,
                                                                (int)srcStride, pLut);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_Lut_S16_S16(void *stream, uint32_t dstWidth, uint32_t dstHeight, int16_t *pDst, uint32_t dstStride,
                                   const int16_t *pSrc, uint32_t srcStride, const int16_t *pLut, uint32_t count,
                                   uint32_t offset)
{
    if (!dstWidth || !dstHeight || !pLut || !count || count > 65536 || offset >= count ||
        !ew_plane_ok(pDst, dstStride, dstWidth) || !ew_plane_ok(pSrc, srcStride, dstWidth))
        return AGOCUDA_INVALID_PARAMS;
    dim3 grd(div_up(dstWidth, kEwBX * 8), div_up(dstHeight, kEwBY));
    k_lut_s16<<<grd, dim3(kEwBX, kEwBY), 0, as_stream(stream)>>>((int)dstWidth, (int)dstHeight, pDst, (int)dstStride, pSrc,
                                                                 (int)srcStride, pLut, (int)count, (int)offset);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

// ---------------------------------------------------------------------------------
// Integral image U8 -> U32 (HafCpu_IntegralImage_U32_U8, ago_haf_cpu_arithmetic.cpp:7057):
// out(x, y) = sum of in(i, j) for i <= x, j <= y, modulo 2^32.  Three launches: row prefix
// sums (a block per row), column totals of 32-row segments, then each segment's rows get
// the totals of the segments above plus their running column sum.
// ---------------------------------------------------------------------------------
namespace {

constexpr int kIiThreads = 256, kIiSeg = 32;

__global__ void __launch_bounds__(kIiThreads)
k_integral_rows(int W, uint32_t *dst, int dstStride, const uint8_t *src, int srcStride)
{
    __shared__ uint32_t warpSum[kIiThreads / 32];
    const int y = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int per = (W + kIiThreads - 1) / kIiThreads, x0 = tid * per, x1 = min(x0 + per, W);
    const uint8_t *s = src + (size_t)y * srcStride;
    uint32_t *d = (uint32_t *)((uint8_t *)dst + (size_t)y * dstStride);
    uint32_t sum = 0;
    for (int x = x0; x < x1; x++) sum += s[x];
    // exclusive prefix of the threads' sums
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) warpSum[warp] = incl;
    __syncthreads();
    uint32_t base = 0;
    for (int w = 0; w < warp; w++) base += warpSum[w];
    uint32_t run = base + incl - sum;
    for (int x = x0; x < x1; x++) { run += s[x]; d[x] = run; }
}

__global__ void __launch_bounds__(kIiThreads)
k_integral_seg_totals(int W, int H, const uint32_t *dst, int dstStride, uint32_t *totals)
{
    const int x = blockIdx.x * kIiThreads + threadIdx.x, seg = blockIdx.y;
    if (x >= W) return;
    const int y0 = seg * kIiSeg, y1 = min(y0 + kIiSeg, H);
    uint32_t t = 0;
    for (int y = y0; y < y1; y++) t += ((const uint32_t *)((const uint8_t *)dst + (size_t)y * dstStride))[x];
    totals[(size_t)seg * W + x] = t;
}

__global__ void __launch_bounds__(kIiThreads)
k_integral_columns(int W, int H, uint32_t *dst, int dstStride, const uint32_t *totals)
{
    const int x = blockIdx.x * kIiThreads + threadIdx.x, seg = blockIdx.y;
    if (x >= W) return;
    uint32_t run = 0;
    for (int s = 0; s < seg; s++) run += totals[(size_t)s * W + x];
    const int y0 = seg * kIiSeg, y1 = min(y0 + kIiSeg, H);
    for (int y = y0; y < y1; y++) {
        uint32_t *p = (uint32_t *)((uint8_t *)dst + (size_t)y * dstStride) + x;
        run += *p;
        *p = run;
    }
}

}  // namespace

extern "C" size_t agocuda_IntegralImage_scratch_size(uint32_t width, uint32_t height)
{
    return (size_t)div_up(height, kIiSeg) * width * sizeof(uint32_t);
}

extern "C" int agocuda_IntegralImage_U32_U8(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint32_t *pDst,
                                            uint32_t dstStride, const uint8_t *pSrc, uint32_t srcStride, void *scratch,
                                            size_t scratchBytes)
{
    const uint32_t W = dstWidth, H = dstHeight;
    if (!W || !H || !pDst || !pSrc || ((uintptr_t)pDst & 3) || (dstStride & 3) || dstStride < 4 * W || srcStride < W ||
        !scratch || scratchBytes < agocuda_IntegralImage_scratch_size(W, H) || H > 65535u * kIiSeg)
        return AGOCUDA_INVALID_PARAMS;
    cudaStream_t s = as_stream(stream);
    uint32_t *tot = (uint32_t *)scratch;
    k_integral_rows<<<H, kIiThreads, 0, s>>>((int)W, pDst, (int)dstStride, pSrc, (int)srcStride);
    const dim3 grd(div_up(W, kIiThreads), div_up(H, kIiSeg));
    k_integral_seg_totals<<<grd, kIiThreads, 0, s>>>((int)W, (int)H, pDst, (int)dstStride, tot);
    k_integral_columns<<<grd, kIiThreads, 0, s>>>((int)W, (int)H, pDst, (int)dstStride, tot);
    agocuda_count_launch(3);
    return agocuda_launch_status();
}

// ---------------------------------------------------------------------------------
// Histogram of a U8 image into a distribution (OpenVX binning: v in [offset, offset+range)
// counts into bin (v - offset) * bins / range).  Blocks count pixel values into per-warp
// 256-entry shared histograms (16 pixels per load), fold them, and add each value's count to
// its bin with one global atomic.
// ---------------------------------------------------------------------------------
namespace {

constexpr int kHistThreads = 256;

__global__ void __launch_bounds__(kHistThreads)
k_histogram(int W, int H, const uint8_t *src, int srcStride, uint32_t *hist, int bins, int offset, int range)
{
    __shared__ uint32_t sub[kHistThreads / 32][256];
    const int tid = threadIdx.x, warp = tid >> 5;
    for (int i = tid; i < (kHistThreads / 32) * 256; i += kHistThreads) (&sub[0][0])[i] = 0;
    __syncthreads();
    const int vecs = (W + 15) / 16;                       // 16-pixel groups per row
    const long long total = (long long)vecs * H;
    for (long long i = (long long)blockIdx.x * kHistThreads + tid; i < total; i += (long long)gridDim.x * kHistThreads) {
        const int y = (int)(i / vecs), x = (int)(i - (long long)y * vecs) * 16;
        const uint8_t *s = src + (size_t)y * srcStride + x;
        if (x + 16 <= W) {
            const uint4 v = __ldg((const uint4 *)s);
            const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int k = 0; k < 4; k++)
#pragma unroll
                for (int b = 0; b < 4; b++) atomicAdd(&sub[warp][(w[k] >> (8 * b)) & 0xff], 1u);
        } else {
            for (int j = 0; j < W - x; j++) atomicAdd(&sub[warp][s[j]], 1u);
        }
    }
    __syncthreads();
    for (int v = tid; v < 256; v += kHistThreads) {
        uint32_t c = 0;
#pragma unroll
        for (int w = 0; w < kHistThreads / 32; w++) c += sub[w][v];
        if (c && v >= offset && v < offset + range) atomicAdd(&hist[(long long)(v - offset) * bins / range], c);
    }
}

}  // namespace

extern "C" int agocuda_Histogram_DATA_U8(void *stream, uint32_t *pHist, uint32_t srcWidth, uint32_t srcHeight,
                                         const uint8_t *pSrc, uint32_t srcStride, uint32_t numBins, int32_t offset,
                                         uint32_t range)
{
    if (!pHist || !pSrc || !srcWidth || !srcHeight || !numBins || !range || numBins > range || srcStride < srcWidth ||
        (((uintptr_t)pSrc | srcStride) & 15) || range > (1u << 30))
        return AGOCUDA_INVALID_PARAMS;
    cudaStream_t s = as_stream(stream);
    if (cudaMemsetAsync(pHist, 0, (size_t)numBins * sizeof(uint32_t), s) != cudaSuccess) return agocuda_launch_status();
    const long long groups = (long long)div_up(srcWidth, 16) * srcHeight;
    const int blocks = (int)std::min<long long>(4 * 148, div_up((unsigned)std::min<long long>(groups, 1ll << 31), kHistThreads));
    k_histogram<<<std::max(1, blocks), kHistThreads, 0, s>>>((int)srcWidth, (int)srcHeight, pSrc, (int)srcStride, pHist,
                                                             (int)numBins, (int)offset, (int)range);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}
