// filters.cu -- 3x3 stencil kernels of the AGO vision path and the fused
// Gaussian -> SobelMagnitude -> ConvertDepth -> Threshold chain, for sm_100a.
//
// Work decomposition shared by the stencil kernels here: one thread owns a 4-pixel
// column group (one 32-bit word of a U8 row) and walks down RPT rows, keeping the
// per-row horizontal partial sums of the rows above in registers, so each input row is
// loaded once per thread (the neighbouring words come from L1).  A warp covers 128
// contiguous bytes per row, so every global access is a full coalesced line.
#include "agocuda_internal.cuh"
#include <math.h>
#include <string.h>

namespace {

constexpr int kBX = 32;      // threads across: 32 x 4 px = 128 columns
constexpr int kBY = 4;       // thread rows per block
constexpr int kRPT = 8;      // output rows per thread

// Pixels p[x-2 .. x+5] of a U8 row, for the 4-pixel group starting at x.
struct Row8 { int p[8]; };
__device__ __forceinline__ Row8 load_row8(const uint8_t *row, int x, int stride)
{
    uint32_t l = load_word_clamped(row, x - 4, stride);
    uint32_t c = load_word_clamped(row, x, stride);
    uint32_t r = load_word_clamped(row, x + 4, stride);
    Row8 o;
    o.p[0] = byte_of(l, 2); o.p[1] = byte_of(l, 3);
    o.p[2] = byte_of(c, 0); o.p[3] = byte_of(c, 1); o.p[4] = byte_of(c, 2); o.p[5] = byte_of(c, 3);
    o.p[6] = byte_of(r, 0); o.p[7] = byte_of(r, 1);
    return o;
}

__device__ __forceinline__ uint32_t pack4(int a, int b, int c, int d)
{
    return (uint32_t)(a & 0xff) | ((uint32_t)(b & 0xff) << 8) | ((uint32_t)(c & 0xff) << 16) | ((uint32_t)(d & 0xff) << 24);
}

// ---------------------------------------------------------------------------------
// Sobel 3x3 GX/GY (HafCpu_Sobel_S16S16_U8_3x3_GXY, ago_haf_cpu_filter.cpp:2237) and
// SobelMagnitude (HafCpu_SobelMagnitude_S16_U8_3x3, ago_haf_cpu_filter.cpp:2468).
// Rolling state per column c in [x-1, x+4]: the row above and the current row.
// ---------------------------------------------------------------------------------
struct SobelRows { int a[6], b[6]; };   // pixel columns x-1..x+4 of rows y-1 and y

__device__ __forceinline__ void sobel_at(const int *pa, const int *pb, const int *pc, int i, int &gx, int &gy)
{
    // columns i-1, i, i+1 in the 6-wide window are indices i, i+1, i+2
    gx = (pa[i + 2] - pa[i]) + 2 * (pb[i + 2] - pb[i]) + (pc[i + 2] - pc[i]);
    gy = (pc[i] + 2 * pc[i + 1] + pc[i + 2]) - (pa[i] + 2 * pa[i + 1] + pa[i + 2]);
}

__device__ __forceinline__ void row6(const Row8 &r, int *o)
{
#pragma unroll
    for (int i = 0; i < 6; i++) o[i] = r.p[i + 1];
}

// round(sqrt(n)) to nearest for integer n in [0, 2^31): exact integer fix-up of a float
// estimate (n is never a perfect half-square, so the rounding direction is exact).
__device__ __forceinline__ int isqrt_round(int n)
{
    int m = __float2int_rn(__fsqrt_rn((float)n));
    long long mm = (long long)m * m;
    if ((long long)n > mm + m) m++;
    else if (m > 0 && (long long)n <= mm - m) m--;   // for m == 0 the lower bound is n >= 0
    return m;
}

__global__ void __launch_bounds__(kBX * kBY)
k_sobel_gxy(int W, int H, int16_t *gxp, int gxStride, int16_t *gyp, int gyStride, const uint8_t *src, int srcStride)
{
    const int x = (blockIdx.x * kBX + threadIdx.x) * 4;
    const int y0 = 1 + (blockIdx.y * kBY + threadIdx.y) * kRPT;
    if (x >= W || y0 >= H - 1) return;
    const int y1 = min(y0 + kRPT, H - 1);
    int pa[6], pb[6], pc[6];
    row6(load_row8(src + (size_t)(y0 - 1) * srcStride, x, srcStride), pa);
    row6(load_row8(src + (size_t)y0 * srcStride, x, srcStride), pb);
    for (int y = y0; y < y1; y++) {
        row6(load_row8(src + (size_t)(y + 1) * srcStride, x, srcStride), pc);
        int gx[4], gy[4];
#pragma unroll
        for (int i = 0; i < 4; i++) sobel_at(pa, pb, pc, i, gx[i], gy[i]);
        uint2 vx, vy;
        vx.x = (uint32_t)(uint16_t)gx[0] | ((uint32_t)(uint16_t)gx[1] << 16);
        vx.y = (uint32_t)(uint16_t)gx[2] | ((uint32_t)(uint16_t)gx[3] << 16);
        vy.x = (uint32_t)(uint16_t)gy[0] | ((uint32_t)(uint16_t)gy[1] << 16);
        vy.y = (uint32_t)(uint16_t)gy[2] | ((uint32_t)(uint16_t)gy[3] << 16);
        *(uint2 *)((uint8_t *)gxp + (size_t)y * gxStride + 2 * x) = vx;
        *(uint2 *)((uint8_t *)gyp + (size_t)y * gyStride + 2 * x) = vy;
#pragma unroll
        for (int i = 0; i < 6; i++) { pa[i] = pb[i]; pb[i] = pc[i]; }
    }
}

__global__ void __launch_bounds__(kBX * kBY)
k_sobel_magnitude(int W, int H, int16_t *dst, int dstStride, const uint8_t *src, int srcStride,
                  int simdBegin, int simdEnd)
{
    const int x = (blockIdx.x * kBX + threadIdx.x) * 4;
    const int y0 = 1 + (blockIdx.y * kBY + threadIdx.y) * kRPT;
    if (x >= W || y0 >= H - 1) return;
    const int y1 = min(y0 + kRPT, H - 1);
    int pa[6], pb[6], pc[6];
    row6(load_row8(src + (size_t)(y0 - 1) * srcStride, x, srcStride), pa);
    row6(load_row8(src + (size_t)y0 * srcStride, x, srcStride), pb);
    for (int y = y0; y < y1; y++) {
        row6(load_row8(src + (size_t)(y + 1) * srcStride, x, srcStride), pc);
        int m[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            int gx, gy;
            sobel_at(pa, pb, pc, i, gx, gy);
            int n = gx * gx + gy * gy;
            int xi = x + i;
            if (xi < simdBegin || xi >= simdEnd)
                m[i] = (int)(int16_t)(int)__fsqrt_rn(__fadd_rn((float)(gx * gx), (float)(gy * gy)));
            else
                m[i] = min(isqrt_round(n), 65535);
        }
        uint2 v;
        v.x = (uint32_t)(uint16_t)m[0] | ((uint32_t)(uint16_t)m[1] << 16);
        v.y = (uint32_t)(uint16_t)m[2] | ((uint32_t)(uint16_t)m[3] << 16);
        *(uint2 *)((uint8_t *)dst + (size_t)y * dstStride + 2 * x) = v;
#pragma unroll
        for (int i = 0; i < 6; i++) { pa[i] = pb[i]; pb[i] = pc[i]; }
    }
}

// ---------------------------------------------------------------------------------
// Pointwise kernels: 4 pixels per thread per row, all rows.
// ---------------------------------------------------------------------------------
__global__ void k_magnitude(int W, int H, int16_t *mag, int magStride, const int16_t *gxp, int gxStride,
                            const int16_t *gyp, int gyStride, int prefix, int tail)
{
    const int x = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    uint2 a = *(const uint2 *)((const uint8_t *)gxp + (size_t)y * gxStride + 2 * x);
    uint2 b = *(const uint2 *)((const uint8_t *)gyp + (size_t)y * gyStride + 2 * x);
    int ga[4] = {(int16_t)(a.x & 0xffff), (int16_t)(a.x >> 16), (int16_t)(a.y & 0xffff), (int16_t)(a.y >> 16)};
    int gb[4] = {(int16_t)(b.x & 0xffff), (int16_t)(b.x >> 16), (int16_t)(b.y & 0xffff), (int16_t)(b.y >> 16)};
    int m[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int xi = x + i;
        int sa = ga[i] * ga[i], sb = gb[i] * gb[i];
        if (xi < prefix) {
            m[i] = (int)(int16_t)(int)__fsqrt_rn(__fadd_rn((float)sa, (float)sb));
        } else if (xi >= tail) {
            float t = __fsqrt_rn(__fadd_rn((float)sa, (float)sb));
            m[i] = (int)(int16_t)(int)round((double)t);
        } else {
            double n = __dadd_rn((double)sa, (double)sb);
            int r = __double2int_rn(__dsqrt_rn(n));
            m[i] = min(r, 32767);
        }
    }
    uint2 v;
    v.x = (uint32_t)(uint16_t)m[0] | ((uint32_t)(uint16_t)m[1] << 16);
    v.y = (uint32_t)(uint16_t)m[2] | ((uint32_t)(uint16_t)m[3] << 16);
    *(uint2 *)((uint8_t *)mag + (size_t)y * magStride + 2 * x) = v;
}

__global__ void k_colordepth_u8_s16_sat(int W, int H, uint8_t *dst, int dstStride, const int16_t *src, int srcStride, int shift)
{
    const int x = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    uint2 a = *(const uint2 *)((const uint8_t *)src + (size_t)y * srcStride + 2 * x);
    int v[4] = {(int16_t)(a.x & 0xffff), (int16_t)(a.x >> 16), (int16_t)(a.y & 0xffff), (int16_t)(a.y >> 16)};
#pragma unroll
    for (int i = 0; i < 4; i++) v[i] = clampi(v[i] >> shift, 0, 255);
    *(uint32_t *)(dst + (size_t)y * dstStride + x) = pack4(v[0], v[1], v[2], v[3]);
}

// ---------------------------------------------------------------------------------
// Fused Gaussian3x3 -> SobelMagnitude -> ColorDepth(SAT, shift) -> Threshold(BINARY, t).
// ColorDepth and Threshold collapse into one comparison on n = gx^2 + gy^2: with
// M = (t + 1) << shift, clamp(mag >> shift, 0, 255) > t  <=>  mag >= M, and
//   SIMD body:  round(sqrt(n)) >= M   <=>  n >= M*M - M + 1
//   scalar tail: trunc(sqrtf(n)) >= M <=>  n >= M*M
// (n < 2^22 here, so sqrtf is exact enough for the second equivalence).
//
// A thread owns 8 columns and walks down its rows.  The Gaussian runs on pairs of columns
// in 16-bit lanes of 32-bit words (horizontal [1 2 1] from byte permutes, vertical sum,
// then the >> 4 kept as a mask, i.e. 16x the Gaussian); the Sobel sums stay in lanes with
// a bias and turn into exact floats, and n >= T is the sign of one exact fused multiply-add
// chain: (16gx)^2 + (16gy)^2 - 256 T, all multiples of 256 below 2^30.
// ---------------------------------------------------------------------------------
constexpr int kC1Rows = 18;     // output rows per thread (a multiple of the 3-way unroll)
constexpr int kC1BX = 32, kC1BY = 4;

// h = p[c-1] + 2 p[c] + p[c+1] on the 5 lane-pair words of 8 columns x..x+7 plus x-1, x+8:
// (x, x+2), (x+1, x+3), (x+4, x+6), (x+5, x+7), (x-1, x+8)
struct C1Row { uint32_t e1, o1, e2, o2, b; };

__device__ __forceinline__ C1Row c1_hsum(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3)
{
    const uint32_t E1 = __byte_perm(w1, 0, 0x4240), O1 = __byte_perm(w1, 0, 0x4341);
    const uint32_t E2 = __byte_perm(w2, 0, 0x4240), O2 = __byte_perm(w2, 0, 0x4341);
    const uint32_t Om1 = __byte_perm(w0, O1, 0x5453), Ep1 = __byte_perm(E1, w2, 0x3432);
    const uint32_t Om2 = __byte_perm(w1, O2, 0x5453), Ep2 = __byte_perm(E2, w3, 0x3432);
    C1Row h;
    h.e1 = Om1 + 2 * E1 + O1;
    h.o1 = E1 + 2 * O1 + Ep1;
    h.e2 = Om2 + 2 * E2 + O2;
    h.o2 = E2 + 2 * O2 + Ep2;
    // columns x-1 and x+8: bytes (x-2, x-1, x) and (x+7, x+8, x+9) weighted 1 2 1
    const uint32_t hl = __dp4a(__funnelshift_r(w0, w1, 16), 0x00010201u, 0u);
    const uint32_t hr = __dp4a(__funnelshift_r(w2, w3, 24), 0x00010201u, 0u);
    h.b = hl | (hr << 16);
    return h;
}

// 16 x Gaussian: ((h0 + 2 h1 + h2) >> 4) << 4, lanes below 4096
__device__ __forceinline__ uint32_t c1_g(uint32_t a, uint32_t b, uint32_t c) { return (a + 2 * b + c) & 0xFFF0FFF0u; }
__device__ __forceinline__ C1Row c1_gauss(const C1Row &a, const C1Row &b, const C1Row &c)
{
    return C1Row{c1_g(a.e1, b.e1, c.e1), c1_g(a.o1, b.o1, c.o1), c1_g(a.e2, b.e2, c.e2), c1_g(a.o2, b.o2, c.o2),
                 c1_g(a.b, b.b, c.b)};
}

// horizontal [1 2 1] of a 16x Gaussian row at the 8 columns, as (x, x+2), (x+1, x+3),
// (x+4, x+6), (x+5, x+7) lane pairs (below 2^16)
struct C1H { uint32_t e1, o1, e2, o2; };
__device__ __forceinline__ C1H c1_hpass(const C1Row &g)
{
    const uint32_t m1 = __byte_perm(g.b, g.o1, 0x5410), p1 = __byte_perm(g.e1, g.e2, 0x5432);
    const uint32_t m2 = __byte_perm(g.o1, g.o2, 0x5432), p2 = __byte_perm(g.e2, g.b, 0x7632);
    return C1H{m1 + 2 * g.e1 + g.o1, g.e1 + 2 * g.o1 + p1, m2 + 2 * g.e2 + g.o2, g.e2 + 2 * g.o2 + p2};
}

// 4 output bytes: 255 where the float is >= 0 (sign bit clear), else 0
__device__ __forceinline__ uint32_t nonneg_bytes(float a, float b, float c, float d)
{
    const uint32_t top = __byte_perm(__byte_perm(__float_as_uint(a), __float_as_uint(b), 0x7373),
                                     __byte_perm(__float_as_uint(c), __float_as_uint(d), 0x7373), 0x5410);
    return ((~top & 0x80808080u) >> 7) * 0xFFu;
}

// lane (value + 16384) of a biased pair word as an exact float value
__device__ __forceinline__ float c1_lo(uint32_t w) { return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7610)) - 8404992.0f; }
__device__ __forceinline__ float c1_hi(uint32_t w) { return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7632)) - 8404992.0f; }

// The rows [y0, y0 + ROWS) of one thread's 8 columns at x (clipped to [2, H-2)).
template <int ROWS>
__device__ __forceinline__ void c1_rows(const agocuda_frame &f, int x, int y0, float tRound, float tTrunc)
{
    const int W = (int)f.width, H = (int)f.height;
    if (x >= W || y0 >= H - 2) return;
    const int y1 = min(y0 + ROWS, H - 2);
    const int ss = (int)f.srcStride;
    const uint8_t *src = f.src;
    float T[8];                                    // -256 T per column (trunc / round span)
#pragma unroll
    for (int j = 0; j < 8; j++) T[j] = (x + j < f.simdBegin || x + j >= f.simdEnd) ? tTrunc : tRound;
    uint32_t nw[4];                                // words of the next input row, loaded a row ahead
    auto fetch = [&](int y) {
        const uint8_t *row = src + (size_t)min(y, H - 1) * ss;
        nw[0] = load_word_clamped(row, x - 4, ss);
        nw[1] = load_word_clamped(row, x, ss);
        nw[2] = load_word_clamped(row, x + 4, ss);
        nw[3] = load_word_clamped(row, x + 8, ss);
    };
    auto hrow = [&](int y) {
        fetch(y);
        return c1_hsum(nw[0], nw[1], nw[2], nw[3]);
    };
    // rolling rows, rotated by the unrolled loop: h of input rows y, y+1; 16x Gaussian of
    // rows y-1, y; horizontal pass of the Gaussian at rows y-1, y
    C1Row h[3], g[3];
    C1H hp[3];
    {
        const C1Row a = hrow(y0 - 2), b = hrow(y0 - 1);
        h[0] = hrow(y0);
        h[1] = hrow(y0 + 1);
        g[0] = c1_gauss(a, b, h[0]);
        g[1] = c1_gauss(b, h[0], h[1]);
        hp[0] = c1_hpass(g[0]);
        hp[1] = c1_hpass(g[1]);
        fetch(y0 + 2);
    }
    auto step = [&](int y, const C1Row &hA, const C1Row &hB, C1Row &hC, const C1Row &gA, const C1Row &gB, C1Row &gC,
                    const C1H &pA, const C1H &pB, C1H &pC) {
        hC = c1_hsum(nw[0], nw[1], nw[2], nw[3]);  // input row y+2, loaded a step earlier
        fetch(y + 3);
        gC = c1_gauss(hA, hB, hC);                 // 16 x Gaussian row y+1
        pC = c1_hpass(gC);
        (void)pB;
        // vertical [1 2 1] of the Gaussian at row y: (x-1, x+8) and the four pairs
        const uint32_t vE1 = gA.e1 + 2 * gB.e1 + gC.e1, vO1 = gA.o1 + 2 * gB.o1 + gC.o1;
        const uint32_t vE2 = gA.e2 + 2 * gB.e2 + gC.e2, vO2 = gA.o2 + 2 * gB.o2 + gC.o2;
        const uint32_t vB = gA.b + 2 * gB.b + gC.b;
        const uint32_t bias = 0x40004000u;
        // 16 gx = V(c+1) - V(c-1), 16 gy = H(y+1) - H(y-1), as biased lane pairs
        const uint32_t gx0 = vO1 + bias - __byte_perm(vB, vO1, 0x5410);     // (x, x+2)
        const uint32_t gx1 = __byte_perm(vE1, vE2, 0x5432) + bias - vE1;    // (x+1, x+3)
        const uint32_t gx2 = vO2 + bias - __byte_perm(vO1, vO2, 0x5432);    // (x+4, x+6)
        const uint32_t gx3 = __byte_perm(vE2, vB, 0x7632) + bias - vE2;     // (x+5, x+7)
        const uint32_t gy0 = pC.e1 + bias - pA.e1, gy1 = pC.o1 + bias - pA.o1;
        const uint32_t gy2 = pC.e2 + bias - pA.e2, gy3 = pC.o2 + bias - pA.o2;
        const float fx[8] = {c1_lo(gx0), c1_lo(gx1), c1_hi(gx0), c1_hi(gx1), c1_lo(gx2), c1_lo(gx3), c1_hi(gx2), c1_hi(gx3)};
        const float fy[8] = {c1_lo(gy0), c1_lo(gy1), c1_hi(gy0), c1_hi(gy1), c1_lo(gy2), c1_lo(gy3), c1_hi(gy2), c1_hi(gy3)};
        float rr[8];
#pragma unroll
        for (int j = 0; j < 8; j++) rr[j] = __fmaf_rn(fx[j], fx[j], __fmaf_rn(fy[j], fy[j], T[j]));
        // 255 where the exact sum is >= 0
        const uint32_t lo = nonneg_bytes(rr[0], rr[1], rr[2], rr[3]);
        const uint32_t hi = nonneg_bytes(rr[4], rr[5], rr[6], rr[7]);
        uint8_t *o = f.dst + (size_t)y * f.dstStride + x;
        *(uint32_t *)o = lo;
        if (x + 4 < W) *(uint32_t *)(o + 4) = hi;
    };
    for (int y = y0; y < y1; y += 3) {             // y is uniform across the thread's loop
        step(y, h[0], h[1], h[2], g[0], g[1], g[2], hp[0], hp[1], hp[2]);
        if (y + 1 >= y1) break;
        step(y + 1, h[1], h[2], h[0], g[1], g[2], g[0], hp[1], hp[2], hp[0]);
        if (y + 2 >= y1) break;
        step(y + 2, h[2], h[0], h[1], g[2], g[0], g[1], hp[2], hp[0], hp[1]);
    }
}

__global__ void __launch_bounds__(kC1BX * kC1BY)
k_fused_gauss_sobelmag_thresh(const agocuda_frame *frames, float tRound, float tTrunc)
{
    const agocuda_frame f = frames[blockIdx.z];
    const int x = (blockIdx.x * kC1BX + threadIdx.x) * 8;
    const int y0 = 2 + (blockIdx.y * kC1BY + threadIdx.y) * kC1Rows;
    c1_rows<kC1Rows>(f, x, y0, tRound, tTrunc);
}

// Persistent form: gridDim.x resident blocks take tiles (256 columns x BY * ROWS rows of one
// frame) from one queue spanning every frame of the batch, whatever their sizes.  tilePrefix
// holds each frame's first tile (numFrames + 1 entries).  queue[0] is the next tile,
// queue[1] counts finished blocks; the last block to finish puts both back to 0, so the
// launch leaves the queue ready for the next one (a launch site owns its queue words).
__device__ __forceinline__ uint32_t frame_of_tile(const uint32_t *prefix, uint32_t n, uint32_t t)
{
    uint32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ uint32_t queue_next(uint32_t *queue)
{
    __shared__ uint32_t next;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) next = atomicAdd(queue, 1u);
    __syncthreads();
    return next;
}

__device__ __forceinline__ void queue_done(uint32_t *queue)
{
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        __threadfence();
        if (atomicAdd(queue + 1, 1u) == gridDim.x - 1) {   // every block has taken its last tile
            atomicExch(queue, 0u);
            atomicExch(queue + 1, 0u);
        }
    }
}

template <int ROWS, int BY>
__global__ void __launch_bounds__(kC1BX * BY)
k_fused_c1_persistent(const agocuda_frame *frames, const uint32_t *tilePrefix, uint32_t numFrames, uint32_t *queue,
                      float tRound, float tTrunc)
{
    const uint32_t total = __ldg(tilePrefix + numFrames);
    for (;;) {
        const uint32_t t = queue_next(queue);
        if (t >= total) break;
        const uint32_t fi = frame_of_tile(tilePrefix, numFrames, t);
        const agocuda_frame f = frames[fi];
        const uint32_t local = t - __ldg(tilePrefix + fi);
        const uint32_t tilesX = (f.width + kC1BX * 8 - 1) / (kC1BX * 8);
        const int x = (int)((local % tilesX) * kC1BX + threadIdx.x) * 8;
        const int y0 = 2 + (int)((local / tilesX) * BY + threadIdx.y) * ROWS;
        c1_rows<ROWS>(f, x, y0, tRound, tTrunc);
    }
    queue_done(queue);
}

// ---------------------------------------------------------------------------------
// TMA-staged form of the chain.  A block of 32 x kC1tBY threads owns 256 columns x
// kC1tBY * kC1tRows output rows of one frame.  One thread copies the block's source box --
// columns x0-16 .. x0+271, rows y0-2 .. y0 + kC1tBY * kC1tRows + 1 -- into shared memory with
// one 2D tensor copy on an mbarrier: the plane is described to TMA as rows of 32-bit
// elements, so a single 72-element box spans the 264 columns the tile reads (a box
// dimension holds at most 256 elements); TMA writes zeros outside the plane.
//
// Each thread owns 8 columns and walks down kC1tRows rows.  The Gaussian stays in 16-bit
// lanes as in the register form; the Sobel and the threshold test run in exact fp32 on the
// FMA pipe instead of in lanes:
//   t  = 6144 + G * 2^-7       the masked 16G lane dropped into the mantissa of 6144 (one permute)
//   gx = [1 2 1]^T (t[c+1] - t[c-1]),  gy = [1 2 1] (t[r+1] - t[r-1])   = k * 2^-7, |k| <= 1020
//   r  = T - gx^2 - gy^2,  T = (n_min - 1/2) * 2^-14                   multiples of 2^-15, |r| < 2^8
// Every value is exact (t in [4096, 8192) has ulp 2^-11), so r < 0 <=> gx^2 + gy^2 >= n_min
// in integers, r is never 0, and the sign byte of r replicated by one permute is the
// output byte (255 where the chain's threshold passes).
// ---------------------------------------------------------------------------------
constexpr int kC1tRows = 36, kC1tBY = 2;              // default shape (rows per warp, warps per block)
constexpr int kC1tBoxW = 72;                            // 32-bit elements: 288 bytes per row
__host__ __device__ constexpr int c1t_box_h(int rows, int by) { return by * rows + 4; }
// resident blocks at 80 registers a thread (the launch bound of each shape)
__host__ __device__ constexpr int c1t_min_blocks(int by) { return 65536 / (32 * by * 80); }
constexpr int kC1tWaitLimit = 1 << 20;                  // bounded mbarrier waits

// t of the lo / hi 16-bit lane of a masked Gaussian word
__device__ __forceinline__ float c1_tlo(uint32_t w) { return __uint_as_float(__byte_perm(w, 0x45C00000u, 0x7610)); }
__device__ __forceinline__ float c1_thi(uint32_t w) { return __uint_as_float(__byte_perm(w, 0x45C00000u, 0x7632)); }

// t at columns x-1 .. x+8 from the lane words (x, x+2), (x+1, x+3), (x+4, x+6), (x+5, x+7), (x-1, x+8)
__device__ __forceinline__ void c1_tcols(const C1Row &g, float *t)
{
    t[0] = c1_tlo(g.b);  t[1] = c1_tlo(g.e1); t[2] = c1_tlo(g.o1); t[3] = c1_thi(g.e1); t[4] = c1_thi(g.o1);
    t[5] = c1_tlo(g.e2); t[6] = c1_tlo(g.o2); t[7] = c1_thi(g.e2); t[8] = c1_thi(g.o2); t[9] = c1_thi(g.b);
}

// bytes 0 and 1: 0xFF where a (resp. b) is negative, else 0 (prmt sign-replicate selectors)
__device__ __forceinline__ uint32_t c1_sign_pair(float a, float b)
{
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, 0xFFFB;" : "=r"(r) : "r"(__float_as_uint(a)), "r"(__float_as_uint(b)));
    return r;
}

// Output rows [ys, ye) of a thread's 8 columns at x (columns from W on are not stored), from
// hrow(y): the lane sums of source row y (rows ys-2 .. ye+1 are asked for once each, in order).
template <class HROW>
__device__ __forceinline__ void c1t_rows(HROW &hrow, int ys, int ye, int x, int W, uint8_t *dst, uint32_t dstStride,
                                         float T)
{
    // rolling rows of output row y: h of input rows y, y+1; t of rows y-1, y; d = t[c+1] - t[c-1]
    // of row y; D = d(y-1) + d(y); all rotated by the 6-way unrolled loop
    C1Row h0, h1, h2;
    float t0[10], t1[10], t2[10], d0[8], d1[8], D0[8], D1[8];
    {
        const C1Row a = hrow(ys - 2), c = hrow(ys - 1);
        h0 = hrow(ys);
        h1 = hrow(ys + 1);
        c1_tcols(c1_gauss(a, c, h0), t0);
        c1_tcols(c1_gauss(c, h0, h1), t1);
#pragma unroll
        for (int j = 0; j < 8; j++) {
            d0[j] = t1[j + 2] - t1[j];
            D0[j] = (t0[j + 2] - t0[j]) + d0[j];
        }
    }
    auto step = [&](int y, const C1Row &hA, const C1Row &hB, C1Row &hC, const float *tA, float *tC, const float *dB,
                    float *dC, const float *DA, float *DB) {
        hC = hrow(y + 2);
        c1_tcols(c1_gauss(hA, hB, hC), tC);               // t of row y+1
        float r[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            dC[j] = tC[j + 2] - tC[j];
            DB[j] = dB[j] + dC[j];
            const float gx = DA[j] + DB[j];
            const float e0 = tC[j] - tA[j], e1 = tC[j + 1] - tA[j + 1], e2 = tC[j + 2] - tA[j + 2];
            const float gy = __fmaf_rn(e1, 2.0f, e0) + e2;
            r[j] = __fmaf_rn(-gx, gx, __fmaf_rn(-gy, gy, T));
        }
        const uint32_t lo = __byte_perm(c1_sign_pair(r[0], r[1]), c1_sign_pair(r[2], r[3]), 0x5410);
        const uint32_t hi = __byte_perm(c1_sign_pair(r[4], r[5]), c1_sign_pair(r[6], r[7]), 0x5410);
        uint8_t *o = dst + (size_t)y * dstStride + x;
        if (x < W) *(uint32_t *)o = lo;
        if (x + 4 < W) *(uint32_t *)(o + 4) = hi;
    };
    for (int y = ys; y < ye; y += 6) {                    // y is uniform across the thread's loop
        step(y, h0, h1, h2, t0, t2, d0, d1, D0, D1);
        if (y + 1 >= ye) break;
        step(y + 1, h1, h2, h0, t1, t0, d1, d0, D1, D0);
        if (y + 2 >= ye) break;
        step(y + 2, h2, h0, h1, t2, t1, d0, d1, D0, D1);
        if (y + 3 >= ye) break;
        step(y + 3, h0, h1, h2, t0, t2, d1, d0, D1, D0);
        if (y + 4 >= ye) break;
        step(y + 4, h1, h2, h0, t1, t0, d0, d1, D0, D1);
        if (y + 5 >= ye) break;
        step(y + 5, h2, h0, h1, t2, t1, d1, d0, D1, D0);
    }
}

template <int ROWS, int BY>
__global__ void __launch_bounds__(32 * BY, c1t_min_blocks(BY))
k_fused_c1_tma(const agocuda_frame *__restrict__ frames, const CUtensorMap *__restrict__ maps, float tRound,
               float tTrunc, uint32_t *status)
{
    constexpr int kC1tBoxH = c1t_box_h(ROWS, BY), kC1tRows = ROWS, kC1tBY = BY;
    __shared__ __align__(128) uint32_t sm[kC1tBoxH * kC1tBoxW];
    __shared__ __align__(8) uint64_t bar;
    const int x0 = blockIdx.x * 256, y0 = 2 + blockIdx.y * (kC1tBY * kC1tRows);
    const int lane = threadIdx.x, tid = threadIdx.x + 32 * threadIdx.y;
    const uint32_t b = smem_addr_u32(&bar);
    // the copy is issued before the frame descriptor arrives (the box depends on the block
    // index only; a box outside a smaller frame of the batch reads zeros)
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(kC1tBoxH * kC1tBoxW * 4)
                     : "memory");
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
            ::"r"(smem_addr_u32(sm)), "l"((uint64_t)(maps + blockIdx.z)), "r"((x0 - 16) / 4), "r"(y0 - 2), "r"(b)
            : "memory");
    }
    const agocuda_frame f = frames[blockIdx.z];
    const int W = (int)f.width, H = (int)f.height;
    __syncthreads();                                      // the barrier is initialised
    bool done = false;
    for (int i = 0; i < kC1tWaitLimit && !done; i++) done = mbarrier_try_wait_parity(b, 0);
    if (!done) {
        // the copy did not complete: report it, give it one more bounded wait, leave
        if (tid == 0) atomicOr(status, AGOCUDA_C1_STATUS_TMA_TIMEOUT);
        for (int i = 0; i < kC1tWaitLimit && !done; i++) done = mbarrier_try_wait_parity(b, 0);
        return;
    }
    if (x0 >= W || y0 >= H - 2) return;                   // uniform over the block
    const int x = x0 + 8 * lane, ys = y0 + (int)threadIdx.y * kC1tRows, ye = min(ys + kC1tRows, H - 2);
    if (x >= W || ys >= ye) return;
    // T of the thread's 8 columns: all in the SIMD body or all in a scalar part (the span's
    // bounds are multiples of 8, checked when the tensor maps are made)
    const float T = (x < f.simdBegin || x >= f.simdEnd) ? tTrunc : tRound;
    // words of columns x-4 .. x+11 of source row yy: shared byte offset 12 + 8 lane in its box row
    const uint32_t *col = sm + 3 + 2 * lane - (y0 - 2) * kC1tBoxW;
    auto hrow = [&](int yy) {
        const uint32_t *p = col + yy * kC1tBoxW;
        const uint2 m = *(const uint2 *)(p + 1);
        return c1_hsum(p[0], m.x, m.y, p[3]);
    };
    c1t_rows(hrow, ys, ye, x, W, f.dst, f.dstStride, T);
}

unsigned long long g_launches = 0;

bool aligned(const void *p, unsigned a) { return ((uintptr_t)p & (a - 1)) == 0; }

// Vector paths need the row base aligned to the word size, the stride a multiple of it
// and at least one full row of pixels.
bool bad_plane(const void *p, uint32_t stride, uint32_t W, unsigned bpp, unsigned word)
{
    return !p || !aligned(p, word) || (stride % word) || stride < W * bpp;
}

}  // namespace

uint64_t agocuda_count_launch(unsigned n) { return __atomic_add_fetch(&g_launches, n, __ATOMIC_RELAXED); }

extern "C" uint64_t agocuda_launch_count(void) { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }
extern "C" int agocuda_abi_version(void) { return 100; }

static dim3 stencil_grid(uint32_t W, uint32_t rows)
{
    return dim3(div_up(W, kBX * 4), div_up(rows, kBY * kRPT), 1);
}

extern "C" int agocuda_Sobel_S16S16_U8_3x3_GXY(void *stream, uint32_t W, uint32_t H, int16_t *pGx, uint32_t gxStride,
                                               int16_t *pGy, uint32_t gyStride, const uint8_t *pSrc, uint32_t srcStride)
{
    if (W < 3 || H < 3 || bad_plane(pGx, gxStride, W, 2, 8) || bad_plane(pGy, gyStride, W, 2, 8) ||
        bad_plane(pSrc, srcStride, W, 1, 4))
        return AGOCUDA_INVALID_PARAMS;
    k_sobel_gxy<<<stencil_grid(W, H - 2), dim3(kBX, kBY), 0, as_stream(stream)>>>((int)W, (int)H, pGx, (int)gxStride, pGy, (int)gyStride, pSrc, (int)srcStride);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_SobelMagnitude_S16_U8_3x3(void *stream, uint32_t W, uint32_t H, int16_t *pDst, uint32_t dstStride,
                                                 const uint8_t *pSrc, uint32_t srcStride)
{
    if (W < 3 || H < 3 || bad_plane(pDst, dstStride, W, 2, 8) || bad_plane(pSrc, srcStride, W, 1, 4))
        return AGOCUDA_INVALID_PARAMS;
    SimdSpan sp = haf_simd_span((const uint8_t *)pDst + dstStride, (int)W);
    k_sobel_magnitude<<<stencil_grid(W, H - 2), dim3(kBX, kBY), 0, as_stream(stream)>>>((int)W, (int)H, pDst, (int)dstStride, pSrc, (int)srcStride, sp.begin, sp.end);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_Magnitude_S16_S16S16(void *stream, uint32_t W, uint32_t H, int16_t *pMag, uint32_t magStride,
                                            const int16_t *pGx, uint32_t gxStride, const int16_t *pGy, uint32_t gyStride)
{
    if (!W || !H || bad_plane(pMag, magStride, W, 2, 8) || bad_plane(pGx, gxStride, W, 2, 8) ||
        bad_plane(pGy, gyStride, W, 2, 8))
        return AGOCUDA_INVALID_PARAMS;
    // HafCpu_Magnitude_S16_S16S16 (ago_haf_cpu_arithmetic.cpp:4989): prefix in pixels
    // from the destination's 16-byte misalignment, 8-wide SIMD body.
    int prefix = (int)((uintptr_t)pMag & 15);
    prefix = (prefix ? 16 - prefix : 0) >> 1;
    int tail = (int)W - (((int)W - prefix) & 7);
    dim3 blk(32, 8);
    dim3 grd(div_up(W, 128), div_up(H, 8));
    k_magnitude<<<grd, blk, 0, as_stream(stream)>>>((int)W, (int)H, pMag, (int)magStride, pGx, (int)gxStride, pGy, (int)gyStride, prefix, tail);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_ColorDepth_U8_S16_Sat(void *stream, uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                             const int16_t *pSrc, uint32_t srcStride, int32_t shift)
{
    if (!W || !H || bad_plane(pDst, dstStride, W, 1, 4) || bad_plane(pSrc, srcStride, W, 2, 8) ||
        shift < 0 || shift > 15)
        return AGOCUDA_INVALID_PARAMS;
    dim3 blk(32, 8);
    dim3 grd(div_up(W, 128), div_up(H, 8));
    k_colordepth_u8_s16_sat<<<grd, blk, 0, as_stream(stream)>>>((int)W, (int)H, pDst, (int)dstStride, pSrc, (int)srcStride, shift);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_fused_GaussSobelMagDepthThresh(void *stream, const agocuda_frame *frames, uint32_t numFrames,
                                                      uint32_t maxWidth, uint32_t maxHeight, int32_t shift, int32_t threshold)
{
    if (!frames || !numFrames || numFrames > 65535 || maxWidth < 5 || maxHeight < 5 || shift < 0 || shift > 15)
        return AGOCUDA_INVALID_PARAMS;
    const int t = (int)(uint8_t)threshold;
    // -256 n_min: (16 gx)^2 + (16 gy)^2 - 256 n_min >= 0 <=> gx^2 + gy^2 >= n_min.  A 3x3 Sobel
    // of a Gaussian has gx^2 + gy^2 <= 2 * 1020^2; thresholds beyond it never pass.
    const double kNever = -256.0 * 4194304.0;
    double tRound = kNever, tTrunc = kNever;
    if (t < 255) {
        long long M = (long long)(t + 1) << shift;
        if (M <= 2048) {
            tRound = -256.0 * (double)(M * M - M + 1);
            tTrunc = -256.0 * (double)(M * M);
        }
    }
    dim3 grd(div_up(maxWidth, kC1BX * 8), div_up(maxHeight - 4, kC1BY * kC1Rows), numFrames);
    k_fused_gauss_sobelmag_thresh<<<grd, dim3(kC1BX, kC1BY), 0, as_stream(stream)>>>(frames, (float)tRound, (float)tTrunc);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

// ---- TMA-staged form
static void c1_thresholds(int32_t shift, int32_t threshold, float &tRound, float &tTrunc)
{
    // T = (n_min - 1/2) * 2^-14 (exact: n_min <= 2^22); never-passing thresholds get a T
    // above the largest gx^2 + gy^2 (2 * 1020^2 * 2^-14 < 128)
    const int t = (int)(uint8_t)threshold;
    tRound = tTrunc = 1024.0f;
    if (t < 255) {
        const long long M = (long long)(t + 1) << shift;
        if (M <= 2048) {
            tRound = (float)(((double)(M * M - M + 1) - 0.5) / 16384.0);
            tTrunc = (float)(((double)(M * M) - 0.5) / 16384.0);
        }
    }
}

extern "C" size_t agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_size(uint32_t numFrames)
{
    return (size_t)numFrames * sizeof(CUtensorMap);
}

// tile shapes of the TMA form (rows per warp, warps per block): the autotuner's space; a
// shape's box (BY * ROWS + 4 rows of 288 bytes) stays within 48 KB of static shared memory
#define C1T_SHAPES(X) X(18, 1) X(24, 1) X(36, 1) X(48, 1) X(18, 2) X(24, 2) X(36, 2) X(48, 2) X(18, 4) X(24, 4) X(36, 4)

static bool c1t_shape_ok(uint32_t rows, uint32_t warps)
{
#define C1T_OK(R, B) if (rows == R && warps == B) return true;
    C1T_SHAPES(C1T_OK)
#undef C1T_OK
    return false;
}

extern "C" int agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_shape(const agocuda_frame *framesHost,
                                                                       uint32_t numFrames, uint32_t rowsPerWarp,
                                                                       uint32_t warpsPerBlock, void *mapsHost,
                                                                       size_t mapsBytes)
{
    if (!framesHost || !numFrames || !mapsHost || ((uintptr_t)mapsHost & 63) || !c1t_shape_ok(rowsPerWarp, warpsPerBlock) ||
        mapsBytes < agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_size(numFrames))
        return AGOCUDA_INVALID_PARAMS;
    const uint32_t boxH = (uint32_t)c1t_box_h((int)rowsPerWarp, (int)warpsPerBlock);
    CUtensorMap *maps = (CUtensorMap *)mapsHost;
    memset(maps, 0, agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_size(numFrames));
    for (uint32_t i = 0; i < numFrames; i++) {
        const agocuda_frame &f = framesHost[i];
        if (f.width < 5 || f.height < 5 || (f.simdBegin & 7) || (f.simdEnd & 7) ||
            !agocuda_u8_as_u32_tensor_map(&maps[i], f.src, f.width, f.height, f.srcStride, kC1tBoxW, boxH))
            return AGOCUDA_INVALID_PARAMS;
    }
    return 0;
}

extern "C" int agocuda_fused_GaussSobelMagDepthThresh_tensor_maps(const agocuda_frame *framesHost, uint32_t numFrames,
                                                                 void *mapsHost, size_t mapsBytes)
{
    return agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_shape(framesHost, numFrames, kC1tRows, kC1tBY, mapsHost,
                                                                    mapsBytes);
}

extern "C" int agocuda_fused_GaussSobelMagDepthThresh_tma_shape(void *stream, const agocuda_frame *frames,
                                                               const void *maps, uint32_t numFrames, uint32_t maxWidth,
                                                               uint32_t maxHeight, int32_t shift, int32_t threshold,
                                                               uint32_t rowsPerWarp, uint32_t warpsPerBlock,
                                                               uint32_t *pStatus)
{
    if (!frames || !maps || ((uintptr_t)maps & 63) || !pStatus || !numFrames || numFrames > 65535 || maxWidth < 5 ||
        maxHeight < 5 || shift < 0 || shift > 15 || !c1t_shape_ok(rowsPerWarp, warpsPerBlock))
        return AGOCUDA_INVALID_PARAMS;
    float tRound, tTrunc;
    c1_thresholds(shift, threshold, tRound, tTrunc);
    cudaStream_t s = as_stream(stream);
    const CUtensorMap *m = (const CUtensorMap *)maps;
#define C1T_LAUNCH(R, B)                                                                                           \
    if (rowsPerWarp == R && warpsPerBlock == B)                                                                    \
        k_fused_c1_tma<R, B><<<dim3(div_up(maxWidth, 256), div_up(maxHeight - 4, B * R), numFrames), dim3(32, B), 0, s>>>( \
            frames, m, tRound, tTrunc, pStatus);
    C1T_SHAPES(C1T_LAUNCH)
#undef C1T_LAUNCH
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_fused_GaussSobelMagDepthThresh_tma(void *stream, const agocuda_frame *frames, const void *maps,
                                                         uint32_t numFrames, uint32_t maxWidth, uint32_t maxHeight,
                                                         int32_t shift, int32_t threshold, uint32_t *pStatus)
{
    return agocuda_fused_GaussSobelMagDepthThresh_tma_shape(stream, frames, maps, numFrames, maxWidth, maxHeight, shift,
                                                           threshold, kC1tRows, kC1tBY, pStatus);
}

// ---- persistent form and its tuning space
static bool c1_shape_ok(uint32_t rows, uint32_t warps)
{
    return (rows == 6 || rows == 12 || rows == 18 || rows == 24) && (warps == 2 || warps == 4 || warps == 8);
}

extern "C" uint32_t agocuda_fused_GaussSobelMagDepthThresh_tiles(uint32_t W, uint32_t H, uint32_t rowsPerThread,
                                                                uint32_t warpsPerBlock)
{
    if (!c1_shape_ok(rowsPerThread, warpsPerBlock) || W < 5 || H < 5) return 0;
    return div_up(W, kC1BX * 8) * div_up(H - 4, warpsPerBlock * rowsPerThread);
}

template <int ROWS, int BY>
static cudaError_t c1_launch(cudaStream_t s, unsigned blocks, const agocuda_frame *frames, const uint32_t *prefix,
                             uint32_t n, uint32_t *queue, float tR, float tT)
{
    k_fused_c1_persistent<ROWS, BY><<<blocks, dim3(kC1BX, BY), 0, s>>>(frames, prefix, n, queue, tR, tT);
    return cudaPeekAtLastError();
}

extern "C" int agocuda_fused_GaussSobelMagDepthThresh_persistent(void *stream, const agocuda_frame *frames,
                                                                 uint32_t numFrames, const uint32_t *tilePrefix,
                                                                 uint32_t *queue, uint32_t rowsPerThread,
                                                                 uint32_t warpsPerBlock, uint32_t blocksPerSM,
                                                                 int32_t shift, int32_t threshold)
{
    if (!frames || !tilePrefix || !queue || !numFrames || !c1_shape_ok(rowsPerThread, warpsPerBlock) || !blocksPerSM ||
        blocksPerSM > 32 || shift < 0 || shift > 15 || ((uintptr_t)queue & 7))
        return AGOCUDA_INVALID_PARAMS;
    const int t = (int)(uint8_t)threshold;
    const double kNever = -256.0 * 4194304.0;
    double tRound = kNever, tTrunc = kNever;
    if (t < 255) {
        long long M = (long long)(t + 1) << shift;
        if (M <= 2048) {
            tRound = -256.0 * (double)(M * M - M + 1);
            tTrunc = -256.0 * (double)(M * M);
        }
    }
    const unsigned blocks = (unsigned)agocuda_sm_count() * blocksPerSM;
    cudaStream_t s = as_stream(stream);
    const float tR = (float)tRound, tT = (float)tTrunc;
    cudaError_t e = cudaErrorInvalidValue;
#define C1_CASE(R, B) \
    if (rowsPerThread == R && warpsPerBlock == B) e = c1_launch<R, B>(s, blocks, frames, tilePrefix, numFrames, queue, tR, tT);
    C1_CASE(6, 2) C1_CASE(6, 4) C1_CASE(6, 8) C1_CASE(12, 2) C1_CASE(12, 4) C1_CASE(12, 8)
    C1_CASE(18, 2) C1_CASE(18, 4) C1_CASE(18, 8) C1_CASE(24, 2) C1_CASE(24, 4) C1_CASE(24, 8)
#undef C1_CASE
    agocuda_count_launch(1);
    return e == cudaSuccess ? agocuda_launch_status() : (int)e;
}
