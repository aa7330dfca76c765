// warp.cu -- WarpPerspective (nearest / bilinear, constant border) and Remap (nearest /
// bilinear, constant and undefined border) on sm_100a, bit-identical to the reference CPU
// kernels ago_haf_cpu_geometric.cpp:1406 / :1579 (perspective) and :72 / :156 / :249 / :372
// (remap).
//
// The reference addresses source taps through a flat byte offset y*pitch + x over AGO's
// buffer (pitch ALIGN16(width), zero padding) and clamps that offset; taps next to a clamped
// or out-of-row offset land in padding or the neighbouring row.  src_tap() resolves a flat
// offset of that layout onto this buffer (any pitch), so border behaviour matches.  Float
// arithmetic keeps the reference's operation order with explicit round-to-nearest intrinsics.
#include "agocuda_internal.cuh"

uint64_t agocuda_count_launch(unsigned n);

namespace {

struct SrcImg {
    const uint8_t *p;
    int stride;          // this buffer's row pitch
    int W, H;
    int pitch;           // AGO row pitch, ALIGN16(W)
};

// byte at flat offset f of the AGO layout (f >= 0): padding and rows past the image read 0
__device__ __forceinline__ uint32_t src_tap(const SrcImg &s, long long f)
{
    const long long r = f / s.pitch, c = f - r * s.pitch;
    return (r < s.H && c < s.W) ? s.p[(size_t)r * s.stride + c] : 0u;
}

// _mm_cvttps_epi32: truncation; NaN and out-of-range values give 0x80000000
__device__ __forceinline__ int32_t cvtt(float f)
{
    return (f >= -2147483648.0f && f < 2147483648.0f) ? __float2int_rz(f) : INT32_MIN;
}

// _mm_packus_epi32 followed by _mm_packus_epi16, one lane
__device__ __forceinline__ uint8_t pack_u8(int32_t v)
{
    const int32_t u16 = v < 0 ? 0 : (v > 65535 ? 65535 : v);
    const int32_t s16 = (int16_t)(uint16_t)u16;
    return (uint8_t)(s16 < 0 ? 0 : (s16 > 255 ? 255 : s16));
}

struct Persp { float a, d, g, b, e, h, c, f, i; };

template <bool BILINEAR>
__global__ void k_warp_perspective(int W, int H, uint8_t *dst, int ds, SrcImg s, Persp m, int border)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const float fy = (float)y, fx = (float)x;
    const float xd = __fadd_rn(__fmul_rn(fy, m.b), m.c), yd = __fadd_rn(__fmul_rn(fy, m.e), m.f);
    const float zd = __fadd_rn(__fmul_rn(fy, m.h), m.i);
    const float z = __fdiv_rn(1.0f, __fadd_rn(__fmul_rn(m.g, fx), zd));
    const float xm = __fmul_rn(__fadd_rn(__fmul_rn(m.a, fx), xd), z);
    const float ym = __fmul_rn(__fadd_rn(__fmul_rn(m.d, fx), yd), z);
    const int32_t srcb = s.H * s.pitch - 1;
    uint8_t out;
    if (!BILINEAR) {
        const bool ok = xm >= 0.f && xm < (float)s.W && ym >= 0.f && ym < (float)s.H;
        int32_t off = (int32_t)((uint32_t)cvtt(ym) * (uint32_t)s.pitch + (uint32_t)cvtt(xm));
        off = off > srcb ? srcb : (off < 0 ? 0 : off);
        out = ok ? (uint8_t)src_tap(s, off) : (uint8_t)border;
    } else {
        const int32_t xi = (int32_t)((uint32_t)cvtt(xm) - (uint32_t)(xm < 0.f));
        const int32_t yi = (int32_t)((uint32_t)cvtt(ym) - (uint32_t)(ym < 0.f));
        const bool ok = xi >= 0 && xi < s.W && yi >= 0 && yi < s.H;
        const bool ok1 = xi >= -1 && xi < s.W && yi >= -1 && yi < s.H;
        const float fxr = __fsub_rn(xm, (float)xi), fyr = __fsub_rn(ym, (float)yi);
        int32_t off = (int32_t)((uint32_t)yi * (uint32_t)s.pitch + (uint32_t)xi);
        off = off > srcb ? srcb : (off < 0 ? 0 : off);
        const float p0 = ok ? (float)src_tap(s, off) : (float)border;
        const float p2 = ok ? (float)src_tap(s, (long long)off + s.pitch) : (float)border;
        const float p1 = ok1 ? (float)src_tap(s, (long long)off + 1) : (float)border;
        const float p3 = ok1 ? (float)src_tap(s, (long long)off + s.pitch + 1) : (float)border;
        const float omx = __fsub_rn(1.0f, fxr), omy = __fsub_rn(1.0f, fyr);
        const float s0 = __fmul_rn(__fmul_rn(p0, omx), omy), s1 = __fmul_rn(__fmul_rn(p1, fxr), omy);
        const float s2 = __fmul_rn(__fmul_rn(p2, omx), fyr), s3 = __fmul_rn(__fmul_rn(p3, fxr), fyr);
        out = pack_u8(cvtt(__fadd_rn(__fadd_rn(__fadd_rn(s0, s1), s2), s3)));
    }
    dst[(size_t)y * ds + x] = out;
}

// Remap table entries: u16 x in the low half, u16 y in the high half, 3 fractional bits,
// 0xFFFF = outside the source.
template <bool CONSTANT>
__global__ void k_remap_bilinear(int W, int H, uint8_t *dst, int ds, SrcImg s, const uint32_t *map, int mapStride,
                                 int border)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const uint32_t e = map[(size_t)y * mapStride + x];
    uint32_t mx = e & 0xFFFF, my = e >> 16;
    const bool bx = mx == 0xFFFF, by = my == 0xFFFF;
    if (bx) mx = CONSTANT ? 0 : 8;
    if (by) my = CONSTANT ? 0 : 8;
    const uint32_t fx = mx & 7, fy = my & 7;
    const long long f = (long long)(my >> 3) * s.pitch + (mx >> 3);
    const uint32_t v = (src_tap(s, f) * (8 - fx) * (8 - fy) + src_tap(s, f + 1) * fx * (8 - fy) +
                        src_tap(s, f + s.pitch) * (8 - fx) * fy + src_tap(s, f + s.pitch + 1) * fx * fy + 32) >> 6;
    dst[(size_t)y * ds + x] = (CONSTANT && bx) ? (uint8_t)border : pack_u8((int32_t)v);
}

// The reference's 4-pixel SIMD body (x < W & ~3) and scalar tail treat 0xFFFF differently.
template <bool CONSTANT>
__global__ void k_remap_nearest(int W, int H, uint8_t *dst, int ds, SrcImg s, const uint32_t *map, int mapStride,
                                int border)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const uint32_t e = map[(size_t)y * mapStride + x];
    const long long srcb = (long long)s.H * s.pitch - 1;
    uint8_t out;
    if (x < (W & ~3)) {
        uint32_t mx = e & 0xFFFF, my = e >> 16;
        const bool bx = mx == 0xFFFF, by = my == 0xFFFF;
        if (bx) mx = CONSTANT ? 0 : 7;
        if (by) my = CONSTANT ? 0 : 7;
        const long long ix = (mx >> 3) + ((mx & 7) > 3), iy = (my >> 3) + ((my & 7) > 3);
        const long long off = iy * s.pitch + ix;
        out = (CONSTANT && (bx || by || off > srcb)) ? (uint8_t)border : (uint8_t)src_tap(s, off);
    } else {
        const int16_t sx = (int16_t)(e & 0xFFFF), sy = (int16_t)(e >> 16);
        const int xx = sx != -1 ? (sx >> 3) + ((sx & 7) >> 2) : (CONSTANT ? border : 0);
        const int yy = sy != -1 ? (sy >> 3) + ((sy & 7) >> 2) : (CONSTANT ? border : 0);
        const long long off = (long long)yy * s.pitch + xx;
        out = (off >= 0 && off <= srcb) ? (uint8_t)src_tap(s, off) : 0;
    }
    dst[(size_t)y * ds + x] = out;
}

bool geometry_ok(uint32_t W, uint32_t H, const void *dst, uint32_t ds, uint32_t sW, uint32_t sH, const void *src,
                 uint32_t ss)
{
    return dst && src && W && H && sW && sH && ds >= W && ss >= sW && sW < 32768 && sH < 32768 && W < 65536 &&
           H < 65536;
}

SrcImg src_img(const uint8_t *p, uint32_t ss, uint32_t sW, uint32_t sH)
{
    return SrcImg{p, (int)ss, (int)sW, (int)sH, (int)((sW + 15) & ~15u)};
}

int launch_perspective(bool bilinear, void *stream, uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                       uint32_t srcW, uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride, const float *m,
                       uint8_t border)
{
    if (!m || !geometry_ok(W, H, pDst, dstStride, srcW, srcH, pSrc, srcStride)) return AGOCUDA_INVALID_PARAMS;
    const Persp p{m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8]};
    const dim3 grd(div_up(W, 128), H);
    const SrcImg s = src_img(pSrc, srcStride, srcW, srcH);
    if (bilinear) k_warp_perspective<true><<<grd, 128, 0, as_stream(stream)>>>((int)W, (int)H, pDst, (int)dstStride, s, p, border);
    else k_warp_perspective<false><<<grd, 128, 0, as_stream(stream)>>>((int)W, (int)H, pDst, (int)dstStride, s, p, border);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

int launch_remap(bool bilinear, bool constant, void *stream, uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                 uint32_t srcW, uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride, const uint32_t *pMap,
                 uint32_t mapStride, uint8_t border)
{
    if (!pMap || (mapStride & 3) || mapStride < 4 * W || !geometry_ok(W, H, pDst, dstStride, srcW, srcH, pSrc, srcStride))
        return AGOCUDA_INVALID_PARAMS;
    const dim3 grd(div_up(W, 128), H);
    const SrcImg s = src_img(pSrc, srcStride, srcW, srcH);
    const int ms = (int)(mapStride / 4);
    cudaStream_t q = as_stream(stream);
    if (bilinear && constant) k_remap_bilinear<true><<<grd, 128, 0, q>>>((int)W, (int)H, pDst, (int)dstStride, s, pMap, ms, border);
    else if (bilinear) k_remap_bilinear<false><<<grd, 128, 0, q>>>((int)W, (int)H, pDst, (int)dstStride, s, pMap, ms, 0);
    else if (constant) k_remap_nearest<true><<<grd, 128, 0, q>>>((int)W, (int)H, pDst, (int)dstStride, s, pMap, ms, border);
    else k_remap_nearest<false><<<grd, 128, 0, q>>>((int)W, (int)H, pDst, (int)dstStride, s, pMap, ms, 0);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

}  // namespace

extern "C" int agocuda_WarpPerspective_U8_U8_Nearest_Constant(void *stream, uint32_t W, uint32_t H, uint8_t *pDst,
                                                              uint32_t dstStride, uint32_t srcW, uint32_t srcH,
                                                              const uint8_t *pSrc, uint32_t srcStride,
                                                              const float *perspectiveMatrix, uint8_t border)
{
    return launch_perspective(false, stream, W, H, pDst, dstStride, srcW, srcH, pSrc, srcStride, perspectiveMatrix, border);
}

extern "C" int agocuda_WarpPerspective_U8_U8_Bilinear_Constant(void *stream, uint32_t W, uint32_t H, uint8_t *pDst,
                                                               uint32_t dstStride, uint32_t srcW, uint32_t srcH,
                                                               const uint8_t *pSrc, uint32_t srcStride,
                                                               const float *perspectiveMatrix, uint8_t border)
{
    return launch_perspective(true, stream, W, H, pDst, dstStride, srcW, srcH, pSrc, srcStride, perspectiveMatrix, border);
}

extern "C" int agocuda_Remap_U8_U8_Nearest(void *stream, uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                           uint32_t srcW, uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride,
                                           const uint32_t *pMap, uint32_t mapStride)
{
    return launch_remap(false, false, stream, W, H, pDst, dstStride, srcW, srcH, pSrc, srcStride, pMap, mapStride, 0);
}

extern "C" int agocuda_Remap_U8_U8_Nearest_Constant(void *stream, uint32_t W, uint32_t H, uint8_t *pDst,
                                                    uint32_t dstStride, uint32_t srcW, uint32_t srcH,
                                                    const uint8_t *pSrc, uint32_t srcStride, const uint32_t *pMap,
                                                    uint32_t mapStride, uint8_t border)
{
    return launch_remap(false, true, stream, W, H, pDst, dstStride, srcW, srcH, pSrc, srcStride, pMap, mapStride, border);
}

extern "C" int agocuda_Remap_U8_U8_Bilinear(void *stream, uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                            uint32_t srcW, uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride,
                                            const uint32_t *pMap, uint32_t mapStride)
{
    return launch_remap(true, false, stream, W, H, pDst, dstStride, srcW, srcH, pSrc, srcStride, pMap, mapStride, 0);
}

extern "C" int agocuda_Remap_U8_U8_Bilinear_Constant(void *stream, uint32_t W, uint32_t H, uint8_t *pDst,
                                                     uint32_t dstStride, uint32_t srcW, uint32_t srcH,
                                                     const uint8_t *pSrc, uint32_t srcStride, const uint32_t *pMap,
                                                     uint32_t mapStride, uint8_t border)
{
    return launch_remap(true, true, stream, W, H, pDst, dstStride, srcW, srcH, pSrc, srcStride, pMap, mapStride, border);
}
