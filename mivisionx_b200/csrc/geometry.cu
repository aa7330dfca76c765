// geometry.cu -- colour conversion RGB -> NV12 / IYUV, ScaleImage (nearest, bilinear,
// area) and WarpAffine (nearest / bilinear, constant border) on sm_100a, plus the fused
// RGB -> {NV12, IYUV, half-size bilinear Y, half-size area Y} kernel.
//
// Float arithmetic keeps the reference's operation order with explicit round-to-nearest
// intrinsics (no contraction), so results are bit-identical to the SSE code.
#include "agocuda_internal.cuh"

uint64_t agocuda_count_launch(unsigned n);

namespace {

__device__ __forceinline__ int ago_px8(const uint8_t *src, int stride, int W, int H, int x, int y)
{
    // pixel as the reference reads it, including one byte past a row (see vision.cu)
    if ((unsigned)y >= (unsigned)H) return 0;
    if (x >= 0 && x < W) return src[(size_t)y * stride + x];
    const bool tight = (W & 15) == 0;
    if (x == -1) return (tight && y > 0) ? src[(size_t)(y - 1) * stride + W - 1] : 0;
    if (x == W) return (tight && y + 1 < H) ? src[(size_t)(y + 1) * stride] : 0;
    return 0;
}

// ------------------------------------------------------------------------------------
// colour conversion (HafCpu_ColorConvert_NV12_RGB color_convert.cpp:2707,
// HafCpu_ColorConvert_IYUV_RGB :2492)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void rgb_yuv(int R, int G, int B, float &y, float &u, float &v)
{
    const float r = (float)R, g = (float)G, b = (float)B;
    y = __fadd_rn(__fadd_rn(__fmul_rn(r, 0.2126f), __fmul_rn(g, 0.7152f)), __fmul_rn(b, 0.0722f));
    u = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(r, -0.1146f), __fmul_rn(g, -0.3854f)), __fmul_rn(b, 0.5f)), 128.0f);
    v = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(r, 0.5f), __fmul_rn(g, -0.4542f)), __fmul_rn(b, -0.0458f)), 128.0f);
}

__device__ __forceinline__ int trunc_sat16(float f)
{
    const int i = __float2int_rz(f);
    return i < 0 ? 0 : (i > 65535 ? 65535 : i);
}

__device__ __forceinline__ int sat8(int v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }

// 2x2 block: the four Y values and the shared U, V.  `simd` selects the SSE body
// arithmetic (x < W & ~3), otherwise the scalar tail's (float sum / 4, double 0.0722).
__device__ __forceinline__ void rgb_block(const int (&px)[4][3], bool simd, int (&y)[4], int &U, int &V)
{
    if (simd) {
        int uu[4], vv[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            float fy, fu, fv;
            rgb_yuv(px[i][0], px[i][1], px[i][2], fy, fu, fv);
            y[i] = sat8(trunc_sat16(fy));
            uu[i] = trunc_sat16(fu);
            vv[i] = trunc_sat16(fv);
        }
        const int ua = (uu[0] + uu[2] + 1) >> 1, ub = (uu[1] + uu[3] + 1) >> 1;
        const int va = (vv[0] + vv[2] + 1) >> 1, vb = (vv[1] + vv[3] + 1) >> 1;
        U = sat8((ua + ub + 1) >> 1);
        V = sat8((va + vb + 1) >> 1);
    } else {
        float u = 0.f, v = 0.f;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float R = (float)px[i][0], G = (float)px[i][1], B = (float)px[i][2];
            const float rg = __fadd_rn(__fmul_rn(R, 0.2126f), __fmul_rn(G, 0.7152f));
            y[i] = (int)(uint8_t)__double2int_rz(__dadd_rn((double)rg, __dmul_rn((double)B, 0.0722)));
            const float uu = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(R, -0.1146f), __fmul_rn(G, -0.3854f)), __fmul_rn(B, 0.5f)), 128.0f);
            const float vv = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(R, 0.5f), __fmul_rn(G, -0.4542f)), __fmul_rn(B, -0.0458f)), 128.0f);
            u = i ? __fadd_rn(u, uu) : uu;
            v = i ? __fadd_rn(v, vv) : vv;
        }
        U = (int)(uint8_t)__float2int_rz(__fdiv_rn(u, 4.0f));
        V = (int)(uint8_t)__float2int_rz(__fdiv_rn(v, 4.0f));
    }
}

// one thread per 2x2 block; planes: Y (full), then either interleaved UV or U and V
__global__ void k_color_rgb_yuv420(int W, int H, const uint8_t *src, int ss, uint8_t *py, int ys, uint8_t *puv, int uvs,
                                   uint8_t *pu, int us, uint8_t *pv, int vs)
{
    const int bx = blockIdx.x * blockDim.x + threadIdx.x, by = blockIdx.y * blockDim.y + threadIdx.y;
    const int x = 2 * bx, y = 2 * by;
    if (x >= W || y >= H) return;
    int px[4][3];
    const uint8_t *s0 = src + (size_t)y * ss + 3 * x, *s1 = s0 + ss;
#pragma unroll
    for (int c = 0; c < 3; c++) { px[0][c] = s0[c]; px[1][c] = s0[3 + c]; px[2][c] = s1[c]; px[3][c] = s1[3 + c]; }
    int yy[4], U, V;
    rgb_block(px, x < (W & ~3), yy, U, V);
    uint8_t *y0 = py + (size_t)y * ys + x;
    y0[0] = (uint8_t)yy[0]; y0[1] = (uint8_t)yy[1]; y0[ys] = (uint8_t)yy[2]; y0[ys + 1] = (uint8_t)yy[3];
    if (puv) { uint8_t *c = puv + (size_t)by * uvs + x; c[0] = (uint8_t)U; c[1] = (uint8_t)V; }
    if (pu) pu[(size_t)by * us + bx] = (uint8_t)U;
    if (pv) pv[(size_t)by * vs + bx] = (uint8_t)V;
}

// ------------------------------------------------------------------------------------
// ScaleImage (ago_haf_cpu_geometric.cpp:1874 nearest, :1977 bilinear, :2491 area)
// ------------------------------------------------------------------------------------
struct ScaleParams { int xinc, yinc, xoffs, yoffs; float xscale, yscale, xoffset, yoffset; };

__global__ void k_scale_nearest(int W, int H, uint8_t *dst, int ds, int sW, int sH, const uint8_t *src, int ss, ScaleParams p)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    int ym = (p.yoffs + y * p.yinc) >> 18, xm = (p.xoffs + x * p.xinc) >> 18;
    ym = ym > sH - 1 ? sH - 1 : (ym < 0 ? 0 : ym);
    xm = xm > sW - 1 ? sW - 1 : (xm < 0 ? 0 : xm);
    dst[(size_t)y * ds + x] = src[(size_t)ym * ss + xm];
}

__global__ void k_scale_bilinear(int W, int H, uint8_t *dst, int ds, int sW, int sH, const uint8_t *src, int ss, ScaleParams p)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const int ypos = p.yoffs + y * p.yinc, xpos = p.xoffs + x * p.xinc;
    int ym = ypos >> 18;
    const int yf = ((ypos & 0x3ffff) + 0x200) >> 10, omy = 0x100 - yf;
    int r1, r2;
    if (ym < 0) r1 = r2 = 0;
    else if (ym >= sH - 1) r1 = r2 = sH - 1;
    else { r1 = ym; r2 = ym + 1; }
    int xm = xpos >> 18;
    if (xm < 0) xm = 0;
    const int xf = ((xpos & 0x3ffff) + 0x200) >> 10, omx = 0x100 - xf;
    const int p1 = ago_px8(src, ss, sW, sH, xm, r1), p2 = ago_px8(src, ss, sW, sH, xm + 1, r1);
    const int p3 = ago_px8(src, ss, sW, sH, xm, r2), p4 = ago_px8(src, ss, sW, sH, xm + 1, r2);
    int o;
    if (x < (W & ~7)) {
        const int t1 = ((((omx * p1) & 0xffff) + ((xf * p2) & 0xffff) + 0x80) & 0xffff) >> 8;
        const int t2 = ((((omx * p3) & 0xffff) + ((xf * p4) & 0xffff) + 0x80) & 0xffff) >> 8;
        o = sat8(((((omy * t1) & 0xffff) + ((yf * t2) & 0xffff) + 0x80) & 0xffff) >> 8);
    } else {
        o = ((omx * omy * p1) + (xf * omy * p2) + (omx * yf * p3) + (xf * yf * p4) + 0x8000) >> 16;
    }
    dst[(size_t)y * ds + x] = (uint8_t)o;
}

// exact 2x area path; columns beyond W & ~7 are not written (as in the reference)
__global__ void k_scale_area2x(int W, int H, uint8_t *dst, int ds, int sW, int sH, const uint8_t *src, int ss, ScaleParams p)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= (W & ~7)) return;
    int r = __float2int_rz(__fadd_rn(p.yoffset, (float)(y * 2)));
    r = r < 0 ? 0 : (r > sH - 2 ? sH - 2 : r);
    const int c = __float2int_rz(p.xoffset) + 2 * x;
    const uint8_t *s0 = src + (size_t)r * ss, *s1 = s0 + ss;
    dst[(size_t)y * ds + x] = (uint8_t)((s0[c] + s0[c + 1] + s1[c] + s1[c + 1] + 2) >> 2);
}

__global__ void k_scale_area1x(int W, int H, uint8_t *dst, int ds, int sW, int sH, const uint8_t *src, int ss, ScaleParams p)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    int r = __float2int_rz(__fadd_rn(p.yoffset, (float)y));
    r = r < 0 ? 0 : (r > H - 1 ? H - 1 : r);
    const int c = __float2int_rz(p.xoffset) + x;
    dst[(size_t)y * ds + x] = src[(size_t)r * ss + (c < 0 ? 0 : c)];
}

// ------------------------------------------------------------------------------------
// WarpAffine, constant border (geometric.cpp:658 nearest, :1100 bilinear)
// ------------------------------------------------------------------------------------
struct AffineParams {
    float r00, r10, r01, r11, c1, c2;
    int border, checkBorder;   // checkBorder: some mapped corner falls outside the source
    float vl, vr, vt, vb;      // source valid rectangle (nearest)
};

// Both warps: a thread owns 4 consecutive output pixels of a row (the reference's 4-pixel
// groups; W4 = W rounded up to 4), computes their source positions with the reference's
// float order, issues all source loads before using any, and stores the 4 bytes as one
// word when the destination allows it.
__device__ __forceinline__ void warp_store4(uint8_t *d, const int v[4], bool word)
{
    if (word) *(uint32_t *)d = (uint32_t)v[0] | ((uint32_t)v[1] << 8) | ((uint32_t)v[2] << 16) | ((uint32_t)v[3] << 24);
    else { d[0] = (uint8_t)v[0]; d[1] = (uint8_t)v[1]; d[2] = (uint8_t)v[2]; d[3] = (uint8_t)v[3]; }
}

__global__ void k_warp_affine_nearest(int W4, int H, uint8_t *dst, int ds, int sW, int sH, const uint8_t *src, int ss,
                                      AffineParams a)
{
    const int x0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x), y = blockIdx.y;
    if (x0 >= W4) return;
    const float xd = __fadd_rn(__fmul_rn((float)y, a.r01), a.c1), yd = __fadd_rn(__fmul_rn((float)y, a.r11), a.c2);
    const long long lim = (long long)sH * ss - 1;
    long long idx[4];
    bool ok[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int x = x0 + k;
        const float xs = __fadd_rn(__fmul_rn(a.r00, (float)x), xd), ys = __fadd_rn(__fmul_rn(a.r10, (float)x), yd);
        idx[k] = (long long)__float2int_rz(ys) * ss + __float2int_rz(xs);
        ok[k] = true;
        if (a.checkBorder) {
            ok[k] = xs >= 0.f && xs < (float)sW && ys >= 0.f && ys < (float)sH && xs >= a.vl && xs < a.vr &&
                    ys >= a.vt && ys < a.vb;
            idx[k] = idx[k] > lim ? lim : (idx[k] < 0 ? 0 : idx[k]);
        }
    }
    int v[4];
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] = src[idx[k]];
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] = ok[k] ? v[k] : a.border;
    uint8_t *d = dst + (size_t)y * ds + x0;
    warp_store4(d, v, ((uintptr_t)d & 3) == 0);
}

// taps (x, y), (x+1, y), (x, y+1), (x+1, y+1) of the flat index the reference forms
struct BilinearTap { const uint8_t *p; int px, py; bool direct; };

__global__ void k_warp_affine_bilinear(int W4, int H, uint8_t *dst, int ds, int sW, int sH, const uint8_t *src, int ss,
                                       AffineParams a)
{
    const int x0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x), y = blockIdx.y;
    if (x0 >= W4) return;
    const float xd = __fadd_rn(__fmul_rn((float)y, a.r01), a.c1), yd = __fadd_rn(__fmul_rn((float)y, a.r11), a.c2);
    const long long lim = (long long)sH * ss - 1;
    float fx[4], fy[4];
    bool ok[4];
    BilinearTap t[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int x = x0 + k;
        const float xs = __fadd_rn(__fmul_rn(a.r00, (float)x), xd), ys = __fadd_rn(__fmul_rn(a.r10, (float)x), yd);
        const int xi = __float2int_rz(xs), yi = __float2int_rz(ys);
        fx[k] = __fsub_rn(xs, (float)xi);
        fy[k] = __fsub_rn(ys, (float)yi);
        ok[k] = !a.checkBorder || (xs >= 0.f && xs < (float)sW && ys >= 0.f && ys < (float)sH);
        int py, pxx;
        if (!ok[k]) {                                          // outside the source: the border value, no reads
            py = 0; pxx = 0;
        } else if (yi >= 0 && yi < sH && xi >= 0 && xi < ss) { // flat index inside, no wrap
            py = yi; pxx = xi;
        } else {                                               // the reference clamps the flat index
            long long idx = (long long)yi * ss + xi;
            idx = idx > lim ? lim : (idx < 0 ? 0 : idx);
            py = (int)(idx / ss); pxx = (int)(idx - (long long)py * ss);
        }
        t[k].px = pxx; t[k].py = py;
        t[k].direct = pxx >= 0 && pxx + 1 < sW && py + 1 < sH;
        t[k].p = src + (size_t)py * ss + pxx;
    }
    int q[4][4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (!ok[k]) {
            q[k][0] = q[k][1] = q[k][2] = q[k][3] = 0;
        } else if (t[k].direct) {
            q[k][0] = t[k].p[0]; q[k][1] = t[k].p[1]; q[k][2] = t[k].p[ss]; q[k][3] = t[k].p[ss + 1];
        } else {   // the reference reads 4 bytes at the (clamped) index and at index + stride
            q[k][0] = ago_px8(src, ss, sW, sH, t[k].px, t[k].py);
            q[k][1] = ago_px8(src, ss, sW, sH, t[k].px + 1, t[k].py);
            q[k][2] = ago_px8(src, ss, sW, sH, t[k].px, t[k].py + 1);
            q[k][3] = ago_px8(src, ss, sW, sH, t[k].px + 1, t[k].py + 1);
        }
    }
    int v[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float omx = __fsub_rn(1.0f, fx[k]), omy = __fsub_rn(1.0f, fy[k]);
        const float f0 = __fmul_rn(__fmul_rn((float)q[k][0], omx), omy), f1 = __fmul_rn(__fmul_rn((float)q[k][1], fx[k]), omy);
        const float f2 = __fmul_rn(__fmul_rn((float)q[k][2], omx), fy[k]), f3 = __fmul_rn(__fmul_rn((float)q[k][3], fx[k]), fy[k]);
        const int val = __float2int_rn(__fadd_rn(__fadd_rn(f0, f1), __fadd_rn(f2, f3)));
        v[k] = sat8(ok[k] ? val : a.border);
    }
    uint8_t *d = dst + (size_t)y * ds + x0;
    warp_store4(d, v, ((uintptr_t)d & 3) == 0);
}

// ------------------------------------------------------------------------------------
// Fused: RGB -> NV12 (Y, UV) + IYUV (Y, U, V) + half-size bilinear and area scaling of Y
// in one pass.  A thread owns a 2x2 RGB block (one scaled output pixel) and also needs
// the Y row above its block for the area scaler's (int)(2y - 0.5) row choice.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ int rgb_y_simd(const uint8_t *p)
{
    float fy, fu, fv;
    rgb_yuv(p[0], p[1], p[2], fy, fu, fv);
    return sat8(trunc_sat16(fy));
}

__global__ void k_fused_rgb_yuv_scale(int W, int H, const uint8_t *src, int ss, uint8_t *y1, int y1s, uint8_t *uv, int uvs,
                                      uint8_t *y2, int y2s, uint8_t *pu, int us, uint8_t *pv, int vs,
                                      uint8_t *outB, int obs, uint8_t *outA, int oas)
{
    const int bx = blockIdx.x * blockDim.x + threadIdx.x, by = blockIdx.y * blockDim.y + threadIdx.y;
    const int x = 2 * bx, y = 2 * by;
    if (x >= W || y >= H) return;
    int px[4][3];
    const uint8_t *s0 = src + (size_t)y * ss + 3 * x, *s1 = s0 + ss;
#pragma unroll
    for (int c = 0; c < 3; c++) { px[0][c] = s0[c]; px[1][c] = s0[3 + c]; px[2][c] = s1[c]; px[3][c] = s1[3 + c]; }
    int yy[4], U, V;
    const bool simd = x < (W & ~3);
    rgb_block(px, simd, yy, U, V);
    uint8_t *a = y1 + (size_t)y * y1s + x, *b = y2 + (size_t)y * y2s + x;
    a[0] = b[0] = (uint8_t)yy[0]; a[1] = b[1] = (uint8_t)yy[1];
    a[y1s] = (uint8_t)yy[2]; a[y1s + 1] = (uint8_t)yy[3];
    b[y2s] = (uint8_t)yy[2]; b[y2s + 1] = (uint8_t)yy[3];
    uint8_t *c = uv + (size_t)by * uvs + x;
    c[0] = (uint8_t)U; c[1] = (uint8_t)V;
    pu[(size_t)by * us + bx] = (uint8_t)U;
    pv[(size_t)by * vs + bx] = (uint8_t)V;
    // bilinear 2x: rows 2y', 2y'+1, columns 2x', 2x'+1, weights 1/2 (xf = yf = 128): two
    // rounded stages in the SIMD body, one (sum*16384 + 0x8000) >> 16 stage in the tail
    if (bx < ((W / 2) & ~7)) {
        const int t1 = (yy[0] + yy[1] + 1) >> 1, t2 = (yy[2] + yy[3] + 1) >> 1;
        outB[(size_t)by * obs + bx] = (uint8_t)((t1 + t2 + 1) >> 1);
    } else {
        outB[(size_t)by * obs + bx] = (uint8_t)((yy[0] + yy[1] + yy[2] + yy[3] + 2) >> 2);
    }
    // area 2x: rows (int)(2y' - 0.5) = 2y' - 1 (0 for y' = 0) and the next one
    if (bx < ((W / 2) & ~7)) {
        int ya, yb;
        if (by == 0) { ya = yy[0] + yy[1]; yb = yy[2] + yy[3]; }
        else {
            const uint8_t *sp = src + (size_t)(y - 1) * ss + 3 * x;
            ya = simd ? rgb_y_simd(sp) + rgb_y_simd(sp + 3) : 0;
            if (!simd) {
                int q[4][3], qy[4], qu, qv;
                for (int cc = 0; cc < 3; cc++) { q[0][cc] = sp[cc]; q[1][cc] = sp[3 + cc]; q[2][cc] = sp[cc]; q[3][cc] = sp[3 + cc]; }
                rgb_block(q, false, qy, qu, qv);
                ya = qy[0] + qy[1];
            }
            yb = yy[0] + yy[1];
        }
        outA[(size_t)by * oas + bx] = (uint8_t)((ya + yb + 2) >> 2);
    }
}

// The same outputs with one thread per 8 columns (four 2x2 blocks) walking down kCsRows block
// rows: 64-bit loads of the 24 RGB bytes of each row and 64/32-bit stores of the planes where
// the group lies in the SIMD body (x + 8 <= W & ~3, buffers aligned), and the Y of the row
// above a block -- the area scaler's first row -- carried from the previous block row instead
// of recomputed.  The arithmetic of each block is rgb_block's, so outputs are identical.
//
// In the SIMD body Y, U and V lie in [0, 256) (the weights of Y are positive and sum to 1; U
// and V are at least 0.5), so trunc_sat16 and sat8 reduce to truncation, done as one
// round-toward-zero add of 2^23 on the FMA pipe instead of a conversion on the XU pipe: the
// word is 0x4B000000 + value.  The integer averages then run on those biased words (every
// bias term divides by the shift that follows, modulo 2^32) and the low bytes are packed.
constexpr int kCsRows = 8;
constexpr uint32_t kBias23 = 0x4B000000u;

__device__ __forceinline__ uint32_t trunc_b(float f) { return __float_as_uint(__fadd_rz(f, 8388608.0f)); }

// Y of one pixel as rgb_block computes it, as a biased word (low byte = Y)
__device__ __forceinline__ uint32_t rgb_y_b(int R, int G, int B, bool simd)
{
    if (simd) {
        float fy, fu, fv;
        rgb_yuv(R, G, B, fy, fu, fv);
        return trunc_b(fy);
    }
    const float rg = __fadd_rn(__fmul_rn((float)R, 0.2126f), __fmul_rn((float)G, 0.7152f));
    return kBias23 + (uint32_t)(uint8_t)__double2int_rz(__dadd_rn((double)rg, __dmul_rn((double)B, 0.0722)));
}

// rgb_block's SIMD body on biased words
__device__ __forceinline__ void rgb_block_b(const int (&px)[4][3], uint32_t (&y)[4], uint32_t &U, uint32_t &V)
{
    uint32_t uu[4], vv[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        float fy, fu, fv;
        rgb_yuv(px[i][0], px[i][1], px[i][2], fy, fu, fv);
        y[i] = trunc_b(fy);
        uu[i] = trunc_b(fu);
        vv[i] = trunc_b(fv);
    }
    const uint32_t ua = (uu[0] + uu[2] + 1) >> 1, ub = (uu[1] + uu[3] + 1) >> 1;
    const uint32_t va = (vv[0] + vv[2] + 1) >> 1, vb = (vv[1] + vv[3] + 1) >> 1;
    U = (ua + ub + 1) >> 1;
    V = (va + vb + 1) >> 1;
}

// the low bytes of four words
__device__ __forceinline__ uint32_t pack_lo4(uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
    return __byte_perm(__byte_perm(a, b, 0x0040), __byte_perm(c, d, 0x0040), 0x5410);
}

__global__ void __launch_bounds__(128)
k_fused_rgb_yuv_scale8(int W, int H, const uint8_t *src, int ss, uint8_t *y1, int y1s, uint8_t *uv, int uvs,
                       uint8_t *y2, int y2s, uint8_t *pu, int us, uint8_t *pv, int vs, uint8_t *outB, int obs,
                       uint8_t *outA, int oas)
{
    const int g = blockIdx.x * 32 + threadIdx.x, x = 8 * g, bx0 = 4 * g;
    const int by0 = (blockIdx.y * 4 + threadIdx.y) * kCsRows, nby = H / 2;
    if (x >= W || by0 >= nby) return;
    const int by1 = min(by0 + kCsRows, nby), simdEnd = W & ~3, scaleEnd = (W / 2) & ~7;
    const bool full = x + 8 <= simdEnd;         // four blocks, SIMD-body arithmetic, vector access
    const bool scaled = bx0 < scaleEnd;         // then all four blocks are below the bound (multiples of 4 / 8)
    const int nb = min(4, (W - x) / 2);         // blocks of the group inside the image (W even)
    uint32_t above[8];                          // Y of row 2 by - 1 (the area scaler's first row), biased
    if (scaled && by0 > 0) {
        const uint8_t *sp = src + (size_t)(2 * by0 - 1) * ss + 3 * x;
#pragma unroll
        for (int j = 0; j < 8; j++) above[j] = rgb_y_b(sp[3 * j], sp[3 * j + 1], sp[3 * j + 2], x + (j & ~1) < simdEnd);
    }
    // the 48 RGB bytes of a block row (full groups), loaded one block row ahead
    uint32_t na[6], nb6[6];
    auto load_rows = [&](int by) {
        const uint8_t *s0 = src + (size_t)(2 * by) * ss + 3 * x, *s1 = s0 + ss;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const uint2 va = *(const uint2 *)(s0 + 8 * k), vb = *(const uint2 *)(s1 + 8 * k);
            na[2 * k] = va.x; na[2 * k + 1] = va.y; nb6[2 * k] = vb.x; nb6[2 * k + 1] = vb.y;
        }
    };
    if (full) load_rows(by0);
    for (int by = by0; by < by1; by++) {
        const int yr = 2 * by;
        const uint8_t *s0 = src + (size_t)yr * ss + 3 * x, *s1 = s0 + ss;
        uint32_t yy[4][4], U[4], V[4];          // biased words
        if (full) {
            uint32_t a[6], b[6];
#pragma unroll
            for (int k = 0; k < 6; k++) { a[k] = na[k]; b[k] = nb6[k]; }
            if (by + 1 < by1) load_rows(by + 1);
            auto byteA = [&](int k) { return (int)((a[k >> 2] >> (8 * (k & 3))) & 0xff); };
            auto byteB = [&](int k) { return (int)((b[k >> 2] >> (8 * (k & 3))) & 0xff); };
#pragma unroll
            for (int i = 0; i < 4; i++) {
                int px[4][3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    px[0][c] = byteA(6 * i + c); px[1][c] = byteA(6 * i + 3 + c);
                    px[2][c] = byteB(6 * i + c); px[3][c] = byteB(6 * i + 3 + c);
                }
                rgb_block_b(px, yy[i], U[i], V[i]);
            }
            const uint2 r0 = make_uint2(pack_lo4(yy[0][0], yy[0][1], yy[1][0], yy[1][1]),
                                        pack_lo4(yy[2][0], yy[2][1], yy[3][0], yy[3][1]));
            const uint2 r1 = make_uint2(pack_lo4(yy[0][2], yy[0][3], yy[1][2], yy[1][3]),
                                        pack_lo4(yy[2][2], yy[2][3], yy[3][2], yy[3][3]));
            *(uint2 *)(y1 + (size_t)yr * y1s + x) = r0;
            *(uint2 *)(y1 + (size_t)(yr + 1) * y1s + x) = r1;
            *(uint2 *)(y2 + (size_t)yr * y2s + x) = r0;
            *(uint2 *)(y2 + (size_t)(yr + 1) * y2s + x) = r1;
            *(uint2 *)(uv + (size_t)by * uvs + x) = make_uint2(pack_lo4(U[0], V[0], U[1], V[1]), pack_lo4(U[2], V[2], U[3], V[3]));
            *(uint32_t *)(pu + (size_t)by * us + bx0) = pack_lo4(U[0], U[1], U[2], U[3]);
            *(uint32_t *)(pv + (size_t)by * vs + bx0) = pack_lo4(V[0], V[1], V[2], V[3]);
        } else {
            for (int i = 0; i < nb; i++) {
                const int xb = x + 2 * i;
                int px[4][3], y4[4], u1, v1;
                const uint8_t *p0 = s0 + 6 * i, *p1 = s1 + 6 * i;
                for (int c = 0; c < 3; c++) { px[0][c] = p0[c]; px[1][c] = p0[3 + c]; px[2][c] = p1[c]; px[3][c] = p1[3 + c]; }
                rgb_block(px, xb < simdEnd, y4, u1, v1);
                for (int k = 0; k < 4; k++) yy[i][k] = kBias23 + (uint32_t)y4[k];
                U[i] = kBias23 + (uint32_t)u1;
                V[i] = kBias23 + (uint32_t)v1;
                uint8_t *ya = y1 + (size_t)yr * y1s + xb, *yb = y2 + (size_t)yr * y2s + xb;
                ya[0] = yb[0] = (uint8_t)y4[0]; ya[1] = yb[1] = (uint8_t)y4[1];
                ya[y1s] = (uint8_t)y4[2]; ya[y1s + 1] = (uint8_t)y4[3];
                yb[y2s] = (uint8_t)y4[2]; yb[y2s + 1] = (uint8_t)y4[3];
                uint8_t *c = uv + (size_t)by * uvs + xb;
                c[0] = (uint8_t)u1; c[1] = (uint8_t)v1;
                pu[(size_t)by * us + bx0 + i] = (uint8_t)u1;
                pv[(size_t)by * vs + bx0 + i] = (uint8_t)v1;
            }
        }
        // half-size bilinear: two rounded stages below the bound, one stage beyond it; area:
        // rows 2 by - 1 (0 for by = 0) and 2 by, below the bound only (biased words: the bias
        // of a sum of two, 150 * 2^24, divides by 2; of four, 300 * 2^24 = 44 * 2^24 modulo 2^32, by 4)
        if (scaled) {
            uint32_t ob[4], oa[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const uint32_t t1 = (yy[i][0] + yy[i][1] + 1) >> 1, t2 = (yy[i][2] + yy[i][3] + 1) >> 1;
                ob[i] = (t1 + t2 + 1) >> 1;
                const uint32_t ya = by == 0 ? yy[i][0] + yy[i][1] : above[2 * i] + above[2 * i + 1];
                const uint32_t yb = by == 0 ? yy[i][2] + yy[i][3] : yy[i][0] + yy[i][1];
                oa[i] = (ya + yb + 2) >> 2;
                above[2 * i] = yy[i][2];
                above[2 * i + 1] = yy[i][3];
            }
            *(uint32_t *)(outB + (size_t)by * obs + bx0) = pack_lo4(ob[0], ob[1], ob[2], ob[3]);
            *(uint32_t *)(outA + (size_t)by * oas + bx0) = pack_lo4(oa[0], oa[1], oa[2], oa[3]);
        } else {
            for (int i = 0; i < nb; i++)
                outB[(size_t)by * obs + bx0 + i] = (uint8_t)((yy[i][0] + yy[i][1] + yy[i][2] + yy[i][3] + 2) >> 2);
        }
    }
}

bool aligned(const void *p, unsigned a) { return ((uintptr_t)p & (a - 1)) == 0; }

ScaleParams scale_params(int kind, uint32_t sW, uint32_t sH, uint32_t dW, uint32_t dH)
{
    // AgoConfigScaleMatrix of the AGO wrappers (ago_kernel_api.cpp:19788, :19908, :20272)
    ScaleParams p;
    p.xscale = (float)((double)sW / (double)dW);
    p.yscale = (float)((double)sH / (double)dH);
    if (kind == 0) { p.xoffset = (float)((double)sW / (double)dW * 0.5); p.yoffset = (float)((double)sH / (double)dH * 0.5); }
    else if (kind == 1) { p.xoffset = (float)((double)sW / (double)dW * 0.5 - 0.5); p.yoffset = (float)((double)sH / (double)dH * 0.5 - 0.5); }
    else { p.xoffset = -0.5f; p.yoffset = -0.5f; }
    const float FPM = (float)(1 << 18);
    p.xinc = (int)(FPM * p.xscale); p.yinc = (int)(FPM * p.yscale);
    p.xoffs = (int)(FPM * p.xoffset); p.yoffs = (int)(FPM * p.yoffset);
    return p;
}

AffineParams affine_params(const float *m, uint32_t dW, uint32_t dH, uint32_t sW, uint32_t sH, uint8_t border,
                           const uint32_t *valid)
{
    AffineParams a;
    a.r00 = m[0]; a.r10 = m[1]; a.r01 = m[2]; a.r11 = m[3]; a.c1 = m[4]; a.c2 = m[5];
    a.border = border;
    // corner test of geometric.cpp:700-716, in host float arithmetic
    volatile float sw = (float)sW, sh = (float)sH;
    bool b = (a.c1 < 0) | (a.c2 < 0) | (a.c1 >= sw) | (a.c2 >= sh);
    volatile float x1 = a.r00 * (float)dW + a.c1, y1 = a.r10 * (float)dW + a.c2;
    b |= (x1 < 0) | (y1 < 0) | (x1 >= sw) | (y1 >= sh);
    x1 = a.r01 * (float)dH + a.c1; y1 = a.r11 * (float)dH + a.c2;
    b |= (x1 < 0) | (y1 < 0) | (x1 >= sw) | (y1 >= sh);
    volatile float t0 = a.r00 * (float)dW, t1 = a.r01 * (float)dH;
    x1 = t0 + t1; x1 = x1 + a.c1;
    volatile float t2 = a.r10 * (float)dW, t3 = a.r11 * (float)dH;
    y1 = t2 + t3; y1 = y1 + a.c2;
    b |= (x1 < 0) | (y1 < 0) | (x1 >= sw) | (y1 >= sh);
    a.checkBorder = b;
    a.vl = valid ? (float)valid[0] : 0.f; a.vt = valid ? (float)valid[1] : 0.f;
    a.vr = valid ? (float)valid[2] : sw; a.vb = valid ? (float)valid[3] : sh;
    return a;
}

}  // namespace

// =====================================================================================
extern "C" int agocuda_ColorConvert_NV12_RGB(void *stream, uint32_t W, uint32_t H, uint8_t *pY, uint32_t yStride,
                                             uint8_t *pUV, uint32_t uvStride, const uint8_t *pSrc, uint32_t srcStride)
{
    if (!pY || !pUV || !pSrc || W < 2 || H < 2 || (W & 1) || (H & 1) || yStride < W || uvStride < W || srcStride < 3 * W)
        return AGOCUDA_INVALID_PARAMS;
    dim3 blk(64, 4), grd(div_up(W / 2, 64), div_up(H / 2, 4));
    k_color_rgb_yuv420<<<grd, blk, 0, as_stream(stream)>>>((int)W, (int)H, pSrc, (int)srcStride, pY, (int)yStride, pUV,
                                                            (int)uvStride, nullptr, 0, nullptr, 0);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_ColorConvert_IYUV_RGB(void *stream, uint32_t W, uint32_t H, uint8_t *pY, uint32_t yStride,
                                             uint8_t *pU, uint32_t uStride, uint8_t *pV, uint32_t vStride,
                                             const uint8_t *pSrc, uint32_t srcStride)
{
    if (!pY || !pU || !pV || !pSrc || W < 2 || H < 2 || (W & 1) || (H & 1) || yStride < W || uStride < W / 2 ||
        vStride < W / 2 || srcStride < 3 * W)
        return AGOCUDA_INVALID_PARAMS;
    dim3 blk(64, 4), grd(div_up(W / 2, 64), div_up(H / 2, 4));
    k_color_rgb_yuv420<<<grd, blk, 0, as_stream(stream)>>>((int)W, (int)H, pSrc, (int)srcStride, pY, (int)yStride, nullptr, 0,
                                                            pU, (int)uStride, pV, (int)vStride);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

static int scale_launch(int kind, void *stream, uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride, uint32_t sW,
                        uint32_t sH, const uint8_t *pSrc, uint32_t srcStride)
{
    if (!pDst || !pSrc || !W || !H || sW < 2 || sH < 2 || dstStride < W || srcStride < sW || sW >= 32768 || sH >= 32768)
        return AGOCUDA_INVALID_PARAMS;
    ScaleParams p = scale_params(kind, sW, sH, W, H);
    dim3 grd(div_up(W, 128), H);
    cudaStream_t s = as_stream(stream);
    if (kind == 0) k_scale_nearest<<<grd, 128, 0, s>>>((int)W, (int)H, pDst, (int)dstStride, (int)sW, (int)sH, pSrc, (int)srcStride, p);
    else if (kind == 1) k_scale_bilinear<<<grd, 128, 0, s>>>((int)W, (int)H, pDst, (int)dstStride, (int)sW, (int)sH, pSrc, (int)srcStride, p);
    else if (p.xscale == 2.0f && p.yscale == 2.0f)
        k_scale_area2x<<<grd, 128, 0, s>>>((int)W, (int)H, pDst, (int)dstStride, (int)sW, (int)sH, pSrc, (int)srcStride, p);
    else if (p.xscale == 1.0f && p.yscale == 1.0f)
        k_scale_area1x<<<grd, 128, 0, s>>>((int)W, (int)H, pDst, (int)dstStride, (int)sW, (int)sH, pSrc, (int)srcStride, p);
    else return -3;   // VX_ERROR_NOT_SUPPORTED: generic area ratios are not implemented on this target
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_ScaleImage_U8_U8_Nearest(void *stream, uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                                uint32_t srcW, uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride)
{ return scale_launch(0, stream, W, H, pDst, dstStride, srcW, srcH, pSrc, srcStride); }

extern "C" int agocuda_ScaleImage_U8_U8_Bilinear(void *stream, uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                                 uint32_t srcW, uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride)
{ return scale_launch(1, stream, W, H, pDst, dstStride, srcW, srcH, pSrc, srcStride); }

extern "C" int agocuda_ScaleImage_U8_U8_Area(void *stream, uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                             uint32_t srcW, uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride)
{ return scale_launch(2, stream, W, H, pDst, dstStride, srcW, srcH, pSrc, srcStride); }

extern "C" int agocuda_WarpAffine_U8_U8_Nearest_Constant(void *stream, uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                                         uint32_t srcW, uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride,
                                                         const float *affineMatrix, uint8_t border, const uint32_t *srcValidRect)
{
    const uint32_t W4 = (W + 3) & ~3u;
    if (!pDst || !pSrc || !affineMatrix || !W || !H || dstStride < W4 || srcStride < srcW || !srcW || !srcH)
        return AGOCUDA_INVALID_PARAMS;
    AffineParams a = affine_params(affineMatrix, W, H, srcW, srcH, border, srcValidRect);
    k_warp_affine_nearest<<<dim3(div_up(W4, 512), H), 128, 0, as_stream(stream)>>>((int)W4, (int)H, pDst, (int)dstStride, (int)srcW,
                                                                                   (int)srcH, pSrc, (int)srcStride, a);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_WarpAffine_U8_U8_Bilinear_Constant(void *stream, uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                                          uint32_t srcW, uint32_t srcH, const uint8_t *pSrc, uint32_t srcStride,
                                                          const float *affineMatrix, uint8_t border)
{
    const uint32_t W4 = (W + 3) & ~3u;
    if (!pDst || !pSrc || !affineMatrix || !W || !H || dstStride < W4 || srcStride < srcW || !srcW || !srcH)
        return AGOCUDA_INVALID_PARAMS;
    AffineParams a = affine_params(affineMatrix, W, H, srcW, srcH, border, nullptr);
    k_warp_affine_bilinear<<<dim3(div_up(W4, 512), H), 128, 0, as_stream(stream)>>>((int)W4, (int)H, pDst, (int)dstStride, (int)srcW,
                                                                                    (int)srcH, pSrc, (int)srcStride, a);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_fused_ColorScale_RGB(void *stream, uint32_t W, uint32_t H, const uint8_t *pSrc, uint32_t srcStride,
                                            uint8_t *pNV12Y, uint32_t nv12YStride, uint8_t *pNV12UV, uint32_t nv12UVStride,
                                            uint8_t *pIYUVY, uint32_t iyuvYStride, uint8_t *pU, uint32_t uStride,
                                            uint8_t *pV, uint32_t vStride, uint8_t *pHalfBilinear, uint32_t hbStride,
                                            uint8_t *pHalfArea, uint32_t haStride)
{
    if (!pSrc || !pNV12Y || !pNV12UV || !pIYUVY || !pU || !pV || !pHalfBilinear || !pHalfArea || W < 16 || H < 4 ||
        (W & 1) || (H & 1) || srcStride < 3 * W)
        return AGOCUDA_INVALID_PARAMS;
    // vector form: 8-byte aligned source, Y and UV rows, 4-byte aligned U, V and scaled rows
    const bool vec = aligned(pSrc, 8) && srcStride % 8 == 0 && aligned(pNV12Y, 8) && nv12YStride % 8 == 0 &&
                     aligned(pNV12UV, 8) && nv12UVStride % 8 == 0 && aligned(pIYUVY, 8) && iyuvYStride % 8 == 0 &&
                     aligned(pU, 4) && uStride % 4 == 0 && aligned(pV, 4) && vStride % 4 == 0 &&
                     aligned(pHalfBilinear, 4) && hbStride % 4 == 0 && aligned(pHalfArea, 4) && haStride % 4 == 0;
    if (vec) {
        dim3 blk(32, 4), grd(div_up(W / 8 + 1, 32), div_up(H / 2, 4 * kCsRows));
        k_fused_rgb_yuv_scale8<<<grd, blk, 0, as_stream(stream)>>>(
            (int)W, (int)H, pSrc, (int)srcStride, pNV12Y, (int)nv12YStride, pNV12UV, (int)nv12UVStride, pIYUVY,
            (int)iyuvYStride, pU, (int)uStride, pV, (int)vStride, pHalfBilinear, (int)hbStride, pHalfArea, (int)haStride);
    } else {
        dim3 blk(64, 4), grd(div_up(W / 2, 64), div_up(H / 2, 4));
        k_fused_rgb_yuv_scale<<<grd, blk, 0, as_stream(stream)>>>((int)W, (int)H, pSrc, (int)srcStride, pNV12Y,
                                                                   (int)nv12YStride, pNV12UV, (int)nv12UVStride, pIYUVY,
                                                                   (int)iyuvYStride, pU, (int)uStride, pV, (int)vStride,
                                                                   pHalfBilinear, (int)hbStride, pHalfArea, (int)haStride);
    }
    agocuda_count_launch(1);
    return agocuda_launch_status();
}
