// vision.cu -- Canny and Harris on sm_100a: per-node kernels (the plain form), fused
// front ends (one HBM pass over the image), union-find hysteresis and the corner pick.
//
// Border semantics.  The reference CPU kernels compute border columns from one byte
// outside the row (x = -1 and x = W).  With AGO's layout (row pitch ALIGN16(W), zero
// padding around each buffer) those bytes are: the last pixel of the previous row / the
// first pixel of the next row when W % 16 == 0, else 0.  The values enter the interior
// through non-maximum suppression and hysteresis, so `ago_px` reproduces them.
#include "agocuda_internal.cuh"
#include <string.h>

#include <cooperative_groups.h>
#include <cuda.h>

#include <mutex>

uint64_t agocuda_count_launch(unsigned n);

namespace {

__device__ __forceinline__ int ago_px(const uint8_t *src, int stride, int W, int H, int x, int y)
{
    if ((unsigned)y >= (unsigned)H) return 0;
    if (x >= 0 && x < W) return src[(size_t)y * stride + x];
    const bool tight = (W & 15) == 0;   // AGO row pitch == W: the neighbouring row's pixel
    if (x == -1) return (tight && y > 0) ? src[(size_t)(y - 1) * stride + W - 1] : 0;
    if (x == W) return (tight && y + 1 < H) ? src[(size_t)(y + 1) * stride] : 0;
    return 0;
}

// ---------------------------------------------------------------------------------
// Canny gradient: ((|gx| + |gy|) << 2) | direction, Gy negated
// (HafCpu_CannySobel_U16_U8_3x3_L1NORM, ago_haf_cpu_canny.cpp:44;
//  HafCpu_FastAtan2_Canny, ago_haf_cpu_arithmetic.cpp:9638)
// ---------------------------------------------------------------------------------
__device__ __forceinline__ int canny_dir(int gx, int gy)
{
    const int ax = abs(gx), ay = abs(gy);
    const float d1 = __fmul_rn((float)ax, 0.4142135623730950488016887242097f);
    const float d2 = __fmul_rn((float)ax, 2.4142135623730950488016887242097f);
    int r = (gx * gy) < 0 ? 3 : 1;
    if ((float)ay <= d1) r = 0;
    if ((float)ay >= d2) r = 2;
    return r;
}

__device__ __forceinline__ uint16_t canny_pack(int gx, int gy)
{
    int16_t t = (int16_t)(abs(gx) + abs(gy));
    t = (int16_t)(t << 2);
    return (uint16_t)(t | canny_dir(gx, gy));
}

// Gradient at one pixel.  `P(dx, dy)` returns the source pixel at (x+dx, y+dy) with
// ago_px semantics.  `simd_x0` selects the reference's SIMD-body formula at x = 0
// (W >= 16), which reads r0[-1] = 0 and r1[-1] = r0[ALIGN16(W)-1]: `r1m` is that value
// (the vertical [1 2 1] sum of column W-1 when W % 16 == 0, else 0).
template <class PX>
__device__ __forceinline__ uint16_t canny_grad(PX P, bool simd_x0, int r1m)
{
    int gx, gy;
    if (simd_x0) {
        const int r0p = P(1, -1) + 2 * P(1, 0) + P(1, 1);
        const int r1c = P(0, 1) - P(0, -1);
        const int r1p = P(1, 1) - P(1, -1);
        gx = (int16_t)r0p;
        gy = (int16_t)(0 - (int16_t)(r1m + 2 * r1c + r1p));
    } else {
        gx = (int16_t)(P(1, -1) - P(-1, -1) + P(1, 1) - P(-1, 1) + 2 * (P(1, 0) - P(-1, 0)));
        gy = (int16_t)(P(-1, 1) + P(1, 1) - P(-1, -1) - P(1, -1) + 2 * (P(0, 1) - P(0, -1)));
        gy = (int16_t)(-gy);
    }
    return canny_pack(gx, gy);
}

// offsets of the two neighbours compared for each direction (canny.cpp:24-29)
__device__ __constant__ int8_t kNOff[4][4] = {{-1, 0, 1, 0}, {1, -1, -1, 1}, {0, -1, 0, 1}, {-1, -1, 1, 1}};

// suppression + double threshold on one pixel of the packed gradient plane G(dx, dy)
template <class GV>
__device__ __forceinline__ int canny_supp(GV G, int lower, int upper)
{
    const int c = G(0, 0);
    const int mag = c >> 2, ang = c & 3;
    const int a = G(kNOff[ang][0], kNOff[ang][1]) >> 2;
    const int b = G(kNOff[ang][2], kNOff[ang][3]) >> 2;
    const int edge = (mag > a && mag > b) ? mag : 0;
    return edge > upper ? 255 : (edge <= lower ? 0 : 127);
}

// warp-aggregated append of one 32-bit item to a list with a device counter
__device__ __forceinline__ void list_append(uint32_t *list, uint32_t *count, uint32_t capacity, uint32_t item, bool pred)
{
    const unsigned m = __ballot_sync(__activemask(), pred);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(m));
    base = __shfl_sync(__activemask(), base, leader);
    if (pred) {
        const uint32_t idx = base + __popc(m & ((1u << lane) - 1));
        if (idx < capacity) list[idx] = item;
    }
}

__global__ void k_canny_sobel(int W, int H, uint16_t *dst, int dstStride, const uint8_t *src, int srcStride)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W) return;
    uint16_t *d = (uint16_t *)((uint8_t *)dst + (size_t)y * dstStride);
    if (y == 0 || y == H - 1) { d[x] = 0; return; }
    auto P = [&](int dx, int dy) { return ago_px(src, srcStride, W, H, x + dx, y + dy); };
    const bool simd_x0 = x == 0 && W >= 16;
    int r1m = 0;
    if (simd_x0 && (W & 15) == 0)
        r1m = ago_px(src, srcStride, W, H, W - 1, y - 1) + 2 * ago_px(src, srcStride, W, H, W - 1, y) +
              ago_px(src, srcStride, W, H, W - 1, y + 1);
    d[x] = canny_grad(P, simd_x0, r1m);
}

// ---------------------------------------------------------------------------------
// Canny gradients with 3x3 L2, 5x5 and 7x7 windows (HafCpu_CannySobel_U16_U8_5x5_L1NORM
// ago_haf_cpu_canny.cpp:145, _7x7_L1NORM :272, _3x3_L2NORM :646, _5x5_L2NORM :756,
// _7x7_L2NORM :893).  The reference splits each row into SIMD columns [0, A - 1),
// A = W - W % 16, computed from per-row vertical sums r0 / r1 held in zeroed node scratch
// (r0 at +16 bytes, r1 right after, ALIGN16(W) entries each), and scalar columns from A - 1
// on; the two formulas differ per variant (16-bit squares for 3x3 L2, a quarter-scale
// saturating body for 7x7, Gy signs, a sign slip in the 5x5 L2 scalar top row), and the
// SIMD part reads r0 / r1 up to R columns outside [0, A).  Each thread evaluates the
// formula of its column, with those scratch reads resolved to the values they find there.
// ---------------------------------------------------------------------------------
template <int G> struct CannyWin;
template <> struct CannyWin<3> { __device__ static int v(int k) { return k == 0 ? 2 : 1; }
                                 __device__ static int d(int k) { return k; } };
template <> struct CannyWin<5> { __device__ static int v(int k) { const int a = k < 0 ? -k : k; return a == 0 ? 6 : (a == 1 ? 4 : 1); }
                                 __device__ static int d(int k) { return k == 0 ? 0 : (k < 0 ? -1 : 1) * ((k < 0 ? -k : k) == 1 ? 2 : 1); } };
template <> struct CannyWin<7> { __device__ static int v(int k) { const int a = k < 0 ? -k : k; return a == 0 ? 20 : (a == 1 ? 15 : (a == 2 ? 6 : 1)); }
                                 __device__ static int d(int k) { const int a = k < 0 ? -k : k; const int m = a == 0 ? 0 : (a == 1 ? 5 : (a == 2 ? 4 : 1)); return k < 0 ? -m : m; } };

__device__ __forceinline__ int16_t cw16(int v) { return (int16_t)v; }
__device__ __forceinline__ int16_t cs16(int v) { return (int16_t)max(-32768, min(32767, v)); }
__device__ __forceinline__ int16_t cabs16(int16_t v) { return (int16_t)(v < 0 ? -(int)v : (int)v); }

// a source pixel as a read at flat offset (y * L + x) of an AGO-laid-out U8 buffer (row
// pitch L = ALIGN16(W), zero padding) finds it; 0 outside the buffer
__device__ __forceinline__ int ago_flat_px(const uint8_t *src, int stride, int W, int H, int L, int x, int y)
{
    const long f = (long)y * L + x;
    if (f < 0 || f >= (long)H * L) return 0;
    const int yy = (int)(f / L), xx = (int)(f - (long)yy * L);
    return xx < W ? src[(size_t)yy * stride + xx] : 0;
}

template <int G>
struct CannyRowSums {
    const uint8_t *s; int stride, y, A, L;
    __device__ int vsum(int c, bool diff) const {
        int a = 0;
#pragma unroll
        for (int k = -G / 2; k <= G / 2; k++)
            a += (diff ? CannyWin<G>::d(k) : CannyWin<G>::v(k)) * s[(size_t)(y + k) * stride + c];
        a = cw16(a);
        return G == 7 ? (a >> 2) : a;
    }
    __device__ int r1(int c) const {
        if (c < 0) { c += L; return c < A ? vsum(c, false) : 0; }   // r1[-k] is r0[L - k]
        return c < A ? vsum(c, true) : 0;                            // unwritten or past r1: zero scratch
    }
    __device__ int r0(int c) const {
        if (c < 0) return 0;                                         // the 16 zero bytes before r0
        if (c < A) return vsum(c, false);
        if (c < L) return 0;
        return r1(c - L);                                            // r0[L + k] is r1[k]
    }
};

__device__ __forceinline__ uint16_t canny_l2_pack(int16_t gx, int16_t gy, bool body3)
{
    float f;
    if (body3)
        f = __fadd_rn((float)(uint16_t)(gx * gx), (float)(uint16_t)(gy * gy));
    else
        f = __int2float_rn((int32_t)((uint32_t)(gx * gx) + (uint32_t)(gy * gy)));
    int m = __float2int_rn(__fsqrt_rn(f));
    m = max(0, min(65535, m));
    return (uint16_t)((uint16_t)(m << 2) | canny_dir(gx, gy));
}

template <int G, bool L2>
__global__ void k_canny_sobel_nxn(int W, int H, uint16_t *dst, int dstStride, const uint8_t *src, int srcStride)
{
    constexpr int R = G / 2;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W) return;
    uint16_t *d = (uint16_t *)((uint8_t *)dst + (size_t)y * dstStride);
    if (y < R || y >= H - R) { d[x] = 0; return; }
    const int L = (W + 15) & ~15, A = W - (W & 15);
    if (x < A - 1) {
        const CannyRowSums<G> sc{src, srcStride, y, A, L};
        int16_t t0, t1;
        if (G == 3) {
            t0 = cw16(sc.r0(x + 1) - sc.r0(x - 1));
            t1 = cw16(0 - cw16(cw16(sc.r1(x - 1) + sc.r1(x + 1)) + cw16(sc.r1(x) << 1)));
        } else if (G == 5) {
            t0 = cs16(cw16(cw16(sc.r0(x + 1) - sc.r0(x - 1)) << 1) + cw16(sc.r0(x + 2) - sc.r0(x - 2)));
            int16_t u = cw16(cw16(cw16(sc.r1(x - 1) + sc.r1(x + 1)) << 2) + cw16(sc.r1(x - 2) + sc.r1(x + 2)));
            u = L2 ? cs16(u + cw16(sc.r1(x) * 6)) : cw16(u + cw16(sc.r1(x) * 6));
            t1 = cw16(0 - u);
        } else {
            const int16_t a = cw16(cs16(sc.r0(x + 2) - sc.r0(x - 2)) << 2);
            const int16_t b = cw16(cs16(sc.r0(x + 1) - sc.r0(x - 1)) * 5);
            t0 = cs16(cs16(a + cs16(sc.r0(x + 3) - sc.r0(x - 3))) + b);
            int16_t u = cs16(cw16(cw16(sc.r1(x - 2) + sc.r1(x + 2)) * 6) + cw16(sc.r1(x) * 20));
            const int16_t v = cw16(cw16(sc.r1(x - 1) + sc.r1(x + 1)) * 15);
            u = cs16(u + cs16(sc.r1(x - 3) + sc.r1(x + 3)));
            u = cs16(u + v);
            t1 = cs16(0 - u);
        }
        if (L2) {
            d[x] = canny_l2_pack(t0, t1, G == 3);
        } else {
            int16_t m = cw16(cabs16(t0) + cabs16(t1));
            if (G == 7 && m > 0x3FFF) m = 0x3FFF;
            d[x] = (uint16_t)((uint16_t)(m << 2) | canny_dir(t0, t1));
        }
        return;
    }
    int gxs = 0, gys = 0;
#pragma unroll
    for (int j = -R; j <= R; j++)
#pragma unroll
        for (int i = -R; i <= R; i++) {
            const int v = ago_flat_px(src, srcStride, W, H, L, x + i, y + j);
            gxs += CannyWin<G>::v(j) * CannyWin<G>::d(i) * v;
            gys += (G == 5 && L2 && j == -R) ? (i == -R ? -1 : 1) * CannyWin<G>::v(i) * v   // canny.cpp:800
                                             : CannyWin<G>::d(j) * CannyWin<G>::v(i) * v;
        }
    const int16_t gx = cw16(gxs);
    int16_t gy = cw16(gys);
    if (!L2 && G != 7) gy = cw16(-gy);
    int16_t t;
    if (L2) {
        const int32_t n = (int32_t)((uint32_t)(gx * gx) + (uint32_t)(gy * gy));
        t = n < 0 ? 0 : cw16((int)__dsqrt_rn((double)n));
    } else {
        t = cw16(abs(gx) + abs(gy));
    }
    t = cw16(t << 2);
    d[x] = (uint16_t)cw16(t | canny_dir(gx, gy));
}

__global__ void k_canny_supp(int W, int H, uint8_t *dst, int dstStride, const uint16_t *g, int gStride,
                             int lower, int upper, uint32_t *stack, uint32_t *stackCount, uint32_t capacity)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const bool in = x >= 1 && x < W - 1 && y >= 1 && y < H - 1;
    int v = 0;
    if (in) {
        auto G = [&](int dx, int dy) { return (int)*(const uint16_t *)((const uint8_t *)g + (size_t)(y + dy) * gStride + 2 * (x + dx)); };
        v = canny_supp(G, lower, upper);
        dst[(size_t)y * dstStride + x] = (uint8_t)v;
    }
    list_append(stack, stackCount, capacity, ((uint32_t)y << 16) | (uint32_t)x, in && v == 255);
}

// ---------------------------------------------------------------------------------
// Hysteresis (HafCpu_CannyEdgeTrace_U8_U8XY, ago_haf_cpu_canny.cpp:598): a pixel ends up
// 255 iff it is 8-connected through non-zero pixels to a strong one -- computed as
// connected components with a lock-free union-find (labels only decrease; a root r has
// L[r] == r), then components holding a strong pixel are marked.  Fixed launch count, so
// the whole Canny node captures into one CUDA graph.
// ---------------------------------------------------------------------------------
constexpr int kFindLimit = 1 << 24;   // bound on pointer chasing; exceeded only on corruption

__device__ __forceinline__ int uf_find(const int *L, int x)
{
    for (int i = 0; i < kFindLimit; i++) {
        const int p = __ldcg(L + x);
        if (p == x) return x;
        x = p;
    }
    return x;
}

// find on a union-find no thread is modifying (after the union pass): L1-cached loads
__device__ __forceinline__ int uf_find_ro(const int *__restrict__ L, int x)
{
    for (int i = 0; i < kFindLimit; i++) {
        const int p = __ldg(L + x);
        if (p == x) return x;
        x = p;
    }
    return x;
}

__device__ __forceinline__ void uf_union(int *L, int a, int b, uint32_t *err)
{
    for (int i = 0; i < kFindLimit; i++) {
        a = uf_find(L, a);
        b = uf_find(L, b);
        if (a == b) return;
        if (a > b) { int t = a; a = b; b = t; }
        const int old = atomicMin(L + b, a);
        if (old == b) return;
        b = old;
    }
    atomicOr(err, 1u);
}

__global__ void k_hyst_init(int W, int H, const uint8_t *E, int eStride, int *L)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const int p = y * W + x;
    const bool m = x >= 1 && x < W - 1 && y >= 1 && y < H - 1 && E[(size_t)y * eStride + x] != 0;
    L[p] = m ? p : -1;
}

__global__ void k_hyst_union(int W, int H, int *L, uint32_t *err)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W || y < 1 || y >= H - 1) return;
    const int p = y * W + x;
    if (__ldcg(L + p) < 0) return;
    // the four neighbours already visited in raster order
    if (x > 0 && __ldcg(L + p - 1) >= 0) uf_union(L, p, p - 1, err);
    if (x > 0 && __ldcg(L + p - W - 1) >= 0) uf_union(L, p, p - W - 1, err);
    if (__ldcg(L + p - W) >= 0) uf_union(L, p, p - W, err);
    if (x + 1 < W && __ldcg(L + p - W + 1) >= 0) uf_union(L, p, p - W + 1, err);
}

// Seeds from the stack.  An entry on an edge-map pixel marks its component.  An entry on a
// pixel outside the map (zero, or on the image border, where labels are -1) marks the
// components of its 8 neighbours instead: the reference's trace grows from every stack entry
// through its neighbours whatever the entry's own value (ago_haf_cpu_canny.cpp:611-625).
// Entries outside the image are skipped and flagged (AGOCUDA_TRACE_STATUS_BAD_ENTRY).
__global__ void k_hyst_mark(int W, int H, const int *L, const uint32_t *strong, const uint32_t *strongCount,
                            uint32_t capacity, uint32_t *rootBits, uint32_t *err)
{
    const uint32_t n = min(*strongCount, capacity);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t xy = strong[i];
        const int x = (int)(xy & 0xffff), y = (int)(xy >> 16);
        if (x >= W || y >= H) { atomicOr(err, AGOCUDA_TRACE_STATUS_BAD_ENTRY); continue; }
        const int p = y * W + x;
        if (L[p] >= 0) {
            const int r = uf_find(L, p);
            atomicOr(rootBits + (r >> 5), 1u << (r & 31));
            continue;
        }
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                const int x1 = x + dx, y1 = y + dy;
                if ((dx | dy) == 0 || x1 < 0 || x1 >= W || y1 < 0 || y1 >= H) continue;
                const int q = y1 * W + x1;
                if (L[q] < 0) continue;
                const int r = uf_find(L, q);
                atomicOr(rootBits + (r >> 5), 1u << (r & 31));
            }
    }
}

__global__ void k_hyst_output(int W, int H, uint8_t *out, int outStride, const int *L, const uint32_t *rootBits)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const int p = y * W + x;
    uint8_t v = 0;
    if (__ldcg(L + p) >= 0) {
        const int r = uf_find(L, p);
        v = (rootBits[r >> 5] >> (r & 31)) & 1 ? 255 : 0;
    }
    out[(size_t)y * outStride + x] = v;
}

// ---------------------------------------------------------------------------------
// Fused Canny: gradient, suppression and double threshold for a 64x32 tile from one read
// of the image, then hysteresis as block-based connected components.  The tile's
// non-zero pixels are labelled in shared memory (lock-free union-find over the W, NW, N
// and NE neighbours, i.e. 8-connectivity).  A component with no pixel on the tile's border
// ring is final in the tile, and so is one holding a strong pixel: the front writes their
// bytes.  The other components ("open": at most 94 per tile) get a slot and a node of a
// compact global union-find (tile * kOpenMax + slot); the ring pixels' slots go to global
// memory for the unions across tile borders, and the runs of open components without a
// strong pixel go to a per-tile list that the last pass sets to 255 where the merged
// component turned out strong.  The result is the same set of 255 pixels as the per-pixel
// union-find above: 8-connected components of the interior non-zero pixels that hold a
// strong (255) pixel.
// ---------------------------------------------------------------------------------
constexpr int kTW = 64, kTH = 32, kTS = kTW * kTH;   // tile and its slot count
constexpr int kIH = kTH + 4;                         // input tile rows (halo 2)
constexpr int kGH = kTH + 2;                         // gradient tile rows (halo 1)
// open components per tile (those touching its 188-pixel border ring: at most 94), runs per
// tile (at most 32 per 64-pixel row), ring pixels per tile
constexpr int kOpenMax = 128, kRunMax = kTS / 2, kBorder = 2 * kTW + 2 * kTH;

// per-tile hysteresis state in global memory: ring labels (open slot or -1; top row, bottom
// row, left column, right column), the union-find over open slots (node = tile * kOpenMax +
// slot), strong bits per node, open-slot counts, and the runs left for the patch pass
struct CannyTiles {
    int16_t *blab;
    int *uf;
    uint32_t *sbits, *nOpen, *runCount, *runs;
    int tilesX, tilesY;
};

// global node of the open component at pixel (x, y), which lies on its tile's border ring;
// -1 where that pixel is not an edge candidate
__device__ __forceinline__ int ring_node(const CannyTiles &T, int x, int y)
{
    const int tx = x / kTW, ty = y / kTH, lx = x - tx * kTW, ly = y - ty * kTH;
    const int tile = ty * T.tilesX + tx;
    int idx;
    if (ly == 0) idx = lx;
    else if (ly == kTH - 1) idx = kTW + lx;
    else if (lx == 0) idx = 2 * kTW + ly;
    else if (lx == kTW - 1) idx = 2 * kTW + kTH + ly;
    else return -1;
    const int s = __ldg(T.blab + (size_t)tile * kBorder + idx);
    return s < 0 ? -1 : tile * kOpenMax + s;
}

__device__ __forceinline__ int sfind(const int *lab, int x)
{
    for (int i = 0; i < kTS; i++) {
        const int p = lab[x];
        if (p == x) return x;
        x = p;
    }
    return x;
}

__device__ __forceinline__ void sunion(int *lab, int a, int b)
{
    for (int i = 0; i < kTS; i++) {
        a = sfind(lab, a);
        b = sfind(lab, b);
        if (a == b) return;
        if (a > b) { const int t = a; a = b; b = t; }
        const int old = atomicMin(lab + b, a);
        if (old == b) return;
        b = old;
    }
}

// --- front end: one block per 64x32 tile, 256 threads -----------------------------
// Input tile as words: rows y0-2 .. y0+33, columns x0-4 .. x0+67 (18 words of 4 pixels);
// gradient tile rows y0-1 .. y0+32 over the same 72 columns (the outer ones are unused).
constexpr int kInWords = (kTW + 8) / 4, kGC = kTW + 8;

// One row's 6 pixels X[-1..4] around a 4-pixel word C (L, R: the words either side) as
// 16-bit lane pairs: E = (X0, X2), O = (X1, X3), Om = (X-1, X1), Ep = (X2, X4).
struct Lanes4 { uint32_t E, O, Om, Ep; };
__device__ __forceinline__ Lanes4 lanes4(uint32_t L, uint32_t C, uint32_t R)
{
    Lanes4 v;
    v.E = __byte_perm(C, 0, 0x4240);
    v.O = __byte_perm(C, 0, 0x4341);
    v.Om = __byte_perm(L, v.O, 0x5453);
    v.Ep = __byte_perm(v.E, R, 0x3432);
    return v;
}

// canny_pack for a gradient held as lanes biased by 1024
__device__ __forceinline__ uint32_t canny_pack_biased(uint32_t bx, uint32_t by)
{
    return canny_pack((int)bx - 1024, (int)by - 1024);
}

__device__ __forceinline__ int sG_mag3(uint32_t g) { return (int)(g | 3u); }   // (mag << 2) | 3: compares as mag

// TMA form of the input tile: one box of 96 x 36 bytes, columns x0-16 .. x0+79 (a TMA box
// starts on a 16-byte column), copied onto an mbarrier; word kInOffTma of a row is column x0-4
constexpr int kInPitchTma = 24, kInOffTma = 3;
constexpr int kCannyWaitLimit = 1 << 20;                 // bounded mbarrier waits

template <bool TMA>
__global__ void __launch_bounds__(256, 6)
k_canny_ccl_front(int W, int H, const uint8_t *__restrict__ src, int srcStride, int lower, int upper,
                  uint8_t *__restrict__ dst, int dstStride, CannyTiles T, uint32_t *__restrict__ err,
                  const __grid_constant__ CUtensorMap map)
{
    constexpr int kPitch = TMA ? kInPitchTma : kInWords, kOff = TMA ? kInOffTma : 0;
    __shared__ __align__(128) uint32_t sIn[kIH][kPitch];
    __shared__ __align__(16) uint16_t sG[kGH][kGC];
    __shared__ __align__(16) int sLab[kTS];
    __shared__ unsigned long long sNZ[kTH], sST[kTH];   // per tile row: non-zero / strong pixels
    __shared__ int16_t sV[kIH];                          // per gradient row: vertical sum of column W-1
    __shared__ uint32_t sStrongRoot[kTS / 32], sOpen[kTS / 32], sOpenPre[kTS / 32], sOpenStrong[kOpenMax / 32];
    __shared__ int sRunN;
    const int x0 = blockIdx.x * kTW, y0 = blockIdx.y * kTH, tid = threadIdx.x;
    const int tile = blockIdx.y * gridDim.x + blockIdx.x;

    // ---- input words; words reaching outside the image follow the reference's reads
    // outside rows (ago_px), byte by byte
    __shared__ __align__(8) uint64_t bar;
    if constexpr (TMA) {
        if (tid == 0) {
            const uint32_t b = smem_addr_u32(&bar);
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(kIH * kPitch * 4) : "memory");
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                ::"r"(smem_addr_u32(&sIn[0][0])), "l"((uint64_t)&map), "r"(x0 - 16), "r"(y0 - 2), "r"(b) : "memory");
        }
    } else {
        const bool al = (((uintptr_t)src | (uintptr_t)srcStride) & 3) == 0;
        static_assert(kIH * kInWords <= 3 * 256, "three words per thread");
#pragma unroll
        for (int it = 0; it < 3; it++) {
            const int i = tid + it * 256;
            if (i >= kIH * kInWords) break;
            const int r = i / kInWords, q = i - r * kInWords;
            const int y = y0 - 2 + r, x = x0 - 4 + 4 * q;
            uint32_t w;
            if (al && (unsigned)y < (unsigned)H && x >= 0 && x + 4 <= W) {
                w = __ldg((const uint32_t *)(src + (size_t)y * srcStride + x));
            } else {
                w = 0;
                for (int k = 0; k < 4; k++) w |= (uint32_t)ago_px(src, srcStride, W, H, x + k, y) << (8 * k);
            }
            sIn[r][q] = w;
        }
    }
    if (tid < kTS / 32) { sStrongRoot[tid] = 0; sOpen[tid] = 0; }
    if (tid < kOpenMax / 32) sOpenStrong[tid] = 0;
    if (tid == 0) sRunN = 0;
    const bool needV = x0 == 0 && (W & 15) == 0 && W >= 16;
    if (needV && tid < kGH) {
        const int y = y0 - 1 + tid;
        sV[tid] = (y >= 1 && y < H - 1)
            ? (int16_t)(ago_px(src, srcStride, W, H, W - 1, y - 1) + 2 * ago_px(src, srcStride, W, H, W - 1, y) +
                        ago_px(src, srcStride, W, H, W - 1, y + 1))
            : 0;
    }
    __syncthreads();
    if constexpr (TMA) {
        const uint32_t b = smem_addr_u32(&bar);
        bool done = false;
        for (int i = 0; i < kCannyWaitLimit && !done; i++) done = mbarrier_try_wait_parity(b, 0);
        if (!__syncthreads_and(done)) {
            // the copy did not complete: report it, give it one more bounded wait, leave
            if (tid == 0) atomicOr(err, AGOCUDA_CANNY_STATUS_TMA_TIMEOUT);
            for (int i = 0; i < kCannyWaitLimit && !done; i++) done = mbarrier_try_wait_parity(b, 0);
            return;
        }
        // TMA writes zeros outside the plane, as ago_px reads except where the row pitch is W
        // (W % 16 == 0): there column -1 is the previous row's last pixel and column W the next
        // row's first
        if ((W & 15) == 0) {
            uint8_t *b8 = (uint8_t *)&sIn[0][0];
            if (x0 == 0 && tid < kIH) {
                const int y = y0 - 2 + tid;
                b8[tid * kPitch * 4 + 15] = (y >= 1 && y < H) ? src[(size_t)(y - 1) * srcStride + W - 1] : 0;
            }
            const int cw = W - (x0 - 16);
            if (cw < kPitch * 4 && tid >= 64 && tid < 64 + kIH) {
                const int r = tid - 64, y = y0 - 2 + r;
                b8[r * kPitch * 4 + cw] = (y >= 0 && y + 1 < H) ? src[(size_t)(y + 1) * srcStride] : 0;
            }
        }
        __syncthreads();
    }

    // ---- packed gradient, 4 columns per item, in 16-bit lanes
    for (int i = tid; i < kGH * kInWords; i += blockDim.x) {
        const int gr = i / kInWords, q = i - gr * kInWords;
        const int y = y0 - 1 + gr, xq = x0 - 4 + 4 * q;
        uint32_t out0 = 0, out1 = 0;
        if (y >= 1 && y < H - 1) {
            Lanes4 t, m, b;
            {
                const uint32_t *r0 = sIn[gr] + kOff, *r1 = sIn[gr + 1] + kOff, *r2 = sIn[gr + 2] + kOff;
                const int ql = q > 0 ? q - 1 : q, qr = q + 1 < kInWords ? q + 1 : q;   // edge items: unused columns
                t = lanes4(r0[ql], r0[q], r0[qr]);
                m = lanes4(r1[ql], r1[q], r1[qr]);
                b = lanes4(r2[ql], r2[q], r2[qr]);
            }
            const uint32_t vE = t.E + 2 * m.E + b.E, vO = t.O + 2 * m.O + b.O;
            const uint32_t vOm = t.Om + 2 * m.Om + b.Om, vEp = t.Ep + 2 * m.Ep + b.Ep;
            const uint32_t bias = 0x04000400u;
            const uint32_t gx02 = vO + bias - vOm, gx13 = vEp + bias - vE;
            const uint32_t ts02 = t.Om + 2 * t.E + t.O, ts13 = t.E + 2 * t.O + t.Ep;
            const uint32_t bs02 = b.Om + 2 * b.E + b.O, bs13 = b.E + 2 * b.O + b.Ep;
            const uint32_t gy02 = ts02 + bias - bs02, gy13 = ts13 + bias - bs13;   // Gy negated (canny.cpp:79)
            uint32_t g0 = canny_pack_biased(gx02 & 0xffff, gy02 & 0xffff);
            uint32_t g1 = canny_pack_biased(gx13 & 0xffff, gy13 & 0xffff);
            uint32_t g2 = canny_pack_biased(gx02 >> 16, gy02 >> 16);
            uint32_t g3 = canny_pack_biased(gx13 >> 16, gy13 >> 16);
            if (xq < 0 || xq + 3 >= W) {   // columns outside the image hold 0
                if ((unsigned)xq >= (unsigned)W) g0 = 0;
                if ((unsigned)(xq + 1) >= (unsigned)W) g1 = 0;
                if ((unsigned)(xq + 2) >= (unsigned)W) g2 = 0;
                if ((unsigned)(xq + 3) >= (unsigned)W) g3 = 0;
            }
            if (xq == 0 && W >= 16) {      // the reference's SIMD-body formula at x = 0
                const uint8_t *b8 = (const uint8_t *)sIn;
                auto P = [&](int dx, int dy) { return (int)b8[(gr + 1 + dy) * (kPitch * 4) + 4 * kOff + 4 + dx]; };
                g0 = canny_grad(P, true, (W & 15) == 0 ? (int)sV[gr] : 0);
            }
            out0 = g0 | (g1 << 16);
            out1 = g2 | (g3 << 16);
        }
        *(uint2 *)&sG[gr][4 * q] = make_uint2(out0, out1);
    }
    __syncthreads();

    // ---- suppression + thresholds: 8 pixels of one row per thread; row masks
    const int r = tid >> 3, sgm = tid & 7, c0 = 8 * sgm;
    const int y = y0 + r;
    {
        int g[3][10];                       // gradient rows y-1 .. y+1, columns c0-1 .. c0+8
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const uint32_t *row = (const uint32_t *)&sG[r + k][c0 + 2];   // columns c0-2 .. c0+9
            uint32_t w[6];
#pragma unroll
            for (int j = 0; j < 6; j++) w[j] = row[j];
            g[k][0] = (int)(w[0] >> 16);
#pragma unroll
            for (int j = 1; j < 5; j++) { g[k][2 * j - 1] = (int)(w[j] & 0xffff); g[k][2 * j] = (int)(w[j] >> 16); }
            g[k][9] = (int)(w[5] & 0xffff);
        }
        uint32_t nz = 0, st = 0;
        const bool rowIn = y >= 1 && y < H - 1;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int x = x0 + c0 + j;
            const int c = g[1][j + 1];
            const int ang = c & 3;
            // neighbours along the direction (kNOff): 0 W/E, 1 NE/SW, 2 N/S, 3 NW/SE
            const int a = (ang & 2) ? ((ang & 1) ? g[0][j] : g[0][j + 1]) : ((ang & 1) ? g[0][j + 2] : g[1][j]);
            const int b = (ang & 2) ? ((ang & 1) ? g[2][j + 2] : g[2][j + 1]) : ((ang & 1) ? g[2][j] : g[1][j + 2]);
            const int mag = c >> 2;
            const bool keep = sG_mag3(c) > sG_mag3(a) && sG_mag3(c) > sG_mag3(b);
            const int edge = keep ? mag : 0;
            const bool in = rowIn && x >= 1 && x < W - 1;
            const bool strong = in && edge > upper;   // 255 (canny_supp), else 0 at <= lower, else 127
            nz |= (uint32_t)(strong || (in && edge > lower)) << j;
            st |= (uint32_t)strong << j;
        }
        ((uint8_t *)&sNZ[r])[sgm] = (uint8_t)nz;
        ((uint8_t *)&sST[r])[sgm] = (uint8_t)st;
    }
    __syncthreads();

    // ---- provisional labels: every pixel points at the first pixel of its run in the row
    const unsigned long long m = sNZ[r];
    const int i0 = r * kTW + c0;
    {
        const unsigned long long below = ~m & ((1ull << c0) - 1ull);
        int start = below ? 64 - __clzll(below) : 0;
        int lab[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int c = c0 + j;
            if (j > 0 && !((m >> (c - 1)) & 1)) start = c;
            lab[j] = ((m >> c) & 1) ? r * kTW + start : -1;
        }
        *(int4 *)&sLab[i0] = make_int4(lab[0], lab[1], lab[2], lab[3]);
        *(int4 *)&sLab[i0 + 4] = make_int4(lab[4], lab[5], lab[6], lab[7]);
    }
    __syncthreads();
    // ---- unions with the row above: one per run of this row and overlapping run above
    // (N if present, unless the left neighbour already covers it; else NW / NE)
    if (r > 0) {
        const unsigned long long a = sNZ[r - 1];
        const unsigned long long uN = m & a & ~((m << 1) & (a << 1));
        const unsigned long long uNW = m & ~a & (a << 1) & ~(m << 1);
        const unsigned long long uNE = m & ~a & (a >> 1) & ~(m >> 1);
        uint32_t bn = (uint32_t)(uN >> c0) & 0xff, bw = (uint32_t)(uNW >> c0) & 0xff, be = (uint32_t)(uNE >> c0) & 0xff;
        while (bn) { const int j = __ffs(bn) - 1; bn &= bn - 1; sunion(sLab, i0 + j, i0 + j - kTW); }
        while (bw) { const int j = __ffs(bw) - 1; bw &= bw - 1; sunion(sLab, i0 + j, i0 + j - kTW - 1); }
        while (be) { const int j = __ffs(be) - 1; be &= be - 1; sunion(sLab, i0 + j, i0 + j - kTW + 1); }
    }
    __syncthreads();

    // ---- roots (the component's smallest pixel index): each run start finds its root and
    // keeps it (no unions run any more), then every pixel reads start -> root in two steps
    {
        uint32_t starts = (uint32_t)((m & ~(m << 1)) >> c0) & 0xff;
        while (starts) {
            const int j = __ffs(starts) - 1;
            starts &= starts - 1;
            sLab[i0 + j] = sfind(sLab, i0 + j);
        }
    }
    __syncthreads();
    int root[8];
    {
        const int4 a = *(const int4 *)&sLab[i0], b = *(const int4 *)&sLab[i0 + 4];
        const int s1[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        const uint32_t stb = (uint32_t)(sST[r] >> c0) & 0xff;
        int lastOr = -1;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            root[j] = s1[j] >= 0 ? sLab[s1[j]] : -1;   // start -> root (a root maps to itself)
            if (((stb >> j) & 1) && root[j] != lastOr) {
                lastOr = root[j];
                atomicOr(&sStrongRoot[lastOr >> 5], 1u << (lastOr & 31));
            }
        }
    }
    // components with a pixel on the tile's border ring are open: they may continue in a
    // neighbouring tile, so they go to the global union-find; the others are final here
    if (r == 0 || r == kTH - 1) {
        int last = -1;
#pragma unroll
        for (int j = 0; j < 8; j++)
            if (root[j] >= 0 && root[j] != last) {
                last = root[j];
                atomicOr(&sOpen[last >> 5], 1u << (last & 31));
            }
    } else {
        if (sgm == 0 && root[0] >= 0) atomicOr(&sOpen[root[0] >> 5], 1u << (root[0] & 31));
        if (sgm == 7 && root[7] >= 0) atomicOr(&sOpen[root[7] >> 5], 1u << (root[7] & 31));
    }
    __syncthreads();
    if (tid < 32) {                       // open slots: exclusive prefix of the 64 words' counts
        const uint32_t n0 = __popc(sOpen[2 * tid]), n1 = __popc(sOpen[2 * tid + 1]);
        uint32_t inc = n0 + n1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
            if (tid >= o) inc += v;
        }
        sOpenPre[2 * tid] = inc - n0 - n1;
        sOpenPre[2 * tid + 1] = inc - n1;
        if (tid == 31) {
            T.nOpen[tile] = min(inc, (uint32_t)kOpenMax);
            if (inc > (uint32_t)kOpenMax) atomicOr(err, 1u);   // not reachable: a ring holds <= 94 components
        }
    }
    __syncthreads();
    auto oslot = [&](int rt) {
        const int w = rt >> 5;
        return (int)(sOpenPre[w] + __popc(sOpen[w] & ((1u << (rt & 31)) - 1u)));
    };
    auto ring_label = [&](int rt) -> int16_t {
        if (rt < 0) return -1;
        const int o = oslot(rt);
        return o < kOpenMax ? (int16_t)o : (int16_t)-1;
    };
    auto is_strong = [&](int rt) { return (sStrongRoot[rt >> 5] >> (rt & 31)) & 1; };

    // edge bytes: 255 for the pixels of components holding a strong pixel of this tile (such a
    // component is strong whatever it joins), else 0; open components without one are
    // patched after the global resolve
    if (y < H && x0 + c0 < W) {
        uint32_t lo = 0, hi = 0;
        int last = -1;
        uint32_t lastV = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if (root[j] < 0) continue;
            if (root[j] != last) { last = root[j]; lastV = is_strong(last) ? 0xFFu : 0u; }
            if (j < 4) lo |= lastV << (8 * j);
            else hi |= lastV << (8 * (j - 4));
        }
        uint8_t *o = dst + (size_t)y * dstStride + x0 + c0;
        const int n = min(8, W - (x0 + c0));
        if (n == 8 && ((uintptr_t)o & 7) == 0) {
            *(uint2 *)o = make_uint2(lo, hi);
        } else {
            for (int j = 0; j < n; j++) o[j] = (uint8_t)((j < 4 ? lo >> (8 * j) : hi >> (8 * (j - 4))) & 0xFF);
        }
    }
    // labels of the ring pixels (open slot or -1): top row, bottom row, left column, right column
    {
        int16_t *bl = T.blab + (size_t)tile * kBorder;
        if (r == 0 || r == kTH - 1) {
#pragma unroll
            for (int j = 0; j < 8; j++) bl[(r == 0 ? 0 : kTW) + c0 + j] = ring_label(root[j]);
        }
        if (sgm == 0) bl[2 * kTW + r] = ring_label(root[0]);
        if (sgm == 7) bl[2 * kTW + kTH + r] = ring_label(root[7]);
    }
    // runs of open components that hold no strong pixel here: (row, column, length, slot),
    // appended with one shared-memory atomic per warp
    {
        uint32_t pend = 0;
        uint32_t sb = (uint32_t)((m & ~(m << 1)) >> c0) & 0xff;
        while (sb) {
            const int j = __ffs(sb) - 1;
            sb &= sb - 1;
            const int rt = sLab[i0 + j];          // a run start holds its root
            if (((sOpen[rt >> 5] >> (rt & 31)) & 1) && !is_strong(rt) && oslot(rt) < kOpenMax) pend |= 1u << j;
        }
        const int lane = tid & 31, cnt = __popc(pend);
        int inc = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += v;
        }
        int base = 0;
        if (lane == 31 && inc) base = atomicAdd(&sRunN, inc);
        base = __shfl_sync(0xffffffffu, base, 31) + inc - cnt;
        while (pend) {
            const int j = __ffs(pend) - 1;
            pend &= pend - 1;
            const int rt = sLab[i0 + j], c = c0 + j;
            const unsigned long long rest = ~(m >> c);
            const int len = rest ? __ffsll((long long)rest) - 1 : kTW - c;
            const uint32_t e = (uint32_t)r | ((uint32_t)c << 5) | ((uint32_t)(len - 1) << 11) | ((uint32_t)oslot(rt) << 17);
            if (base < kRunMax) T.runs[(size_t)tile * kRunMax + base] = e;
            base++;
        }
    }
    // union-find nodes of the open slots, and which of them hold a strong pixel
    if (tid < kTS / 32) {
        uint32_t ow = sOpen[tid];
        const uint32_t sw = sStrongRoot[tid];
        int o = (int)sOpenPre[tid];
        while (ow) {
            const int b = __ffs(ow) - 1;
            ow &= ow - 1;
            if (o < kOpenMax) {
                T.uf[(size_t)tile * kOpenMax + o] = tile * kOpenMax + o;
                if ((sw >> b) & 1) atomicOr(&sOpenStrong[o >> 5], 1u << (o & 31));
            }
            o++;
        }
    }
    __syncthreads();
    if (tid < kOpenMax / 32) T.sbits[(size_t)tile * (kOpenMax / 32) + tid] = sOpenStrong[tid];
    if (tid == 0) T.runCount[tile] = (uint32_t)min(sRunN, kRunMax);
}

// unions across tile borders: the W / NW / N / NE neighbours of a tile's left column, top
// row and right column that lie in another tile (both ends are ring pixels of their tiles)
__global__ void k_canny_ccl_border(int W, int H, CannyTiles T, uint32_t *err)
{
    constexpr int kPer = kTH + kTW + kTH;
    const int tile = blockIdx.y, b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= kPer) return;
    const int x0 = (tile % T.tilesX) * kTW, y0 = (tile / T.tilesX) * kTH;
    int x, y;
    if (b < kTH) { x = x0; y = y0 + b; }
    else if (b < kTH + kTW) { x = x0 + b - kTH; y = y0; }
    else { x = x0 + kTW - 1; y = y0 + b - kTH - kTW; }
    if (x >= W || y >= H) return;
    const int sp = ring_node(T, x, y);
    if (sp < 0) return;
    const int dx[4] = {-1, -1, 0, 1}, dy[4] = {0, -1, -1, -1};
    for (int k = 0; k < 4; k++) {
        const int nx = x + dx[k], ny = y + dy[k];
        if (nx < 0 || ny < 0 || nx >= W) continue;
        if (nx >= x0 && nx < x0 + kTW && ny >= y0) continue;     // same tile: done locally
        const int sq = ring_node(T, nx, ny);
        if (sq >= 0) uf_union(T.uf, sp, sq, err);
    }
}

// after the unions: every open node points straight at its component's root (path
// compression; concurrent readers see the old parent or the root, both lead to the root),
// and a node holding a strong pixel sets its root's strong bit.  One thread per node.
__global__ void k_canny_ccl_flatten(CannyTiles T, int nodes)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    const int tile = i / kOpenMax, o = i - tile * kOpenMax;
    if (o >= (int)__ldg(T.nOpen + tile)) return;
    const int rt = uf_find(T.uf, i);
    if (rt != i) {
        T.uf[i] = rt;
        if ((__ldcg(T.sbits + (i >> 5)) >> (i & 31)) & 1) atomicOr(T.sbits + (rt >> 5), 1u << (rt & 31));
    }
}

// the runs of open components without a strong pixel in their tile: 255 where the merged
// component is strong (the front wrote 0); a warp per tile
__global__ void __launch_bounds__(256) k_canny_ccl_patch(int tiles, CannyTiles T, uint8_t *__restrict__ dst, int dstStride)
{
    const int tile = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (tile >= tiles) return;
    const int n = (int)T.runCount[tile];
    const int x0 = (tile % T.tilesX) * kTW, y0 = (tile / T.tilesX) * kTH;
    for (int k = lane; k < n; k += 32) {
        const uint32_t e = T.runs[(size_t)tile * kRunMax + k];
        const int r = (int)(e & 31), c = (int)((e >> 5) & 63), len = (int)((e >> 11) & 63) + 1, s = (int)(e >> 17);
        const int g = __ldg(T.uf + tile * kOpenMax + s);          // flattened: the component's root
        if ((__ldg(T.sbits + (g >> 5)) >> (g & 31)) & 1) {
            uint8_t *o = dst + (size_t)(y0 + r) * dstStride + x0 + c;
            for (int q = 0; q < len; q++) o[q] = 255;
        }
    }
}

// ---------------------------------------------------------------------------------
// Harris (ago_haf_cpu_harris.cpp): HG3 = {gx*gx, gx*gy, gy*gy} of the integer 3x3 Sobel
// (exact in float), 3x3 window sums (exact: integers below 2^24), then the score in
// round-to-nearest float with the reference's operation order (no FMA).
// ---------------------------------------------------------------------------------
__device__ __forceinline__ float harris_score(float gx2, float gxy2, float gy2, float k, float Tc, float norm)
{
    const float traceA = __fadd_rn(gx2, gy2);
    const float detA = __fsub_rn(__fmul_rn(gx2, gy2), __fmul_rn(gxy2, gxy2));
    float Mc = __fsub_rn(detA, __fmul_rn(__fmul_rn(k, traceA), traceA));
    Mc = __fdiv_rn(Mc, norm);
    return Mc > Tc ? Mc : 0.0f;
}

template <class PX>
__device__ __forceinline__ void harris_grad(PX P, float &gxx, float &gxy, float &gyy)
{
    const int gx = (int16_t)((P(1, 1) - P(-1, 1)) + (P(1, -1) - P(-1, -1)) + 2 * (P(1, 0) - P(-1, 0)));
    const int gy = (int16_t)((P(-1, 1) + 2 * P(0, 1) + P(1, 1)) - (P(-1, -1) + 2 * P(0, -1) + P(1, -1)));
    gxx = __fmul_rn((float)gx, (float)gx);
    gxy = __fmul_rn((float)gx, (float)gy);
    gyy = __fmul_rn((float)gy, (float)gy);
}

__global__ void k_harris_sobel(int W, int H, float *dst, int dstStride, const uint8_t *src, int srcStride)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    float *d = (float *)((uint8_t *)dst + (size_t)y * dstStride) + 3 * x;
    if (y == 0 || y == H - 1) { d[0] = d[1] = d[2] = 0.f; return; }
    auto P = [&](int dx, int dy) { return ago_px(src, srcStride, W, H, x + dx, y + dy); };
    harris_grad(P, d[0], d[1], d[2]);
}

__global__ void k_harris_score(int W, int H, float *dst, int dstStride, const float *hg, int hgStride, float k, float Tc, float norm)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    float v = 0.f;
    if (x >= 1 && x < W - 1 && y >= 1 && y < H - 1) {
        float s0 = 0.f, s1 = 0.f, s2 = 0.f;
        for (int j = -1; j <= 1; j++) {
            const float *r = (const float *)((const uint8_t *)hg + (size_t)(y + j) * hgStride);
            for (int i = -1; i <= 1; i++) {
                s0 = __fadd_rn(s0, r[3 * (x + i)]);
                s1 = __fadd_rn(s1, r[3 * (x + i) + 1]);
                s2 = __fadd_rn(s2, r[3 * (x + i) + 2]);
            }
        }
        v = harris_score(s0, s1, s2, k, Tc, norm);
    }
    *(float *)((uint8_t *)dst + (size_t)y * dstStride + 4 * x) = v;
}

// XYS record (ago_keypoint_xys_t): int16 x, int16 y, float s -- 8 bytes, read as one int64
// sort key (strength bits, then y, then x), exactly how the reference sorts it.
__device__ __forceinline__ uint64_t xys_pack(int x, int y, float s)
{
    return (uint64_t)(uint16_t)x | ((uint64_t)(uint16_t)y << 16) | ((uint64_t)__float_as_uint(s) << 32);
}

// non-maximum suppression rule of HafCpu_NonMaxSupp_XY_ANY_3x3 (harris.cpp:882)
template <class SV>
__device__ __forceinline__ bool harris_nms(SV S)
{
    const float v = S(0, 0);
    return v >= S(-1, -1) && v >= S(0, -1) && v >= S(1, -1) && v >= S(-1, 0) && v > S(1, 0) &&
           v > S(-1, 1) && v > S(0, 1) && v > S(1, 1);
}

__device__ __forceinline__ void xys_append(uint64_t *list, uint32_t *count, uint32_t capacity, uint64_t item, bool pred)
{
    const unsigned m = __ballot_sync(__activemask(), pred);
    if (!m) return;
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(m));
    base = __shfl_sync(__activemask(), base, leader);
    if (pred) {
        const uint32_t idx = base + __popc(m & ((1u << lane) - 1));
        if (idx < capacity) list[idx] = item;
    }
}

__global__ void k_harris_nms(int W, int H, const float *sc, int scStride, uint64_t *list, uint32_t *count, uint32_t capacity)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    const bool in = x >= 1 && x < W - 1 && y >= 1 && y < H - 1;
    bool keep = false;
    float v = 0.f;
    if (in) {
        auto S = [&](int dx, int dy) { return *(const float *)((const uint8_t *)sc + (size_t)(y + dy) * scStride + 4 * (x + dx)); };
        keep = harris_nms(S);
        v = S(0, 0);
    }
    xys_append(list, count, capacity, xys_pack(x, y, v), keep);
}

// Harris front end as column strips: a warp owns 120 output columns (lanes 1..30, four
// columns each; lanes 0 and 31 carry the halo) and walks down 32 output rows with rolling
// registers.  Per input row a lane loads one word; the Sobel sums run in 16-bit lanes
// (four columns in four registers), the products and window sums in float -- integers
// below 2^24, i.e. exactly the float sums the reference forms in any order.  The score
// keeps the reference's float operation order, and its division is skipped only where the
// result cannot exceed the threshold.
constexpr int kHRows = 64, kHCols = 120;

__device__ __forceinline__ uint32_t harris_word(const uint8_t *src, int stride, int W, int H, int x, int y, bool fast)
{
    if (fast && y >= 0 && y < H) return __ldg((const uint32_t *)(src + (size_t)y * stride + x));
    uint32_t w = 0;
    for (int k = 0; k < 4; k++) w |= (uint32_t)ago_px(src, stride, W, H, x + k, y) << (8 * k);
    return w;
}

// biased 16-bit lane (value + 1024) as an exact float
__device__ __forceinline__ float lane_lo(uint32_t w) { return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7610)) - 8389632.0f; }
__device__ __forceinline__ float lane_hi(uint32_t w) { return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7632)) - 8389632.0f; }

// TMA form: each warp copies its source rows ys-3 .. ys+kHRows+2, columns from (xs-4) rounded
// down to 16 bytes, 144 bytes wide, into shared memory with one tensor copy on its own
// mbarrier (the warps of a block are independent)
constexpr int kHBoxW = 144, kHBoxH = kHRows + 6;
constexpr int kHBoxSlot = (kHBoxH * kHBoxW + 127) & ~127;   // a TMA destination starts on 128 bytes

template <bool TMA>
__global__ void __launch_bounds__(128)
k_harris_rows(int W, int H, const uint8_t *__restrict__ src, int srcStride, float k, float Tc, float norm,
              uint64_t *list, uint32_t *count, uint32_t capacity, uint32_t *pStatus, const __grid_constant__ CUtensorMap map)
{
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int xs = (blockIdx.x * (blockDim.x >> 5) + wib) * kHCols;
    if (xs >= W) return;                                   // warp-uniform
    const int xl = xs - 4 + 4 * lane;                      // this lane's columns xl .. xl+3
    const int ys = blockIdx.y * kHRows, yEnd = min(ys + kHRows, H);
    const bool fast = ((((uintptr_t)src | (uintptr_t)srcStride) & 3) == 0) && xl >= 0 && xl + 4 <= W;
    __shared__ __align__(128) uint8_t sBox[TMA ? 4 : 1][TMA ? kHBoxSlot : 16];
    static_assert(kHBoxSlot % 128 == 0, "each warp's box starts on a 128-byte boundary");
    __shared__ __align__(8) uint64_t sBar[4];
    const int bx = (xs - 4) & ~15;                         // box start column
    if constexpr (TMA) {
        const uint32_t b = smem_addr_u32(&sBar[wib]);
        if (lane == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(kHBoxH * kHBoxW) : "memory");
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                ::"r"(smem_addr_u32(sBox[wib])), "l"((uint64_t)&map), "r"(bx), "r"(ys - 3), "r"(b) : "memory");
        }
        __syncwarp();
        bool done = false;
        for (int i = 0; i < kCannyWaitLimit && !done; i++) done = mbarrier_try_wait_parity(b, 0);
        if (!__all_sync(0xffffffffu, done)) {
            // the copy did not complete: report it, give it one more bounded wait, leave
            if (lane == 0) atomicOr(pStatus, AGOCUDA_HARRIS_STATUS_TMA_TIMEOUT);
            for (int i = 0; i < kCannyWaitLimit && !done; i++) done = mbarrier_try_wait_parity(b, 0);
            return;
        }
        // TMA writes zeros outside the plane, as ago_px reads except where the row pitch is W
        // (W % 16 == 0): column -1 is the previous row's last pixel, column W the next row's first
        if ((W & 15) == 0) {
            uint8_t *row = sBox[wib];
            for (int i = lane; i < kHBoxH; i += 32) {
                const int y = ys - 3 + i;
                if (bx < 0) row[i * kHBoxW - 1 - bx] = (y >= 1 && y < H) ? src[(size_t)(y - 1) * srcStride + W - 1] : 0;
                if (W - bx < kHBoxW) row[i * kHBoxW + W - bx] = (y >= 0 && y + 1 < H) ? src[(size_t)(y + 1) * srcStride] : 0;
            }
        }
        __syncwarp();
    }
    // source word of this lane at row y
    auto word = [&](int y) -> uint32_t {
        if constexpr (TMA) return *(const uint32_t *)(sBox[wib] + (y - (ys - 3)) * kHBoxW + (xl - bx));
        else return harris_word(src, srcStride, W, H, xl, y, fast);
    };
    const bool outLane = lane >= 1 && lane <= 30;
    bool gradCol[4], scoreCol[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        gradCol[c] = xl + c >= 0 && xl + c < W;
        scoreCol[c] = xl + c >= 1 && xl + c < W - 1;
    }
    // the score is 0 without the division where Mc < zLess or Mc <= zLessEq:
    // Tc > 0: Mc < 0.999 Tc norm (the quotient cannot exceed Tc); Tc == 0: Mc <= 0
    const float cut = Tc > 0.f ? __fmul_rn(0.999f, __fmul_rn(Tc, norm)) : 0.f;
    const float zLess = Tc > 0.f ? cut : -INFINITY, zLessEq = Tc == 0.f ? 0.f : -INFINITY;
    // rolling state, rotated by the unrolled loop: input rows as 16-bit lanes, products of
    // gradient rows, scores (columns -1 .. 4) of score rows
    Lanes4 X[3] = {};
    float P[3][3][4] = {};
    float S[3][6] = {};
    uint32_t next = word(ys - 3);
    const int rLast = yEnd + 2;

    // one input row r: t, m = rows r-2, r-1 (b receives row r); v0, v1 = products at
    // gradient rows g-2, g-1 (p receives g = r-1); sA, sB = scores at rows s-2, s-1 (sc
    // receives s = g-1); suppression at n = s-1
    auto step = [&](int r, const Lanes4 &t, const Lanes4 &m, Lanes4 &b, const float (&v0)[3][4],
                    const float (&v1)[3][4], float (&p)[3][4], const float (&sA)[6], const float (&sB)[6],
                    float (&sc)[6]) {
        const uint32_t cur = next;
        if (r + 1 <= rLast) next = word(r + 1);
        b = lanes4(__shfl_up_sync(0xffffffffu, cur, 1), cur, __shfl_down_sync(0xffffffffu, cur, 1));
        // gradient at g = r - 1 (HafCpu_HarrisSobel_HG3_U8_3x3, harris.cpp:85)
        const int g = r - 1;
        {
            const uint32_t bias = 0x04000400u;
            const uint32_t vE = t.E + 2 * m.E + b.E, vO = t.O + 2 * m.O + b.O;
            const uint32_t vOm = t.Om + 2 * m.Om + b.Om, vEp = t.Ep + 2 * m.Ep + b.Ep;
            const uint32_t gx02 = vO + bias - vOm, gx13 = vEp + bias - vE;
            const uint32_t gy02 = (b.Om + 2 * b.E + b.O) + bias - (t.Om + 2 * t.E + t.O);
            const uint32_t gy13 = (b.E + 2 * b.O + b.Ep) + bias - (t.E + 2 * t.O + t.Ep);
            const float gx[4] = {lane_lo(gx02), lane_lo(gx13), lane_hi(gx02), lane_hi(gx13)};
            const float gy[4] = {lane_lo(gy02), lane_lo(gy13), lane_hi(gy02), lane_hi(gy13)};
            const bool rowOk = g >= 1 && g < H - 1;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const bool ok = rowOk && gradCol[c];
                p[0][c] = ok ? __fmul_rn(gx[c], gx[c]) : 0.f;
                p[1][c] = ok ? __fmul_rn(gx[c], gy[c]) : 0.f;
                p[2][c] = ok ? __fmul_rn(gy[c], gy[c]) : 0.f;
            }
        }
        // window sums at s = g - 1 over gradient rows g-2 .. g (HafCpu_HarrisScore_HVC_HG3_3x3)
        float vs[3][6];
#pragma unroll
        for (int q = 0; q < 3; q++) {
#pragma unroll
            for (int c = 0; c < 4; c++) vs[q][c + 1] = __fadd_rn(__fadd_rn(v0[q][c], v1[q][c]), p[q][c]);
            vs[q][0] = __shfl_up_sync(0xffffffffu, vs[q][4], 1);
            vs[q][5] = __shfl_down_sync(0xffffffffu, vs[q][1], 1);
        }
        const int srow = g - 1;
        const bool sRowOk = srow >= 1 && srow < H - 1;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const float gx2 = __fadd_rn(__fadd_rn(vs[0][c], vs[0][c + 1]), vs[0][c + 2]);
            const float gxy2 = __fadd_rn(__fadd_rn(vs[1][c], vs[1][c + 1]), vs[1][c + 2]);
            const float gy2 = __fadd_rn(__fadd_rn(vs[2][c], vs[2][c + 1]), vs[2][c + 2]);
            const float traceA = __fadd_rn(gx2, gy2);
            const float detA = __fsub_rn(__fmul_rn(gx2, gy2), __fmul_rn(gxy2, gxy2));
            const float Mc = __fsub_rn(detA, __fmul_rn(__fmul_rn(k, traceA), traceA));
            float v = 0.f;
            if (sRowOk && scoreCol[c] && !(Mc < zLess || Mc <= zLessEq)) {
                const float q = __fdiv_rn(Mc, norm);
                v = q > Tc ? q : 0.f;
            }
            sc[c + 1] = v;
        }
        sc[0] = __shfl_up_sync(0xffffffffu, sc[4], 1);
        sc[5] = __shfl_down_sync(0xffffffffu, sc[1], 1);
        // non-maximum suppression at n = s - 1 (HafCpu_NonMaxSupp_XY_ANY_3x3, harris.cpp:882):
        // >= the row above and the left neighbour, > the right neighbour and the row below
        const int n = srow - 1;
        const bool rowOut = n >= ys && n < yEnd && n >= 1 && n < H - 1;
        uint32_t keep = 0;
        if (outLane && rowOut) {
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const float v = sB[c + 1];
                const float above = fmaxf(fmaxf(sA[c], sA[c + 1]), sA[c + 2]);
                const float below = fmaxf(fmaxf(sc[c], sc[c + 1]), sc[c + 2]);
                const bool kc = scoreCol[c] && v >= above && v >= sB[c] && v > sB[c + 2] && v > below;
                keep |= (uint32_t)kc << c;
            }
        }
        if (rowOut && __any_sync(0xffffffffu, keep != 0)) {
#pragma unroll
            for (int c = 0; c < 4; c++)
                xys_append(list, count, capacity, xys_pack(xl + c, n, sB[c + 1]), (keep >> c) & 1);
        }
    };
    for (int r = ys - 3; r <= rLast; r += 3) {             // r is warp-uniform
        step(r, X[0], X[1], X[2], P[0], P[1], P[2], S[0], S[1], S[2]);
        if (r + 1 > rLast) break;
        step(r + 1, X[1], X[2], X[0], P[1], P[2], P[0], S[1], S[2], S[0]);
        if (r + 2 > rLast) break;
        step(r + 2, X[2], X[0], X[1], P[2], P[0], P[1], S[2], S[0], S[1]);
    }
}

// ---------------------------------------------------------------------------------
// Corner pick (HafCpu_HarrisMergeSortAndPick_XY_XYS, harris.cpp:923).  Reference: sort the
// candidates descending as int64, then walk them in order keeping a point when its grid cell
// is empty and no kept point in the 5x5 cells around is closer than min_dist2.  That is the
// greedy maximal independent set of the conflict graph (same cell, or within the cell
// window and closer than min_dist2) in sorted order; it is computed here in rounds: a
// candidate is kept once every conflicting predecessor is rejected, and rejected as soon as
// one is kept -- the same set, in parallel.  One CTA; candidates sit in shared memory.
// ---------------------------------------------------------------------------------
constexpr int kPickMax = 8192;                 // candidates held in shared memory
constexpr int kPickHash = 2 * kPickMax;        // open-addressing cell table

struct PickSmem {
    uint64_t key[kPickMax];
    int next[kPickMax];
    int head[kPickHash];
    uint8_t state[kPickMax];   // 0 undecided, 1 kept, 2 rejected
    int changed, undecided, kept;
};

__device__ __forceinline__ int kx(uint64_t k) { return (int)(int16_t)(k & 0xffff); }
__device__ __forceinline__ int ky(uint64_t k) { return (int)(int16_t)((k >> 16) & 0xffff); }
__device__ __forceinline__ float ks(uint64_t k) { return __uint_as_float((uint32_t)(k >> 32)); }
__device__ __forceinline__ uint32_t hcell(int cx, int cy) { return ((uint32_t)cx * 73856093u) ^ ((uint32_t)cy * 19349663u); }

__global__ void __launch_bounds__(1024)
k_harris_pick(const uint64_t *list, const uint32_t *listCount, uint32_t listCapacity, float minDistance,
              int cell, int gridW, int gridH, vx_keypoint_like *out, uint32_t outCapacity, uint32_t *outCount,
              uint32_t *numCorners, uint32_t *status, bool clusterPath)
{
    extern __shared__ __align__(16) uint8_t smem_raw[];
    PickSmem &S = *reinterpret_cast<PickSmem *>(smem_raw);
    const int tid = threadIdx.x, nt = blockDim.x;
    const int n = (int)min(*listCount, listCapacity);
    if (n > kPickMax) {
        // more candidates than this kernel holds: the cluster kernel after it takes them, or,
        // without its scratch, report and emit nothing
        if (!clusterPath && tid == 0) { atomicOr(status, 2u); *outCount = 0; if (numCorners) *numCorners = 0; }
        return;
    }
    int np2 = 1;
    while (np2 < n) np2 <<= 1;
    for (int i = tid; i < np2; i += nt) S.key[i] = i < n ? list[i] : 0;   // 0 sorts last (descending)
    __syncthreads();
    // bitonic sort, descending by the signed int64 value
    for (int k = 2; k <= np2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < np2; i += nt) {
                const int l = i ^ j;
                if (l > i) {
                    const int64_t a = (int64_t)S.key[i], b = (int64_t)S.key[l];
                    const bool desc = (i & k) == 0;
                    if (desc ? (a < b) : (a > b)) { S.key[i] = (uint64_t)b; S.key[l] = (uint64_t)a; }
                }
            }
            __syncthreads();
        }
    const bool useGrid = minDistance > 2.0f;
    if (useGrid) {
        for (int i = tid; i < kPickHash; i += nt) S.head[i] = -1;
        for (int i = tid; i < n; i += nt) { S.next[i] = -1; S.state[i] = 0; }
        __syncthreads();
        // cell lists (any order inside a cell; priorities come from sorted indices)
        for (int i = tid; i < n; i += nt) {
            const int cx = kx(S.key[i]) / cell, cy = ky(S.key[i]) / cell;
            uint32_t h = hcell(cx, cy) & (kPickHash - 1);
            for (int probe = 0; probe < kPickHash; probe++, h = (h + 1) & (kPickHash - 1)) {
                int cur = atomicCAS(&S.head[h], -1, i);
                if (cur == -1) break;                       // new cell: i heads it
                const int ccx = kx(S.key[cur]) / cell, ccy = ky(S.key[cur]) / cell;
                if (ccx == cx && ccy == cy) {               // same cell: push i in front of its list
                    int prev = S.head[h];
                    for (int t = 0; t < kPickMax; t++) {
                        S.next[i] = prev;
                        const int got = atomicCAS(&S.head[h], prev, i);
                        if (got == prev) break;
                        prev = got;
                    }
                    break;
                }
            }
        }
        __syncthreads();
        const int md2 = (int)ceilf(__fmul_rn(minDistance, minDistance));
        for (int round = 0; round <= n; round++) {
            if (tid == 0) S.changed = 0;
            __syncthreads();
            for (int i = tid; i < n; i += nt) {
                if (S.state[i]) continue;
                const int x = kx(S.key[i]), y = ky(S.key[i]);
                const int cx = x / cell, cy = y / cell;
                bool blocked = false, waiting = false;
                for (int yy = max(cy - 2, 0); yy <= min(cy + 2, gridH - 1) && !blocked; yy++)
                    for (int xx = max(cx - 2, 0); xx <= min(cx + 2, gridW - 1) && !blocked; xx++) {
                        uint32_t h = hcell(xx, yy) & (kPickHash - 1);
                        int j = -1;
                        for (int probe = 0; probe < kPickHash; probe++, h = (h + 1) & (kPickHash - 1)) {
                            const int c = S.head[h];
                            if (c < 0) break;
                            if (kx(S.key[c]) / cell == xx && ky(S.key[c]) / cell == yy) { j = c; break; }
                        }
                        for (; j >= 0; j = S.next[j]) {
                            if (j >= i) continue;   // only higher-priority candidates matter
                            const int dx = kx(S.key[j]) - x, dy = ky(S.key[j]) - y;
                            const bool conflict = (xx == cx && yy == cy) || (dx * dx + dy * dy < md2);
                            if (!conflict) continue;
                            const uint8_t sj = S.state[j];
                            if (sj == 1) { blocked = true; break; }
                            if (sj == 0) waiting = true;
                        }
                    }
                if (blocked) { S.state[i] = 2; S.changed = 1; }
                else if (!waiting) { S.state[i] = 1; S.changed = 1; }
            }
            __syncthreads();
            const int ch = S.changed;
            __syncthreads();
            if (!ch) break;
        }
    } else {
        for (int i = tid; i < n; i += nt) S.state[i] = 1;
        __syncthreads();
    }
    // compact kept candidates in sorted order (block-wide scan in chunks of nt)
    if (tid == 0) S.kept = 0;
    __syncthreads();
    __shared__ int warpSums[32];
    for (int base = 0; base < n; base += nt) {
        const int i = base + tid;
        const int f = (i < n && S.state[i] == 1) ? 1 : 0;
        const unsigned m = __ballot_sync(0xffffffffu, f);
        const int lane = tid & 31, w = tid >> 5;
        if (lane == 0) warpSums[w] = __popc(m);
        __syncthreads();
        int off = 0;
        for (int q = 0; q < w; q++) off += warpSums[q];
        const int pos = S.kept + off + __popc(m & ((1u << lane) - 1));
        if (f && pos < (int)outCapacity) {
            const uint64_t kk = S.key[i];
            vx_keypoint_like kp;
            kp.x = kx(kk); kp.y = ky(kk); kp.strength = ks(kk);
            kp.scale = 0.f; kp.orientation = 0.f; kp.tracking_status = 1; kp.error = 0.f;
            out[pos] = kp;
        }
        __syncthreads();
        if (tid == 0) { int t = 0; for (int q = 0; q < (nt + 31) / 32; q++) t += warpSums[q]; S.kept += t; }
        __syncthreads();
    }
    if (tid == 0) {
        *outCount = min((uint32_t)S.kept, outCapacity);
        if (numCorners) *numCorners = (uint32_t)S.kept;
    }
}

// ---------------------------------------------------------------------------------
// Dense candidate sets (more than kPickMax; the reference's list holds up to W*H entries,
// ago_drama_divide.cpp:1726): the same greedy pick by one cluster of kPCtas CTAs over
// global scratch.  The hardware schedules a cluster's CTAs together, so cluster barriers
// (no software spin) separate the phases:
//   1. LSD radix sort, 8 passes of 8 bits, of the keys mapped so that ascending unsigned
//      order is the reference's descending int64 order; each pass is stable (per-CTA digit
//      counts in global memory, per-tile warp ranks from __match_any_sync);
//   2. a dense cell grid (head per cell, next per candidate);
//   3. the rounds of decisions of the shared-memory kernel over the whole cluster, until no
//      candidate is undecided (each round decides at least the highest-priority undecided
//      candidate, so at most n rounds);
//   4. compaction of the kept candidates in sorted order.
// ---------------------------------------------------------------------------------
constexpr int kPCtas = 8, kPThreads = 512, kPWarps = kPThreads / 32;
constexpr uint64_t kSignBit = 0x8000000000000000ull;

struct PickScratch { uint64_t *a, *b; uint32_t *hist; int *head, *next; uint8_t *state; uint32_t *flags; };

static size_t pick_align(size_t v) { return (v + 255) & ~(size_t)255; }

static size_t pick_scratch_layout(uint32_t W, uint32_t H, uint32_t listCapacity, float minDistance, void *base,
                                  PickScratch *ps, int *cellOut, int *gwOut, int *ghOut)
{
    int cell = 1, gw = 1, gh = 1;
    if (minDistance > 2.0f) {   // grid geometry of ago_kernel_api.cpp:20806-20809
        cell = (int)floor((double)minDistance / 1.41421356237309504880);
        gw = (int)((W + cell - 1) / cell);
        gh = (int)((H + cell - 1) / cell);
    }
    if (cellOut) { *cellOut = cell; *gwOut = gw; *ghOut = gh; }
    const size_t n = listCapacity;
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off += pick_align(bytes); return o; };
    const size_t oa = take(n * 8), ob = take(n * 8), oh = take(kPCtas * 256 * 4), ohead = take((size_t)gw * gh * 4),
                 onext = take(n * 4), ost = take(n), ofl = take(64);
    if (ps && base) {
        uint8_t *b = (uint8_t *)base;
        ps->a = (uint64_t *)(b + oa); ps->b = (uint64_t *)(b + ob); ps->hist = (uint32_t *)(b + oh);
        ps->head = (int *)(b + ohead); ps->next = (int *)(b + onext); ps->state = b + ost; ps->flags = (uint32_t *)(b + ofl);
    }
    return off;
}

__device__ __forceinline__ uint64_t pick_unmap(uint64_t t) { return ~t ^ kSignBit; }

__global__ void __cluster_dims__(kPCtas, 1, 1) __launch_bounds__(kPThreads)
k_harris_pick_cluster(const uint64_t *list, const uint32_t *listCount, uint32_t listCapacity, float minDistance,
                      int cell, int gridW, int gridH, vx_keypoint_like *out, uint32_t outCapacity, uint32_t *outCount,
                      uint32_t *numCorners, uint32_t *status, PickScratch P)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int n = (int)min(*listCount, listCapacity);
    if (n <= kPickMax) return;                       // the shared-memory kernel took this list
    const int rank = (int)cluster.block_rank(), tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int gtid = rank * kPThreads + tid, gstride = kPCtas * kPThreads;
    const int per = (n + kPCtas - 1) / kPCtas;
    const int c0 = min(rank * per, n), c1 = min(c0 + per, n);   // this CTA's contiguous chunk
    __shared__ uint32_t hist[256], base[256];
    __shared__ uint16_t wc[kPWarps][256];
    __shared__ int kept;

    // ---- 1. radix sort (the 8th pass leaves the keys in P.a)
    for (int i = c0 + tid; i < c1; i += kPThreads) P.a[i] = ~(list[i] ^ kSignBit);
    uint64_t *src = P.a, *dst = P.b;
    for (int pass = 0; pass < 8; pass++) {
        const int shift = pass * 8;
        if (tid < 256) hist[tid] = 0;
        __syncthreads();
        for (int i = c0 + tid; i < c1; i += kPThreads) atomicAdd(&hist[(src[i] >> shift) & 255], 1u);
        __syncthreads();
        if (tid < 256) P.hist[rank * 256 + tid] = hist[tid];
        __threadfence();
        cluster.sync();
        if (tid < 256) {   // digit d of this CTA starts after every smaller digit and after d in lower ranks
            uint32_t tot = 0, lower = 0;
            for (int c = 0; c < kPCtas; c++) {
                const uint32_t v = __ldcg(&P.hist[c * 256 + tid]);
                tot += v;
                if (c < rank) lower += v;
            }
            hist[tid] = tot;
            base[tid] = lower;
        }
        __syncthreads();
        if (tid == 0) { uint32_t run = 0; for (int d = 0; d < 256; d++) { const uint32_t t = hist[d]; hist[d] = run; run += t; } }
        __syncthreads();
        if (tid < 256) base[tid] += hist[tid];
        __syncthreads();
        for (int t0 = c0; t0 < c1; t0 += kPThreads) {   // stable scatter, one tile of kPThreads keys at a time
            const int i = t0 + tid;
            const bool valid = i < c1;
            const uint64_t key = valid ? src[i] : 0;
            const int d = valid ? (int)((key >> shift) & 255) : 256;
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            const int r = __popc(peers & ((1u << lane) - 1));
            for (int k = tid; k < kPWarps * 256; k += kPThreads) (&wc[0][0])[k] = 0;
            __syncthreads();
            if (valid && r == 0) wc[w][d] = (uint16_t)__popc(peers);
            __syncthreads();
            if (tid < 256) {
                uint32_t run = 0;
                for (int q = 0; q < kPWarps; q++) { const uint32_t c = wc[q][tid]; wc[q][tid] = (uint16_t)run; run += c; }
                hist[tid] = run;
            }
            __syncthreads();
            if (valid) dst[base[d] + wc[w][d] + r] = key;
            __syncthreads();
            if (tid < 256) base[tid] += hist[tid];
            __syncthreads();
        }
        __threadfence();
        cluster.sync();
        uint64_t *t = src; src = dst; dst = t;
    }
    const uint64_t *key = src;

    // ---- 2./3. grid and rounds of decisions
    const bool useGrid = minDistance > 2.0f;
    if (useGrid) {
        for (int c = gtid; c < gridW * gridH; c += gstride) P.head[c] = -1;
        for (int i = gtid; i < n; i += gstride) P.state[i] = 0;
        if (gtid < 3) P.flags[gtid] = 0;
        __threadfence();
        cluster.sync();
        for (int i = gtid; i < n; i += gstride) {
            const uint64_t k = pick_unmap(key[i]);
            const int x = kx(k), y = ky(k);
            const int cx = x / cell, cy = y / cell;
            if (x < 0 || y < 0 || cx >= gridW || cy >= gridH) {   // outside the image the grid covers
                P.state[i] = 2;
                atomicOr(status, AGOCUDA_PICK_STATUS_BAD_ENTRY);
                continue;
            }
            P.next[i] = atomicExch(&P.head[cy * gridW + cx], i);
        }
        __threadfence();
        cluster.sync();
        const int md2 = (int)ceilf(__fmul_rn(minDistance, minDistance));
        for (int round = 0; round <= n; round++) {
            if (gtid == 0) P.flags[(round + 1) % 3] = 0;
            bool undecided = false;
            for (int i = gtid; i < n; i += gstride) {
                if (__ldcg(&P.state[i])) continue;
                const uint64_t k = pick_unmap(key[i]);
                const int x = kx(k), y = ky(k), cx = x / cell, cy = y / cell;
                bool blocked = false, waiting = false;
                for (int yy = max(cy - 2, 0); yy <= min(cy + 2, gridH - 1) && !blocked; yy++)
                    for (int xx = max(cx - 2, 0); xx <= min(cx + 2, gridW - 1) && !blocked; xx++)
                        for (int j = __ldcg(&P.head[yy * gridW + xx]); j >= 0; j = __ldcg(&P.next[j])) {
                            if (j >= i) continue;   // only higher-priority candidates matter
                            const uint64_t kj = pick_unmap(key[j]);
                            const int dx = kx(kj) - x, dy = ky(kj) - y;
                            if (!((xx == cx && yy == cy) || (dx * dx + dy * dy < md2))) continue;
                            const uint8_t sj = __ldcg(&P.state[j]);
                            if (sj == 1) { blocked = true; break; }
                            if (sj == 0) waiting = true;
                        }
                if (blocked) __stcg(&P.state[i], (uint8_t)2);
                else if (!waiting) __stcg(&P.state[i], (uint8_t)1);
                else undecided = true;
            }
            if (__syncthreads_or(undecided) && tid == 0) atomicOr(&P.flags[round % 3], 1u);
            __threadfence();
            cluster.sync();
            if (__ldcg(&P.flags[round % 3]) == 0) break;   // the same value for every thread of the cluster
        }
    } else {
        for (int i = gtid; i < n; i += gstride) P.state[i] = 1;
        __threadfence();
        cluster.sync();
    }

    // ---- 4. kept candidates in sorted order: per-CTA counts, then tile scans of the chunk
    int mine = 0;
    for (int t0 = c0; t0 < c1; t0 += kPThreads) {
        const int i = t0 + tid;
        mine += __syncthreads_count(i < c1 && __ldcg(&P.state[i]) == 1);
    }
    if (tid == 0) P.hist[rank] = (uint32_t)mine;
    __threadfence();
    cluster.sync();
    if (tid == 0) {
        int before = 0, total = 0;
        for (int c = 0; c < kPCtas; c++) { const int v = (int)__ldcg(&P.hist[c]); total += v; if (c < rank) before += v; }
        kept = before;
        if (rank == 0) { *outCount = min((uint32_t)total, outCapacity); if (numCorners) *numCorners = (uint32_t)total; }
    }
    __syncthreads();
    __shared__ int warpSums[kPWarps];
    for (int t0 = c0; t0 < c1; t0 += kPThreads) {
        const int i = t0 + tid;
        const int f = (i < c1 && __ldcg(&P.state[i]) == 1) ? 1 : 0;
        const unsigned m = __ballot_sync(0xffffffffu, f);
        if (lane == 0) warpSums[w] = __popc(m);
        __syncthreads();
        int off = 0;
        for (int q = 0; q < w; q++) off += warpSums[q];
        const int pos = kept + off + __popc(m & ((1u << lane) - 1));
        if (f && pos < (int)outCapacity) {
            const uint64_t kk = pick_unmap(key[i]);
            vx_keypoint_like kp;
            kp.x = kx(kk); kp.y = ky(kk); kp.strength = ks(kk);
            kp.scale = 0.f; kp.orientation = 0.f; kp.tracking_status = 1; kp.error = 0.f;
            out[pos] = kp;
        }
        __syncthreads();
        if (tid == 0) { int t = 0; for (int q = 0; q < kPWarps; q++) t += warpSums[q]; kept += t; }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------
// Harris with 5x5 / 7x7 gradients (HafCpu_HarrisSobel_HG3_U8_{5x5,7x7}, ago_haf_cpu_harris.cpp:
// 333, :455) and 5x5 / 7x7 blocks (HafCpu_HarrisScore_HVC_HG3_{5x5,7x7}, :661, :731), one
// thread per pixel.  Gradients: separable integer taps over every column (the taps leaving
// the row read the neighbouring rows' bytes as AGO lays them out), products rounded to
// float; rows within gs/2 of the top and bottom written 0 (never written by the reference,
// zero in its buffers).  Scores: window sums in the reference's (row, column) order, no
// fused multiply-adds; the 7x7 kernel stores column x's score at x - 1 as the reference does
// (it writes its third border zero without advancing its output pointer).
// ---------------------------------------------------------------------------------
template <int G>
__global__ void __launch_bounds__(256) k_harris_sobel_nxn(int W, int H, float *dst, int dstStride, const uint8_t *src,
                                                         int srcStride)
{
    const int x = blockIdx.x * 64 + (threadIdx.x & 63), y = blockIdx.y * 4 + (threadIdx.x >> 6);
    if (x >= W || y >= H) return;
    constexpr int R = G / 2;
    float *o = (float *)((uint8_t *)dst + (size_t)y * dstStride) + 3 * x;
    if (y < R || y >= H - R) { o[0] = 0.f; o[1] = 0.f; o[2] = 0.f; return; }
    const int d5[5] = {-1, -2, 0, 2, 1}, s5[5] = {1, 4, 6, 4, 1};
    const int d7[7] = {-1, -4, -5, 0, 5, 4, 1}, s7[7] = {1, 6, 15, 20, 15, 6, 1};
    const bool inside = x >= R && x < W - R;
    int gx = 0, gy = 0;
#pragma unroll
    for (int v = -R; v <= R; v++) {
        int hd = 0, hs = 0;
        const uint8_t *row = src + (size_t)(y + v) * srcStride;
#pragma unroll
        for (int u = -R; u <= R; u++) {
            const int p = inside ? (int)row[x + u] : (int)ago_byte(src, (size_t)srcStride, W, H, y + v, x + u);
            hd += (G == 5 ? d5[u + R] : d7[u + R]) * p;
            hs += (G == 5 ? s5[u + R] : s7[u + R]) * p;
        }
        gx += (G == 5 ? s5[v + R] : s7[v + R]) * hd;
        gy += (G == 5 ? d5[v + R] : d7[v + R]) * hs;
    }
    const float fx = (float)gx, fy = (float)gy;
    o[0] = __fmul_rn(fx, fx);
    o[1] = __fmul_rn(fx, fy);
    o[2] = __fmul_rn(fy, fy);
}

template <int B>
__global__ void __launch_bounds__(256) k_harris_score_nxn(int W, int H, float *dst, int dstStride, const float *src,
                                                         int srcStride, float k, float Tc, float norm)
{
    const int x = blockIdx.x * 64 + (threadIdx.x & 63), y = blockIdx.y * 4 + (threadIdx.x >> 6);
    if (x >= W || y >= H) return;
    constexpr int R = B / 2, SHIFT = B == 7 ? 1 : 0;
    // output column x holds the score of column x + SHIFT
    const int c = x + SHIFT;
    float v = 0.f;
    if (y >= R && y < H - R && c >= R && c < W - R) {
        float gx2 = 0.f, gy2 = 0.f, gxy2 = 0.f;
#pragma unroll
        for (int j = -R; j <= R; j++) {
            const float *t = (const float *)((const uint8_t *)src + (size_t)(y + j) * srcStride);
#pragma unroll
            for (int i = -R; i <= R; i++) {
                gx2 = __fadd_rn(gx2, t[3 * (c + i) + 0]);
                gxy2 = __fadd_rn(gxy2, t[3 * (c + i) + 1]);
                gy2 = __fadd_rn(gy2, t[3 * (c + i) + 2]);
            }
        }
        const float traceA = __fadd_rn(gx2, gy2);
        const float detA = __fsub_rn(__fmul_rn(gx2, gy2), __fmul_rn(gxy2, gxy2));
        float Mc = __fsub_rn(detA, __fmul_rn(__fmul_rn(k, traceA), traceA));
        Mc = __fdiv_rn(Mc, norm);
        v = Mc > Tc ? Mc : 0.f;
    }
    *(float *)((uint8_t *)dst + (size_t)y * dstStride + 4 * (size_t)x) = v;
}

bool aligned(const void *p, unsigned a) { return ((uintptr_t)p & (a - 1)) == 0; }

}  // namespace

// =====================================================================================
// C ABI
// =====================================================================================
static dim3 row_grid(uint32_t W, uint32_t H, unsigned bx) { return dim3(div_up(W, bx), H, 1); }

extern "C" int agocuda_CannySobel_U16_U8_3x3_L1NORM(void *stream, uint32_t W, uint32_t H, uint16_t *pDst, uint32_t dstStride,
                                                    const uint8_t *pSrc, uint32_t srcStride)
{
    if (!pDst || !pSrc || W < 3 || H < 3 || dstStride < 2 * W || srcStride < W || !aligned(pDst, 2) || (dstStride & 1))
        return AGOCUDA_INVALID_PARAMS;
    k_canny_sobel<<<row_grid(W, H, 128), 128, 0, as_stream(stream)>>>((int)W, (int)H, pDst, (int)dstStride, pSrc, (int)srcStride);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

#define CANNY_NXN(NAME, G, L2)                                                                                  \
    extern "C" int NAME(void *stream, uint32_t W, uint32_t H, uint16_t *pDst, uint32_t dstStride,              \
                        const uint8_t *pSrc, uint32_t srcStride)                                                \
    {                                                                                                           \
        if (!pDst || !pSrc || W < G || H < G || dstStride < 2 * W || srcStride < W || !aligned(pDst, 2) ||   \
            (dstStride & 1))                                                                                    \
            return AGOCUDA_INVALID_PARAMS;                                                                      \
        k_canny_sobel_nxn<G, L2><<<row_grid(W, H, 128), 128, 0, as_stream(stream)>>>((int)W, (int)H, pDst,    \
                                                                                     (int)dstStride, pSrc,     \
                                                                                     (int)srcStride);          \
        agocuda_count_launch(1);                                                                                \
        return agocuda_launch_status();                                                                         \
    }
CANNY_NXN(agocuda_CannySobel_U16_U8_3x3_L2NORM, 3, true)
CANNY_NXN(agocuda_CannySobel_U16_U8_5x5_L1NORM, 5, false)
CANNY_NXN(agocuda_CannySobel_U16_U8_5x5_L2NORM, 5, true)
CANNY_NXN(agocuda_CannySobel_U16_U8_7x7_L1NORM, 7, false)
CANNY_NXN(agocuda_CannySobel_U16_U8_7x7_L2NORM, 7, true)
#undef CANNY_NXN

extern "C" int agocuda_CannySuppThreshold_U8XY_U16_3x3(void *stream, uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                                       const uint16_t *pSrc, uint32_t srcStride, uint32_t *pStack,
                                                       uint32_t *pStackCount, uint32_t stackCapacity,
                                                       uint16_t hystLower, uint16_t hystUpper)
{
    if (!pDst || !pSrc || !pStack || !pStackCount || W < 3 || H < 3 || dstStride < W || srcStride < 2 * W)
        return AGOCUDA_INVALID_PARAMS;
    cudaMemsetAsync(pStackCount, 0, sizeof(uint32_t), as_stream(stream));
    k_canny_supp<<<row_grid(W, H, 128), 128, 0, as_stream(stream)>>>((int)W, (int)H, pDst, (int)dstStride, pSrc, (int)srcStride,
                                                                      hystLower, hystUpper, pStack, pStackCount, stackCapacity);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" size_t agocuda_CannyEdgeTrace_scratch_size(uint32_t W, uint32_t H)
{
    const size_t n = (size_t)W * H;
    return n * sizeof(int) + ((n + 31) / 32) * sizeof(uint32_t) + 256;
}

// shared by the per-node edge trace and the fused Canny
static int hysteresis_tail(cudaStream_t s, int W, int H, uint8_t *out, int outStride, int *L, uint32_t *bits,
                           const uint32_t *strong, const uint32_t *strongCount, uint32_t capacity, uint32_t *err)
{
    const size_t n = (size_t)W * H;
    cudaMemsetAsync(bits, 0, ((n + 31) / 32) * sizeof(uint32_t), s);
    k_hyst_union<<<row_grid(W, H, 256), 256, 0, s>>>(W, H, L, err);
    k_hyst_mark<<<1184, 256, 0, s>>>(W, H, L, strong, strongCount, capacity, bits, err);
    k_hyst_output<<<row_grid(W, H, 256), 256, 0, s>>>(W, H, out, outStride, L, bits);
    agocuda_count_launch(3);
    return agocuda_launch_status();
}

extern "C" int agocuda_CannyEdgeTrace_U8_U8XY(void *stream, uint32_t W, uint32_t H, uint8_t *pImg, uint32_t stride,
                                              const uint32_t *pStack, const uint32_t *pStackCount, uint32_t stackCapacity,
                                              void *scratch, size_t scratchBytes, uint32_t *pStatus)
{
    if (!pImg || !pStack || !pStackCount || !scratch || !pStatus || W < 3 || H < 3 || stride < W || W > 65535 || H > 65535 ||
        (size_t)W * H >= (1ull << 31) || scratchBytes < agocuda_CannyEdgeTrace_scratch_size(W, H) || !aligned(scratch, 256))
        return AGOCUDA_INVALID_PARAMS;
    int *L = (int *)scratch;
    uint32_t *bits = (uint32_t *)((uint8_t *)scratch + (((size_t)W * H * sizeof(int) + 255) & ~(size_t)255));
    cudaStream_t s = as_stream(stream);
    k_hyst_init<<<row_grid(W, H, 256), 256, 0, s>>>((int)W, (int)H, pImg, (int)stride, L);
    agocuda_count_launch(1);
    return hysteresis_tail(s, (int)W, (int)H, pImg, (int)stride, L, bits, pStack, pStackCount, stackCapacity, pStatus);
}

// ---------------------------------------------------------------------------------
// Hysteresis without any allocation.  The union-find labels and the root bitmap live in a
// file-scope device array of fixed size (every GPU that loads this library holds it until
// the process exits), so a caller that must not allocate device memory can still run the
// edge trace.  Host code may not use the array's name as a device address: the address is
// looked up once per device with cudaGetSymbolAddress, with that device current.
// ---------------------------------------------------------------------------------
constexpr size_t kNoAllocMaxPixels = (size_t)1 << 21;                 // 2,097,152 pixels
constexpr size_t kNoAllocLabelBytes = kNoAllocMaxPixels * sizeof(int);   // 8 MiB
constexpr size_t kNoAllocBitBytes = kNoAllocMaxPixels / 8;               // 256 KiB
static __device__ __align__(256) uint8_t g_noalloc_trace_scratch[kNoAllocLabelBytes + kNoAllocBitBytes];

// The array's device address, per device, together with the context it was looked up in:
// after cudaDeviceReset the device gets a new primary context and the module may load at
// another address, so a changed context means a fresh lookup.
static std::mutex g_noalloc_mu;
static void *g_noalloc_ptr[256];
static CUcontext g_noalloc_ctx[256];

// cuCtxGetCurrent through the runtime's entry-point query: the library does not link the
// driver library itself, so it still loads on a host without a GPU driver.
static CUresult current_context(CUcontext *ctx)
{
    using Fn = CUresult (*)(CUcontext *);
    static Fn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (Fn) nullptr;
        return (Fn)p;
    }();
    return fn ? fn(ctx) : CUDA_ERROR_NOT_FOUND;
}

extern "C" int agocuda_CannyEdgeTrace_U8_U8XY_noalloc(void *stream, uint32_t W, uint32_t H, uint8_t *pImg, uint32_t stride,
                                                      const uint32_t *pStack, const uint32_t *pStackCount,
                                                      uint32_t stackCapacity, uint32_t *pStatus)
{
    if (!pImg || !pStack || !pStackCount || !pStatus || W < 3 || H < 3 || stride < W || W > 65535 || H > 65535)
        return AGOCUDA_INVALID_PARAMS;
    if ((size_t)W * H > kNoAllocMaxPixels) return AGOCUDA_TOO_LARGE;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return (int)e;
    if (dev < 0 || dev >= 256) return AGOCUDA_INVALID_PARAMS;
    void *base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        CUcontext cur = nullptr;
        if (!g_noalloc_ptr[dev] || current_context(&cur) != CUDA_SUCCESS || cur != g_noalloc_ctx[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_trace_scratch);   // makes the primary context current
            if (e != cudaSuccess || !p) return e != cudaSuccess ? (int)e : AGOCUDA_INVALID_PARAMS;
            if (current_context(&cur) != CUDA_SUCCESS) return AGOCUDA_INVALID_PARAMS;
            g_noalloc_ptr[dev] = p;
            g_noalloc_ctx[dev] = cur;
        }
        base = g_noalloc_ptr[dev];
    }
    int *L = (int *)base;
    uint32_t *bits = (uint32_t *)((uint8_t *)base + kNoAllocLabelBytes);
    cudaStream_t s = as_stream(stream);
    // labels are rewritten for every pixel and the bitmap is cleared: nothing carries over
    k_hyst_init<<<row_grid(W, H, 256), 256, 0, s>>>((int)W, (int)H, pImg, (int)stride, L);
    agocuda_count_launch(1);
    return hysteresis_tail(s, (int)W, (int)H, pImg, (int)stride, L, bits, pStack, pStackCount, stackCapacity, pStatus);
}

extern "C" size_t agocuda_CannyEdgeTrace_noalloc_max_pixels(void) { return kNoAllocMaxPixels; }

// scratch of the fused Canny: the per-tile state of CannyTiles, each array 256-byte aligned
static size_t canny_tiles_layout(uint32_t W, uint32_t H, void *base, CannyTiles *T)
{
    CannyTiles c{};
    c.tilesX = (int)div_up(W, kTW);
    c.tilesY = (int)div_up(H, kTH);
    const size_t tiles = (size_t)c.tilesX * c.tilesY;
    auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
    const size_t sizes[6] = {al(tiles * kBorder * 2), al(tiles * kOpenMax * 4), al(tiles * (kOpenMax / 8)),
                             al(tiles * 4), al(tiles * 4), al(tiles * kRunMax * 4)};
    size_t off[6], o = 0;
    for (int i = 0; i < 6; i++) { off[i] = o; o += sizes[i]; }
    if (base && T) {
        uint8_t *p = (uint8_t *)base;
        c.blab = (int16_t *)(p + off[0]);
        c.uf = (int *)(p + off[1]);
        c.sbits = (uint32_t *)(p + off[2]);
        c.nOpen = (uint32_t *)(p + off[3]);
        c.runCount = (uint32_t *)(p + off[4]);
        c.runs = (uint32_t *)(p + off[5]);
        *T = c;
    }
    return o;
}

extern "C" int agocuda_fused_CannyEdgeDetector_3x3_L1(void *stream, uint32_t W, uint32_t H, uint8_t *pDst, uint32_t dstStride,
                                                      const uint8_t *pSrc, uint32_t srcStride, uint16_t hystLower,
                                                      uint16_t hystUpper, void *scratch, size_t scratchBytes, uint32_t *pStatus)
{
    if (!pDst || !pSrc || !scratch || !pStatus || W < 3 || H < 3 || dstStride < W || srcStride < W || W > 65535 ||
        H > 65535 || !aligned(scratch, 256))
        return AGOCUDA_INVALID_PARAMS;
    CannyTiles T{};
    if (scratchBytes < canny_tiles_layout(W, H, scratch, &T)) return AGOCUDA_INVALID_PARAMS;
    cudaStream_t s = as_stream(stream);
    const int tiles = T.tilesX * T.tilesY, nodes = tiles * kOpenMax;
    // the input tiles come by TMA where the plane allows a tensor map (16-byte aligned rows);
    // the map is a kernel parameter, so a captured launch keeps it
    CUtensorMap map;
    memset(&map, 0, sizeof(map));
    if (agocuda_u8_tensor_map(&map, pSrc, W, H, srcStride, kInPitchTma * 4, kIH))
        k_canny_ccl_front<true><<<dim3(T.tilesX, T.tilesY), 256, 0, s>>>(
            (int)W, (int)H, pSrc, (int)srcStride, hystLower, hystUpper, pDst, (int)dstStride, T, pStatus, map);
    else
        k_canny_ccl_front<false><<<dim3(T.tilesX, T.tilesY), 256, 0, s>>>(
            (int)W, (int)H, pSrc, (int)srcStride, hystLower, hystUpper, pDst, (int)dstStride, T, pStatus, map);
    constexpr int kPer = kTH + kTW + kTH;
    k_canny_ccl_border<<<dim3(div_up(kPer, 128), tiles), 128, 0, s>>>((int)W, (int)H, T, pStatus);
    k_canny_ccl_flatten<<<div_up(nodes, 256), 256, 0, s>>>(T, nodes);
    k_canny_ccl_patch<<<div_up(tiles, 8), 256, 0, s>>>(tiles, T, pDst, (int)dstStride);
    agocuda_count_launch(4);
    return agocuda_launch_status();
}

extern "C" size_t agocuda_fused_CannyEdgeDetector_scratch_size(uint32_t W, uint32_t H)
{
    return canny_tiles_layout(W, H, nullptr, nullptr) + 256;   // + room to align an arbitrary base to 256
}

extern "C" int agocuda_HarrisSobel_HG3_U8_3x3(void *stream, uint32_t W, uint32_t H, float *pDst, uint32_t dstStride,
                                              const uint8_t *pSrc, uint32_t srcStride)
{
    if (!pDst || !pSrc || W < 3 || H < 3 || dstStride < 12 * W || srcStride < W || !aligned(pDst, 4) || (dstStride & 3))
        return AGOCUDA_INVALID_PARAMS;
    k_harris_sobel<<<row_grid(W, H, 128), 128, 0, as_stream(stream)>>>((int)W, (int)H, pDst, (int)dstStride, pSrc, (int)srcStride);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_HarrisScore_HVC_HG3_3x3(void *stream, uint32_t W, uint32_t H, float *pDst, uint32_t dstStride,
                                               const float *pSrc, uint32_t srcStride, float sensitivity,
                                               float strengthThreshold, float normFactor)
{
    if (!pDst || !pSrc || W < 3 || H < 3 || dstStride < 4 * W || srcStride < 12 * W || !aligned(pDst, 4) || !aligned(pSrc, 4))
        return AGOCUDA_INVALID_PARAMS;
    k_harris_score<<<row_grid(W, H, 128), 128, 0, as_stream(stream)>>>((int)W, (int)H, pDst, (int)dstStride, pSrc, (int)srcStride,
                                                                       sensitivity, strengthThreshold, normFactor);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_NonMaxSupp_XY_ANY_3x3(void *stream, uint32_t W, uint32_t H, const float *pSrc, uint32_t srcStride,
                                             uint64_t *pList, uint32_t *pListCount, uint32_t listCapacity)
{
    if (!pSrc || !pList || !pListCount || W < 3 || H < 3 || srcStride < 4 * W || !aligned(pSrc, 4))
        return AGOCUDA_INVALID_PARAMS;
    cudaMemsetAsync(pListCount, 0, 4, as_stream(stream));
    k_harris_nms<<<row_grid(W, H, 128), 128, 0, as_stream(stream)>>>((int)W, (int)H, pSrc, (int)srcStride, pList, pListCount, listCapacity);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" size_t agocuda_HarrisMergeSortAndPick_scratch_size(uint32_t W, uint32_t H, uint32_t listCapacity,
                                                              float minDistance)
{
    return pick_scratch_layout(W, H, listCapacity, minDistance, nullptr, nullptr, nullptr, nullptr, nullptr);
}

extern "C" int agocuda_HarrisMergeSortAndPick_XY_XYS(void *stream, uint32_t W, uint32_t H, const uint64_t *pList,
                                                     const uint32_t *pListCount, uint32_t listCapacity, float minDistance,
                                                     void *pCorners, uint32_t cornerCapacity, uint32_t *pCornerCount,
                                                     uint32_t *pNumCorners, void *scratch, size_t scratchBytes,
                                                     uint32_t *pStatus)
{
    if (!pList || !pListCount || !pCorners || !pCornerCount || !pStatus || !W || !H || !(minDistance > 0.0f))
        return AGOCUDA_INVALID_PARAMS;
    int cell = 1, gw = 1, gh = 1;
    PickScratch ps{};
    const size_t need = pick_scratch_layout(W, H, listCapacity, minDistance, scratch, &ps, &cell, &gw, &gh);
    const bool cluster = scratch != nullptr && listCapacity > (uint32_t)kPickMax;
    if (cluster && (scratchBytes < need || !aligned(scratch, 256))) return AGOCUDA_INVALID_PARAMS;
    static bool attr = false;
    const int smem = (int)sizeof(PickSmem);
    if (!attr) {
        if (cudaFuncSetAttribute(k_harris_pick, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
            return agocuda_launch_status();
        attr = true;
    }
    cudaStream_t s = as_stream(stream);
    k_harris_pick<<<1, 1024, smem, s>>>(pList, pListCount, listCapacity, minDistance, cell, gw, gh,
                                        (vx_keypoint_like *)pCorners, cornerCapacity, pCornerCount, pNumCorners, pStatus,
                                        cluster);
    agocuda_count_launch(1);
    if (cluster) {
        k_harris_pick_cluster<<<kPCtas, kPThreads, 0, s>>>(pList, pListCount, listCapacity, minDistance, cell, gw, gh,
                                                           (vx_keypoint_like *)pCorners, cornerCapacity, pCornerCount,
                                                           pNumCorners, pStatus, ps);
        agocuda_count_launch(1);
    }
    return agocuda_launch_status();
}

// Candidate list capacity of the fused Harris: the suppression keeps no two 8-adjacent
// pixels (>= towards the left and upper row, > towards the right and lower row), so at most
// one pixel of every 2x2 block survives.
static uint32_t harris_list_capacity(uint32_t W, uint32_t H) { return ((W + 1) / 2) * ((H + 1) / 2); }

extern "C" int agocuda_fused_HarrisCorners_3x3(void *stream, uint32_t W, uint32_t H, const uint8_t *pSrc, uint32_t srcStride,
                                               float sensitivity, float strengthThreshold, float normFactor, float minDistance,
                                               void *pCorners, uint32_t cornerCapacity, uint32_t *pCornerCount,
                                               uint32_t *pNumCorners, void *scratch, size_t scratchBytes, uint32_t *pStatus)
{
    const uint32_t cap = harris_list_capacity(W, H);
    const size_t listBytes = pick_align((size_t)cap * 8);
    if (!pSrc || !pCorners || !pCornerCount || !scratch || !pStatus || W < 3 || H < 3 || srcStride < W ||
        scratchBytes < agocuda_fused_HarrisCorners_scratch_size(W, H, minDistance) || !aligned(scratch, 256))
        return AGOCUDA_INVALID_PARAMS;
    uint32_t *cnt = (uint32_t *)scratch;
    uint64_t *list = (uint64_t *)((uint8_t *)scratch + 256);
    void *pickScratch = (uint8_t *)scratch + 256 + listBytes;
    cudaStream_t s = as_stream(stream);
    cudaMemsetAsync(cnt, 0, 4, s);
    const int strips = (int)div_up(W, kHCols);
    // the source rows come by TMA where the plane allows a tensor map (16-byte aligned rows);
    // the map is a kernel parameter, so a captured launch keeps it
    CUtensorMap map;
    memset(&map, 0, sizeof(map));
    const dim3 grd(div_up(strips, 4), div_up(H, kHRows));
    if (agocuda_u8_tensor_map(&map, pSrc, W, H, srcStride, kHBoxW, kHBoxH))
        k_harris_rows<true><<<grd, 128, 0, s>>>((int)W, (int)H, pSrc, (int)srcStride, sensitivity, strengthThreshold,
                                                normFactor, list, cnt, cap, pStatus, map);
    else
        k_harris_rows<false><<<grd, 128, 0, s>>>((int)W, (int)H, pSrc, (int)srcStride, sensitivity, strengthThreshold,
                                                 normFactor, list, cnt, cap, pStatus, map);
    agocuda_count_launch(1);
    int rc = agocuda_launch_status();
    if (rc) return rc;
    return agocuda_HarrisMergeSortAndPick_XY_XYS(stream, W, H, list, cnt, cap, minDistance, pCorners, cornerCapacity,
                                                 pCornerCount, pNumCorners, pickScratch,
                                                 agocuda_HarrisMergeSortAndPick_scratch_size(W, H, cap, minDistance), pStatus);
}

extern "C" size_t agocuda_fused_HarrisCorners_scratch_size(uint32_t W, uint32_t H, float minDistance)
{
    const uint32_t cap = harris_list_capacity(W, H);
    return 256 + pick_align((size_t)cap * 8) + agocuda_HarrisMergeSortAndPick_scratch_size(W, H, cap, minDistance);
}

extern "C" int agocuda_HarrisSobel_HG3_U8_NxN(void *stream, uint32_t W, uint32_t H, float *pDst, uint32_t dstStride,
                                              const uint8_t *pSrc, uint32_t srcStride, uint32_t gradientSize)
{
    if (!pDst || !pSrc || (gradientSize != 5 && gradientSize != 7) || W < gradientSize || H < gradientSize ||
        dstStride < 12 * W || srcStride < W || !aligned(pDst, 4) || (dstStride & 3))
        return AGOCUDA_INVALID_PARAMS;
    const dim3 grd(div_up(W, 64), div_up(H, 4));
    if (gradientSize == 5)
        k_harris_sobel_nxn<5><<<grd, 256, 0, as_stream(stream)>>>((int)W, (int)H, pDst, (int)dstStride, pSrc, (int)srcStride);
    else
        k_harris_sobel_nxn<7><<<grd, 256, 0, as_stream(stream)>>>((int)W, (int)H, pDst, (int)dstStride, pSrc, (int)srcStride);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_HarrisScore_HVC_HG3_NxN(void *stream, uint32_t W, uint32_t H, float *pDst, uint32_t dstStride,
                                               const float *pSrc, uint32_t srcStride, float sensitivity,
                                               float strengthThreshold, float normFactor, uint32_t blockSize)
{
    if (!pDst || !pSrc || (blockSize != 5 && blockSize != 7) || W < blockSize || H < blockSize || dstStride < 4 * W ||
        srcStride < 12 * W || !aligned(pDst, 4) || !aligned(pSrc, 4) || (dstStride & 3) || (srcStride & 3))
        return AGOCUDA_INVALID_PARAMS;
    const dim3 grd(div_up(W, 64), div_up(H, 4));
    if (blockSize == 5)
        k_harris_score_nxn<5><<<grd, 256, 0, as_stream(stream)>>>((int)W, (int)H, pDst, (int)dstStride, pSrc, (int)srcStride,
                                                                  sensitivity, strengthThreshold, normFactor);
    else
        k_harris_score_nxn<7><<<grd, 256, 0, as_stream(stream)>>>((int)W, (int)H, pDst, (int)dstStride, pSrc, (int)srcStride,
                                                                  sensitivity, strengthThreshold, normFactor);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}
