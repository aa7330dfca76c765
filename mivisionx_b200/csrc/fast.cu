// fast.cu -- vxFastCornersNode (org.khronos.openvx.fast_corners) on sm_100a: FAST-9 corners of
// a U8 image with and without non-maximum suppression, as a raster-ordered vx_keypoint_t list.
//
// Reference arithmetic (HafCpu_FastCorners_XY_U8_{NoSupression,Supression},
// ago_haf_cpu_fast_corners.cpp:414, :599): a pixel c is a corner when 9 contiguous pixels of
// the 16-pixel radius-3 circle are all > c + t or all < c - t (16-bit compares, t =
// floor(strength_threshold)).  Without suppression rows 3 .. H-4 and EVERY column are tested
// (the circle of the outer three columns reads across the row end in AGO's layout) and each
// corner's strength is the threshold.  With suppression rows 3 .. H-4 and columns 3 .. W-4
// get a strength -- the reference's binary search (:216) for the largest threshold that
// still gives a corner, which is (max over 9-arcs of the arc's minimum contrast) - 1 on each
// side, the larger side kept -- and a corner survives when its strength is >= its upper and
// left neighbours and > its right and lower ones.  The list is in raster order; the count
// scalar holds every corner, the array min(count, capacity).  The reference's GPU path
// appends with atomics; this one keeps the CPU path's order.
//
// Four launches: k_fast_map (strengths / flags, one 128x8 tile per CTA staged in shared
// memory), k_fast_rows (a warp per row: suppression, ballot bitmap and row count),
// k_fast_scan (one CTA: row offsets and counts) and k_fast_emit (a warp per row writes its
// keypoints at its offset).
#include "agocuda_internal.cuh"

uint64_t agocuda_count_launch(unsigned n);

namespace {

constexpr int kFtX = 128, kFtY = 8, kFtHalo = 4;
constexpr int kFtSW = kFtX + 2 * kFtHalo, kFtSH = kFtY + 6;   // 136 x 14 bytes

__device__ __constant__ int8_t kCircleDx[16] = {0, 1, 2, 3, 3, 3, 2, 1, 0, -1, -2, -3, -3, -3, -2, -1};
__device__ __constant__ int8_t kCircleDy[16] = {-3, -3, -2, -1, 0, 1, 2, 3, 3, 3, 2, 1, 0, -1, -2, -3};

// bit i: circle pixels i .. i+8 (mod 16) all set in m
__device__ __forceinline__ bool arc9(uint32_t m)
{
    const uint32_t r = m | (m << 16);
    uint32_t a = r & (r >> 1);
    a &= a >> 2;
    a &= a >> 4;
    a &= r >> 8;
    return (a & 0xFFFFu) != 0;
}

// max over the 16 circular windows of 9 of the window minimum of d
__device__ __forceinline__ int best_arc_min(const int d[16])
{
    int m1[16], m2[16], m4[16];
#pragma unroll
    for (int i = 0; i < 16; i++) m1[i] = min(d[i], d[(i + 1) & 15]);
#pragma unroll
    for (int i = 0; i < 16; i++) m2[i] = min(m1[i], m1[(i + 2) & 15]);
#pragma unroll
    for (int i = 0; i < 16; i++) m4[i] = min(m2[i], m2[(i + 4) & 15]);
    int best = -1 << 20;
#pragma unroll
    for (int i = 0; i < 16; i++) best = max(best, min(m4[i], d[(i + 8) & 15]));
    return best;
}

// map: suppression -> strength (0 = no corner) for rows 3..H-4, columns 3..W-4; otherwise 1 for
// a corner in rows 3..H-4 (every column).  Every other pixel of the map is written 0.
template <bool SUP>
__global__ void __launch_bounds__(256) k_fast_map(int W, int H, const uint8_t *src, int srcStride, int t, uint8_t *map,
                                                 int mapStride)
{
    __shared__ __align__(16) uint8_t tile[kFtSH][kFtSW];
    const int x0 = blockIdx.x * kFtX, y0 = blockIdx.y * kFtY;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const bool edge = x0 - kFtHalo < 0 || x0 + kFtX + kFtHalo > W || y0 - 3 < 0 || y0 + kFtY + 3 > H;
    if (!edge) {
        for (int i = tid; i < kFtSH * (kFtSW / 4); i += 256) {
            const int r = i / (kFtSW / 4), w = i - r * (kFtSW / 4);
            *(uint32_t *)&tile[r][4 * w] = ldg_u32(src + (size_t)(y0 - 3 + r) * srcStride + x0 - kFtHalo + 4 * w);
        }
    } else {
        // image-edge tiles: bytes as AGO's layout holds them (across row ends, zero outside)
        for (int i = tid; i < kFtSH * kFtSW; i += 256) {
            const int r = i / kFtSW, c = i - r * kFtSW;
            tile[r][c] = (uint8_t)ago_byte(src, (size_t)srcStride, W, H, y0 - 3 + r, x0 - kFtHalo + c);
        }
    }
    __syncthreads();
    const int y = y0 + threadIdx.y;
    if (y >= H) return;
    const int lx0 = 4 * threadIdx.x;
    uint32_t out = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int x = x0 + lx0 + q;
        const bool cand = y >= 3 && y < H - 3 && x < W && (!SUP || (x >= 3 && x < W - 3));
        int v = 0;
        if (cand) {
            const int cx = kFtHalo + lx0 + q, cy = 3 + threadIdx.y;
            const int c = tile[cy][cx];
            int b[16];
#pragma unroll
            for (int i = 0; i < 16; i++) b[i] = tile[cy + kCircleDy[i]][cx + kCircleDx[i]];
            const int hi = (int16_t)(c + t), lo = (int16_t)(c - t);
            uint32_t plus = 0, minus = 0;
#pragma unroll
            for (int i = 0; i < 16; i++) {
                plus |= (uint32_t)(b[i] > hi) << i;
                minus |= (uint32_t)(b[i] < lo) << i;
            }
            const bool cp = arc9(plus), cm = arc9(minus);
            if (!SUP) {
                v = cp || cm;
            } else if (cp || cm) {
                int d[16];
                int sp = 0, sn = 0;
                if (cp) {
#pragma unroll
                    for (int i = 0; i < 16; i++) d[i] = b[i] - c;
                    sp = best_arc_min(d) - 1;
                }
                if (cm) {
#pragma unroll
                    for (int i = 0; i < 16; i++) d[i] = c - b[i];
                    sn = best_arc_min(d) - 1;
                }
                v = (uint8_t)max(sp, sn);
            }
        }
        out |= (uint32_t)(v & 0xff) << (8 * q);
    }
    const int x = x0 + lx0;
    uint8_t *d = map + (size_t)y * mapStride + x;
    if (x + 4 <= mapStride) *(uint32_t *)d = out;
    else for (int q = 0; q < mapStride - x; q++) d[q] = (uint8_t)(out >> (8 * q));
}

// one warp per row: the surviving corners of the row as a bitmap and their count
template <bool SUP>
__global__ void __launch_bounds__(256) k_fast_rows(int W, int H, const uint8_t *map, int mapStride, uint32_t *bitmap,
                                                  int words, uint32_t *rowCount)
{
    const int y = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (y >= H) return;
    uint32_t count = 0;
    const uint8_t *row = map + (size_t)y * mapStride;
    for (int w = 0; w < words; w++) {
        const int x = 32 * w + lane;
        bool keep = false;
        if (y >= 3 && y < H - 3 && x < W) {
            const int v = row[x];
            if (!SUP) {
                keep = v != 0;
            } else if (v && x >= 3 && x < W - 3) {
                const uint8_t *u = row - mapStride, *d = row + mapStride;
                keep = v >= u[x - 1] && v >= u[x] && v >= u[x + 1] && v >= row[x - 1] && v > row[x + 1] && v > d[x - 1] &&
                       v > d[x] && v > d[x + 1];
            }
        }
        const uint32_t bits = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) bitmap[(size_t)y * words + w] = bits;
        count += __popc(bits);
    }
    if (lane == 0) rowCount[y] = count;
}

// one CTA of 1024 threads: exclusive scan of the row counts; the totals
__global__ void __launch_bounds__(1024) k_fast_scan(int H, const uint32_t *rowCount, uint32_t *rowStart, uint32_t capacity,
                                                   uint32_t *pCornerCount, uint32_t *pNumCorners)
{
    __shared__ uint32_t warpSum[32];
    const int per = (H + 1023) / 1024, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int r0 = min(H, tid * per), r1 = min(H, r0 + per);
    uint32_t s = 0;
    for (int r = r0; r < r1; r++) s += rowCount[r];
    uint32_t inc = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t n = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += n;
    }
    if (lane == 31) warpSum[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        uint32_t v = warpSum[lane], x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t n = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += n;
        }
        warpSum[lane] = x - v;     // exclusive prefix of the warps
    }
    __syncthreads();
    uint32_t run = warpSum[wid] + inc - s;
    for (int r = r0; r < r1; r++) {
        rowStart[r] = run;
        run += rowCount[r];
    }
    if (tid == 1023) {
        const uint32_t total = warpSum[wid] + inc;
        if (pNumCorners) *pNumCorners = total;
        if (pCornerCount) *pCornerCount = min(total, capacity);
    }
}

template <bool SUP>
__global__ void __launch_bounds__(256) k_fast_emit(int W, int H, const uint8_t *map, int mapStride, const uint32_t *bitmap,
                                                  int words, const uint32_t *rowStart, uint32_t capacity,
                                                  vx_keypoint_like *corners, float threshold)
{
    const int y = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (y >= H) return;
    uint32_t at = rowStart[y];
    if (at >= capacity) return;
    const uint32_t below = (1u << lane) - 1u;
    for (int w = 0; w < words && at < capacity; w++) {
        const uint32_t bits = bitmap[(size_t)y * words + w];
        if ((bits >> lane) & 1u) {
            const uint32_t i = at + __popc(bits & below);
            if (i < capacity) {
                const int x = 32 * w + lane;
                vx_keypoint_like k;
                k.x = x;
                k.y = y;
                k.strength = SUP ? (float)map[(size_t)y * mapStride + x] : threshold;
                k.scale = 0.f;
                k.orientation = 0.f;
                k.tracking_status = 1;
                k.error = 0.f;
                corners[i] = k;
            }
        }
        at += __popc(bits);
    }
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

struct FastScratch {
    uint8_t *map;
    uint32_t *bitmap, *rowCount, *rowStart;
    int mapStride, words;
    size_t bytes;
};

FastScratch fast_layout(uint32_t W, uint32_t H, void *base)
{
    FastScratch s{};
    s.mapStride = (int)((W + 15) & ~15u);
    s.words = (int)((W + 31) / 32);
    uint8_t *p = (uint8_t *)base;
    size_t o = 0;
    s.map = p + o; o += align256((size_t)s.mapStride * H);
    s.bitmap = (uint32_t *)(p + o); o += align256((size_t)s.words * H * 4);
    s.rowCount = (uint32_t *)(p + o); o += align256((size_t)H * 4);
    s.rowStart = (uint32_t *)(p + o); o += align256((size_t)H * 4);
    s.bytes = o;
    return s;
}

}  // namespace

extern "C" size_t agocuda_FastCorners_scratch_size(uint32_t width, uint32_t height)
{
    return fast_layout(width, height, nullptr).bytes;
}

extern "C" int agocuda_FastCorners_XY_U8(void *stream, uint32_t W, uint32_t H, const uint8_t *pSrc, uint32_t srcStride,
                                         float strengthThreshold, int32_t nonmaxSuppression, void *pCorners,
                                         uint32_t cornerCapacity, uint32_t *pCornerCount, uint32_t *pNumCorners,
                                         void *scratch, size_t scratchBytes)
{
    if (!pSrc || !scratch || W < 7 || H < 7 || W > (1u << 20) || H > (1u << 20) || srcStride < W || (srcStride & 3) ||
        ((uintptr_t)pSrc & 3) || ((uintptr_t)scratch & 255) || (cornerCapacity && !pCorners) ||
        !(strengthThreshold > -32768.f && strengthThreshold < 32768.f))
        return AGOCUDA_INVALID_PARAMS;
    const FastScratch s = fast_layout(W, H, scratch);
    if (scratchBytes < s.bytes) return AGOCUDA_INVALID_PARAMS;
    const int t = (int16_t)floorf(strengthThreshold);
    cudaStream_t q = as_stream(stream);
    const dim3 g1(div_up(W, kFtX), div_up(H, kFtY)), b1(32, kFtY);
    const unsigned g2 = div_up(H, 8);
    vx_keypoint_like *kp = (vx_keypoint_like *)pCorners;
    if (nonmaxSuppression) {
        k_fast_map<true><<<g1, b1, 0, q>>>((int)W, (int)H, pSrc, (int)srcStride, t, s.map, s.mapStride);
        k_fast_rows<true><<<g2, 256, 0, q>>>((int)W, (int)H, s.map, s.mapStride, s.bitmap, s.words, s.rowCount);
    } else {
        k_fast_map<false><<<g1, b1, 0, q>>>((int)W, (int)H, pSrc, (int)srcStride, t, s.map, s.mapStride);
        k_fast_rows<false><<<g2, 256, 0, q>>>((int)W, (int)H, s.map, s.mapStride, s.bitmap, s.words, s.rowCount);
    }
    k_fast_scan<<<1, 1024, 0, q>>>((int)H, s.rowCount, s.rowStart, cornerCapacity, pCornerCount, pNumCorners);
    if (nonmaxSuppression)
        k_fast_emit<true><<<g2, 256, 0, q>>>((int)W, (int)H, s.map, s.mapStride, s.bitmap, s.words, s.rowStart,
                                             cornerCapacity, kp, strengthThreshold);
    else
        k_fast_emit<false><<<g2, 256, 0, q>>>((int)W, (int)H, s.map, s.mapStride, s.bitmap, s.words, s.rowStart,
                                              cornerCapacity, kp, strengthThreshold);
    agocuda_count_launch(4);
    return agocuda_launch_status();
}
