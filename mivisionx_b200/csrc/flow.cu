// flow.cu -- Gaussian pyramid levels and pyramidal Lucas-Kanade tracking on sm_100a.
//
// Pyramid level: HafCpu_ScaleGaussianHalf_U8_U8_5x5 (ago_haf_cpu_pyramid.cpp:94), called by
// agoKernel_ScaleGaussianHalf_U8_U8_5x5 (ago_kernel_api.cpp:15420) for destination rows
// 1..H-2; rows 0 and H-1 of a level are never written by the reference (zero in AGO's
// zero-initialised buffers) and are written 0 here.  The 5x5 stencil reads two columns
// outside the row at both image edges; those reads follow AGO's buffer layout (row pitch
// ALIGN16(width), zero padding), so edge threads resolve them with ago_byte().
//
// LK: HafCpu_OpticalFlowPyrLK_XY_XY_Generic (ago_haf_cpu_opticalflow.cpp:153), CPU-only in
// the reference.  One warp tracks one keypoint through every level.  The reference's float
// accumulations run in 4-lane SSE registers in a fixed order; the warp reproduces that order
// exactly: per-pixel work is spread over the lanes and each reference accumulator lane is
// summed sequentially by one lane.  The Scharr derivatives are computed on the fly for the
// window; the few derivative values the reference takes from scratch memory it did not
// write in the current level (column 0's left neighbour of the vertical difference, the
// right neighbour of column W&~7 - 1, derivative row 0) are reproduced: k_lk_prep replays
// the reference's row-buffer writes into a persistent per-node array.
#include "agocuda_internal.cuh"

uint64_t agocuda_count_launch(unsigned n);

namespace {

// ---------------------------------------------------------------------------------
// ScaleGaussianHalf 5x5.  A thread produces 8 output pixels x 8 output rows.  Pixel
// pairs live in the two 16-bit halves of a 32-bit register (horizontal sums <= 4080,
// vertical sums <= 65280, so halves never carry into each other).
// ---------------------------------------------------------------------------------
constexpr int kHalfThreads = 32;
constexpr int kHalfCols = 8 * kHalfThreads;     // output columns per tile
constexpr int kHalfRows = 8;                    // output rows per tile

// One word of a row whose 4 columns [c, c+4) reach outside [0, W): ago_byte() per byte,
// kept out of line (inlined at every call site it made the kernel's code large enough to
// thrash the instruction cache).  Columns within one AGO row pitch of the row (W >= 24)
// skip the division, and the 4 loads issue back to back.
__device__ __noinline__ uint32_t half_edge_word(const uint8_t *src, int stride, int W, int H, int r, int c)
{
    uint32_t out = 0;
    if (W >= 24) {
        const int S = (W + 15) & ~15;
        const uint8_t *ptr[4];
        bool ok[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int cc0 = c + k;
            int rr = r, cc = cc0;
            bool v = true;
            if (cc0 < 0) { rr = r - 1; cc = cc0 + S; v = r > 0 && cc < W; }
            else if (cc0 >= W) { rr = r + 1; cc = cc0 - S; v = cc0 >= S && r + 1 < H && cc < W; }
            ok[k] = v;
            ptr[k] = v ? src + (size_t)rr * stride + cc : src;
        }
        uint32_t px[4];
#pragma unroll
        for (int k = 0; k < 4; k++) px[k] = *ptr[k];
#pragma unroll
        for (int k = 0; k < 4; k++) out |= (ok[k] ? px[k] : 0u) << (8 * k);
        return out;
    }
#pragma unroll 1
    for (int k = 0; k < 4; k++) out |= ago_byte(src, stride, W, H, r, c + k) << (8 * k);
    return out;
}

// Six words covering source bytes [x0, x0 + 24) of row r, x0 = 2*ox - 4 (a multiple of 4):
// words inside the row load directly, the border ones go through half_edge_word
__device__ __forceinline__ void half_load_row(const agocuda_half_job &J, int r, int x0, bool edge, uint32_t w[6])
{
    const uint8_t *p = J.src + (size_t)r * J.srcStride + x0;
    if (!edge) {
        w[0] = *(const uint32_t *)p;
        const uint4 m = *(const uint4 *)(p + 4);
        w[1] = m.x; w[2] = m.y; w[3] = m.z; w[4] = m.w;
        w[5] = *(const uint32_t *)(p + 20);
    } else {
        const int W = (int)J.srcW;
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const int c = x0 + 4 * k;
            w[k] = (c >= 0 && c + 4 <= W) ? *(const uint32_t *)(p + 4 * k)
                                          : half_edge_word(J.src, (int)J.srcStride, W, (int)J.srcH, r, c);
        }
    }
}

// Horizontal [1 4 6 4 1] sums of one source row at the 8 sample columns of a thread,
// as 4 packed pairs.  CO = sample column parity (1: samples at odd offsets).
template <int CO>
__device__ __forceinline__ void half_hsum(const uint32_t w[6], uint32_t h[4])
{
    uint32_t E[6], O[6];
#pragma unroll
    for (int k = 0; k < 6; k++) { E[k] = w[k] & 0x00FF00FFu; O[k] = (w[k] >> 8) & 0x00FF00FFu; }
    const uint32_t *C = CO ? O : E, *N = CO ? E : O;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const uint32_t c0 = C[q + 1];
        const uint32_t cm = __funnelshift_r(C[q], C[q + 1], 16);
        const uint32_t cp = __funnelshift_r(C[q + 1], C[q + 2], 16);
        const uint32_t nm = CO ? N[q + 1] : __funnelshift_r(N[q], N[q + 1], 16);
        const uint32_t np = CO ? __funnelshift_r(N[q + 1], N[q + 2], 16) : N[q + 1];
        h[q] = cm + cp + 6u * c0 + 4u * (nm + np);
    }
}

template <int CO, int ROWS = kHalfRows>
__device__ __forceinline__ void half_tile(const agocuda_half_job &J, int ox, int oy0)
{
    const int oW = (int)J.dstW, oH = (int)J.dstH;
    const int ro = (J.srcH & 1) ? 0 : 1;              // centre row parity (sampleFirstRow = H odd)
    const int x0 = 2 * ox - 4;
    const bool edge = (ox == 0) || (x0 + 24 > (int)J.srcW);
    const int yEnd = min(oy0 + ROWS, oH);
    uint32_t h[5][4];
    int have = 0;                                    // rows of h[] valid for the current output row
    for (int oy = oy0; oy < yEnd; oy++) {
        uint8_t *d = J.dst + (size_t)oy * J.dstStride + ox;
        uint32_t out0 = 0, out1 = 0;
        if (oy >= 1 && oy <= oH - 2) {
            const int rc = 2 * oy + ro;              // centre source row
            if (have == 0) {
#pragma unroll
                for (int i = 0; i < 5; i++) {
                    uint32_t w[6];
                    half_load_row(J, rc - 2 + i, x0, edge, w);
                    half_hsum<CO>(w, h[i]);
                }
            } else {
#pragma unroll
                for (int q = 0; q < 4; q++) { h[0][q] = h[2][q]; h[1][q] = h[3][q]; h[2][q] = h[4][q]; }
#pragma unroll
                for (int i = 3; i < 5; i++) {
                    uint32_t w[6];
                    half_load_row(J, rc - 2 + i, x0, edge, w);
                    half_hsum<CO>(w, h[i]);
                }
            }
            have = 1;
            uint32_t b[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint32_t v = h[0][q] + h[4][q] + 6u * h[2][q] + 4u * (h[1][q] + h[3][q]);
                b[q] = (v >> 8) & 0x00FF00FFu;
            }
            out0 = __byte_perm(b[0], b[1], 0x6420);
            out1 = __byte_perm(b[2], b[3], 0x6420);
        } else {
            have = 0;
        }
        if (ox + 8 <= oW) {
            *(uint2 *)d = make_uint2(out0, out1);
        } else {
            for (int i = 0; ox + i < oW; i++) d[i] = (uint8_t)((i < 4 ? out0 >> (8 * i) : out1 >> (8 * (i - 4))) & 0xFF);
        }
    }
}

__global__ void __launch_bounds__(kHalfThreads) k_gauss_half(const agocuda_half_job *jobs, uint32_t numJobs)
{
    // find the job owning this tile (jobs are sorted by tileBegin)
    uint32_t lo = 0, hi = numJobs - 1;
    const uint32_t t = blockIdx.x;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (jobs[mid].tileBegin <= t) lo = mid; else hi = mid - 1;
    }
    const agocuda_half_job J = jobs[lo];               // by value: dst stores may alias a reference
    const uint32_t local = t - J.tileBegin;
    const uint32_t tilesX = (J.dstW + kHalfCols - 1) / kHalfCols;
    const int ox = (int)(local % tilesX) * kHalfCols + 8 * (int)threadIdx.x;
    const int oy0 = (int)(local / tilesX) * kHalfRows;
    if (ox >= (int)J.dstW) return;
    if (J.srcW & 1) half_tile<0>(J, ox, oy0);
    else half_tile<1>(J, ox, oy0);
}

// Persistent form with a tunable tile: THREADS threads x 8 columns wide, ROWS rows high.
// Blocks take tiles from one queue over the jobs' tiles (job j's tiles start at
// jobs[j].tileBegin for this tile shape); queue words as in the config-1 chain.
template <int THREADS, int ROWS>
__global__ void __launch_bounds__(THREADS) k_gauss_half_persistent(const agocuda_half_job *jobs, uint32_t numJobs,
                                                                    uint32_t totalTiles, uint32_t *queue)
{
    __shared__ uint32_t next;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) next = atomicAdd(queue, 1u);
        __syncthreads();
        const uint32_t t = next;
        if (t >= totalTiles) break;
        uint32_t lo = 0, hi = numJobs - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (jobs[mid].tileBegin <= t) lo = mid; else hi = mid - 1;
        }
        const agocuda_half_job J = jobs[lo];
        const uint32_t local = t - J.tileBegin;
        const uint32_t tilesX = (J.dstW + 8 * THREADS - 1) / (8 * THREADS);
        const int ox = (int)(local % tilesX) * 8 * THREADS + 8 * (int)threadIdx.x;
        const int oy0 = (int)(local / tilesX) * ROWS;
        if (ox < (int)J.dstW) {
            if (J.srcW & 1) half_tile<0, ROWS>(J, ox, oy0);
            else half_tile<1, ROWS>(J, ox, oy0);
        }
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(queue + 1, 1u) == gridDim.x - 1) {
            atomicExch(queue, 0u);
            atomicExch(queue + 1, 0u);
        }
    }
}

__global__ void __launch_bounds__(kHalfThreads) k_gauss_half_one(const agocuda_half_job J)
{
    const uint32_t tilesX = (J.dstW + kHalfCols - 1) / kHalfCols;
    const int ox = (int)(blockIdx.x % tilesX) * kHalfCols + 8 * (int)threadIdx.x;
    const int oy0 = (int)(blockIdx.x / tilesX) * kHalfRows;
    if (ox >= (int)J.dstW) return;
    if (J.srcW & 1) half_tile<0>(J, ox, oy0);
    else half_tile<1>(J, ox, oy0);
}

// ---------------------------------------------------------------------------------
// TMA-staged form: a block of 112 threads produces 112 output columns x 32 output rows of one
// level.  One tensor copy brings the source box -- columns 2*ox0-16 .. 2*ox0+239, rows
// 2*oy0+ro-2 .. +67 -- into shared memory (completion on an mbarrier, bounded wait; the box
// start column is a multiple of 16 bytes); box columns outside the row are then rewritten with
// the bytes AGO's buffer layout holds there (ago_byte), so every output equals the register
// form's.  A thread computes 8 output columns x 4 output rows from shared-memory words.
// ---------------------------------------------------------------------------------
constexpr int kHtCols = 112, kHtRows = 32, kHtThreads = 112;
constexpr int kHtGroups = kHtCols / 8;                  // 14 column groups of 8 outputs
constexpr int kHtRowsPerThread = kHtRows / (kHtThreads / kHtGroups);   // 4
constexpr int kHtBoxW = 256, kHtBoxH = 2 * kHtRows + 4;
constexpr int kHtWaitLimit = 1 << 20;

template <int CO>
__device__ __forceinline__ void half_rows_smem(const agocuda_half_job &J, const uint8_t (*tile)[kHtBoxW], int sx0,
                                               int sy0, int ox, int oyA, int oyB)
{
    const int oW = (int)J.dstW, oH = (int)J.dstH;
    const int ro = (J.srcH & 1) ? 0 : 1;
    const int c0 = 2 * ox - 4 - sx0;                    // tile column of the thread's first word
    uint32_t h[5][4];
    int have = 0;
    auto row_sum = [&](int r, uint32_t hq[4]) {
        const uint32_t *p = (const uint32_t *)&tile[r][c0];
        uint32_t w[6];
#pragma unroll
        for (int k = 0; k < 6; k++) w[k] = p[k];
        half_hsum<CO>(w, hq);
    };
    for (int oy = oyA; oy < oyB; oy++) {
        uint8_t *d = J.dst + (size_t)oy * J.dstStride + ox;
        uint32_t out0 = 0, out1 = 0;
        if (oy >= 1 && oy <= oH - 2) {
            const int rc = 2 * oy + ro - sy0;           // centre source row, in the tile
            if (have == 0) {
#pragma unroll
                for (int i = 0; i < 5; i++) row_sum(rc - 2 + i, h[i]);
            } else {
#pragma unroll
                for (int q = 0; q < 4; q++) { h[0][q] = h[2][q]; h[1][q] = h[3][q]; h[2][q] = h[4][q]; }
                row_sum(rc + 1, h[3]);
                row_sum(rc + 2, h[4]);
            }
            have = 1;
            uint32_t b[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint32_t v = h[0][q] + h[4][q] + 6u * h[2][q] + 4u * (h[1][q] + h[3][q]);
                b[q] = (v >> 8) & 0x00FF00FFu;
            }
            out0 = __byte_perm(b[0], b[1], 0x6420);
            out1 = __byte_perm(b[2], b[3], 0x6420);
        } else {
            have = 0;
        }
        if (ox + 8 <= oW) {
            *(uint2 *)d = make_uint2(out0, out1);
        } else {
            for (int i = 0; ox + i < oW; i++) d[i] = (uint8_t)((i < 4 ? out0 >> (8 * i) : out1 >> (8 * (i - 4))) & 0xFF);
        }
    }
}

__global__ void __launch_bounds__(kHtThreads) k_gauss_half_tma(const agocuda_half_job *jobs, const CUtensorMap *maps,
                                                               uint32_t numJobs, uint32_t *status)
{
    __shared__ __align__(128) uint8_t tile[kHtBoxH][kHtBoxW];
    __shared__ __align__(8) uint64_t bar;
    uint32_t lo = 0, hi = numJobs - 1;
    const uint32_t t = blockIdx.x;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (jobs[mid].tileBegin <= t) lo = mid; else hi = mid - 1;
    }
    const agocuda_half_job J = jobs[lo];
    const uint32_t local = t - J.tileBegin;
    const uint32_t tilesX = (J.dstW + kHtCols - 1) / kHtCols;
    const int ox0 = (int)(local % tilesX) * kHtCols, oy0 = (int)(local / tilesX) * kHtRows;
    const int ro = (J.srcH & 1) ? 0 : 1;
    const int sx0 = 2 * ox0 - 16, sy0 = 2 * oy0 + ro - 2;
    const int tid = threadIdx.x;
    const uint32_t b = smem_addr_u32(&bar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(kHtBoxW * kHtBoxH) : "memory");
        asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                     ::"r"(smem_addr_u32(&tile[0][0])), "l"((uint64_t)(maps + lo)), "r"(sx0), "r"(sy0), "r"(b) : "memory");
    }
    bool done = false;
    for (int i = 0; i < kHtWaitLimit && !done; i++) done = mbarrier_try_wait_parity(b, 0);
    if (!done) {
        if (tid == 0) atomicOr(status, AGOCUDA_HALF_STATUS_TMA_TIMEOUT);
        for (int i = 0; i < kHtWaitLimit && !done; i++) done = mbarrier_try_wait_parity(b, 0);
        return;
    }
    // box columns the tile reads that lie outside the row take AGO's bytes: 16 on the left at
    // most, on the right from the row end to the last column read
    const int W = (int)J.srcW, H = (int)J.srcH;
    const int cEnd = min(kHtBoxW, 2 * (min(ox0 + kHtCols, (int)J.dstW) - ox0) + 36);
    const int lEnd = max(0, min(-sx0, cEnd)), rBeg = max(W - sx0, 0);
    const int nL = lEnd, nR = max(0, cEnd - rBeg), per = nL + nR;
    if (per > 0) {
        const int rows = min(kHtBoxH, 2 * (min(oy0 + kHtRows, (int)J.dstH) - oy0) + 4);
        for (int i = tid; i < rows * per; i += kHtThreads) {
            const int r = i / per, k = i - r * per;
            const int c = k < nL ? k : rBeg + (k - nL);
            tile[r][c] = (uint8_t)ago_byte(J.src, (size_t)J.srcStride, W, H, sy0 + r, sx0 + c);
        }
        __syncthreads();
    }
    const int ox = ox0 + 8 * (tid % kHtGroups);
    const int oyA = oy0 + kHtRowsPerThread * (tid / kHtGroups);
    const int oyB = min(oyA + kHtRowsPerThread, (int)J.dstH);
    if (ox >= (int)J.dstW || oyA >= oyB) return;
    if (J.srcW & 1) half_rows_smem<0>(J, tile, sx0, sy0, ox, oyA, oyB);
    else half_rows_smem<1>(J, tile, sx0, sy0, ox, oyA, oyB);
}

// ---------------------------------------------------------------------------------
// Pyramidal LK
// ---------------------------------------------------------------------------------
constexpr int kLkWarps = 8;
constexpr int kWin = AGOCUDA_LK_MAX_WINDOW;
constexpr int kWBits = 14;
constexpr int kPatchPerLane = ((kWin + 3) * (kWin + 3) + 31) / 32;   // image patch bytes per lane
constexpr int kJPerLane = ((kWin + 1) * (kWin + 1) + 31) / 32;       // J window bytes per lane
constexpr float kFltScale = 1.f / (1 << 20);
constexpr int kTermEpsilon = 0xF001, kTermBoth = 0xF002;   // VX_TERM_CRITERIA_EPSILON / _BOTH

struct LkWarpSmem {
    int16_t I[kWin * kWin + 1];
    int16_t dI[2 * kWin * kWin + 2];
    union {
        struct { uint8_t img[(kWin + 3) * (kWin + 3) + 2]; int16_t deriv[2 * (kWin + 1) * (kWin + 1)]; } s;
        struct { uint8_t J[(kWin + 1) * (kWin + 1)]; int32_t prod[2 * kWin * kWin]; } it;
    } u;
};

__device__ __forceinline__ int descale(int v, int n) { return (v + (1 << (n - 1))) >> n; }
__device__ __forceinline__ int sat16(int v) { return max(-32768, min(32767, v)); }

// bilinear weights as the reference computes them (opticalflow.cpp:327): float products,
// + 0.5 in double, truncation
__device__ __forceinline__ void lk_weights(float a, float b, int w[4])
{
    const float s = (float)(1 << kWBits);
    w[0] = (int)__dadd_rn((double)__fmul_rn(__fmul_rn(__fsub_rn(1.f, a), __fsub_rn(1.f, b)), s), 0.5);
    w[1] = (int)__dadd_rn((double)__fmul_rn(__fmul_rn(a, __fsub_rn(1.f, b)), s), 0.5);
    w[2] = (int)__dadd_rn((double)__fmul_rn(__fmul_rn(__fsub_rn(1.f, a), b), s), 0.5);
    w[3] = (1 << kWBits) - w[0] - w[1] - w[2];
}

constexpr unsigned kWrX = 1, kWrY = 2, kWrStrength = 4, kWrStatus = 8, kWrError = 16;

// WIN > 0: the window size as a compile-time constant (index arithmetic without divisions);
// WIN == 0: any window size from the frame descriptor
template <int WIN>
__device__ void lk_track_point(const agocuda_lk_frame &F, uint32_t pt, LkWarpSmem &S, int lane, uint32_t *pStatus)
{
    const vx_keypoint_like *oldKP = (const vx_keypoint_like *)F.oldPoints;
    const vx_keypoint_like *estKP = (const vx_keypoint_like *)F.estPoints;
    vx_keypoint_like *outKP = (vx_keypoint_like *)F.newPoints;
    const int win = WIN > 0 ? WIN : F.windowDimension;
    const float fHalf = (float)(win >> 1);
    const vx_keypoint_like o = oldKP[pt];
    if (!o.tracking_status) {                          // untracked input: copied (opticalflow.cpp:199)
        if (lane == 0) {
            vx_keypoint_like &d = outKP[pt];
            d.x = o.x; d.y = o.y; d.strength = o.strength; d.tracking_status = o.tracking_status;
            d.scale = o.scale; d.error = o.error;
        }
        return;
    }
    int32_t ox = 0, oy = 0, ost = 0;
    float ostr = 0.f, oerr = 0.f;
    unsigned wr = 0;
    float carryX = 0.f, carryY = 0.f;                 // the reference's per-point next-level estimate
    const int top = (int)F.levels - 1;
    // 4-pixel SIMD groups of the covariance pass, 8-pixel group of the mismatch pass
    const int ngA = win >= 4 ? (win - 4) / 4 + 1 : 0;          // x <= win-4  (interpolated path)
    const int ngZ = win > 4 ? (win - 5) / 4 + 1 : 0;           // x <  win-4  (integer path)
    const int ng8 = win >= 8 ? 1 : 0;                          // x <= win-8, win <= 15

    for (int level = top; level >= 0; level--) {
        const agocuda_pyramid_level LI = F.oldPyr[level], LJ = F.newPyr[level];
        const float ptScale = ldexpf(1.0f, -level);
        float px = __fmul_rn((float)o.x, ptScale), py = __fmul_rn((float)o.y, ptScale);
        float nx, ny;
        if (level == top) {
            if (F.useInitialEstimate) {
                const vx_keypoint_like e = estKP[pt];
                nx = __fmul_rn((float)e.x, ptScale); ny = __fmul_rn((float)e.y, ptScale);
                ostr = e.strength; ost = e.tracking_status; oerr = e.error;
                wr |= kWrStrength | kWrStatus | kWrError;
            } else {
                nx = px; ny = py;
                ost = o.tracking_status; ostr = o.strength;
                wr |= kWrStatus | kWrStrength;
            }
            carryX = nx; carryY = ny;
        } else {
            carryX = __fmul_rn(carryX, 2.0f); carryY = __fmul_rn(carryY, 2.0f);
            nx = carryX; ny = carryY;
        }
        if (!ost) continue;
        px = __fsub_rn(px, fHalf); py = __fsub_rn(py, fHalf);
        nx = __fsub_rn(nx, fHalf); ny = __fsub_rn(ny, fHalf);
        const int ipx = (int)floorf(px), ipy = (int)floorf(py);
        const int limX = (int)(LI.width - 2u - (uint32_t)win), limY = (int)(LI.height - 2u - (uint32_t)win);
        if (ipx < 0 || ipx >= limX || ipy < 0 || ipy >= limY) {
            if (!level) { ox = (int)nx; oy = (int)ny; ost = 0; oerr = 0.f; wr |= kWrX | kWrY | kWrStatus | kWrError; }
            continue;
        }
        float a = __fsub_rn(px, (float)ipx), b = __fsub_rn(py, (float)ipy);

        // ---- image patch rows ipy-1 .. ipy+win+1, cols ipx-1 .. ipx+win+1
        const int P = win + 3, Q = win + 1;
        __syncwarp();
        {
            uint8_t v[kPatchPerLane];
#pragma unroll
            for (int k = 0; k < kPatchPerLane; k++) {
                const int i = lane + 32 * k, r = ipy - 1 + i / P, c = ipx - 1 + i % P;
                v[k] = (i < P * P && r >= 0 && c >= 0) ? LI.image[(size_t)r * LI.stride + c] : 0;
            }
#pragma unroll
            for (int k = 0; k < kPatchPerLane; k++)
                if (lane + 32 * k < P * P) S.u.s.img[lane + 32 * k] = v[k];
        }
        __syncwarp();
        // ---- Scharr (gx, gy) at window positions (ipy + y, ipx + x), y, x in [0, win]
        {
            const int W8 = (int)(LI.width & ~7u);
            const int tL = (int)(F.scharrWords[level][0] & 0xFFFF);
            const int t0R = (int)(F.scharrWords[level][1] & 0xFFFF), t1R = (int)(F.scharrWords[level][1] >> 16);
            for (int i = lane; i < Q * Q; i += 32) {
                const int y = i / Q, x = i % Q, gr = ipy + y, gc = ipx + x;
                int gx = 0, gy = 0;
                if (gr > 0 && gc >= W8 && level > 0) {   // the previous call's level-0 derivative here
                    const int j = gc - W8;
                    if (F.carry && j < AGOCUDA_LK_CARRY_COLUMNS && gr < (int)F.carryRows) {
                        const int32_t v = F.carry[((level - 1) * AGOCUDA_LK_CARRY_COLUMNS + j) * (int)F.carryRows + gr];
                        gx = (int16_t)(v & 0xFFFF);
                        gy = (int16_t)((uint32_t)v >> 16);
                    }
                } else if (gr > 0 && gc < W8) {
                    const uint8_t *r0 = &S.u.s.img[y * P + x + 1], *r1 = r0 + P, *r2 = r1 + P;  // column gc
                    const int v1c = (int)r2[0] - (int)r0[0];
                    int v0l, v1l, v0r, v1r;
                    if (gc == 0) { v0l = 0; v1l = tL; }
                    else { v0l = 3 * ((int)r0[-1] + r2[-1]) + 10 * r1[-1]; v1l = (int)r2[-1] - (int)r0[-1]; }
                    if (gc + 1 == W8) { v0r = t0R; v1r = t1R; }
                    else { v0r = 3 * ((int)r0[1] + r2[1]) + 10 * r1[1]; v1r = (int)r2[1] - (int)r0[1]; }
                    gx = (int16_t)(uint16_t)(v0r - v0l);
                    gy = (int16_t)(uint16_t)(3 * (v1l + v1r) + 10 * v1c);
                }
                S.u.s.deriv[2 * i] = (int16_t)gx;
                S.u.s.deriv[2 * i + 1] = (int16_t)gy;
            }
        }
        __syncwarp();
        // ---- window values and the covariance matrix
        const bool whole = (a == 0.0f && b == 0.0f);
        int w[4];
        lk_weights(a, b, w);
        for (int p = lane; p < win * win; p += 32) {
            const int y = p / win, x = p % win;
            const uint8_t *s0 = &S.u.s.img[(y + 1) * P + x + 1], *s1 = s0 + P;
            const int16_t *d0 = &S.u.s.deriv[2 * (y * Q + x)], *d1 = d0 + 2 * Q;
            int iv, ix, iy;
            if (whole) {
                iv = s0[0] << 5; ix = d0[0]; iy = d0[1];
            } else {
                iv = descale(s0[0] * w[0] + s0[1] * w[1] + s1[0] * w[2] + s1[1] * w[3], kWBits - 5);
                ix = descale(d0[0] * w[0] + d0[2] * w[1] + d1[0] * w[2] + d1[2] * w[3], kWBits);
                iy = descale(d0[1] * w[0] + d0[3] * w[1] + d1[1] * w[2] + d1[3] * w[3], kWBits);
                if (x < 4 * ngA) { iv = sat16(iv); ix = sat16(ix); iy = sat16(iy); }
            }
            S.I[p] = (int16_t)iv;
            S.dI[2 * p] = (int16_t)ix;
            S.dI[2 * p + 1] = (int16_t)iy;
        }
        __syncwarp();
        float A11, A12, A22;
        {
            // lanes 0..11: SIMD lanes (entry q = lane/4, lane k = lane%4); 12..14: scalar sums
            float acc = 0.f;
            if (whole) {
                if (lane < 3) {
                    for (int y = 0; y < win; y++) {
                        const int16_t *dr = &S.dI[2 * y * win];
                        int x = 0;
                        for (int g = 0; g < ngZ; g++, x += 4) {
                            int s = 0;
                            for (int k = 0; k < 4; k++) {
                                const int gx = dr[2 * (x + k)], gy = dr[2 * (x + k) + 1];
                                s += lane == 0 ? gx * gx : (lane == 1 ? gx * gy : gy * gy);
                            }
                            acc = __fadd_rn(acc, (float)s);
                        }
                        for (; x < win; x++) {
                            const int gx = dr[2 * x], gy = dr[2 * x + 1];
                            acc = __fadd_rn(acc, (float)(lane == 0 ? gx * gx : (lane == 1 ? gx * gy : gy * gy)));
                        }
                    }
                }
                A11 = __shfl_sync(0xffffffffu, acc, 0);
                A12 = __shfl_sync(0xffffffffu, acc, 1);
                A22 = __shfl_sync(0xffffffffu, acc, 2);
            } else {
                if (lane < 12) {
                    const int q = lane >> 2, k = lane & 3;
                    for (int y = 0; y < win; y++)
                        for (int g = 0; g < ngA; g++) {
                            const int p = y * win + 4 * g + k;
                            const float fx = (float)S.dI[2 * p], fy = (float)S.dI[2 * p + 1];
                            acc = __fadd_rn(acc, q == 0 ? __fmul_rn(fx, fx) : (q == 1 ? __fmul_rn(fx, fy) : __fmul_rn(fy, fy)));
                        }
                } else if (lane < 15) {
                    const int q = lane - 12;
                    for (int y = 0; y < win; y++)
                        for (int x = 4 * ngA; x < win; x++) {
                            const int gx = S.dI[2 * (y * win + x)], gy = S.dI[2 * (y * win + x) + 1];
                            acc = __fadd_rn(acc, (float)(q == 0 ? gx * gx : (q == 1 ? gx * gy : gy * gy)));
                        }
                }
                float l[12];
#pragma unroll
                for (int i = 0; i < 12; i++) l[i] = __shfl_sync(0xffffffffu, acc, i);
                A11 = __shfl_sync(0xffffffffu, acc, 12);
                A12 = __shfl_sync(0xffffffffu, acc, 13);
                A22 = __shfl_sync(0xffffffffu, acc, 14);
                if (win >= 4) {
                    A11 = __fadd_rn(A11, __fadd_rn(__fadd_rn(__fadd_rn(l[0], l[1]), l[2]), l[3]));
                    A12 = __fadd_rn(A12, __fadd_rn(__fadd_rn(__fadd_rn(l[4], l[5]), l[6]), l[7]));
                    A22 = __fadd_rn(A22, __fadd_rn(__fadd_rn(__fadd_rn(l[8], l[9]), l[10]), l[11]));
                }
            }
        }
        A11 = __fmul_rn(A11, kFltScale);
        A12 = __fmul_rn(A12, kFltScale);
        A22 = __fmul_rn(A22, kFltScale);
        float D = __fsub_rn(__fmul_rn(A11, A22), __fmul_rn(A12, A12));
        const float t = __fadd_rn(__fmul_rn(__fsub_rn(A11, A22), __fsub_rn(A11, A22)), __fmul_rn(__fmul_rn(4.f, A12), A12));
        const float minEig = __fdiv_rn(__fsub_rn(__fadd_rn(A22, A11), __fsqrt_rn(t)), (float)(2 * win * win));
        if (minEig < 1.0e-04F || D < 1.0e-07F) {
            if (!level) { ox = (int)nx; oy = (int)ny; ost = 0; oerr = 0.f; wr |= kWrX | kWrY | kWrStatus | kWrError; }
            continue;
        }
        D = __fdiv_rn(1.f, D);

        // ---- Gauss-Newton iterations
        float prevDx = 0.f, prevDy = 0.f, ddx = 0.f, ddy = 0.f;
        int jx = INT32_MIN, jy = INT32_MIN;               // integer position of the staged J window
        const bool epsOnly = F.termination == kTermEpsilon;
        const bool epsTest = epsOnly || F.termination == kTermBoth;
        for (unsigned j = 0; j < F.numIterations || (epsOnly && j < AGOCUDA_LK_EPSILON_ONLY_MAX_ITERATIONS);) {
            const int inx = (int)floorf(nx), iny = (int)floorf(ny);
            const int jlimX = (int)(LJ.width - (uint32_t)win), jlimY = (int)(LJ.height - (uint32_t)win);
            if (inx < 0 || inx >= jlimX || iny < 0 || iny >= jlimY) {
                if (!level) { ost = 0; oerr = 0.f; wr |= kWrStatus | kWrError; }
                break;
            }
            a = __fsub_rn(nx, (float)inx);
            b = __fsub_rn(ny, (float)iny);
            lk_weights(a, b, w);
            __syncwarp();
            if (inx != jx || iny != jy) {                 // the J window only moves with the integer position
                uint8_t v[kJPerLane];
#pragma unroll
                for (int k = 0; k < kJPerLane; k++) {
                    const int i = lane + 32 * k;
                    v[k] = i < Q * Q ? LJ.image[(size_t)(iny + i / Q) * LJ.stride + inx + i % Q] : 0;
                }
#pragma unroll
                for (int k = 0; k < kJPerLane; k++)
                    if (lane + 32 * k < Q * Q) S.u.it.J[lane + 32 * k] = v[k];
                jx = inx;
                jy = iny;
            }
            __syncwarp();
            for (int p = lane; p < win * win; p += 32) {
                const int y = p / win, x = p % win;
                const uint8_t *j0 = &S.u.it.J[y * Q + x], *j1 = j0 + Q;
                int jv = descale(j0[0] * w[0] + j0[1] * w[1] + j1[0] * w[2] + j1[1] * w[3], kWBits - 5);
                const int it = x < 8 * ng8 ? sat16(sat16(jv) - S.I[p]) : jv - S.I[p];
                S.u.it.prod[2 * p] = S.dI[2 * p] * it;
                S.u.it.prod[2 * p + 1] = S.dI[2 * p + 1] * it;
            }
            __syncwarp();
            // lanes 0..7: SIMD accumulators qb0 (lanes 0-3) and qb1 (lanes 4-7); lanes 8, 9:
            // the double scalar sums of the pixels after the 8-pixel group
            float acc = 0.f;
            double dacc = 0.0;
            if (lane < 8) {
                if (ng8) {
                    const int col = 2 * (lane >> 2) + ((lane & 3) >> 1), comp = lane & 1;
                    for (int y = 0; y < win; y++) {
                        acc = __fadd_rn(acc, (float)S.u.it.prod[2 * (y * win + col) + comp]);
                        acc = __fadd_rn(acc, (float)S.u.it.prod[2 * (y * win + col + 4) + comp]);
                    }
                }
            } else if (lane < 10) {
                const int comp = lane - 8;
                for (int y = 0; y < win; y++)
                    for (int x = 8 * ng8; x < win; x++)
                        dacc = __dadd_rn(dacc, (double)(float)S.u.it.prod[2 * (y * win + x) + comp]);
            }
            float q[8];
#pragma unroll
            for (int i = 0; i < 8; i++) q[i] = __shfl_sync(0xffffffffu, acc, i);
            double ib1 = __shfl_sync(0xffffffffu, dacc, 8), ib2 = __shfl_sync(0xffffffffu, dacc, 9);
            if (ng8) {
                ib1 = __dadd_rn(ib1, (double)__fadd_rn(__fadd_rn(q[0], q[4]), __fadd_rn(q[2], q[6])));
                ib2 = __dadd_rn(ib2, (double)__fadd_rn(__fadd_rn(q[1], q[5]), __fadd_rn(q[3], q[7])));
            }
            const float b1 = __double2float_rn(__dmul_rn(ib1, (double)kFltScale));
            const float b2 = __double2float_rn(__dmul_rn(ib2, (double)kFltScale));
            const float dx = __fmul_rn(__fsub_rn(__fmul_rn(A12, b2), __fmul_rn(A22, b1)), D);
            const float dy = __fmul_rn(__fsub_rn(__fmul_rn(A12, b1), __fmul_rn(A11, b2)), D);
            nx = __fadd_rn(nx, dx);
            ny = __fadd_rn(ny, dy);
            if (__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)) <= F.epsilon && epsTest) break;
            if (j > 0 && (double)fabsf(__fadd_rn(dx, prevDx)) < 0.01 && (double)fabsf(__fadd_rn(dy, prevDy)) < 0.01) {
                ddx = __fmul_rn(dx, 0.5f);
                ddy = __fmul_rn(dy, 0.5f);
                break;
            }
            prevDx = dx;
            prevDy = dy;
            j++;
        }
        if (!level) {
            ox = (int)__fadd_rn(__fsub_rn(__fadd_rn(nx, fHalf), ddx), 0.5f);
            oy = (int)__fadd_rn(__fsub_rn(__fadd_rn(ny, fHalf), ddy), 0.5f);
            wr |= kWrX | kWrY;
        } else {
            carryX = __fsub_rn(__fadd_rn(nx, fHalf), ddx);
            carryY = __fsub_rn(__fadd_rn(ny, fHalf), ddy);
        }
    }
    if (lane == 0) {
        vx_keypoint_like &d = outKP[pt];
        if (wr & kWrX) d.x = ox;
        if (wr & kWrY) d.y = oy;
        if (wr & kWrStrength) d.strength = ostr;
        if (wr & kWrStatus) d.tracking_status = ost;
        if (wr & kWrError) d.error = oerr;
    }
    (void)pStatus;
}

// 8 resident blocks (64 warps per SM, 32 registers): the tracking loop is latency-bound (its
// sums keep the reference's addition order, so each is one dependent chain), and more warps
// beat the register spills this costs (measured: 2.79 ms per pyramid + LK step at 4 blocks,
// 2.61 at 6, 2.55 at 8)
__global__ void __launch_bounds__(kLkWarps * 32, 8) k_lk_track(agocuda_lk_frame *frames, uint32_t *pStatus)
{
    __shared__ LkWarpSmem smem[kLkWarps];
    const agocuda_lk_frame &F = frames[blockIdx.y];
    const uint32_t pt = blockIdx.x * kLkWarps + (threadIdx.x >> 5);
    if (pt >= F.count) return;
    if (F.windowDimension == 9) lk_track_point<9>(F, pt, smem[threadIdx.x >> 5], threadIdx.x & 31, pStatus);
    else lk_track_point<0>(F, pt, smem[threadIdx.x >> 5], threadIdx.x & 31, pStatus);
}

// Replays the reference's Scharr row-buffer writes (ComputeSharr, opticalflow.cpp:65): per
// level, the buffer words the level reads but does not write are captured first, then the
// level's last processed row is written into the buffer.  The buffer persists per node, so
// the top level sees what the previous execution's level 0 left.  Also checks the point
// counts (ago_kernel_api.cpp:20603).
__global__ void __launch_bounds__(256) k_lk_prep(agocuda_lk_frame *frames, uint32_t *pStatus)
{
    agocuda_lk_frame &F = frames[blockIdx.x];
    if (threadIdx.x == 0) {
        const uint32_t n = *F.pOldCount;
        const bool bad = n != *F.pEstCount || n > F.newCapacity;
        F.count = bad ? 0 : n;
        if (bad) atomicOr(pStatus, AGOCUDA_LK_STATUS_BAD_COUNT);
        else *F.pNewCount = n;
    }
    uint16_t *T = F.scharrRows;
    for (int level = (int)F.levels - 1; level >= 0; level--) {
        const agocuda_pyramid_level L = F.oldPyr[level];
        const uint32_t W8 = L.width & ~7u, A = (L.width + 2 + 7) & ~7u;
        __syncthreads();
        if (threadIdx.x == 0) {
            F.scharrWords[level][0] = T[A - 1];
            F.scharrWords[level][1] = (uint32_t)T[W8] | ((uint32_t)T[A + W8] << 16);
        }
        __syncthreads();
        if (L.height >= 3) {
            const uint8_t *r0 = L.image + (size_t)(L.height - 3) * L.stride, *r1 = r0 + L.stride, *r2 = r1 + L.stride;
            for (uint32_t c = threadIdx.x; c < W8; c += blockDim.x) {
                T[c] = (uint16_t)(3 * (r0[c] + r2[c]) + 10 * r1[c]);
                T[A + c] = (uint16_t)((int)r2[c] - (int)r0[c]);
            }
        }
    }
}

// After tracking: the level-0 Scharr derivative of this call's old image at the columns
// [W_l & ~7, W_l - 3] of every level l >= 1, which the next call's level l reads (the
// reference's derivative buffer has the level-0 row pitch at every level, and only level 0
// reaches those words).  Rows 1 .. H_l - 3; row 0 is never written and stays 0.
__global__ void __launch_bounds__(256) k_lk_carry(const agocuda_lk_frame *frames)
{
    const agocuda_lk_frame &F = frames[blockIdx.x];
    if (!F.carry) return;
    const agocuda_pyramid_level L0 = F.oldPyr[0];
    for (int level = 1; level < (int)F.levels; level++) {
        const int Wl = (int)F.oldPyr[level].width, Hl = (int)F.oldPyr[level].height, W8 = Wl & ~7;
        const int cols = min(Wl - 2 - W8, AGOCUDA_LK_CARRY_COLUMNS), rows = min(Hl - 2, (int)F.carryRows);
        if (cols <= 0 || rows <= 1) continue;
        for (int i = threadIdx.x; i < cols * rows; i += blockDim.x) {
            const int j = i / rows, y = i - j * rows, x = W8 + j;
            int32_t v = 0;
            if (y >= 1) {
                const uint8_t *r0 = L0.image + (size_t)(y - 1) * L0.stride, *r1 = r0 + L0.stride, *r2 = r1 + L0.stride;
                const int t0l = 3 * (r0[x - 1] + r2[x - 1]) + 10 * r1[x - 1], t0r = 3 * (r0[x + 1] + r2[x + 1]) + 10 * r1[x + 1];
                const int t1l = (int)r2[x - 1] - (int)r0[x - 1], t1c = (int)r2[x] - (int)r0[x], t1r = (int)r2[x + 1] - (int)r0[x + 1];
                const uint32_t gx = (uint16_t)(t0r - t0l), gy = (uint16_t)(3 * (t1l + t1r) + 10 * t1c);
                v = (int32_t)(gx | (gy << 16));
            }
            F.carry[((level - 1) * AGOCUDA_LK_CARRY_COLUMNS + j) * (int)F.carryRows + y] = v;
        }
    }
}

__global__ void k_lk_store_frame(const agocuda_lk_frame F, agocuda_lk_frame *dst)
{
    if (threadIdx.x == 0) {
        // keep the kernel-written fields of an earlier call (count is rewritten by prep)
        const uint32_t n = dst->count;
        *dst = F;
        dst->count = n;
    }
}

bool half_job_ok(uint32_t dstW, uint32_t dstH, const void *dst, uint32_t dstStride, uint32_t srcW, uint32_t srcH,
                 const void *src, uint32_t srcStride)
{
    return dst && src && srcW >= 5 && srcH >= 5 && dstW == (srcW + 1) / 2 && dstH == (srcH + 1) / 2 && dstW >= 3 &&
           dstH >= 3 && ((uintptr_t)dst & 15) == 0 && ((uintptr_t)src & 15) == 0 && (dstStride & 15) == 0 &&
           (srcStride & 15) == 0 && dstStride >= dstW && srcStride >= srcW;
}

}  // namespace

// ---------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------
extern "C" int agocuda_ScaleGaussianHalf_U8_U8_5x5(void *stream, uint32_t dstWidth, uint32_t dstHeight, uint8_t *pDst,
                                                   uint32_t dstStride, uint32_t srcWidth, uint32_t srcHeight,
                                                   const uint8_t *pSrc, uint32_t srcStride)
{
    if (!half_job_ok(dstWidth, dstHeight, pDst, dstStride, srcWidth, srcHeight, pSrc, srcStride))
        return AGOCUDA_INVALID_PARAMS;
    agocuda_half_job J{pSrc, pDst, srcWidth, srcHeight, srcStride, dstWidth, dstHeight, dstStride, 0, 0};
    k_gauss_half_one<<<agocuda_ScaleGaussianHalf_tiles(dstWidth, dstHeight), kHalfThreads, 0, as_stream(stream)>>>(J);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_fused_ScaleGaussianHalf_batch(void *stream, const agocuda_half_job *jobs, uint32_t numJobs,
                                                     uint32_t totalTiles)
{
    if (!jobs || !numJobs || !totalTiles) return AGOCUDA_INVALID_PARAMS;
    k_gauss_half<<<totalTiles, kHalfThreads, 0, as_stream(stream)>>>(jobs, numJobs);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" uint32_t agocuda_ScaleGaussianHalf_tiles_tma(uint32_t dstWidth, uint32_t dstHeight)
{
    return ((dstWidth + kHtCols - 1) / kHtCols) * ((dstHeight + kHtRows - 1) / kHtRows);
}

extern "C" int agocuda_ScaleGaussianHalf_tensor_maps(const agocuda_half_job *jobsHost, uint32_t numJobs, void *mapsHost,
                                                     size_t mapsBytes)
{
    if (!jobsHost || !numJobs || !mapsHost || ((uintptr_t)mapsHost & 63) || mapsBytes < numJobs * sizeof(CUtensorMap))
        return AGOCUDA_INVALID_PARAMS;
    CUtensorMap *maps = (CUtensorMap *)mapsHost;
    for (uint32_t i = 0; i < numJobs; i++) {
        const agocuda_half_job &j = jobsHost[i];
        if (!half_job_ok(j.dstW, j.dstH, j.dst, j.dstStride, j.srcW, j.srcH, j.src, j.srcStride) ||
            !agocuda_u8_tensor_map(&maps[i], j.src, j.srcW, j.srcH, j.srcStride, kHtBoxW, kHtBoxH))
            return AGOCUDA_INVALID_PARAMS;
    }
    return 0;
}

extern "C" int agocuda_fused_ScaleGaussianHalf_tma(void *stream, const agocuda_half_job *jobs, const void *maps,
                                                   uint32_t numJobs, uint32_t totalTiles, uint32_t *pStatus)
{
    if (!jobs || !maps || ((uintptr_t)maps & 63) || !numJobs || !totalTiles || !pStatus) return AGOCUDA_INVALID_PARAMS;
    k_gauss_half_tma<<<totalTiles, kHtThreads, 0, as_stream(stream)>>>(jobs, (const CUtensorMap *)maps, numJobs, pStatus);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" uint32_t agocuda_ScaleGaussianHalf_tiles(uint32_t dstWidth, uint32_t dstHeight)
{
    return ((dstWidth + kHalfCols - 1) / kHalfCols) * ((dstHeight + kHalfRows - 1) / kHalfRows);
}

static bool half_shape_ok(uint32_t threads, uint32_t rows)
{
    return (threads == 32 || threads == 64 || threads == 128) && (rows == 2 || rows == 4 || rows == 8);
}

extern "C" uint32_t agocuda_ScaleGaussianHalf_tiles_shape(uint32_t dstWidth, uint32_t dstHeight, uint32_t threads,
                                                         uint32_t rows)
{
    if (!half_shape_ok(threads, rows)) return 0;
    return ((dstWidth + 8 * threads - 1) / (8 * threads)) * ((dstHeight + rows - 1) / rows);
}

template <int T, int R>
static void half_persistent_launch(cudaStream_t s, unsigned blocks, const agocuda_half_job *jobs, uint32_t n,
                                   uint32_t total, uint32_t *queue)
{
    k_gauss_half_persistent<T, R><<<blocks, T, 0, s>>>(jobs, n, total, queue);
}

extern "C" int agocuda_fused_ScaleGaussianHalf_persistent(void *stream, const agocuda_half_job *jobs, uint32_t numJobs,
                                                          uint32_t totalTiles, uint32_t *queue, uint32_t threads,
                                                          uint32_t rows, uint32_t blocksPerSM)
{
    if (!jobs || !numJobs || !totalTiles || !queue || ((uintptr_t)queue & 7) || !half_shape_ok(threads, rows) ||
        !blocksPerSM || blocksPerSM > 32)
        return AGOCUDA_INVALID_PARAMS;
    const unsigned blocks = (unsigned)agocuda_sm_count() * blocksPerSM;
    cudaStream_t s = as_stream(stream);
#define HALF_CASE(T, R) if (threads == T && rows == R) half_persistent_launch<T, R>(s, blocks, jobs, numJobs, totalTiles, queue);
    HALF_CASE(32, 2) HALF_CASE(32, 4) HALF_CASE(32, 8) HALF_CASE(64, 2) HALF_CASE(64, 4) HALF_CASE(64, 8)
    HALF_CASE(128, 2) HALF_CASE(128, 4) HALF_CASE(128, 8)
#undef HALF_CASE
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" size_t agocuda_OpticalFlowPyrLK_scharr_rows_size(uint32_t width0)
{
    return ((size_t)2 * width0 + 32) * sizeof(uint16_t);
}

extern "C" int agocuda_OpticalFlowPyrLK_batch(void *stream, agocuda_lk_frame *frames, uint32_t numFrames,
                                              uint32_t maxPoints, uint32_t *pStatus)
{
    if (!frames || !numFrames || !pStatus) return AGOCUDA_INVALID_PARAMS;
    cudaStream_t s = as_stream(stream);
    k_lk_prep<<<numFrames, 256, 0, s>>>(frames, pStatus);
    agocuda_count_launch(1);
    if (maxPoints) {
        k_lk_track<<<dim3((maxPoints + kLkWarps - 1) / kLkWarps, numFrames), kLkWarps * 32, 0, s>>>(frames, pStatus);
        agocuda_count_launch(1);
    }
    k_lk_carry<<<numFrames, 256, 0, s>>>(frames);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" size_t agocuda_OpticalFlowPyrLK_carry_size(uint32_t levels, uint32_t height1)
{
    return levels > 1 ? (size_t)(levels - 1) * AGOCUDA_LK_CARRY_COLUMNS * height1 * sizeof(int32_t) : 0;
}

extern "C" size_t agocuda_OpticalFlowPyrLK_scratch_size_carry(uint32_t width0, uint32_t height0, uint32_t levels)
{
    return ((agocuda_OpticalFlowPyrLK_scratch_size(width0) + 255) & ~(size_t)255) +
           agocuda_OpticalFlowPyrLK_carry_size(levels, (height0 + 1) / 2);
}

extern "C" size_t agocuda_OpticalFlowPyrLK_scratch_size(uint32_t width0)
{
    return ((sizeof(agocuda_lk_frame) + 255) & ~(size_t)255) + agocuda_OpticalFlowPyrLK_scharr_rows_size(width0);
}

extern "C" int agocuda_OpticalFlowPyrLK_XY_XY(void *stream, void *newKeyPoint, uint32_t newCapacity, uint32_t *pNewCount,
                                              float pyramidScale, uint32_t levels,
                                              const agocuda_pyramid_level *oldPyramid,
                                              const agocuda_pyramid_level *newPyramid, const uint32_t *pKeyPointCount,
                                              const void *oldKeyPoint, const uint32_t *pEstimateCount,
                                              const void *newKeyPointEstimate, int32_t termination, float epsilon,
                                              uint32_t numIterations, int32_t useInitialEstimate,
                                              int32_t windowDimension, void *scratch, size_t scratchBytes,
                                              uint32_t *pStatus)
{
    if (!newKeyPoint || !pNewCount || !oldPyramid || !newPyramid || !pKeyPointCount || !oldKeyPoint ||
        !pEstimateCount || !newKeyPointEstimate || !scratch || !pStatus || ((uintptr_t)scratch & 255))
        return AGOCUDA_INVALID_PARAMS;
    if (pyramidScale != 0.5f || levels < 1 || levels > AGOCUDA_LK_MAX_LEVELS || windowDimension < 3 ||
        windowDimension > AGOCUDA_LK_MAX_WINDOW)
        return AGOCUDA_INVALID_PARAMS;
    if (scratchBytes < agocuda_OpticalFlowPyrLK_scratch_size(oldPyramid[0].width)) return AGOCUDA_INVALID_PARAMS;
    agocuda_lk_frame F;
    memset(&F, 0, sizeof(F));
    for (uint32_t l = 0; l < levels; l++) {
        const agocuda_pyramid_level &a = oldPyramid[l], &b = newPyramid[l];
        if (!a.image || !b.image || a.width < 8 || a.width != b.width || a.height != b.height || a.height < 3)
            return AGOCUDA_INVALID_PARAMS;
        F.oldPyr[l] = a;
        F.newPyr[l] = b;
    }
    F.oldPoints = oldKeyPoint;
    F.estPoints = newKeyPointEstimate;
    F.newPoints = newKeyPoint;
    F.pOldCount = pKeyPointCount;
    F.pEstCount = pEstimateCount;
    F.pNewCount = pNewCount;
    F.newCapacity = newCapacity;
    F.levels = levels;
    F.termination = termination;
    F.epsilon = epsilon;
    F.numIterations = numIterations;
    F.useInitialEstimate = useInitialEstimate;
    F.windowDimension = windowDimension;
    auto *dev = (agocuda_lk_frame *)scratch;
    F.scharrRows = (uint16_t *)((uint8_t *)scratch + ((sizeof(agocuda_lk_frame) + 255) & ~(size_t)255));
    if (levels > 1 && scratchBytes >= agocuda_OpticalFlowPyrLK_scratch_size_carry(oldPyramid[0].width, oldPyramid[0].height, levels)) {
        F.carry = (int32_t *)((uint8_t *)scratch + ((agocuda_OpticalFlowPyrLK_scratch_size(oldPyramid[0].width) + 255) & ~(size_t)255));
        F.carryRows = oldPyramid[1].height;
    }
    cudaStream_t s = as_stream(stream);
    k_lk_store_frame<<<1, 32, 0, s>>>(F, dev);
    agocuda_count_launch(1);
    const int rc = agocuda_launch_status();
    if (rc) return rc;
    return agocuda_OpticalFlowPyrLK_batch(stream, dev, 1, newCapacity, pStatus);
}
