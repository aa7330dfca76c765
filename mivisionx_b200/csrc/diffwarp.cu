// diffwarp.cu -- differentiable F32 warps on sm_100a: bilinear WarpAffine, WarpPerspective
// and Remap with a constant border, their adjoints, and fused "warp + L2 loss + adjoint"
// steps.
//
// The reference has no F32 warp (its warps validate U8 only, ago_kernel_api.cpp:19255); the
// coordinate conventions are those of its U8 warps.  WarpAffine (ago_haf_cpu_geometric.cpp:
// 679-684, ago_affine_matrix_t m[3][2]):  xs = m00*x + m10*y + m20,  ys = m01*x + m11*y + m21,
// theta holding (m00, m01, m10, m11, m20, m21).  WarpPerspective (ago_haf_cpu_geometric.cpp:
// 1594-1602, ago_perspective_matrix_t m[3][3]):  z = m02*x + m12*y + m22,
// xs = (m00*x + m10*y + m20) / z,  ys = (m01*x + m11*y + m21) / z, theta holding the nine
// entries in storage order; z == 0 samples the border.  Bilinear interpolation from
// floor(xs), floor(ys); each of the four taps outside the source reads the border value.
//
// Adjoint: d/dsrc scatters gout times the tap weights (red.global.add on the source
// gradient); d/dtheta sums gout * (dout/dxs * dxs/dtheta + dout/dys * dys/dtheta) with
// double sums per warp and block (atomicAdd double per block and image).
#include "agocuda_internal.cuh"

uint64_t agocuda_count_launch(unsigned n);

namespace {

struct Taps {
    int x0, y0;
    float fx, fy;
    float p00, p01, p10, p11;
    bool k00, k01, k10, k11;
};

// Positions are formed in double: a float position near x = 1000 is only good to ~6e-5 px,
// and the theta gradient is a strongly cancelling sum over every pixel.
__device__ __forceinline__ Taps taps(const float *src, int stride, int W, int H, double xs, double ys, float border)
{
    Taps t;
    const double fx0 = floor(xs), fy0 = floor(ys);
    t.fx = (float)(xs - fx0);
    t.fy = (float)(ys - fy0);
    // positions far outside the source (or NaN): every tap reads the border
    const bool far = !(fx0 > -2.0 && fx0 < (double)W + 1.0 && fy0 > -2.0 && fy0 < (double)H + 1.0);
    t.x0 = far ? -2 : (int)fx0;
    t.y0 = far ? -2 : (int)fy0;
    if (far) { t.fx = 0.f; t.fy = 0.f; }     // NaN / infinite positions: the border, exactly
    const int x1 = t.x0 + 1, y1 = t.y0 + 1;
    const bool cx0 = t.x0 >= 0 && t.x0 < W, cx1 = x1 >= 0 && x1 < W, cy0 = t.y0 >= 0 && t.y0 < H, cy1 = y1 >= 0 && y1 < H;
    t.k00 = cx0 && cy0; t.k01 = cx1 && cy0; t.k10 = cx0 && cy1; t.k11 = cx1 && cy1;
    t.p00 = t.k00 ? __ldg(src + (size_t)t.y0 * stride + t.x0) : border;
    t.p01 = t.k01 ? __ldg(src + (size_t)t.y0 * stride + x1) : border;
    t.p10 = t.k10 ? __ldg(src + (size_t)y1 * stride + t.x0) : border;
    t.p11 = t.k11 ? __ldg(src + (size_t)y1 * stride + x1) : border;
    return t;
}

__device__ __forceinline__ float interp(const Taps &t)
{
    return (t.p00 * (1.f - t.fx) + t.p01 * t.fx) * (1.f - t.fy) + (t.p10 * (1.f - t.fx) + t.p11 * t.fx) * t.fy;
}

// scatter g times the tap weights into the source gradient
__device__ __forceinline__ void scatter(float *gsrc, int stride, const Taps &t, float g)
{
    if (t.k00) atomicAdd(gsrc + (size_t)t.y0 * stride + t.x0, g * (1.f - t.fx) * (1.f - t.fy));
    if (t.k01) atomicAdd(gsrc + (size_t)t.y0 * stride + t.x0 + 1, g * t.fx * (1.f - t.fy));
    if (t.k10) atomicAdd(gsrc + (size_t)(t.y0 + 1) * stride + t.x0, g * (1.f - t.fx) * t.fy);
    if (t.k11) atomicAdd(gsrc + (size_t)(t.y0 + 1) * stride + t.x0 + 1, g * t.fx * t.fy);
}

__device__ __forceinline__ float dout_dxs(const Taps &t) { return (1.f - t.fy) * (t.p01 - t.p00) + t.fy * (t.p11 - t.p10); }
__device__ __forceinline__ float dout_dys(const Taps &t) { return (1.f - t.fx) * (t.p10 - t.p00) + t.fx * (t.p11 - t.p01); }

// block reduction of N per-thread terms into double atomics at dst[0..N), summed in double
// from the first addition (the theta gradient cancels strongly across pixels)
template <int N>
__device__ __forceinline__ void block_add(const float (&v)[N], double *dst)
{
    __shared__ double red[N][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < N; k++) {
        double s = (double)v[k];
#pragma unroll
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red[k][warp] = (double)s;
    }
    __syncthreads();
    if (threadIdx.x < N) {
        double s = 0.0;
        for (int w = 0; w < nw; w++) s += red[threadIdx.x][w];
        atomicAdd(dst + threadIdx.x, s);
    }
}

struct Img32 {
    float *p;                 // image 0 (image i at p + i * batch)
    long long batch;
    int stride, W, H;
};

enum Mode { kForward = 0, kAdjoint = 1, kFusedL2 = 2 };

// One thread per output pixel of image blockIdx.z.  Modes: forward (out), adjoint (gout ->
// gsrc, gtheta), fused L2 step (target -> gsrc, gtheta and loss with gout = 2 (out - target)).
// NT = 6: affine; NT = 9: perspective.  Per image the adjoint adds NT theta gradients, the
// fused step NT gradients and then the loss.
template <int MODE, int NT>
__global__ void __launch_bounds__(256)
k_warp_f32(int W, int H, Img32 src, Img32 out, Img32 aux, const float *theta, float border, Img32 gsrc, double *gtheta)
{
    const int x = blockIdx.x * 32 + (threadIdx.x & 31), y = blockIdx.y * 8 + (threadIdx.x >> 5), n = blockIdx.z;
    const float *th = theta + NT * n;
    float acc[NT + 1];
#pragma unroll
    for (int k = 0; k <= NT; k++) acc[k] = 0.f;
    if (x < W && y < H) {
        const float fx = (float)x, fy = (float)y;
        double xs, ys, iz = 1.0;
        if (NT == 6) {
            xs = (double)th[0] * x + (double)th[2] * y + (double)th[4];
            ys = (double)th[1] * x + (double)th[3] * y + (double)th[5];
        } else {
            const double z = (double)th[2] * x + (double)th[5] * y + (double)th[8];
            iz = z != 0.0 ? 1.0 / z : 0.0;
            xs = z != 0.0 ? ((double)th[0] * x + (double)th[3] * y + (double)th[6]) * iz : __longlong_as_double(0x7ff8000000000000ll);
            ys = z != 0.0 ? ((double)th[1] * x + (double)th[4] * y + (double)th[7]) * iz : xs;
        }
        const Taps t = taps(src.p + src.batch * n, src.stride, src.W, src.H, xs, ys, border);
        if (MODE == kForward) {
            out.p[out.batch * n + (size_t)y * out.stride + x] = interp(t);
        } else {
            float g;
            if (MODE == kAdjoint) {
                g = aux.p[aux.batch * n + (size_t)y * aux.stride + x];
            } else {
                const float r = interp(t) - aux.p[aux.batch * n + (size_t)y * aux.stride + x];
                acc[NT] = r * r;
                g = 2.f * r;
            }
            scatter(gsrc.p + gsrc.batch * n, gsrc.stride, t, g);
            const float gx = g * dout_dxs(t), gy = g * dout_dys(t);
            if (NT == 6) {
                acc[0] = gx * fx; acc[1] = gy * fx; acc[2] = gx * fy; acc[3] = gy * fy; acc[4] = gx; acc[5] = gy;
            } else if (iz != 0.0 && (gx != 0.f || gy != 0.f)) {   // a sample on the border has no theta term
                // d(xs)/d(m00, m10, m20) = (x, y, 1) / z; d(xs)/d(m02, m12, m22) = -xs (x, y, 1) / z; same for ys
                const double gxz = gx * iz, gyz = gy * iz, q = -((double)gx * xs + (double)gy * ys) * iz;
                acc[0] = (float)(gxz * x); acc[1] = (float)(gyz * x); acc[2] = (float)(q * x);
                acc[3] = (float)(gxz * y); acc[4] = (float)(gyz * y); acc[5] = (float)(q * y);
                acc[6] = (float)gxz; acc[7] = (float)gyz; acc[8] = (float)q;
            }
        }
    }
    if (MODE == kAdjoint) {
        float v[NT];
#pragma unroll
        for (int k = 0; k < NT; k++) v[k] = acc[k];
        block_add<NT>(v, gtheta + NT * n);
    } else if (MODE == kFusedL2) {
        block_add<NT + 1>(acc, gtheta + (NT + 1) * n);
    }
}

// Remap: sample at (x + field[y][x].x, y + field[y][x].y); the adjoint writes gfield per pixel.
template <int MODE>
__global__ void __launch_bounds__(256)
k_remap_f32(int W, int H, Img32 src, Img32 out, Img32 aux, const float2 *field, long long fieldBatch, int fieldStride,
            float border, Img32 gsrc, float2 *gfield)
{
    const int x = blockIdx.x * 32 + (threadIdx.x & 31), y = blockIdx.y * 8 + (threadIdx.x >> 5), n = blockIdx.z;
    if (x >= W || y >= H) return;
    const size_t fi = fieldBatch * n + (size_t)y * fieldStride + x;
    const float2 d = field[fi];
    const Taps t = taps(src.p + src.batch * n, src.stride, src.W, src.H, (double)x + d.x, (double)y + d.y, border);
    if (MODE == kForward) {
        out.p[out.batch * n + (size_t)y * out.stride + x] = interp(t);
    } else {
        const float g = aux.p[aux.batch * n + (size_t)y * aux.stride + x];
        scatter(gsrc.p + gsrc.batch * n, gsrc.stride, t, g);
        gfield[fi] = make_float2(g * dout_dxs(t), g * dout_dys(t));
    }
}

Img32 img32(const float *p, long long batch, int stride, int W, int H) { return Img32{(float *)p, batch, stride, W, H}; }

bool batch_ok(int n, int W, int H, int sW, int sH)
{
    return n > 0 && n <= 65535 && W > 0 && H > 0 && sW > 0 && sH > 0 && W < (1 << 24) && H < (1 << 24) &&
           sW < (1 << 24) && sH < (1 << 24);
}

}  // namespace

extern "C" int agocuda_WarpAffine_F32_Bilinear_Constant_batch(void *stream, int n, int W, int H, float *pDst,
                                                              long long dstBatch, int dstStride, int srcW, int srcH,
                                                              const float *pSrc, long long srcBatch, int srcStride,
                                                              const float *theta, float border)
{
    if (!pDst || !pSrc || !theta || !batch_ok(n, W, H, srcW, srcH) || dstStride < W || srcStride < srcW)
        return AGOCUDA_INVALID_PARAMS;
    const dim3 grd(div_up(W, 32), div_up(H, 8), n);
    k_warp_f32<kForward, 6><<<grd, 256, 0, as_stream(stream)>>>(
        W, H, img32(pSrc, srcBatch, srcStride, srcW, srcH), img32(pDst, dstBatch, dstStride, W, H), Img32{}, theta, border,
        Img32{}, nullptr);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_WarpAffine_F32_Bilinear_Constant_adjoint_batch(void *stream, int n, int W, int H,
                                                                      const float *pGradOut, long long goBatch, int goStride,
                                                                      int srcW, int srcH, const float *pSrc,
                                                                      long long srcBatch, int srcStride, const float *theta,
                                                                      float border, float *pGradSrc, double *pGradTheta)
{
    if (!pGradOut || !pSrc || !theta || !pGradSrc || !pGradTheta || !batch_ok(n, W, H, srcW, srcH) || goStride < W ||
        srcStride < srcW)
        return AGOCUDA_INVALID_PARAMS;
    const dim3 grd(div_up(W, 32), div_up(H, 8), n);
    k_warp_f32<kAdjoint, 6><<<grd, 256, 0, as_stream(stream)>>>(
        W, H, img32(pSrc, srcBatch, srcStride, srcW, srcH), Img32{}, img32(pGradOut, goBatch, goStride, W, H), theta, border,
        img32(pGradSrc, srcBatch, srcStride, srcW, srcH), pGradTheta);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_WarpAffine_F32_L2_step_batch(void *stream, int n, int W, int H, const float *pTarget, long long tBatch,
                                                    int tStride, int srcW, int srcH, const float *pSrc, long long srcBatch,
                                                    int srcStride, const float *theta, float border, float *pGradSrc,
                                                    double *pGradThetaLoss)
{
    if (!pTarget || !pSrc || !theta || !pGradSrc || !pGradThetaLoss || !batch_ok(n, W, H, srcW, srcH) || tStride < W ||
        srcStride < srcW)
        return AGOCUDA_INVALID_PARAMS;
    const dim3 grd(div_up(W, 32), div_up(H, 8), n);
    k_warp_f32<kFusedL2, 6><<<grd, 256, 0, as_stream(stream)>>>(
        W, H, img32(pSrc, srcBatch, srcStride, srcW, srcH), Img32{}, img32(pTarget, tBatch, tStride, W, H), theta, border,
        img32(pGradSrc, srcBatch, srcStride, srcW, srcH), pGradThetaLoss);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_Remap_F32_Bilinear_Constant_batch(void *stream, int n, int W, int H, float *pDst, long long dstBatch,
                                                         int dstStride, int srcW, int srcH, const float *pSrc,
                                                         long long srcBatch, int srcStride, const float *pField,
                                                         long long fieldBatch, int fieldStride, float border)
{
    if (!pDst || !pSrc || !pField || !batch_ok(n, W, H, srcW, srcH) || dstStride < W || srcStride < srcW ||
        fieldStride < W || ((uintptr_t)pField & 7))
        return AGOCUDA_INVALID_PARAMS;
    const dim3 grd(div_up(W, 32), div_up(H, 8), n);
    k_remap_f32<kForward><<<grd, 256, 0, as_stream(stream)>>>(
        W, H, img32(pSrc, srcBatch, srcStride, srcW, srcH), img32(pDst, dstBatch, dstStride, W, H), Img32{},
        (const float2 *)pField, fieldBatch, fieldStride, border, Img32{}, nullptr);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_Remap_F32_Bilinear_Constant_adjoint_batch(void *stream, int n, int W, int H, const float *pGradOut,
                                                                 long long goBatch, int goStride, int srcW, int srcH,
                                                                 const float *pSrc, long long srcBatch, int srcStride,
                                                                 const float *pField, long long fieldBatch, int fieldStride,
                                                                 float border, float *pGradSrc, float *pGradField)
{
    if (!pGradOut || !pSrc || !pField || !pGradSrc || !pGradField || !batch_ok(n, W, H, srcW, srcH) || goStride < W ||
        srcStride < srcW || fieldStride < W || ((uintptr_t)pField & 7) || ((uintptr_t)pGradField & 7))
        return AGOCUDA_INVALID_PARAMS;
    const dim3 grd(div_up(W, 32), div_up(H, 8), n);
    k_remap_f32<kAdjoint><<<grd, 256, 0, as_stream(stream)>>>(
        W, H, img32(pSrc, srcBatch, srcStride, srcW, srcH), Img32{}, img32(pGradOut, goBatch, goStride, W, H),
        (const float2 *)pField, fieldBatch, fieldStride, border, img32(pGradSrc, srcBatch, srcStride, srcW, srcH),
        (float2 *)pGradField);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_WarpPerspective_F32_Bilinear_Constant_batch(void *stream, int n, int W, int H, float *pDst,
                                                                   long long dstBatch, int dstStride, int srcW, int srcH,
                                                                   const float *pSrc, long long srcBatch, int srcStride,
                                                                   const float *theta, float border)
{
    if (!pDst || !pSrc || !theta || !batch_ok(n, W, H, srcW, srcH) || dstStride < W || srcStride < srcW)
        return AGOCUDA_INVALID_PARAMS;
    const dim3 grd(div_up(W, 32), div_up(H, 8), n);
    k_warp_f32<kForward, 9><<<grd, 256, 0, as_stream(stream)>>>(
        W, H, img32(pSrc, srcBatch, srcStride, srcW, srcH), img32(pDst, dstBatch, dstStride, W, H), Img32{}, theta, border,
        Img32{}, nullptr);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_WarpPerspective_F32_Bilinear_Constant_adjoint_batch(void *stream, int n, int W, int H,
                                                                           const float *pGradOut, long long goBatch,
                                                                           int goStride, int srcW, int srcH,
                                                                           const float *pSrc, long long srcBatch,
                                                                           int srcStride, const float *theta, float border,
                                                                           float *pGradSrc, double *pGradTheta)
{
    if (!pGradOut || !pSrc || !theta || !pGradSrc || !pGradTheta || !batch_ok(n, W, H, srcW, srcH) || goStride < W ||
        srcStride < srcW)
        return AGOCUDA_INVALID_PARAMS;
    const dim3 grd(div_up(W, 32), div_up(H, 8), n);
    k_warp_f32<kAdjoint, 9><<<grd, 256, 0, as_stream(stream)>>>(
        W, H, img32(pSrc, srcBatch, srcStride, srcW, srcH), Img32{}, img32(pGradOut, goBatch, goStride, W, H), theta, border,
        img32(pGradSrc, srcBatch, srcStride, srcW, srcH), pGradTheta);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}

extern "C" int agocuda_WarpPerspective_F32_L2_step_batch(void *stream, int n, int W, int H, const float *pTarget,
                                                         long long tBatch, int tStride, int srcW, int srcH, const float *pSrc,
                                                         long long srcBatch, int srcStride, const float *theta, float border,
                                                         float *pGradSrc, double *pGradThetaLoss)
{
    if (!pTarget || !pSrc || !theta || !pGradSrc || !pGradThetaLoss || !batch_ok(n, W, H, srcW, srcH) || tStride < W ||
        srcStride < srcW)
        return AGOCUDA_INVALID_PARAMS;
    const dim3 grd(div_up(W, 32), div_up(H, 8), n);
    k_warp_f32<kFusedL2, 9><<<grd, 256, 0, as_stream(stream)>>>(
        W, H, img32(pSrc, srcBatch, srcStride, srcW, srcH), Img32{}, img32(pTarget, tBatch, tStride, W, H), theta, border,
        img32(pGradSrc, srcBatch, srcStride, srcW, srcH), pGradThetaLoss);
    agocuda_count_launch(1);
    return agocuda_launch_status();
}
