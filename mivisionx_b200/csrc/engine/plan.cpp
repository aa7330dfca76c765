// plan.cpp -- turns the lowered graph into device work.
//
// The reference HIP target launches one kernel per lowered node on one stream
// (ago/ago_util_hip.cpp:686) and cannot fuse (agoGpuHipSuperNodeLaunch returns -1, :740).
// Here the planner (1) matches chains of lowered nodes whose intermediates are virtual and
// private to the chain and replaces each chain by one fused kernel that keeps the
// intermediates on chip, (2) batches identical fused chains of independent sub-graphs
// (same kernel, same by-value parameters, any frame sizes) into ONE launch over a frame
// table, and (3) emits the remaining nodes one launch each.  With
// VX_GRAPH_ATTRIBUTE_AMD_OPTIMIZER_FLAGS bit kOptNoFusion set, every node is its own
// launch: that is the "plain" one-launch-per-node form the fused form is measured against.
#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <set>
#include <sstream>

#include "vx_internal.h"

namespace agovx {

bool lnode_is_output(const LNode &ln, size_t i);

static cudaStream_t S(cudaStream_t s) { return s; }

std::vector<uint32_t> tune_lookup(const char *kernel, uint32_t w, uint32_t h, const std::vector<uint32_t> &dflt);

static uint8_t *dptr(Ref *r) { return IMG(r)->planes[0].dev; }
static uint32_t dstride(Ref *r) { return IMG(r)->planes[0].dev_stride; }
static uint32_t W(Ref *r) { return IMG(r)->width; }
static uint32_t H(Ref *r) { return IMG(r)->height; }

static void *scratch(Graph *g, size_t bytes)
{
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, bytes);
    g->dev_scratch.push_back(p);
    return p;
}

// number of lowered nodes that read `d` (excluding `self`)
static int readers(Graph *g, Ref *d, const LNode *self = nullptr)
{
    int n = 0;
    for (const LNode &ln : g->lnodes) {
        if (&ln == self) continue;
        for (size_t i = 0; i < ln.p.size(); i++) if (!lnode_is_output(ln, i) && ln.p[i] == d) n++;
    }
    return n;
}

static bool private_virtual(Graph *g, Ref *d) { return d && d->is_virtual && readers(g, d) == 1; }

static const LNode *reader_of(Graph *g, Ref *d)
{
    for (const LNode &ln : g->lnodes)
        for (size_t i = 0; i < ln.p.size(); i++) if (!lnode_is_output(ln, i) && ln.p[i] == d) return &ln;
    return nullptr;
}

// Harris score normalisation of the AGO wrappers (ago_kernel_api.cpp:16941-16942 for 3x3
// blocks, :17012-17013 for 5x5, :17083-17084 for 7x7), in float: ((f*f)*f)*f with
// f = 255 * 2^(gradient_size-1) * block_size.
static float harris_norm(int32_t gs, int32_t bs = 3)
{
    const float f0 = 255.0f * (float)(1 << (gs - 1)) * (float)bs;
    volatile float f = f0 * f0;
    f = f * f0;
    f = f * f0;
    return f;
}

// ------------------------------------------------------------------------------------
// The remap table the reference kernels read: vxSetRemapPoint (api/vx_api.cpp:7884) stores
// each float source point as u16 fixed point, (u16)(v * 2^bits + 0.5f) in float, with
// ago_util.cpp:2451's fractional bits, and 0xFFFF in both coordinates for a point outside
// [0, W-1) x [0, H-1).  One uint32 per destination pixel: x | y << 16.
// ------------------------------------------------------------------------------------
static std::vector<uint32_t> remap_fixed_table(const Remap *r)
{
    int bits = 3;
    if (r->src_width >= (1u << 15) || r->src_height >= (1u << 15)) bits = 0;
    else if (r->src_width >= (1u << 14) || r->src_height >= (1u << 14)) bits = 1;
    else if (r->src_width >= (1u << 13) || r->src_height >= (1u << 13)) bits = 2;
    const float sc = (float)(1 << bits), wl = (float)(r->src_width - 1), hl = (float)(r->src_height - 1);
    // float -> u16 as x86 converts it: to int32 with truncation (0x80000000 when out of range)
    auto to_u16 = [](float v) -> uint32_t {
        const int32_t i = (v >= -2147483648.0f && v < 2147483648.0f) ? (int32_t)v : INT32_MIN;
        return (uint32_t)i & 0xFFFF;
    };
    std::vector<uint32_t> out(r->table.size());
    for (size_t k = 0; k < out.size(); k++) {
        const float sx = r->table[k].x, sy = r->table[k].y;
        if (sx < 0.0f || sy < 0.0f || sx >= wl || sy >= hl) out[k] = 0xFFFFFFFFu;
        else out[k] = to_u16(sx * sc + 0.5f) | (to_u16(sy * sc + 0.5f) << 16);
    }
    return out;
}

// ------------------------------------------------------------------------------------
// pyramidal LK: device descriptors of OPTICAL_FLOW_PYR_LK_XY_XY nodes
// (AGO order: new points, old pyramid, new pyramid, old points, estimates, termination,
//  epsilon, num_iterations, use_initial_estimate, window_dimension)
// ------------------------------------------------------------------------------------
// a pyramid level as the kernels see it: a virtual level-0 copy removed by the copy-removal
// pass reads its source image (ago_drama_remove.cpp:926)
static const Image *pyr_level(Graph *g, Pyramid *py, size_t l)
{
    auto it = g->replaced.find(py->level[l]);
    return it == g->replaced.end() ? py->level[l] : IMG(it->second);
}

// Batched steps launch over groups of this many frames: a group's kernels can start while
// later frames are still being uploaded, and groups spread over the capture lanes.
constexpr size_t kGroupFrames = 8;

static vx_status lk_frame(Graph *g, LNode &ln, agocuda_lk_frame &F, uint32_t &cap)
{
    auto &p = ln.p;
    memset(&F, 0, sizeof F);
    Pyramid *po = static_cast<Pyramid *>(p[1]), *pn = static_cast<Pyramid *>(p[2]);
    if (po->levels > AGOCUDA_LK_MAX_LEVELS) return VX_ERROR_NOT_SUPPORTED;
    for (size_t l = 0; l < po->levels; l++) {
        const Image *a = pyr_level(g, po, l), *b = pyr_level(g, pn, l);
        F.oldPyr[l] = agocuda_pyramid_level{a->planes[0].dev, a->width, a->height, a->planes[0].dev_stride, 0};
        F.newPyr[l] = agocuda_pyramid_level{b->planes[0].dev, b->width, b->height, b->planes[0].dev_stride, 0};
    }
    Array *out = static_cast<Array *>(p[0]), *old = static_cast<Array *>(p[3]), *est = static_cast<Array *>(p[4]);
    F.oldPoints = old->dev; F.estPoints = est->dev; F.newPoints = out->dev;
    F.pOldCount = old->dev_count; F.pEstCount = est->dev_count; F.pNewCount = out->dev_count;
    F.newCapacity = (uint32_t)out->capacity;
    F.levels = (uint32_t)po->levels;
    F.termination = sc_enum(p[5]);
    F.epsilon = sc_f32(p[6]);
    F.numIterations = static_cast<Scalar *>(p[7])->v.u32;
    F.useInitialEstimate = static_cast<Scalar *>(p[8])->v.b ? 1 : 0;
    F.windowDimension = (int32_t)static_cast<Scalar *>(p[9])->v.sz;
    // the node's Scharr row-buffer state starts zeroed and persists across executions and
    // re-plans, like the reference's node scratch
    Node *nd = ln.origin;
    void *rows = nd->node_state(0, agocuda_OpticalFlowPyrLK_scharr_rows_size(po->level[0]->width));
    if (!rows) return VX_ERROR_NO_MEMORY;
    F.scharrRows = (uint16_t *)rows;
    if (po->levels > 1) {   // level-0 derivative columns carried to the next execution (zeroed: none yet)
        const uint32_t h1 = pyr_level(g, po, 1)->height;
        void *carry = nd->node_state(1, agocuda_OpticalFlowPyrLK_carry_size((uint32_t)po->levels, h1));
        if (!carry) return VX_ERROR_NO_MEMORY;
        F.carry = (int32_t *)carry;
        F.carryRows = h1;
    }
    cap = (uint32_t)old->capacity;
    return VX_SUCCESS;
}

static vx_status lk_batch_step(Graph *g, const std::vector<LNode *> &nodes, Step &st)
{
    std::vector<agocuda_lk_frame> fr(nodes.size());
    std::vector<uint32_t> cap(nodes.size(), 0);
    for (size_t i = 0; i < nodes.size(); i++)
        if (vx_status s = lk_frame(g, *nodes[i], fr[i], cap[i])) return s;
    void *dev = scratch(g, fr.size() * sizeof(agocuda_lk_frame));
    if (!dev) return VX_ERROR_NO_MEMORY;
    if (cudaMemcpy(dev, fr.data(), fr.size() * sizeof(agocuda_lk_frame), cudaMemcpyHostToDevice) != cudaSuccess)
        return VX_FAILURE;
    uint32_t *status = g->status_dev;
    std::vector<std::function<int(cudaStream_t)>> fns;
    for (size_t k0 = 0; k0 < fr.size(); k0 += kGroupFrames) {
        const size_t k1 = std::min(fr.size(), k0 + kGroupFrames);
        const uint32_t pts = *std::max_element(cap.begin() + k0, cap.begin() + k1);
        agocuda_lk_frame *d0 = (agocuda_lk_frame *)dev + k0;
        const uint32_t n = (uint32_t)(k1 - k0);
        fns.push_back([=](cudaStream_t q) { return agocuda_OpticalFlowPyrLK_batch(S(q), d0, n, pts, status); });
        st.parts.push_back(Part{fns.back(), std::vector<LNode *>(nodes.begin() + k0, nodes.begin() + k1)});
    }
    st.num_kernels = 3 * (int)fns.size();
    st.launch = [fns](cudaStream_t q) {
        for (auto &f : fns) { int rc = f(q); if (rc) return rc; }
        return 0;
    };
    return VX_SUCCESS;
}

// ScaleGaussianHalf levels of many images in one launch (one job per lowered node)
// The TMA-staged batch: one launch per group of levels, source boxes copied by TMA through a
// tensor map per level encoded here.  False when a level's planes cannot be mapped.
static bool half_batch_tma(Graph *g, const std::vector<LNode *> &nodes, Step &st, vx_status &err)
{
    // groups of 16 levels: the groups are separate branches of the captured graph, and with
    // frames from application buffers the first groups start while later frames upload
    const size_t kGroupJobs = 2 * kGroupFrames;
    std::vector<agocuda_half_job> jobs;
    std::vector<uint32_t> group_tiles;
    uint32_t tiles = 0;
    for (size_t i = 0; i < nodes.size(); i++) {
        if (i % kGroupJobs == 0 && i) { group_tiles.push_back(tiles); tiles = 0; }
        const Image *d = IMG(nodes[i]->p[0]), *s = IMG(nodes[i]->p[1]);
        jobs.push_back(agocuda_half_job{s->planes[0].dev, d->planes[0].dev, s->width, s->height, s->planes[0].dev_stride,
                                        d->width, d->height, d->planes[0].dev_stride, tiles, 0});
        tiles += agocuda_ScaleGaussianHalf_tiles_tma(d->width, d->height);
    }
    group_tiles.push_back(tiles);
    const size_t mb = jobs.size() * 128;
    std::vector<uint64_t> host(mb / 8 + 8);
    void *h = (void *)(((uintptr_t)host.data() + 63) & ~(uintptr_t)63);
    if (agocuda_ScaleGaussianHalf_tensor_maps(jobs.data(), (uint32_t)jobs.size(), h, mb) != 0) return false;
    agocuda_half_job *dev = (agocuda_half_job *)scratch(g, jobs.size() * sizeof(agocuda_half_job));
    uint8_t *maps = (uint8_t *)scratch(g, mb);
    if (!dev || !maps) { err = VX_ERROR_NO_MEMORY; return true; }
    if (cudaMemcpy(dev, jobs.data(), jobs.size() * sizeof(agocuda_half_job), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(maps, h, mb, cudaMemcpyHostToDevice) != cudaSuccess) {
        err = VX_FAILURE;
        return true;
    }
    uint32_t *status = g->status_dev;
    std::vector<std::function<int(cudaStream_t)>> fns;
    for (size_t k0 = 0, gi = 0; k0 < jobs.size(); k0 += kGroupJobs, gi++) {
        const size_t k1 = std::min(jobs.size(), k0 + kGroupJobs);
        const agocuda_half_job *d0 = dev + k0;
        const uint8_t *m0 = maps + k0 * 128;
        const uint32_t n = (uint32_t)(k1 - k0), t = group_tiles[gi];
        fns.push_back([=](cudaStream_t q) { return agocuda_fused_ScaleGaussianHalf_tma(S(q), d0, m0, n, t, status); });
        st.parts.push_back(Part{fns.back(), std::vector<LNode *>(nodes.begin() + k0, nodes.begin() + k1)});
    }
    st.num_kernels = (int)fns.size();
    st.launch = [fns](cudaStream_t q) {
        for (auto &f : fns) { int rc = f(q); if (rc) return rc; }
        return 0;
    };
    err = VX_SUCCESS;
    return true;
}

static vx_status half_batch_step(Graph *g, const std::vector<LNode *> &nodes, Step &st)
{
    // launch shape from the autotuner's table (largest output of the batch): threads per
    // block, rows per thread, resident blocks per SM, persistent queue or one block per tile
    uint32_t bw = 0, bh = 0;
    bool streamed = false;
    for (LNode *n : nodes) {
        const Image *d = IMG(n->p[0]), *s0 = IMG(n->p[1]);
        if ((uint64_t)d->width * d->height > (uint64_t)bw * bh) { bw = d->width; bh = d->height; }
        const Image *root = s0->parent ? s0->parent : s0;
        if (root->import_type == VX_MEMORY_TYPE_HOST) streamed = true;
    }
    if (!(g->optimizer_flags & kOptNoTma)) {
        vx_status err = VX_SUCCESS;
        if (half_batch_tma(g, nodes, st, err)) return err;
    }
    std::vector<uint32_t> cfg = tune_lookup("ScaleGaussianHalf_U8_U8_5x5", bw, bh, {32, 8, 1, 0});
    if (cfg[3] && !agocuda_ScaleGaussianHalf_tiles_shape(bw, bh, cfg[0], cfg[1])) cfg = {32, 8, 1, 0};
    const bool persistent = cfg[3] != 0;
    auto tiles_of = [&](const Image *d) {
        return persistent ? agocuda_ScaleGaussianHalf_tiles_shape(d->width, d->height, cfg[0], cfg[1])
                          : agocuda_ScaleGaussianHalf_tiles(d->width, d->height);
    };
    // launches over groups of images (tile numbering restarts in every group); images uploaded
    // from application buffers go in groups so the first ones compute while the rest arrive
    const size_t kGroupJobs = (streamed || !persistent) ? 2 * kGroupFrames : nodes.size();
    std::vector<agocuda_half_job> jobs;
    std::vector<uint32_t> group_tiles;
    uint32_t tiles = 0;
    for (size_t i = 0; i < nodes.size(); i++) {
        if (i % kGroupJobs == 0 && i) { group_tiles.push_back(tiles); tiles = 0; }
        const Image *d = IMG(nodes[i]->p[0]), *s = IMG(nodes[i]->p[1]);
        agocuda_half_job j{s->planes[0].dev, d->planes[0].dev, s->width, s->height, s->planes[0].dev_stride,
                           d->width, d->height, d->planes[0].dev_stride, tiles, 0};
        tiles += tiles_of(d);
        jobs.push_back(j);
    }
    group_tiles.push_back(tiles);
    agocuda_half_job *dev = (agocuda_half_job *)scratch(g, jobs.size() * sizeof(agocuda_half_job));
    if (!dev) return VX_ERROR_NO_MEMORY;
    if (cudaMemcpy(dev, jobs.data(), jobs.size() * sizeof(agocuda_half_job), cudaMemcpyHostToDevice) != cudaSuccess)
        return VX_FAILURE;
    std::vector<std::function<int(cudaStream_t)>> fns;
    uint32_t *queues = nullptr;
    if (persistent) {
        queues = (uint32_t *)scratch(g, 2 * sizeof(uint32_t) * group_tiles.size());
        if (!queues) return VX_ERROR_NO_MEMORY;
    }
    const uint32_t threads = cfg[0], rows = cfg[1], bps = cfg[2];
    for (size_t k0 = 0, gi = 0; k0 < jobs.size(); k0 += kGroupJobs, gi++) {
        const size_t k1 = std::min(jobs.size(), k0 + kGroupJobs);
        const agocuda_half_job *d0 = dev + k0;
        const uint32_t n = (uint32_t)(k1 - k0), t = group_tiles[gi];
        if (persistent) {
            uint32_t *queue = queues + 2 * gi;
            fns.push_back([=](cudaStream_t q) {
                return agocuda_fused_ScaleGaussianHalf_persistent(S(q), d0, n, t, queue, threads, rows, bps);
            });
        } else {
            fns.push_back([=](cudaStream_t q) { return agocuda_fused_ScaleGaussianHalf_batch(S(q), d0, n, t); });
        }
        st.parts.push_back(Part{fns.back(), std::vector<LNode *>(nodes.begin() + k0, nodes.begin() + k1)});
    }
    st.num_kernels = (int)fns.size();
    st.launch = [fns](cudaStream_t q) {
        for (auto &f : fns) { int rc = f(q); if (rc) return rc; }
        return 0;
    };
    return VX_SUCCESS;
}

// ------------------------------------------------------------------------------------
// plain (one launch per lowered node) steps
// ------------------------------------------------------------------------------------
static vx_status plain_step(Graph *g, LNode &ln, Step &st)
{
    auto &p = ln.p;
    st.name = lk_name(ln.k);
    st.nodes = {&ln};
    switch (ln.k) {
    case LK::GAUSSIAN_U8_U8_3x3: {
        uint8_t *d = dptr(p[0]); const uint8_t *s = dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        st.launch = [=](cudaStream_t q) { return agocuda_Gaussian_U8_U8_3x3(S(q), w, h, d, ds, s, ss); };
        return VX_SUCCESS;
    }
    case LK::SOBEL_S16S16_U8_3x3_GXY: case LK::SOBEL_S16_U8_3x3_GX: case LK::SOBEL_S16_U8_3x3_GY: {
        const bool gxy = ln.k == LK::SOBEL_S16S16_U8_3x3_GXY;
        Ref *src = gxy ? p[2] : p[1];
        uint32_t w = W(src), h = H(src);
        uint32_t tmp_stride = align_up(w * 2, 64);
        int16_t *gx, *gy; uint32_t gxs, gys;
        if (gxy) { gx = (int16_t *)dptr(p[0]); gxs = dstride(p[0]); gy = (int16_t *)dptr(p[1]); gys = dstride(p[1]); }
        else {
            int16_t *t = (int16_t *)scratch(g, (size_t)tmp_stride * h);
            if (!t) return VX_ERROR_NO_MEMORY;
            if (ln.k == LK::SOBEL_S16_U8_3x3_GX) { gx = (int16_t *)dptr(p[0]); gxs = dstride(p[0]); gy = t; gys = tmp_stride; }
            else { gy = (int16_t *)dptr(p[0]); gys = dstride(p[0]); gx = t; gxs = tmp_stride; }
        }
        const uint8_t *s = dptr(src); uint32_t ss = dstride(src);
        st.launch = [=](cudaStream_t q) { return agocuda_Sobel_S16S16_U8_3x3_GXY(S(q), w, h, gx, gxs, gy, gys, s, ss); };
        return VX_SUCCESS;
    }
    case LK::SOBEL_MAGNITUDE_S16_U8_3x3: {
        int16_t *d = (int16_t *)dptr(p[0]); const uint8_t *s = dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        st.launch = [=](cudaStream_t q) { return agocuda_SobelMagnitude_S16_U8_3x3(S(q), w, h, d, ds, s, ss); };
        return VX_SUCCESS;
    }
    case LK::MAGNITUDE_S16_S16S16: {
        int16_t *d = (int16_t *)dptr(p[0]); const int16_t *a = (const int16_t *)dptr(p[1]), *b = (const int16_t *)dptr(p[2]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), as_ = dstride(p[1]), bs = dstride(p[2]);
        st.launch = [=](cudaStream_t q) { return agocuda_Magnitude_S16_S16S16(S(q), w, h, d, ds, a, as_, b, bs); };
        return VX_SUCCESS;
    }
    case LK::COLOR_DEPTH_U8_S16_SAT: {
        uint8_t *d = dptr(p[0]); const int16_t *s = (const int16_t *)dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        int32_t shift = sc_i32(p[2]);
        st.launch = [=](cudaStream_t q) { return agocuda_ColorDepth_U8_S16_Sat(S(q), w, h, d, ds, s, ss, shift); };
        return VX_SUCCESS;
    }
    case LK::THRESHOLD_U8_U8_BINARY: {
        uint8_t *d = dptr(p[0]); const uint8_t *s = dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        int32_t thr = static_cast<Threshold *>(p[2])->value.U8;   // threshold_value.U1 (ago_kernel_api.cpp:3442)
        st.launch = [=](cudaStream_t q) { return agocuda_Threshold_U8_U8_Binary(S(q), w, h, d, ds, s, ss, thr); };
        return VX_SUCCESS;
    }
    case LK::COLOR_DEPTH_U8_S16_WRAP: {
        uint8_t *d = dptr(p[0]); const int16_t *s = (const int16_t *)dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        int32_t shift = sc_i32(p[2]);
        st.launch = [=](cudaStream_t q) { return agocuda_ColorDepth_U8_S16_Wrap(S(q), w, h, d, ds, s, ss, shift); };
        return VX_SUCCESS;
    }
    case LK::COLOR_DEPTH_S16_U8: {
        int16_t *d = (int16_t *)dptr(p[0]); const uint8_t *s = dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        int32_t shift = sc_i32(p[2]);
        st.launch = [=](cudaStream_t q) { return agocuda_ColorDepth_S16_U8(S(q), w, h, d, ds, s, ss, shift); };
        return VX_SUCCESS;
    }
    case LK::CHANNEL_EXTRACT_U8_U16_POS0: case LK::CHANNEL_EXTRACT_U8_U16_POS1: case LK::CHANNEL_EXTRACT_U8_U24_POS0:
    case LK::CHANNEL_EXTRACT_U8_U24_POS1: case LK::CHANNEL_EXTRACT_U8_U24_POS2: case LK::CHANNEL_EXTRACT_U8_U32_POS0:
    case LK::CHANNEL_EXTRACT_U8_U32_POS1: case LK::CHANNEL_EXTRACT_U8_U32_POS2: case LK::CHANNEL_EXTRACT_U8_U32_POS3: {
        using Fn = int (*)(void *, uint32_t, uint32_t, uint8_t *, uint32_t, const uint8_t *, uint32_t);
        static const Fn fns[] = {agocuda_ChannelExtract_U8_U16_Pos0, agocuda_ChannelExtract_U8_U16_Pos1,
                                 agocuda_ChannelExtract_U8_U24_Pos0, agocuda_ChannelExtract_U8_U24_Pos1,
                                 agocuda_ChannelExtract_U8_U24_Pos2, agocuda_ChannelExtract_U8_U32_Pos0,
                                 agocuda_ChannelExtract_U8_U32_Pos1, agocuda_ChannelExtract_U8_U32_Pos2,
                                 agocuda_ChannelExtract_U8_U32_Pos3};
        const Fn fn = fns[(int)ln.k - (int)LK::CHANNEL_EXTRACT_U8_U16_POS0];
        uint8_t *d = dptr(p[0]); const uint8_t *s = dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        st.launch = [=](cudaStream_t q) { return fn(S(q), w, h, d, ds, s, ss); };
        return VX_SUCCESS;
    }
    case LK::CHANNEL_COMBINE_U16_U8U8: {
        uint8_t *d = dptr(p[0]); const uint8_t *a = dptr(p[1]), *b = dptr(p[2]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), as_ = dstride(p[1]), bs = dstride(p[2]);
        st.launch = [=](cudaStream_t q) { return agocuda_ChannelCombine_U16_U8U8(S(q), w, h, d, ds, a, as_, b, bs); };
        return VX_SUCCESS;
    }
    case LK::CHANNEL_COMBINE_U24_U8U8U8_RGB: case LK::CHANNEL_COMBINE_U32_U8U8U8_UYVY: case LK::CHANNEL_COMBINE_U32_U8U8U8_YUYV: {
        using Fn = int (*)(void *, uint32_t, uint32_t, uint8_t *, uint32_t, const uint8_t *, uint32_t, const uint8_t *,
                           uint32_t, const uint8_t *, uint32_t);
        const Fn fn = ln.k == LK::CHANNEL_COMBINE_U24_U8U8U8_RGB ? agocuda_ChannelCombine_U24_U8U8U8_RGB
                    : ln.k == LK::CHANNEL_COMBINE_U32_U8U8U8_UYVY ? agocuda_ChannelCombine_U32_U8U8U8_UYVY
                                                                  : agocuda_ChannelCombine_U32_U8U8U8_YUYV;
        uint8_t *d = dptr(p[0]); const uint8_t *a = dptr(p[1]), *b = dptr(p[2]), *c = dptr(p[3]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), as_ = dstride(p[1]), bs = dstride(p[2]), cs = dstride(p[3]);
        st.launch = [=](cudaStream_t q) { return fn(S(q), w, h, d, ds, a, as_, b, bs, c, cs); };
        return VX_SUCCESS;
    }
    case LK::CHANNEL_COMBINE_U32_U8U8U8U8_RGBX: {
        uint8_t *d = dptr(p[0]); const uint8_t *a = dptr(p[1]), *b = dptr(p[2]), *c = dptr(p[3]), *e = dptr(p[4]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), as_ = dstride(p[1]), bs = dstride(p[2]), cs = dstride(p[3]),
                 es = dstride(p[4]);
        st.launch = [=](cudaStream_t q) {
            return agocuda_ChannelCombine_U32_U8U8U8U8_RGBX(S(q), w, h, d, ds, a, as_, b, bs, c, cs, e, es);
        };
        return VX_SUCCESS;
    }
    case LK::HISTOGRAM_DATA_U8: {
        Distribution *dist = static_cast<Distribution *>(p[0]);
        if (!dist->dev && cudaMalloc((void **)&dist->dev, dist->bins * sizeof(uint32_t)) != cudaSuccess) return VX_ERROR_NO_MEMORY;
        uint32_t *hist = dist->dev;
        const uint8_t *s = dptr(p[1]);
        const uint32_t w = W(p[1]), h = H(p[1]), ss = dstride(p[1]), bins = (uint32_t)dist->bins, range = dist->range;
        const int32_t off = dist->offset;
        st.launch = [=](cudaStream_t q) { return agocuda_Histogram_DATA_U8(S(q), hist, w, h, s, ss, bins, off, range); };
        return VX_SUCCESS;
    }
    case LK::INTEGRAL_IMAGE_U32_U8: {
        uint32_t *d = (uint32_t *)dptr(p[0]); const uint8_t *s = dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        const size_t sb = agocuda_IntegralImage_scratch_size(w, h);
        void *scr = scratch(g, sb);
        if (!scr) return VX_ERROR_NO_MEMORY;
        st.num_kernels = 3;
        st.launch = [=](cudaStream_t q) { return agocuda_IntegralImage_U32_U8(S(q), w, h, d, ds, s, ss, scr, sb); };
        return VX_SUCCESS;
    }
    case LK::CONVOLVE_U8_U8: case LK::CONVOLVE_S16_U8: {
        // coefficients and shift by value: a change re-plans (the convolution's version is
        // part of the graph's parameter hash)
        const Convolution *cv = static_cast<Convolution *>(p[2]);
        const uint32_t cols = (uint32_t)cv->columns, rows = (uint32_t)cv->rows;
        std::vector<int16_t> k = cv->coeffs;
        int32_t shift = 0;
        while (shift < 31 && (1u << shift) < cv->scale) shift++;
        uint8_t *d = dptr(p[0]); const uint8_t *s = dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        // AGO rows are 16-byte aligned: SIMD body [0, W - W % 16), scalar tail after it
        const int32_t sb = 0, se = (int32_t)(w - (w & 15));
        if (ln.k == LK::CONVOLVE_U8_U8)
            st.launch = [=](cudaStream_t q) { return agocuda_Convolve_U8_U8(S(q), w, h, d, ds, s, ss, k.data(), cols, rows, shift, sb, se); };
        else
            st.launch = [=](cudaStream_t q) {
                return agocuda_Convolve_S16_U8(S(q), w, h, (int16_t *)d, ds, s, ss, k.data(), cols, rows, shift, sb, se);
            };
        return VX_SUCCESS;
    }
    case LK::LUT_U8_U8: case LK::LUT_S16_S16: {
        // the table's current contents go to device memory with the plan; a changed table
        // changes the graph's parameter hash and re-plans
        const Lut *l = static_cast<Lut *>(p[2]);
        void *tab = scratch(g, l->data.size());
        if (!tab || cudaMemcpy(tab, l->data.data(), l->data.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            return VX_ERROR_NO_MEMORY;
        uint8_t *d = dptr(p[0]); const uint8_t *s = dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        if (ln.k == LK::LUT_U8_U8) {
            const uint8_t *t = (const uint8_t *)tab;
            st.launch = [=](cudaStream_t q) { return agocuda_Lut_U8_U8(S(q), w, h, d, ds, s, ss, t); };
        } else {
            const int16_t *t = (const int16_t *)tab;
            const uint32_t cnt = (uint32_t)l->count, off = l->offset;
            st.launch = [=](cudaStream_t q) {
                return agocuda_Lut_S16_S16(S(q), w, h, (int16_t *)d, ds, (const int16_t *)s, ss, t, cnt, off);
            };
        }
        return VX_SUCCESS;
    }
    case LK::THRESHOLD_U8_U8_RANGE: {
        uint8_t *d = dptr(p[0]); const uint8_t *s = dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        Threshold *t = static_cast<Threshold *>(p[2]);
        int32_t lo = t->lower.U8, hi = t->upper.U8;   // threshold_lower/upper.U1 as vx_uint8 (ago_kernel_api.cpp:3511)
        st.launch = [=](cudaStream_t q) { return agocuda_Threshold_U8_U8_Range(S(q), w, h, d, ds, s, ss, lo, hi); };
        return VX_SUCCESS;
    }
    case LK::BOX_U8_U8_3x3: case LK::DILATE_U8_U8_3x3: case LK::ERODE_U8_U8_3x3: case LK::MEDIAN_U8_U8_3x3:
    case LK::NOT_U8_U8: {
        using Fn = int (*)(void *, uint32_t, uint32_t, uint8_t *, uint32_t, const uint8_t *, uint32_t);
        const Fn fn = ln.k == LK::BOX_U8_U8_3x3 ? agocuda_Box_U8_U8_3x3 : ln.k == LK::DILATE_U8_U8_3x3 ? agocuda_Dilate_U8_U8_3x3
                    : ln.k == LK::ERODE_U8_U8_3x3 ? agocuda_Erode_U8_U8_3x3 : ln.k == LK::MEDIAN_U8_U8_3x3 ? agocuda_Median_U8_U8_3x3
                    : agocuda_Not_U8_U8;
        uint8_t *d = dptr(p[0]); const uint8_t *s = dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        st.launch = [=](cudaStream_t q) { return fn(S(q), w, h, d, ds, s, ss); };
        return VX_SUCCESS;
    }
#define EW(KIND, FN, TO, TA, TB)                                                                     \
    case LK::KIND: {                                                                                \
        TO *d = (TO *)dptr(p[0]); const TA *a = (const TA *)dptr(p[1]); const TB *b = (const TB *)dptr(p[2]); \
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), as_ = dstride(p[1]), bs = dstride(p[2]);   \
        st.launch = [=](cudaStream_t q) { return FN(S(q), w, h, d, ds, a, as_, b, bs); };            \
        return VX_SUCCESS;                                                                          \
    }
    EW(ABS_DIFF_U8_U8U8, agocuda_AbsDiff_U8_U8U8, uint8_t, uint8_t, uint8_t)
    EW(ABS_DIFF_S16_S16S16_SAT, agocuda_AbsDiff_S16_S16S16_Sat, int16_t, int16_t, int16_t)
    EW(ADD_U8_U8U8_WRAP, agocuda_Add_U8_U8U8_Wrap, uint8_t, uint8_t, uint8_t)
    EW(ADD_U8_U8U8_SAT, agocuda_Add_U8_U8U8_Sat, uint8_t, uint8_t, uint8_t)
    EW(ADD_S16_U8U8, agocuda_Add_S16_U8U8, int16_t, uint8_t, uint8_t)
    EW(ADD_S16_S16U8_WRAP, agocuda_Add_S16_S16U8_Wrap, int16_t, int16_t, uint8_t)
    EW(ADD_S16_S16U8_SAT, agocuda_Add_S16_S16U8_Sat, int16_t, int16_t, uint8_t)
    EW(ADD_S16_S16S16_WRAP, agocuda_Add_S16_S16S16_Wrap, int16_t, int16_t, int16_t)
    EW(ADD_S16_S16S16_SAT, agocuda_Add_S16_S16S16_Sat, int16_t, int16_t, int16_t)
    EW(SUB_U8_U8U8_WRAP, agocuda_Sub_U8_U8U8_Wrap, uint8_t, uint8_t, uint8_t)
    EW(SUB_U8_U8U8_SAT, agocuda_Sub_U8_U8U8_Sat, uint8_t, uint8_t, uint8_t)
    EW(SUB_S16_U8U8, agocuda_Sub_S16_U8U8, int16_t, uint8_t, uint8_t)
    EW(SUB_S16_S16U8_WRAP, agocuda_Sub_S16_S16U8_Wrap, int16_t, int16_t, uint8_t)
    EW(SUB_S16_S16U8_SAT, agocuda_Sub_S16_S16U8_Sat, int16_t, int16_t, uint8_t)
    EW(SUB_S16_U8S16_WRAP, agocuda_Sub_S16_U8S16_Wrap, int16_t, uint8_t, int16_t)
    EW(SUB_S16_U8S16_SAT, agocuda_Sub_S16_U8S16_Sat, int16_t, uint8_t, int16_t)
    EW(SUB_S16_S16S16_WRAP, agocuda_Sub_S16_S16S16_Wrap, int16_t, int16_t, int16_t)
    EW(SUB_S16_S16S16_SAT, agocuda_Sub_S16_S16S16_Sat, int16_t, int16_t, int16_t)
    EW(AND_U8_U8U8, agocuda_And_U8_U8U8, uint8_t, uint8_t, uint8_t)
    EW(OR_U8_U8U8, agocuda_Or_U8_U8U8, uint8_t, uint8_t, uint8_t)
    EW(XOR_U8_U8U8, agocuda_Xor_U8_U8U8, uint8_t, uint8_t, uint8_t)
#undef EW
    case LK::CANNY_SOBEL_U16_U8_3x3_L1NORM: {
        uint16_t *d = (uint16_t *)dptr(p[0]); const uint8_t *s = dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        st.launch = [=](cudaStream_t q) { return agocuda_CannySobel_U16_U8_3x3_L1NORM(S(q), w, h, d, ds, s, ss); };
        return VX_SUCCESS;
    }
#define CANNY_SOBEL(K, FN)                                                                                      \
    case LK::K: {                                                                                               \
        uint16_t *d = (uint16_t *)dptr(p[0]); const uint8_t *s = dptr(p[1]);                                   \
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);                             \
        st.launch = [=](cudaStream_t q) { return FN(S(q), w, h, d, ds, s, ss); };                              \
        return VX_SUCCESS;                                                                                      \
    }
    CANNY_SOBEL(CANNY_SOBEL_U16_U8_3x3_L2NORM, agocuda_CannySobel_U16_U8_3x3_L2NORM)
    CANNY_SOBEL(CANNY_SOBEL_U16_U8_5x5_L1NORM, agocuda_CannySobel_U16_U8_5x5_L1NORM)
    CANNY_SOBEL(CANNY_SOBEL_U16_U8_5x5_L2NORM, agocuda_CannySobel_U16_U8_5x5_L2NORM)
    CANNY_SOBEL(CANNY_SOBEL_U16_U8_7x7_L1NORM, agocuda_CannySobel_U16_U8_7x7_L1NORM)
    CANNY_SOBEL(CANNY_SOBEL_U16_U8_7x7_L2NORM, agocuda_CannySobel_U16_U8_7x7_L2NORM)
#undef CANNY_SOBEL
    case LK::CANNY_SUPP_THRESHOLD_U8XY_U16_3x3: case LK::CANNY_SUPP_THRESHOLD_U8XY_U16_7x7: {
        uint8_t *d = dptr(p[0]); Array *stk = static_cast<Array *>(p[1]); const uint16_t *s = (const uint16_t *)dptr(p[2]);
        Threshold *t = static_cast<Threshold *>(p[3]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[2]);
        // threshold_lower/upper .U1 passed as vx_uint16 (ago_kernel_api.cpp:17967); the 7x7
        // variant divides both by 4 first (ago_kernel_api.cpp:18035)
        const int32_t q4 = ln.k == LK::CANNY_SUPP_THRESHOLD_U8XY_U16_7x7 ? 4 : 1;
        uint16_t lo = (uint16_t)((int32_t)t->lower.U32 / q4), hi = (uint16_t)((int32_t)t->upper.U32 / q4);
        uint32_t *stack = (uint32_t *)stk->dev, *cnt = stk->dev_count; uint32_t cap = (uint32_t)stk->capacity;
        st.launch = [=](cudaStream_t q) {
            return agocuda_CannySuppThreshold_U8XY_U16_3x3(S(q), w, h, d, ds, s, ss, stack, cnt, cap, lo, hi);
        };
        return VX_SUCCESS;
    }
    case LK::CANNY_EDGE_TRACE_U8_U8XY: {
        uint8_t *d = dptr(p[0]); Array *stk = static_cast<Array *>(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]);
        size_t sb = agocuda_CannyEdgeTrace_scratch_size(w, h);
        void *scr = scratch(g, sb);
        if (!scr) return VX_ERROR_NO_MEMORY;
        const uint32_t *stack = (const uint32_t *)stk->dev, *cnt = stk->dev_count; uint32_t cap = (uint32_t)stk->capacity;
        uint32_t *status = g->status_dev;
        st.num_kernels = 4;
        st.launch = [=](cudaStream_t q) {
            return agocuda_CannyEdgeTrace_U8_U8XY(S(q), w, h, d, ds, stack, cnt, cap, scr, sb, status);
        };
        return VX_SUCCESS;
    }
    case LK::HARRIS_SOBEL_HG3_U8_3x3: {
        float *d = (float *)dptr(p[0]); const uint8_t *s = dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        st.launch = [=](cudaStream_t q) { return agocuda_HarrisSobel_HG3_U8_3x3(S(q), w, h, d, ds, s, ss); };
        return VX_SUCCESS;
    }
    case LK::HARRIS_SCORE_HVC_HG3_3x3: {
        float *d = (float *)dptr(p[0]); const float *s = (const float *)dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        float k = sc_f32(p[2]), tc = sc_f32(p[3]);
        float norm = harris_norm(sc_i32(p[4]));
        st.launch = [=](cudaStream_t q) { return agocuda_HarrisScore_HVC_HG3_3x3(S(q), w, h, d, ds, s, ss, k, tc, norm); };
        return VX_SUCCESS;
    }
    case LK::HARRIS_SOBEL_HG3_U8_5x5: case LK::HARRIS_SOBEL_HG3_U8_7x7: {
        float *d = (float *)dptr(p[0]); const uint8_t *s = dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        const uint32_t gs = ln.k == LK::HARRIS_SOBEL_HG3_U8_5x5 ? 5 : 7;
        st.launch = [=](cudaStream_t q) { return agocuda_HarrisSobel_HG3_U8_NxN(S(q), w, h, d, ds, s, ss, gs); };
        return VX_SUCCESS;
    }
    case LK::HARRIS_SCORE_HVC_HG3_5x5: case LK::HARRIS_SCORE_HVC_HG3_7x7: {
        float *d = (float *)dptr(p[0]); const float *s = (const float *)dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        float k = sc_f32(p[2]), tc = sc_f32(p[3]);
        const uint32_t bs = ln.k == LK::HARRIS_SCORE_HVC_HG3_5x5 ? 5 : 7;
        float norm = harris_norm(sc_i32(p[4]), (int32_t)bs);
        st.launch = [=](cudaStream_t q) { return agocuda_HarrisScore_HVC_HG3_NxN(S(q), w, h, d, ds, s, ss, k, tc, norm, bs); };
        return VX_SUCCESS;
    }
    case LK::NON_MAX_SUPP_XY_ANY_3x3: {
        Array *lst = static_cast<Array *>(p[0]); const float *s = (const float *)dptr(p[1]);
        uint32_t w = W(p[1]), h = H(p[1]), ss = dstride(p[1]);
        uint64_t *l = (uint64_t *)lst->dev; uint32_t *cnt = lst->dev_count; uint32_t cap = (uint32_t)lst->capacity;
        st.launch = [=](cudaStream_t q) { return agocuda_NonMaxSupp_XY_ANY_3x3(S(q), w, h, s, ss, l, cnt, cap); };
        return VX_SUCCESS;
    }
    case LK::HARRIS_MERGE_SORT_AND_PICK_XY_XYS: {
        Array *corners = static_cast<Array *>(p[0]);
        Scalar *num = p[1] ? static_cast<Scalar *>(p[1]) : nullptr;
        Array *lst = static_cast<Array *>(p[2]);
        float mind = sc_f32(p[3]);
        uint32_t w = static_cast<Scalar *>(p[4])->v.u32, h = static_cast<Scalar *>(p[5])->v.u32;
        if (num && scalar_alloc_device(num)) return VX_ERROR_NO_MEMORY;
        const uint64_t *l = (const uint64_t *)lst->dev; const uint32_t *lc = lst->dev_count; uint32_t lcap = (uint32_t)lst->capacity;
        void *out = corners->dev; uint32_t ocap = (uint32_t)corners->capacity; uint32_t *oc = corners->dev_count;
        uint32_t *nc = num ? num->dev : nullptr;
        uint32_t *status = g->status_dev;
        const size_t sb = agocuda_HarrisMergeSortAndPick_scratch_size(w, h, lcap, mind);
        void *scr = scratch(g, sb);
        if (!scr) return VX_ERROR_NO_MEMORY;
        st.num_kernels = 2;
        st.launch = [=](cudaStream_t q) {
            return agocuda_HarrisMergeSortAndPick_XY_XYS(S(q), w, h, l, lc, lcap, mind, out, ocap, oc, nc, scr, sb, status);
        };
        return VX_SUCCESS;
    }
    case LK::USER_KERNEL: {
        // the node's kernel_f on the host, between the device steps (launches are not captured)
        Node *n = ln.origin;
        g->host_steps = true;
        st.num_kernels = 0;
        st.name = "user:" + n->ukernel->kname;
        st.launch = [g, n](cudaStream_t q) { return run_user_node(g, n, q); };
        return VX_SUCCESS;
    }
    case LK::FAST_CORNERS_XY_U8_SUPRESSION: case LK::FAST_CORNERS_XY_U8_NOSUPRESSION: {
        Array *corners = static_cast<Array *>(p[0]);
        Scalar *num = p[1] ? static_cast<Scalar *>(p[1]) : nullptr;
        if (num && scalar_alloc_device(num)) return VX_ERROR_NO_MEMORY;
        const uint8_t *s = dptr(p[2]);
        uint32_t w = W(p[2]), h = H(p[2]), ss = dstride(p[2]);
        const float thr = sc_f32(p[3]);
        const int32_t sup = ln.k == LK::FAST_CORNERS_XY_U8_SUPRESSION;
        void *out = corners->dev; uint32_t ocap = (uint32_t)corners->capacity; uint32_t *oc = corners->dev_count;
        uint32_t *nc = num ? num->dev : nullptr;
        const size_t sb = agocuda_FastCorners_scratch_size(w, h);
        void *scr = scratch(g, sb);
        if (!scr) return VX_ERROR_NO_MEMORY;
        st.num_kernels = 4;
        st.launch = [=](cudaStream_t q) {
            return agocuda_FastCorners_XY_U8(S(q), w, h, s, ss, thr, sup, out, ocap, oc, nc, scr, sb);
        };
        return VX_SUCCESS;
    }
    case LK::COLOR_CONVERT_NV12_RGB: {
        uint8_t *y = dptr(p[0]), *uv = dptr(p[1]); const uint8_t *s = dptr(p[2]);
        uint32_t w = W(p[2]), h = H(p[2]), ys = dstride(p[0]), uvs = dstride(p[1]), ss = dstride(p[2]);
        st.launch = [=](cudaStream_t q) { return agocuda_ColorConvert_NV12_RGB(S(q), w, h, y, ys, uv, uvs, s, ss); };
        return VX_SUCCESS;
    }
    case LK::COLOR_CONVERT_IYUV_RGB: {
        uint8_t *y = dptr(p[0]), *u = dptr(p[1]), *v = dptr(p[2]); const uint8_t *s = dptr(p[3]);
        uint32_t w = W(p[3]), h = H(p[3]), ys = dstride(p[0]), us = dstride(p[1]), vs = dstride(p[2]), ss = dstride(p[3]);
        st.launch = [=](cudaStream_t q) { return agocuda_ColorConvert_IYUV_RGB(S(q), w, h, y, ys, u, us, v, vs, s, ss); };
        return VX_SUCCESS;
    }
    case LK::SCALE_IMAGE_U8_U8_NEAREST: case LK::SCALE_IMAGE_U8_U8_BILINEAR: case LK::SCALE_IMAGE_U8_U8_AREA: {
        uint8_t *d = dptr(p[0]); const uint8_t *s = dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), sw = W(p[1]), sh = H(p[1]), ss = dstride(p[1]);
        if (ln.k == LK::SCALE_IMAGE_U8_U8_AREA && !((sw == 2 * w && sh == 2 * h) || (sw == w && sh == h))) {
            log_error(g, VX_ERROR_NOT_SUPPORTED, "ERROR: area scaling %ux%u -> %ux%u: only the 1x and 2x ratios are implemented\n", sw, sh, w, h);
            return VX_ERROR_NOT_SUPPORTED;
        }
        const LK k = ln.k;
        st.launch = [=](cudaStream_t q) {
            if (k == LK::SCALE_IMAGE_U8_U8_NEAREST) return agocuda_ScaleImage_U8_U8_Nearest(S(q), w, h, d, ds, sw, sh, s, ss);
            if (k == LK::SCALE_IMAGE_U8_U8_BILINEAR) return agocuda_ScaleImage_U8_U8_Bilinear(S(q), w, h, d, ds, sw, sh, s, ss);
            return agocuda_ScaleImage_U8_U8_Area(S(q), w, h, d, ds, sw, sh, s, ss);
        };
        return VX_SUCCESS;
    }
    case LK::WARP_AFFINE_U8_U8_NEAREST_CONSTANT: case LK::WARP_AFFINE_U8_U8_BILINEAR_CONSTANT: {
        uint8_t *d = dptr(p[0]); const uint8_t *s = dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), sw = W(p[1]), sh = H(p[1]), ss = dstride(p[1]);
        Matrix *m = static_cast<Matrix *>(p[2]);
        std::array<float, 6> mat;
        memcpy(mat.data(), m->data.data(), sizeof(float) * 6);
        const uint8_t border = static_cast<Scalar *>(p[3])->v.u8;
        const vx_rectangle_t vr = IMG(p[1])->valid;   // the nearest kernel masks by the source valid rect
        const bool nn = ln.k == LK::WARP_AFFINE_U8_U8_NEAREST_CONSTANT;
        st.launch = [=](cudaStream_t q) {
            const uint32_t rect[4] = {vr.start_x, vr.start_y, vr.end_x, vr.end_y};
            return nn ? agocuda_WarpAffine_U8_U8_Nearest_Constant(S(q), w, h, d, ds, sw, sh, s, ss, mat.data(), border, rect)
                      : agocuda_WarpAffine_U8_U8_Bilinear_Constant(S(q), w, h, d, ds, sw, sh, s, ss, mat.data(), border);
        };
        return VX_SUCCESS;
    }
    case LK::CHANNEL_COPY_U8_U8: {
        uint8_t *d = dptr(p[0]); const uint8_t *s = dptr(p[1]);
        uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), ss = dstride(p[1]);
        st.num_kernels = 0;   // a copy-engine transfer, not a kernel
        st.launch = [=](cudaStream_t q) {
            return cudaMemcpy2DAsync(d, ds, s, ss, w, h, cudaMemcpyDeviceToDevice, q) == cudaSuccess ? 0 : -1;
        };
        return VX_SUCCESS;
    }
    case LK::WARP_PERSPECTIVE_U8_U8_NEAREST_CONSTANT: case LK::WARP_PERSPECTIVE_U8_U8_BILINEAR_CONSTANT:
    case LK::WARP_PERSPECTIVE_U8_U8_NEAREST: case LK::WARP_PERSPECTIVE_U8_U8_BILINEAR: {
        uint8_t *d = dptr(p[0]); const uint8_t *s = dptr(p[1]);
        const uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), sw = W(p[1]), sh = H(p[1]), ss = dstride(p[1]);
        std::array<float, 9> mat;
        memcpy(mat.data(), static_cast<Matrix *>(p[2])->data.data(), sizeof(float) * 9);
        // the undefined-border kernels are the constant ones with border 0 (geometric.cpp:1372, :1560)
        const bool cst = ln.k == LK::WARP_PERSPECTIVE_U8_U8_NEAREST_CONSTANT || ln.k == LK::WARP_PERSPECTIVE_U8_U8_BILINEAR_CONSTANT;
        const uint8_t border = cst ? static_cast<Scalar *>(p[3])->v.u8 : 0;
        const bool bl = ln.k == LK::WARP_PERSPECTIVE_U8_U8_BILINEAR_CONSTANT || ln.k == LK::WARP_PERSPECTIVE_U8_U8_BILINEAR;
        st.launch = [=](cudaStream_t q) {
            return bl ? agocuda_WarpPerspective_U8_U8_Bilinear_Constant(S(q), w, h, d, ds, sw, sh, s, ss, mat.data(), border)
                      : agocuda_WarpPerspective_U8_U8_Nearest_Constant(S(q), w, h, d, ds, sw, sh, s, ss, mat.data(), border);
        };
        return VX_SUCCESS;
    }
    case LK::REMAP_U8_U8_NEAREST_CONSTANT: case LK::REMAP_U8_U8_BILINEAR_CONSTANT:
    case LK::REMAP_U8_U8_NEAREST: case LK::REMAP_U8_U8_BILINEAR: {
        uint8_t *d = dptr(p[0]); const uint8_t *s = dptr(p[1]);
        const uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), sw = W(p[1]), sh = H(p[1]), ss = dstride(p[1]);
        const Remap *r = static_cast<Remap *>(p[2]);
        const std::vector<uint32_t> fixed = remap_fixed_table(r);
        void *map = scratch(g, fixed.size() * sizeof(uint32_t));
        if (!map) return VX_ERROR_NO_MEMORY;
        if (cudaMemcpy(map, fixed.data(), fixed.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess)
            return VX_FAILURE;
        const uint32_t ms = r->dst_width * 4;
        const LK k = ln.k;
        const uint8_t border = (k == LK::REMAP_U8_U8_NEAREST_CONSTANT || k == LK::REMAP_U8_U8_BILINEAR_CONSTANT)
                                   ? static_cast<Scalar *>(p[3])->v.u8 : 0;
        const uint32_t *m = (const uint32_t *)map;
        st.launch = [=](cudaStream_t q) {
            switch (k) {
            case LK::REMAP_U8_U8_NEAREST: return agocuda_Remap_U8_U8_Nearest(S(q), w, h, d, ds, sw, sh, s, ss, m, ms);
            case LK::REMAP_U8_U8_BILINEAR: return agocuda_Remap_U8_U8_Bilinear(S(q), w, h, d, ds, sw, sh, s, ss, m, ms);
            case LK::REMAP_U8_U8_NEAREST_CONSTANT:
                return agocuda_Remap_U8_U8_Nearest_Constant(S(q), w, h, d, ds, sw, sh, s, ss, m, ms, border);
            default: return agocuda_Remap_U8_U8_Bilinear_Constant(S(q), w, h, d, ds, sw, sh, s, ss, m, ms, border);
            }
        };
        return VX_SUCCESS;
    }
    case LK::SCALE_GAUSSIAN_HALF_U8_U8_5x5: {                    // ago_kernel_api.cpp:15420
        uint8_t *d = dptr(p[0]); const uint8_t *s = dptr(p[1]);
        const uint32_t w = W(p[0]), h = H(p[0]), ds = dstride(p[0]), sw = W(p[1]), sh = H(p[1]), ss = dstride(p[1]);
        st.launch = [=](cudaStream_t q) { return agocuda_ScaleGaussianHalf_U8_U8_5x5(S(q), w, h, d, ds, sw, sh, s, ss); };
        return VX_SUCCESS;
    }
    case LK::OPTICAL_FLOW_PYR_LK_XY_XY:                           // ago_kernel_api.cpp:20587
        return lk_batch_step(g, {&ln}, st);
    default:
        log_error(g, VX_ERROR_NOT_IMPLEMENTED, "ERROR: kernel %s has no device implementation yet\n", lk_name(ln.k));
        return VX_ERROR_NOT_IMPLEMENTED;
    }
}

// ------------------------------------------------------------------------------------
// fused chains
// ------------------------------------------------------------------------------------
struct Chain {
    std::string kind;                 // pattern name
    std::vector<LNode *> nodes;
    std::vector<int64_t> key;         // by-value parameters: chains with equal keys batch
    Ref *src = nullptr, *dst = nullptr;
    std::vector<Ref *> elide;         // intermediates the fused kernel keeps on chip
    agocuda_pixel_program prog{};     // fused_PixelChain: the ops
    std::vector<Ref *> sides;         // fused_PixelChain: second operands of binary ops
};

// U8 -> U8 kernels the fused pixel-chain kernel runs (0: not one of them)
static int px_code(LK k)
{
    switch (k) {
    case LK::NOT_U8_U8: return AGOCUDA_PX_NOT;
    case LK::AND_U8_U8U8: return AGOCUDA_PX_AND;
    case LK::OR_U8_U8U8: return AGOCUDA_PX_OR;
    case LK::XOR_U8_U8U8: return AGOCUDA_PX_XOR;
    case LK::ABS_DIFF_U8_U8U8: return AGOCUDA_PX_ABSDIFF;
    case LK::ADD_U8_U8U8_WRAP: return AGOCUDA_PX_ADD_WRAP;
    case LK::ADD_U8_U8U8_SAT: return AGOCUDA_PX_ADD_SAT;
    case LK::SUB_U8_U8U8_WRAP: return AGOCUDA_PX_SUB_WRAP;
    case LK::SUB_U8_U8U8_SAT: return AGOCUDA_PX_SUB_SAT;
    case LK::THRESHOLD_U8_U8_BINARY: return AGOCUDA_PX_THRESHOLD_BINARY;
    case LK::THRESHOLD_U8_U8_RANGE: return AGOCUDA_PX_THRESHOLD_RANGE;
    case LK::BOX_U8_U8_3x3: return AGOCUDA_PX_BOX3x3;
    case LK::MEDIAN_U8_U8_3x3: return AGOCUDA_PX_MEDIAN3x3;
    case LK::DILATE_U8_U8_3x3: return AGOCUDA_PX_DILATE3x3;
    case LK::ERODE_U8_U8_3x3: return AGOCUDA_PX_ERODE3x3;
    case LK::GAUSSIAN_U8_U8_3x3: return AGOCUDA_PX_GAUSSIAN3x3;
    default: return 0;
    }
}
static bool px_binary(int code) { return code >= AGOCUDA_PX_AND && code <= AGOCUDA_PX_SUB_SAT; }
static bool px_stencil(int code) { return code >= AGOCUDA_PX_BOX3x3; }

static int writer_level(Graph *g, Ref *d)
{
    int lv = -1;
    for (const LNode &ln : g->lnodes) {
        if (ln.removed) continue;
        for (size_t i = 0; i < ln.p.size(); i++)
            if (lnode_is_output(ln, i) && ln.p[i] == d) lv = std::max(lv, ln.level);
    }
    return lv;
}

// A maximal run of U8 pixel kernels linked by private virtual images (two or more nodes).
// The second operands of binary kernels become side inputs; each must be ready before the
// chain's first node runs (written at a lower level, or a graph input).
static bool match_pixel_chain(Graph *g, LNode &a, const std::set<LNode *> &taken, Chain &c)
{
    const int code0 = px_code(a.k);
    if (!code0) return false;
    agocuda_pixel_program P{};
    std::vector<Ref *> sides, elide;
    std::vector<LNode *> nodes;
    int stencils = 0;
    auto add_op = [&](const LNode &n, int code, Ref *other, int first) -> bool {
        if (P.numOps >= AGOCUDA_PX_MAX_OPS) return false;
        if (px_stencil(code) && stencils >= AGOCUDA_PX_MAX_STENCILS) return false;
        agocuda_pixel_op op{code, -1, first, 0, 0};
        if (px_binary(code)) {
            if (!other || other->type != VX_TYPE_IMAGE || IMG(other)->format != VX_DF_IMAGE_U8) return false;
            if (writer_level(g, other) >= a.level) return false;
            size_t k = std::find(sides.begin(), sides.end(), other) - sides.begin();
            if (k == sides.size()) {
                if (sides.size() >= AGOCUDA_PX_MAX_SIDES) return false;
                sides.push_back(other);
            }
            op.side = (int32_t)k;
        }
        if (code == AGOCUDA_PX_THRESHOLD_BINARY) op.p0 = static_cast<Threshold *>(n.p[2])->value.U8;
        if (code == AGOCUDA_PX_THRESHOLD_RANGE) {
            op.p0 = static_cast<Threshold *>(n.p[2])->lower.U8;
            op.p1 = static_cast<Threshold *>(n.p[2])->upper.U8;
        }
        if (px_stencil(code)) stencils++;
        P.ops[P.numOps++] = op;
        return true;
    };
    Ref *src = a.p[1];
    if (!add_op(a, code0, px_binary(code0) ? a.p[2] : nullptr, 0)) return false;
    nodes.push_back(&a);
    Ref *out = a.p[0];
    for (;;) {
        if (!private_virtual(g, out) || IMG(out)->parent) break;
        LNode *n = const_cast<LNode *>(reader_of(g, out));
        if (!n || n->removed || taken.count(n)) break;
        const int cd = px_code(n->k);
        if (!cd) break;
        Ref *other = nullptr;
        int first = 0;
        if (px_binary(cd)) {
            if (n->p[1] == out && n->p[2] != out) other = n->p[2];
            else if (n->p[2] == out && n->p[1] != out) { other = n->p[1]; first = 1; }
            else break;
        } else if (n->p[1] != out) {
            break;
        }
        const agocuda_pixel_program keep = P;
        const size_t nsides = sides.size();
        const int kst = stencils;
        if (!add_op(*n, cd, other, first)) { P = keep; sides.resize(nsides); stencils = kst; break; }
        elide.push_back(out);
        nodes.push_back(n);
        out = n->p[0];
    }
    if (nodes.size() < 2) return false;
    Image *s = IMG(src), *d = IMG(out);
    if (s->width != d->width || s->height != d->height || s->width < 4 || s->height < 3) return false;
    // the kernel copies src / side rows in 16-byte chunks (images imported from device
    // pointers may not allow that: they run per node)
    auto a16 = [](Ref *r) {
        const Plane &pl = IMG(r)->planes[0];
        return IMG(r)->import_type != VX_MEMORY_TYPE_HIP || (((uintptr_t)pl.dev | pl.dev_stride) & 15) == 0;
    };
    auto a4 = [](Ref *r) {
        const Plane &pl = IMG(r)->planes[0];
        return IMG(r)->import_type != VX_MEMORY_TYPE_HIP || (((uintptr_t)pl.dev | pl.dev_stride) & 3) == 0;
    };
    if (!a16(src) || !a4(out)) return false;
    for (Ref *sd : sides) if (!a16(sd)) return false;
    c.kind = "fused_PixelChain";
    c.nodes = nodes;
    c.src = src; c.dst = out;
    c.elide = elide;
    c.prog = P;
    c.sides = sides;
    c.key = {P.numOps, (int64_t)sides.size()};
    for (int k = 0; k < P.numOps; k++) {
        const agocuda_pixel_op &op = P.ops[k];
        c.key.insert(c.key.end(), {op.code, op.side, op.sideFirst, op.p0, op.p1});
    }
    return true;
}

// Gaussian3x3 -> SobelMagnitude -> ColorDepth_U8_S16_Sat -> Threshold_U8_U8_Binary
static bool match_gauss_sobelmag_thresh(Graph *g, LNode &a, Chain &c)
{
    if (a.k != LK::GAUSSIAN_U8_U8_3x3 || !private_virtual(g, a.p[0])) return false;
    LNode *b = const_cast<LNode *>(reader_of(g, a.p[0]));
    if (!b || b->removed || b->k != LK::SOBEL_MAGNITUDE_S16_U8_3x3 || !private_virtual(g, b->p[0])) return false;
    LNode *d = const_cast<LNode *>(reader_of(g, b->p[0]));
    if (!d || d->k != LK::COLOR_DEPTH_U8_S16_SAT || !private_virtual(g, d->p[0])) return false;
    LNode *t = const_cast<LNode *>(reader_of(g, d->p[0]));
    if (!t || t->k != LK::THRESHOLD_U8_U8_BINARY) return false;
    Image *src = IMG(a.p[1]), *dst = IMG(t->p[0]);
    if (src->width < 5 || src->height < 5) return false;
    c.kind = "fused_GaussSobelMagDepthThresh";
    c.nodes = {&a, b, d, t};
    c.key = {sc_i32(d->p[2]), static_cast<Threshold *>(t->p[2])->value.U8};
    c.src = src; c.dst = dst;
    c.elide = {a.p[0], b->p[0], d->p[0]};
    return true;
}

// CannySobel -> CannySuppThreshold -> CannyEdgeTrace (one vxCannyEdgeDetectorNode)
static bool match_canny(Graph *g, LNode &a, Chain &c)
{
    if (a.k != LK::CANNY_SOBEL_U16_U8_3x3_L1NORM || !private_virtual(g, a.p[0])) return false;
    LNode *b = const_cast<LNode *>(reader_of(g, a.p[0]));
    if (!b || b->k != LK::CANNY_SUPP_THRESHOLD_U8XY_U16_3x3 || !b->p[1]->is_virtual) return false;
    LNode *t = const_cast<LNode *>(reader_of(g, b->p[1]));
    if (!t || t->k != LK::CANNY_EDGE_TRACE_U8_U8XY || t->p[0] != b->p[0]) return false;
    Threshold *th = static_cast<Threshold *>(b->p[3]);
    c.kind = "fused_CannyEdgeDetector";
    c.nodes = {&a, b, t};
    c.key = {(int64_t)(uint16_t)th->lower.U32, (int64_t)(uint16_t)th->upper.U32};
    c.src = a.p[1]; c.dst = b->p[0];
    c.elide = {a.p[0], b->p[1]};
    return true;
}

// HarrisSobel -> HarrisScore -> NonMaxSupp -> HarrisMergeSortAndPick (one vxHarrisCornersNode)
static bool match_harris(Graph *g, LNode &a, Chain &c)
{
    if (a.k != LK::HARRIS_SOBEL_HG3_U8_3x3 || !private_virtual(g, a.p[0])) return false;
    LNode *b = const_cast<LNode *>(reader_of(g, a.p[0]));
    if (!b || b->k != LK::HARRIS_SCORE_HVC_HG3_3x3 || !private_virtual(g, b->p[0])) return false;
    LNode *n = const_cast<LNode *>(reader_of(g, b->p[0]));
    if (!n || n->k != LK::NON_MAX_SUPP_XY_ANY_3x3 || !private_virtual(g, n->p[0])) return false;
    LNode *pk = const_cast<LNode *>(reader_of(g, n->p[0]));
    if (!pk || pk->k != LK::HARRIS_MERGE_SORT_AND_PICK_XY_XYS) return false;
    c.kind = "fused_HarrisCorners";
    c.nodes = {&a, b, n, pk};
    c.src = a.p[1]; c.dst = pk->p[0];
    c.elide = {a.p[0], b->p[0], n->p[0]};
    return true;
}

// ColorConvert_NV12_RGB + ColorConvert_IYUV_RGB of one RGB image, and a bilinear and an area
// ScaleImage of (either) Y plane to exactly half size: one pass over the RGB frame.
static bool match_color_scale(Graph *g, LNode &a, Chain &c)
{
    if (a.k != LK::COLOR_CONVERT_NV12_RGB) return false;
    Ref *rgb = a.p[2];
    Image *ri = IMG(rgb);
    if (ri->width < 16 || (ri->width & 1) || (ri->height & 1)) return false;
    LNode *iy = nullptr, *sb = nullptr, *sa = nullptr;
    for (LNode &n : g->lnodes) {
        if (n.removed) continue;
        if (n.k == LK::COLOR_CONVERT_IYUV_RGB && n.p[3] == rgb && !iy) iy = &n;
    }
    if (!iy) return false;
    for (LNode &n : g->lnodes) {
        if (n.removed || (n.p.size() < 2)) continue;
        if (n.p[1] != a.p[0] && n.p[1] != iy->p[0]) continue;
        Image *o = IMG(n.p[0]);
        if (o->width * 2 != ri->width || o->height * 2 != ri->height) continue;
        if (n.k == LK::SCALE_IMAGE_U8_U8_BILINEAR && !sb) sb = &n;
        if (n.k == LK::SCALE_IMAGE_U8_U8_AREA && !sa) sa = &n;
    }
    if (!sb || !sa) return false;
    c.kind = "fused_ColorScale";
    c.nodes = {&a, iy, sb, sa};
    c.src = rgb; c.dst = nullptr;
    return true;
}

static vx_status build_fused_batch(Graph *g, std::vector<Chain> &chains, Step &st)
{
    if (chains[0].kind == "batch_ScaleGaussianHalf" || chains[0].kind == "batch_OpticalFlowPyrLK") {
        std::vector<LNode *> nodes;
        for (Chain &c : chains) nodes.push_back(c.nodes[0]);
        st.name = chains[0].kind + " x" + std::to_string(chains.size());
        st.nodes = nodes;
        return chains[0].kind == "batch_ScaleGaussianHalf" ? half_batch_step(g, nodes, st) : lk_batch_step(g, nodes, st);
    }
    if (chains[0].kind == "fused_ColorScale") {
        std::vector<std::function<int(cudaStream_t)>> fns;
        st.name = chains[0].kind + " x" + std::to_string(chains.size());
        st.num_kernels = (int)chains.size();
        for (Chain &c : chains) {
            for (LNode *n : c.nodes) st.nodes.push_back(n);
            LNode *nv = c.nodes[0], *iy = c.nodes[1], *sb = c.nodes[2], *sa = c.nodes[3];
            Image *s = IMG(c.src);
            const uint32_t w = s->width, h = s->height, ss = s->planes[0].dev_stride;
            const uint8_t *src = s->planes[0].dev;
            uint8_t *y1 = dptr(nv->p[0]), *uv = dptr(nv->p[1]), *y2 = dptr(iy->p[0]), *u = dptr(iy->p[1]), *v = dptr(iy->p[2]);
            uint8_t *ob = dptr(sb->p[0]), *oa = dptr(sa->p[0]);
            const uint32_t y1s = dstride(nv->p[0]), uvs = dstride(nv->p[1]), y2s = dstride(iy->p[0]), us = dstride(iy->p[1]),
                           vs = dstride(iy->p[2]), obs = dstride(sb->p[0]), oas = dstride(sa->p[0]);
            fns.push_back([=](cudaStream_t q) {
                return agocuda_fused_ColorScale_RGB(S(q), w, h, src, ss, y1, y1s, uv, uvs, y2, y2s, u, us, v, vs, ob, obs, oa, oas);
            });
            st.parts.push_back(Part{fns.back(), c.nodes});
        }
        st.launch = [fns](cudaStream_t q) {
            for (auto &f : fns) { int rc = f(q); if (rc) return rc; }
            return 0;
        };
        return VX_SUCCESS;
    }
    if (chains[0].kind == "fused_CannyEdgeDetector" || chains[0].kind == "fused_HarrisCorners") {
        // one step holding every frame's launches (one CUDA graph segment)
        std::vector<std::function<int(cudaStream_t)>> fns;
        st.name = chains[0].kind + " x" + std::to_string(chains.size());
        st.num_kernels = 0;
        uint32_t *status = g->status_dev;
        for (Chain &c : chains) {
            for (LNode *n : c.nodes) st.nodes.push_back(n);
            Image *s = IMG(c.src);
            const uint32_t w = s->width, h = s->height, ss = s->planes[0].dev_stride;
            const uint8_t *src = s->planes[0].dev;
            if (c.kind == "fused_CannyEdgeDetector") {
                Image *d = IMG(c.dst);
                uint8_t *dst = d->planes[0].dev; const uint32_t ds = d->planes[0].dev_stride;
                const size_t sb = agocuda_fused_CannyEdgeDetector_scratch_size(w, h);
                void *scr = scratch(g, sb);
                if (!scr) return VX_ERROR_NO_MEMORY;
                const uint16_t lo = (uint16_t)c.key[0], hi = (uint16_t)c.key[1];
                fns.push_back([=](cudaStream_t q) {
                    return agocuda_fused_CannyEdgeDetector_3x3_L1(S(q), w, h, dst, ds, src, ss, lo, hi, scr, sb, status);
                });
                st.parts.push_back(Part{fns.back(), c.nodes});
                st.num_kernels += 4;
            } else {
                LNode *sc = c.nodes[1], *pk = c.nodes[3];
                const float k = sc_f32(sc->p[2]), tc = sc_f32(sc->p[3]), norm = harris_norm(sc_i32(sc->p[4]));
                const float mind = sc_f32(pk->p[3]);
                Array *corners = static_cast<Array *>(pk->p[0]);
                Scalar *num = pk->p[1] ? static_cast<Scalar *>(pk->p[1]) : nullptr;
                if (num && scalar_alloc_device(num)) return VX_ERROR_NO_MEMORY;
                void *out = corners->dev; const uint32_t ocap = (uint32_t)corners->capacity; uint32_t *oc = corners->dev_count;
                uint32_t *nc = num ? num->dev : nullptr;
                const size_t sb = agocuda_fused_HarrisCorners_scratch_size(w, h, mind);
                void *scr = scratch(g, sb);
                if (!scr) return VX_ERROR_NO_MEMORY;
                fns.push_back([=](cudaStream_t q) {
                    return agocuda_fused_HarrisCorners_3x3(S(q), w, h, src, ss, k, tc, norm, mind, out, ocap, oc, nc, scr, sb, status);
                });
                st.parts.push_back(Part{fns.back(), c.nodes});
                st.num_kernels += 3;
            }
        }
        st.launch = [fns](cudaStream_t q) {
            for (auto &f : fns) { int rc = f(q); if (rc) return rc; }
            return 0;
        };
        return VX_SUCCESS;
    }
    const Chain &c0 = chains[0];
    st.name = c0.kind + " x" + std::to_string(chains.size());
    for (Chain &c : chains) for (LNode *n : c.nodes) st.nodes.push_back(n);
    if (c0.kind == "fused_PixelChain") {
        std::vector<agocuda_pixel_frame> fr;
        for (Chain &c : chains) {
            Image *s = IMG(c.src), *d = IMG(c.dst);
            agocuda_pixel_frame f{};
            f.src = s->planes[0].dev; f.srcStride = s->planes[0].dev_stride;
            f.dst = d->planes[0].dev; f.dstStride = d->planes[0].dev_stride;
            f.width = d->width; f.height = d->height;
            for (size_t k = 0; k < c.sides.size(); k++) {
                Image *sd = IMG(c.sides[k]);
                if (sd->width != d->width || sd->height != d->height) return VX_ERROR_INVALID_DIMENSION;
                f.side[k] = sd->planes[0].dev; f.sideStride[k] = sd->planes[0].dev_stride;
            }
            fr.push_back(f);
        }
        agocuda_pixel_frame *dev = (agocuda_pixel_frame *)scratch(g, fr.size() * sizeof(agocuda_pixel_frame));
        if (!dev) return VX_ERROR_NO_MEMORY;
        cudaMemcpy(dev, fr.data(), fr.size() * sizeof(agocuda_pixel_frame), cudaMemcpyHostToDevice);
        const agocuda_pixel_program prog = c0.prog;
        // TMA staging: one tensor map per plane of every frame, encoded now, kept on the device
        uint8_t *maps = nullptr;
        const size_t mapsPerFrame = agocuda_PixelChain_tensor_maps_size(1);
        if (!(g->optimizer_flags & kOptNoTma)) {
            const size_t mb = agocuda_PixelChain_tensor_maps_size((uint32_t)fr.size());
            std::vector<uint64_t> host((mb + 7) / 8 + 8);
            void *h = (void *)(((uintptr_t)host.data() + 63) & ~(uintptr_t)63);
            if (agocuda_PixelChain_tensor_maps(&prog, fr.data(), (uint32_t)fr.size(), h, mb) == 0) {
                maps = (uint8_t *)scratch(g, mb);
                if (!maps) return VX_ERROR_NO_MEMORY;
                cudaMemcpy(maps, h, mb, cudaMemcpyHostToDevice);
            }
        }
        uint32_t *status = g->status_dev;
        std::vector<std::function<int(cudaStream_t)>> fns;
        for (size_t k0 = 0; k0 < fr.size(); k0 += kGroupFrames) {
            const size_t k1 = std::min(fr.size(), k0 + kGroupFrames);
            uint32_t gw = 0, gh = 0;
            for (size_t k = k0; k < k1; k++) { gw = std::max(gw, fr[k].width); gh = std::max(gh, fr[k].height); }
            const agocuda_pixel_frame *d0 = dev + k0;
            const uint32_t n = (uint32_t)(k1 - k0);
            if (maps) {
                const uint8_t *m0 = maps + k0 * mapsPerFrame;
                fns.push_back([=](cudaStream_t q) {
                    return agocuda_fused_PixelChain_U8_tma(S(q), &prog, d0, m0, n, gw, gh, status);
                });
            } else {
                fns.push_back([=](cudaStream_t q) { return agocuda_fused_PixelChain_U8(S(q), &prog, d0, n, gw, gh); });
            }
            Part pt{fns.back(), {}};
            for (size_t k = k0; k < k1; k++) for (LNode *nd : chains[k].nodes) pt.nodes.push_back(nd);
            st.parts.push_back(std::move(pt));
        }
        st.num_kernels = (int)fns.size();
        st.launch = [fns](cudaStream_t q) {
            for (auto &f : fns) { int rc = f(q); if (rc) return rc; }
            return 0;
        };
        return VX_SUCCESS;
    }
    if (c0.kind == "fused_GaussSobelMagDepthThresh") {
        std::vector<agocuda_frame> fr;
        for (Chain &c : chains) {
            Image *s = IMG(c.src), *d = IMG(c.dst);
            agocuda_frame f{};
            f.src = s->planes[0].dev; f.dst = d->planes[0].dev;
            f.width = s->width; f.height = s->height;
            f.srcStride = s->planes[0].dev_stride; f.dstStride = d->planes[0].dev_stride;
            // the virtual SobelMagnitude output AGO allocates is 16-byte aligned: SIMD body
            // [0, W - W % 16) (ago_haf_cpu_filter.cpp:2480-2483)
            f.simdBegin = 0; f.simdEnd = (int32_t)(s->width - (s->width & 15));
            fr.push_back(f);
        }
        agocuda_frame *dev = (agocuda_frame *)scratch(g, fr.size() * sizeof(agocuda_frame));
        if (!dev) return VX_ERROR_NO_MEMORY;
        cudaMemcpy(dev, fr.data(), fr.size() * sizeof(agocuda_frame), cudaMemcpyHostToDevice);
        const int32_t shift = (int32_t)c0.key[0], thr = (int32_t)c0.key[1];
        // launch shape from the autotuner's table (largest frame of the batch): rows per
        // thread, warps per block, resident blocks per SM, persistent tile queue or grid
        uint32_t bw = 0, bh = 0;
        for (const agocuda_frame &f : fr)
            if ((uint64_t)f.width * f.height > (uint64_t)bw * bh) { bw = f.width; bh = f.height; }
        std::vector<uint32_t> cfg = tune_lookup("fused_GaussSobelMagDepthThresh", bw, bh, {18, 4, 6, 1});
        if (!agocuda_fused_GaussSobelMagDepthThresh_tiles(bw, bh, cfg[0], cfg[1])) cfg = {18, 4, 6, 1};
        // frames uploaded from application buffers inside the CUDA graph go in groups, so the
        // first group computes while later frames are on the bus; resident frames share one queue
        bool streamed = false;
        for (Chain &c : chains) {
            Image *s0 = IMG(c.src), *root = s0->parent ? s0->parent : s0;
            if (root->import_type == VX_MEMORY_TYPE_HOST) streamed = true;
        }
        const size_t group = streamed ? kGroupFrames : fr.size();
        // TMA staging (the default): one tensor map per frame, encoded now, kept on the device
        uint8_t *maps = nullptr;
        const size_t mapBytes = agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_size(1);
        // its tile shape from the autotuner's table (rows per warp, warps per block)
        std::vector<uint32_t> tshape = tune_lookup("fused_GaussSobelMagDepthThresh_tma", bw, bh, {36, 2});
        if (!(g->optimizer_flags & kOptNoTma)) {
            const size_t mb = agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_size((uint32_t)fr.size());
            std::vector<uint64_t> host((mb + 7) / 8 + 8);
            void *h = (void *)(((uintptr_t)host.data() + 63) & ~(uintptr_t)63);
            int rc = agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_shape(fr.data(), (uint32_t)fr.size(), tshape[0],
                                                                              tshape[1], h, mb);
            if (rc != 0 && (tshape[0] != 36 || tshape[1] != 2)) {   // a shape this library does not build
                tshape = {36, 2};
                rc = agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_shape(fr.data(), (uint32_t)fr.size(), 36, 2, h, mb);
            }
            if (rc == 0) {
                maps = (uint8_t *)scratch(g, mb);
                if (!maps) return VX_ERROR_NO_MEMORY;
                cudaMemcpy(maps, h, mb, cudaMemcpyHostToDevice);
            }
        }
        uint32_t *status = g->status_dev;
        std::vector<std::function<int(cudaStream_t)>> fns;
        for (size_t k0 = 0; k0 < fr.size(); k0 += group) {
            const size_t k1 = std::min(fr.size(), k0 + group);
            uint32_t gw = 0, gh = 0;
            for (size_t k = k0; k < k1; k++) { gw = std::max(gw, fr[k].width); gh = std::max(gh, fr[k].height); }
            const agocuda_frame *d0 = dev + k0;
            const uint32_t n = (uint32_t)(k1 - k0);
            if (maps) {
                const uint8_t *m0 = maps + k0 * mapBytes;
                const uint32_t tr = tshape[0], tw = tshape[1];
                fns.push_back([=](cudaStream_t q) {
                    return agocuda_fused_GaussSobelMagDepthThresh_tma_shape(S(q), d0, m0, n, gw, gh, shift, thr, tr, tw,
                                                                           status);
                });
            } else if (cfg[3]) {
                // tile prefix of the group's frames, then the queue words
                std::vector<uint32_t> pre(n + 1 + 2, 0);
                for (uint32_t k = 0; k < n; k++)
                    pre[k + 1] = pre[k] + agocuda_fused_GaussSobelMagDepthThresh_tiles(fr[k0 + k].width, fr[k0 + k].height,
                                                                                       cfg[0], cfg[1]);
                if (pre.size() % 2) pre.push_back(0);
                uint32_t *dpre = (uint32_t *)scratch(g, pre.size() * sizeof(uint32_t));
                if (!dpre) return VX_ERROR_NO_MEMORY;
                cudaMemcpy(dpre, pre.data(), pre.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
                uint32_t *queue = dpre + ((n + 1 + 1) & ~1u);        // 8-byte aligned, zero
                const uint32_t rows = cfg[0], warps = cfg[1], bps = cfg[2];
                fns.push_back([=](cudaStream_t q) {
                    return agocuda_fused_GaussSobelMagDepthThresh_persistent(S(q), d0, n, dpre, queue, rows, warps, bps,
                                                                             shift, thr);
                });
            } else {
                fns.push_back([=](cudaStream_t q) {
                    return agocuda_fused_GaussSobelMagDepthThresh(S(q), d0, n, gw, gh, shift, thr);
                });
            }
            Part pt{fns.back(), {}};
            for (size_t k = k0; k < k1; k++) for (LNode *nd : chains[k].nodes) pt.nodes.push_back(nd);
            st.parts.push_back(std::move(pt));
        }
        st.num_kernels = (int)fns.size();
        st.launch = [fns](cudaStream_t q) {
            for (auto &f : fns) { int rc = f(q); if (rc) return rc; }
            return 0;
        };
        return VX_SUCCESS;
    }
    return VX_ERROR_NOT_IMPLEMENTED;
}

// ------------------------------------------------------------------------------------
vx_status plan_graph(Graph *g)
{
    for (void *p : g->dev_scratch) cudaFree(p);
    g->dev_scratch.clear();
    g->steps.clear();
    g->host_steps = false;
    g->inputs.clear();
    g->outputs.clear();

    // graph inputs / outputs and device allocation of every image the plan touches
    std::set<Ref *> written, read;
    for (LNode &ln : g->lnodes)
        for (size_t i = 0; i < ln.p.size(); i++) {
            Ref *r = ln.p[i];
            if (!r) continue;
            (lnode_is_output(ln, i) ? written : read).insert(r);
            if (ln.k == LK::CANNY_EDGE_TRACE_U8_U8XY && i == 0) written.insert(r);
        }
    auto root = [](Ref *r) -> Ref * { return (r->type == VX_TYPE_IMAGE && IMG(r)->parent) ? IMG(r)->parent : r; };
    // by root, each once: the planes of a multi-plane image are images of their own (AGO children)
    std::set<Ref *> seen_in, seen_out;
    for (Ref *r : read)
        if (!r->is_virtual && (r->type == VX_TYPE_IMAGE || r->type == VX_TYPE_ARRAY || r->type == VX_TYPE_PYRAMID) &&
            !written.count(r) && seen_in.insert(root(r)).second)
            g->inputs.push_back(root(r));
    for (Ref *r : written)
        if (!r->is_virtual && seen_out.insert(root(r)).second) g->outputs.push_back(root(r));

    // fusion
    std::set<LNode *> fused;
    std::map<std::vector<int64_t>, std::vector<Chain>> groups;   // (pattern id, level, key...) -> chains
    std::vector<std::vector<int64_t>> group_order;
    if (!(g->optimizer_flags & kOptNoFusion)) {
        for (LNode &ln : g->lnodes) {
            Chain c;
            if (fused.count(&ln)) continue;
            int pattern = 0;
            if (match_gauss_sobelmag_thresh(g, ln, c)) pattern = 1;
            else if (match_canny(g, ln, c)) pattern = 2;
            else if (match_harris(g, ln, c)) pattern = 3;
            else if (match_color_scale(g, ln, c)) pattern = 4;
            else if (ln.k == LK::SCALE_GAUSSIAN_HALF_U8_U8_5x5) { c.kind = "batch_ScaleGaussianHalf"; c.nodes = {&ln}; pattern = 5; }
            else if (ln.k == LK::OPTICAL_FLOW_PYR_LK_XY_XY) { c.kind = "batch_OpticalFlowPyrLK"; c.nodes = {&ln}; pattern = 6; }
            else if (match_pixel_chain(g, ln, fused, c)) pattern = 7;
            for (LNode *n : c.nodes) if (pattern && fused.count(n)) pattern = 0;   // a node joins one chain
            if (pattern) {
                std::vector<int64_t> gk{pattern, ln.level};
                gk.insert(gk.end(), c.key.begin(), c.key.end());
                if (!groups.count(gk)) group_order.push_back(gk);
                groups[gk].push_back(c);
                for (LNode *n : c.nodes) fused.insert(n);
            }
        }
    }
    // images eliminated by fusion need no memory; everything else is allocated now
    std::set<Ref *> elided;
    for (auto &kv : groups)
        for (Chain &c : kv.second)
            for (Ref *r : c.elide) elided.insert(r);
    for (LNode &ln : g->lnodes)
        for (Ref *r : ln.p) {
            if (!r || elided.count(r)) continue;
            if (r->type == VX_TYPE_IMAGE) { if (image_alloc_device(IMG(r))) return VX_ERROR_NO_MEMORY; }
            else if (r->type == VX_TYPE_ARRAY) { if (array_alloc_device(static_cast<Array *>(r))) return VX_ERROR_NO_MEMORY; }
            else if (r->type == VX_TYPE_PYRAMID) {
                for (Image *lv : static_cast<Pyramid *>(r)->level)
                    if (!g->replaced.count(lv) && image_alloc_device(lv)) return VX_ERROR_NO_MEMORY;
            }
            else if (r->type == VX_TYPE_SCALAR && r->is_virtual == false) { /* host value */ }
        }

    // steps in level order: a fused group is emitted where its first node sits
    std::map<LNode *, std::vector<int64_t>> first_of_group;
    for (auto &gk : group_order) first_of_group[groups[gk][0].nodes[0]] = gk;
    std::ostringstream txt;
    for (LNode &ln : g->lnodes) {
        Step st;
        if (fused.count(&ln)) {
            auto it = first_of_group.find(&ln);
            if (it == first_of_group.end()) continue;
            vx_status s = build_fused_batch(g, groups[it->second], st);
            if (s) return s;
        } else {
            vx_status s = plain_step(g, ln, st);
            if (s) return s;
        }
        txt << st.name << "\t" << st.num_kernels << "\n";
        g->steps.push_back(std::move(st));
    }
    g->plan_text = txt.str();
    return VX_SUCCESS;
}

}  // namespace agovx
