// vx_graph.cpp -- graphs, nodes, node factories, vxVerifyGraph and vxProcessGraph.
//
// vxVerifyGraph (reference: api/vx_api.cpp:2934 -> agoVerifyGraph/agoOptimizeGraph/
// agoInitializeGraph) here: validates nodes and infers virtual meta, lowers the graph to
// AGO low-level kernels with AGO's merge rules, propagates valid rectangles, plans the
// device work (fused multi-node kernels, batched launches over independent same-kernel
// nodes), allocates device buffers and captures the whole launch sequence into one CUDA
// graph.  vxProcessGraph uploads stale inputs, replays the CUDA graph and waits.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <set>

#include "vx_internal.h"

using namespace agovx;

namespace agovx {

static void plan_state_free(PlanState &ps)
{
    if (ps.cexec) cudaGraphExecDestroy(ps.cexec);
    if (ps.cgraph) cudaGraphDestroy(ps.cgraph);
    for (void *p : ps.dev_scratch) cudaFree(p);
    ps = PlanState{};
}

// move the graph's current plan into `ps` (and the other way round)
static void plan_state_swap(Graph *g, PlanState &ps)
{
    std::swap(g->steps, ps.steps);
    std::swap(g->dev_scratch, ps.dev_scratch);
    std::swap(g->cgraph, ps.cgraph);
    std::swap(g->cexec, ps.cexec);
    std::swap(g->inputs, ps.inputs);
    std::swap(g->outputs, ps.outputs);
    std::swap(g->streamed_in, ps.streamed_in);
    std::swap(g->streamed_out, ps.streamed_out);
    std::swap(g->staged_in, ps.staged_in);
    std::swap(g->staged_out, ps.staged_out);
    std::swap(g->plan_text, ps.plan_text);
}

void graph_plan_cache_clear(Graph *g)
{
    for (auto &kv : g->plan_cache) plan_state_free(kv.second);
    g->plan_cache.clear();
}

void graph_invalidate(Graph *g)
{
    graph_plan_cache_clear(g);
    g->verified = false;
    g->state = VX_GRAPH_STATE_UNVERIFIED;
    if (g->cexec) { cudaGraphExecDestroy(g->cexec); g->cexec = nullptr; }
    if (g->cgraph) { cudaGraphDestroy(g->cgraph); g->cgraph = nullptr; }
    g->streamed_in.clear();
    g->streamed_out.clear();
    g->steps.clear();
}

static uint64_t fnv(uint64_t h, const void *p, size_t n)
{
    const uint8_t *b = (const uint8_t *)p;
    for (size_t i = 0; i < n; i++) { h ^= b[i]; h *= 1099511628211ull; }
    return h;
}

// Kernel parameters passed by value are baked into the captured CUDA graph: a change of
// any of them (scalar, threshold, matrix, remap table, valid rectangle) re-plans.
static uint64_t param_signature(Graph *g)
{
    uint64_t h = 1469598103934665603ull;
    for (LNode &ln : g->lnodes) {
        for (Ref *r : ln.p) {
            if (!r) continue;
            switch (r->type) {
            case VX_TYPE_SCALAR: h = fnv(h, &static_cast<Scalar *>(r)->version, 8); h = fnv(h, static_cast<Scalar *>(r)->v.raw, 8); break;
            case VX_TYPE_THRESHOLD: h = fnv(h, &static_cast<Threshold *>(r)->version, 8); break;
            case VX_TYPE_MATRIX: h = fnv(h, &static_cast<Matrix *>(r)->version, 8); break;
            case VX_TYPE_LUT: h = fnv(h, &static_cast<Lut *>(r)->version, 8); break;
            case VX_TYPE_CONVOLUTION: h = fnv(h, &static_cast<Convolution *>(r)->version, 8); break;
            case VX_TYPE_REMAP: h = fnv(h, &static_cast<Remap *>(r)->version, 8); break;
            case VX_TYPE_IMAGE: {
                Image *img = IMG(r);
                h = fnv(h, &img->valid, sizeof(img->valid));
                for (int i = 0; i < img->num_planes; i++) h = fnv(h, &img->planes[i].dev, sizeof(void *));
                break;
            }
            // storage that ageing a delay moves between objects
            case VX_TYPE_ARRAY: h = fnv(h, &static_cast<Array *>(r)->dev, sizeof(void *)); break;
            case VX_TYPE_PYRAMID:
                for (Image *lv : static_cast<Pyramid *>(r)->level) h = fnv(h, &lv->planes[0].dev, sizeof(void *));
                break;
            default: break;
            }
        }
    }
    return h;
}

// ---- capture ------------------------------------------------------------------------
// The plan's steps -- split into their per-frame parts where a step batches independent
// frames -- become the nodes of a dependency graph over the data each one reads and
// writes.  Stream capture over a few lanes (streams forked from the graph's stream and
// joined back to it) turns that into a CUDA graph whose independent branches run
// concurrently: one frame's single-CTA corner pick beside another frame's stencils, the
// upload of frame i+1 beside the kernels of frame i.  Host-imported images whose memory is
// page-locked are uploaded and downloaded inside the CUDA graph, on lanes of their own, so
// vxProcessGraph overlaps the PCIe copies with the kernels.
constexpr int kComputeLanes = 8;
// image uploads and downloads (copy engines) and array transfers (small kernels reading or
// writing mapped host memory) get lanes of their own, so none waits behind another kind
// (two lanes each way: copies of a few MB finish below PCIe rate one at a time)
constexpr int kUploadLane = kComputeLanes, kDownloadLane = kComputeLanes + 2, kArrayLane = kComputeLanes + 4;
constexpr int kNumLanes = kComputeLanes + 5;

struct CapPart {
    std::function<int(cudaStream_t)> launch;
    std::vector<Ref *> rd, wr;
    bool barrier = false;          // touches unknown data: ordered after and before everything
    int lane = 0;
    std::vector<int> deps;
    cudaEvent_t done = nullptr;    // recorded after the part when another lane waits for it
};

static bool host_pinned(const void *p)
{
    cudaPointerAttributes a{};
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
    return a.type == cudaMemoryTypeHost;
}

// Host-imported image that can be copied inside the CUDA graph.
static bool streamable(Image *root)
{
    if (root->import_type != VX_MEMORY_TYPE_HOST || !root->allocated()) return false;
    for (int i = 0; i < root->num_planes; i++)
        if (!host_pinned(root->planes[i].host)) return false;
    return true;
}

static void collect_touches(Graph *g, const std::vector<LNode *> &nodes, const std::map<Image *, Ref *> &level_of,
                            CapPart &cp)
{
    auto key = [&](Ref *r) -> Ref * {
        auto rp = g->replaced.find(r);
        if (rp != g->replaced.end()) r = rp->second;
        if (r->type == VX_TYPE_IMAGE) {
            Image *img = IMG(r);
            auto lv = level_of.find(img);
            if (lv != level_of.end()) return lv->second;
            return img->parent ? img->parent : img;
        }
        return r;
    };
    if (nodes.empty()) { cp.barrier = true; return; }
    for (LNode *ln : nodes)
        for (size_t i = 0; i < ln->p.size(); i++) {
            Ref *r = ln->p[i];
            if (!r) continue;
            const bool w = lnode_is_output(*ln, i) || (ln->k == LK::CANNY_EDGE_TRACE_U8_U8XY && i == 0);
            (w ? cp.wr : cp.rd).push_back(key(r));
            if (r->type == VX_TYPE_PYRAMID)   // levels aliased to other images (copy removal)
                for (Image *lv : static_cast<Pyramid *>(r)->level) {
                    auto rp = g->replaced.find(lv);
                    if (rp != g->replaced.end()) (w ? cp.wr : cp.rd).push_back(key(rp->second));
                }
        }
}

// Array whose items can cross PCIe inside the CUDA graph: its host buffer (allocated at
// capacity when the array is created) is page-locked and mapped once, here.
static bool stageable(Array *a)
{
    if (a->is_virtual || !a->dev || !a->dev_count || a->host.empty() || a->host.size() < a->capacity * a->item_size)
        return false;
    if (!a->host_mapped) {
        if (cudaHostRegister(a->host.data(), a->host.size(), cudaHostRegisterMapped) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        void *d = nullptr;
        if (cudaHostGetDevicePointer(&d, a->host.data(), 0) != cudaSuccess) {
            cudaHostUnregister(a->host.data());
            cudaGetLastError();
            return false;
        }
        a->host_mapped = (uint8_t *)d;
    }
    return true;
}

// host <-> device copy of one plane; one linear copy when both layouts are packed
static cudaError_t plane_copy(const Plane &p, cudaMemcpyKind kind, cudaStream_t q)
{
    const size_t row = (size_t)p.width * p.bpp;
    const bool h2d = kind == cudaMemcpyHostToDevice;
    void *dst = h2d ? (void *)p.dev : (void *)p.host;
    const void *src = h2d ? (const void *)p.host : (const void *)p.dev;
    if (p.host_stride == row && p.dev_stride == row) return cudaMemcpyAsync(dst, src, row * p.height, kind, q);
    return h2d ? cudaMemcpy2DAsync(dst, p.dev_stride, src, p.host_stride, row, p.height, kind, q)
               : cudaMemcpy2DAsync(dst, p.host_stride, src, p.dev_stride, row, p.height, kind, q);
}

constexpr size_t kIoSlots = 1024;   // count slots per graph (arrays staged beyond this use blocking copies)

static void release_capture(Graph *g)
{
    if (g->cexec) { cudaGraphExecDestroy(g->cexec); g->cexec = nullptr; }
    if (g->cgraph) { cudaGraphDestroy(g->cgraph); g->cgraph = nullptr; }
    for (cudaEvent_t e : g->cap_events) cudaEventDestroy(e);
    g->cap_events.clear();
    g->streamed_in.clear();
    g->streamed_out.clear();
    g->staged_in.clear();
    g->staged_out.clear();
}

static cudaEvent_t cap_event(Graph *g)
{
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
    g->cap_events.push_back(e);
    return e;
}

static vx_status capture(Graph *g)
{
    release_capture(g);
    // user kernels run on the host between launches: such plans launch step by step
    if ((g->optimizer_flags & kOptNoGraphCapture) || g->host_steps) return VX_SUCCESS;
    const bool serial = (g->optimizer_flags & (kOptSerial | kOptNoFusion)) != 0;

    // ---- parts, in plan order, with the data they touch
    std::map<Image *, Ref *> level_of;
    for (LNode &ln : g->lnodes)
        for (Ref *r : ln.p)
            if (r && r->type == VX_TYPE_PYRAMID)
                for (Image *lv : static_cast<Pyramid *>(r)->level) level_of[lv] = r;
    std::vector<CapPart> parts;
    if (!serial && !g->io_slots_host) {
        if (cudaHostAlloc((void **)&g->io_slots_host, kIoSlots * sizeof(uint32_t), cudaHostAllocMapped) != cudaSuccess ||
            cudaHostGetDevicePointer((void **)&g->io_slots_dev, g->io_slots_host, 0) != cudaSuccess)
            return VX_ERROR_NO_MEMORY;
    }
    auto slot_free = [&]() { return g->staged_in.size() + g->staged_out.size() < kIoSlots; };
    if (!serial) {   // all input arrays in one launch (a table in device memory)
        std::vector<agocuda_array_xfer> xf;
        CapPart cp;
        for (Ref *r : g->inputs)
            if (r->type == VX_TYPE_ARRAY && slot_free() && stageable(static_cast<Array *>(r))) {
                Array *a = static_cast<Array *>(r);
                xf.push_back(agocuda_array_xfer{a->dev, a->dev_count, a->host_mapped, g->io_slots_dev + g->staged_in.size(),
                                                (uint32_t)a->item_size, (uint32_t)a->capacity});
                cp.wr.push_back(a);
                g->staged_in.push_back(a);
            }
        if (!xf.empty()) {
            void *table = nullptr;
            if (cudaMalloc(&table, xf.size() * sizeof(agocuda_array_xfer)) != cudaSuccess) return VX_ERROR_NO_MEMORY;
            g->dev_scratch.push_back(table);
            if (cudaMemcpy(table, xf.data(), xf.size() * sizeof(agocuda_array_xfer), cudaMemcpyHostToDevice) != cudaSuccess)
                return VX_FAILURE;
            const uint32_t n = (uint32_t)xf.size();
            cp.lane = kArrayLane;
            cp.launch = [table, n](cudaStream_t q) {
                return agocuda_array_upload_batch(q, (const agocuda_array_xfer *)table, n);
            };
            parts.push_back(std::move(cp));
        }
    }
    if (!serial)
        for (Ref *r : g->inputs)
            if (r->type == VX_TYPE_IMAGE && streamable(IMG(r))) {
                Image *img = IMG(r);
                CapPart cp;
                cp.wr = {img};
                cp.lane = kUploadLane + (int)(g->streamed_in.size() & 1);
                cp.launch = [img](cudaStream_t q) {
                    for (int i = 0; i < img->num_planes; i++)
                        if (plane_copy(img->planes[i], cudaMemcpyHostToDevice, q) != cudaSuccess) return -1;
                    return 0;
                };
                parts.push_back(std::move(cp));
                g->streamed_in.push_back(img);
            }
    for (Step &st : g->steps) {
        if (st.parts.empty() || serial) {
            CapPart cp;
            cp.launch = st.launch;
            collect_touches(g, st.nodes, level_of, cp);
            parts.push_back(std::move(cp));
        } else {
            for (Part &pt : st.parts) {
                CapPart cp;
                cp.launch = pt.launch;
                collect_touches(g, pt.nodes, level_of, cp);
                parts.push_back(std::move(cp));
            }
        }
    }
    if (!serial)
        for (Ref *r : g->outputs)
            if (r->type == VX_TYPE_IMAGE && streamable(IMG(r))) {
                Image *img = IMG(r);
                CapPart cp;
                cp.rd = {img};
                cp.lane = kDownloadLane + (int)(g->streamed_out.size() & 1);
                cp.launch = [img](cudaStream_t q) {
                    for (int i = 0; i < img->num_planes; i++)
                        if (plane_copy(img->planes[i], cudaMemcpyDeviceToHost, q) != cudaSuccess) return -1;
                    return 0;
                };
                parts.push_back(std::move(cp));
                g->streamed_out.push_back(img);
            }
    if (!serial)
        for (Ref *r : g->outputs)
            if (r->type == VX_TYPE_ARRAY && slot_free() && stageable(static_cast<Array *>(r))) {
                Array *a = static_cast<Array *>(r);
                uint32_t *slot = g->io_slots_dev + g->staged_in.size() + g->staged_out.size();
                CapPart cp;
                cp.rd = {a};
                cp.lane = kArrayLane;
                cp.launch = [a, slot](cudaStream_t q) {
                    return agocuda_array_download(q, a->host_mapped, slot, a->dev, a->dev_count, (uint32_t)a->item_size,
                                                  (uint32_t)a->capacity);
                };
                parts.push_back(std::move(cp));
                g->staged_out.push_back(a);
            }

    // the array transfers are kernels of the CUDA graph too: list them with the plan
    if (!g->staged_in.empty()) g->plan_text += "array_upload_batch\t1\n";
    if (!g->staged_out.empty())
        g->plan_text += "array_download x" + std::to_string(g->staged_out.size()) + "\t" +
                        std::to_string(g->staged_out.size()) + "\n";

    // ---- dependencies: read-after-write, write-after-write, write-after-read
    std::map<Ref *, int> last_writer;
    std::map<Ref *, std::vector<int>> readers;
    int last_barrier = -1;
    for (int j = 0; j < (int)parts.size(); j++) {
        CapPart &cp = parts[j];
        std::set<int> d;
        if (cp.barrier) {
            for (int i = 0; i < j; i++) d.insert(i);
            last_barrier = j;
        } else {
            if (last_barrier >= 0) d.insert(last_barrier);
            for (Ref *r : cp.rd) { auto w = last_writer.find(r); if (w != last_writer.end()) d.insert(w->second); }
            for (Ref *r : cp.wr) {
                auto w = last_writer.find(r);
                if (w != last_writer.end()) d.insert(w->second);
                for (int i : readers[r]) d.insert(i);
            }
        }
        d.erase(j);
        cp.deps.assign(d.begin(), d.end());
        for (Ref *r : cp.rd) readers[r].push_back(j);
        for (Ref *r : cp.wr) { last_writer[r] = j; readers[r].clear(); }
        if (cp.barrier) { last_writer.clear(); readers.clear(); }
    }

    // ---- emission order: by the latest upload a part waits for (a stable topological
    // order, since uploads are sources), so each lane's FIFO takes frames as they arrive
    std::vector<int> rank(parts.size(), 0), order(parts.size());
    for (int j = 0, up = 0; j < (int)parts.size(); j++) {
        if (parts[j].lane == kUploadLane || parts[j].lane == kUploadLane + 1) { rank[j] = ++up; continue; }
        for (int i : parts[j].deps) rank[j] = std::max(rank[j], rank[i]);
    }
    for (int j = 0; j < (int)parts.size(); j++) order[j] = j;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return rank[a] < rank[b]; });
    // compute lanes in emission order: follow the latest compute dependency (no extra
    // ordering), else take the next lane round-robin
    int rr = 0;
    for (int j : order) {
        CapPart &cp = parts[j];
        if (cp.lane >= kComputeLanes) continue;
        if (serial) { cp.lane = 0; continue; }
        int lane = -1, latest = -1;
        for (int i : cp.deps)
            if (parts[i].lane < kComputeLanes && i > latest) { latest = i; lane = parts[i].lane; }
        cp.lane = lane >= 0 ? lane : (rr++ % kComputeLanes);
    }

    // ---- record
    cudaSetDevice(g->ctx->device);
    while ((int)g->lanes.size() < kNumLanes - 1) {
        cudaStream_t s = nullptr;
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return VX_ERROR_NO_RESOURCES;
        g->lanes.push_back(s);
    }
    std::vector<cudaStream_t> lane(kNumLanes);
    lane[0] = g->stream;   // lane 0 is the graph's own stream
    for (int i = 1; i < kNumLanes; i++) lane[i] = g->lanes[i - 1];
    std::vector<bool> used(kNumLanes, false);
    for (CapPart &cp : parts)
        for (int i : cp.deps)
            if (parts[i].lane != cp.lane && !parts[i].done && !(parts[i].done = cap_event(g))) return VX_ERROR_NO_RESOURCES;
    cudaEvent_t fork = cap_event(g);
    if (!fork) return VX_ERROR_NO_RESOURCES;

    if (cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return VX_FAILURE;
    int rc = 0;
    cudaEventRecord(fork, g->stream);
    used[0] = true;
    for (size_t o = 0; o < order.size() && !rc; o++) {
        CapPart &cp = parts[order[o]];
        cudaStream_t q = lane[cp.lane];
        if (!used[cp.lane]) { cudaStreamWaitEvent(q, fork, 0); used[cp.lane] = true; }
        for (int i : cp.deps)
            if (parts[i].lane != cp.lane) cudaStreamWaitEvent(q, parts[i].done, 0);
        rc = cp.launch(q);
        if (cp.done) cudaEventRecord(cp.done, q);
    }
    for (int l = 1; l < kNumLanes && !rc; l++) {
        if (!used[l]) continue;
        cudaEvent_t e = cap_event(g);
        if (!e) { rc = -1; break; }
        cudaEventRecord(e, lane[l]);
        cudaStreamWaitEvent(g->stream, e, 0);
    }
    cudaGraph_t cg = nullptr;
    cudaError_t e = cudaStreamEndCapture(g->stream, &cg);
    if (rc || e != cudaSuccess) {
        if (cg) cudaGraphDestroy(cg);
        cudaGetLastError();
        g->streamed_in.clear();
        g->streamed_out.clear();
        g->staged_in.clear();
        g->staged_out.clear();
        log_error(g, VX_FAILURE, "ERROR: CUDA graph capture failed (step rc=%d, %s)\n", rc, cudaGetErrorString(e));
        return VX_FAILURE;
    }
    if (cudaGraphInstantiate(&g->cexec, cg, 0) != cudaSuccess) { cudaGraphDestroy(cg); return VX_FAILURE; }
    g->cgraph = cg;
    return VX_SUCCESS;
}

// User-kernel nodes: deinitialize (agoShutdownNode) before a re-verification and at
// teardown, initialize (agoInitializeNode) after a verification, allocating
// VX_KERNEL_LOCAL_DATA_SIZE bytes of node local data first.
void user_nodes_deinit(Graph *g)
{
    for (Node *n : g->nodes) {
        if (!n->ukernel || !n->initialized) continue;
        if (n->ukernel->deinit)
            n->ukernel->deinit((vx_node)n, (const vx_reference *)n->params.data(), (vx_uint32)n->params.size());
        if (n->local_owned) { free(n->local_ptr); n->local_ptr = nullptr; n->local_size = 0; n->local_owned = false; }
        n->initialized = false;
    }
}

static vx_status user_nodes_init(Graph *g)
{
    for (Node *n : g->nodes) {
        if (!n->ukernel || n->removed || n->initialized) continue;
        Kernel *k = n->ukernel;
        if (k->local_size) {
            n->local_ptr = calloc(1, k->local_size);
            if (!n->local_ptr) return VX_ERROR_NO_MEMORY;
            n->local_size = k->local_size;
            n->local_owned = true;
        }
        n->initialized = true;
        if (k->init) {
            const vx_status s = k->init((vx_node)n, (const vx_reference *)n->params.data(), (vx_uint32)n->params.size());
            if (s) {
                log_error(n, s, "ERROR: vxVerifyGraph: kernel %s: initialize failed (%d)\n", k->kname.c_str(), s);
                return s;
            }
        }
    }
    return VX_SUCCESS;
}

// The data a user kernel's node reads are current on the device (every earlier step ran
// there, and host-written outputs of earlier user nodes were uploaded): host copies refresh on
// access.
static void mark_device_current(Ref *r)
{
    if (r->type == VX_TYPE_IMAGE) {
        Image *root = IMG(r)->parent ? IMG(r)->parent : IMG(r);
        if (root->num_planes && root->planes[0].dev) { root->dev_valid = true; root->host_valid = false; }
    } else if (r->type == VX_TYPE_ARRAY) {
        Array *a = static_cast<Array *>(r);
        if (a->dev) { a->dev_valid = true; a->host_valid = false; }
    } else if (r->type == VX_TYPE_PYRAMID) {
        for (Image *lv : static_cast<Pyramid *>(r)->level) mark_device_current(lv);
    } else if (r->type == VX_TYPE_SCALAR) {
        Scalar *sc = static_cast<Scalar *>(r);
        if (sc->dev) sc->dev_newer = true;
    }
}

// host-written outputs of a user node go to the device before the next step reads them
static vx_status upload_written(Ref *r, cudaStream_t q)
{
    if (r->type == VX_TYPE_IMAGE) return image_sync_to_device(IMG(r)->parent ? IMG(r)->parent : IMG(r), q);
    if (r->type == VX_TYPE_ARRAY) return array_sync_to_device(static_cast<Array *>(r), q);
    if (r->type == VX_TYPE_PYRAMID) {
        for (Image *lv : static_cast<Pyramid *>(r)->level)
            if (vx_status s = image_sync_to_device(lv, q)) return s;
    }
    return VX_SUCCESS;
}

// A user kernel's node at execution time (ago_interface.cpp:2432, ago_util_hip.cpp:708).
// Host kernels: the stream drains, the kernel reads through the host access calls and its
// outputs are uploaded afterwards.  Device-buffer kernels: the kernel enqueues its own work
// on the graph's stream (VX_NODE_ATTRIBUTE_AMD_HIP_STREAM) and the stream keeps the order.
int run_user_node(Graph *g, Node *n, cudaStream_t q)
{
    Kernel *k = n->ukernel;
    const size_t np = n->params.size();
    auto dir = [&](size_t i) { return i < k->uparams.size() ? k->uparams[i].dir : (vx_enum)VX_INPUT; };
    if (!k->gpu_access && cudaStreamSynchronize(q) != cudaSuccess) return -1;
    for (size_t i = 0; i < np; i++)
        if (n->params[i] && dir(i) != VX_OUTPUT) mark_device_current(n->params[i]);
    g->ctx->in_user_kernel++;
    const vx_status s = k->func((vx_node)n, (const vx_reference *)n->params.data(), (vx_uint32)np);
    g->ctx->in_user_kernel--;
    n->status = s;
    if (s != VX_SUCCESS) {
        log_error(n, s, "ERROR: kernel %s exec failed (%d)\n", k->kname.c_str(), s);
        return -2;
    }
    for (size_t i = 0; i < np; i++) {
        Ref *r = n->params[i];
        if (!r || dir(i) == VX_INPUT) continue;
        if (k->gpu_access) mark_device_current(r);
        else if (upload_written(r, q)) return -3;
    }
    return 0;
}

vx_status graph_verify(Graph *g)
{
    std::lock_guard<std::recursive_mutex> lk(g->lock);
    user_nodes_deinit(g);
    graph_invalidate(g);
    cudaSetDevice(g->ctx->device);
    if (!g->stream && cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess) return VX_ERROR_NO_RESOURCES;
    if (!g->ev0) { cudaEventCreate(&g->ev0); cudaEventCreate(&g->ev1); }
    if (!g->status_host) {
        if (cudaHostAlloc((void **)&g->status_host, 64, cudaHostAllocMapped) != cudaSuccess) return VX_ERROR_NO_MEMORY;
        *g->status_host = 0;
        if (cudaHostGetDevicePointer((void **)&g->status_dev, g->status_host, 0) != cudaSuccess) return VX_ERROR_NO_RESOURCES;
    }
    vx_status s = lower_graph(g);
    if (s) return s;
    s = propagate_valid_rects(g);
    if (s) return s;
    s = plan_graph(g);
    if (s) return s;
    g->param_signature = param_signature(g);
    s = capture(g);
    if (s) return s;
    s = user_nodes_init(g);
    if (s) return s;
    g->verified = true;
    g->state = VX_GRAPH_STATE_VERIFIED;
    return VX_SUCCESS;
}

static uint64_t now_ns()
{
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
        std::chrono::high_resolution_clock::now().time_since_epoch()).count();
}

vx_status graph_process(Graph *g, bool wait)
{
    std::lock_guard<std::recursive_mutex> lk(g->lock);
    const uint64_t t0 = now_ns();
    if (!g->verified) { vx_status s = graph_verify(g); if (s) return s; }
    // by-value parameters or storage (delay ageing) changed since capture: switch to the
    // plan made for this signature before, else re-plan (valid rects and sizes stay put)
    if (param_signature(g) != g->param_signature) {
        vx_status s = propagate_valid_rects(g);
        if (s) return s;
        const uint64_t sig = param_signature(g);
        if (sig != g->param_signature) {
            constexpr size_t kCachedPlans = 3;
            PlanState &old = g->plan_cache[g->param_signature];
            plan_state_free(old);
            plan_state_swap(g, old);                    // the graph now holds no plan
            old.use = ++g->plan_uses;
            auto it = g->plan_cache.find(sig);
            if (it != g->plan_cache.end()) {
                plan_state_swap(g, it->second);
                g->plan_cache.erase(it);
            } else {
                s = plan_graph(g);
                if (!s) s = capture(g);
            }
            g->param_signature = sig;
            while (g->plan_cache.size() > kCachedPlans) {
                auto lru = g->plan_cache.begin();
                for (auto i = g->plan_cache.begin(); i != g->plan_cache.end(); ++i)
                    if (i->second.use < lru->second.use) lru = i;
                plan_state_free(lru->second);
                g->plan_cache.erase(lru);
            }
            if (s) return s;
        }
    }
    cudaSetDevice(g->ctx->device);
    for (Ref *r : g->inputs) {
        vx_status s = VX_SUCCESS;
        const bool streamed = std::find(g->streamed_in.begin(), g->streamed_in.end(), r) != g->streamed_in.end();
        if (streamed) {
            // the CUDA graph uploads the application's buffer: make sure that buffer is current
            Image *img = IMG(r);
            if (!img->host_valid && img->dev_valid) s = image_sync_to_host(img);
            if (s) return s;
            continue;
        }
        if (r->type == VX_TYPE_IMAGE) s = image_sync_to_device(IMG(r), g->stream);
        else if (r->type == VX_TYPE_ARRAY) {
            Array *a = static_cast<Array *>(r);
            auto it = std::find(g->staged_in.begin(), g->staged_in.end(), a);
            if (it != g->staged_in.end()) {
                // the CUDA graph uploads the host items unless the device copy is current
                g->io_slots_host[it - g->staged_in.begin()] =
                    a->dev_valid ? AGOCUDA_ARRAY_SKIP : (uint32_t)std::min(a->num_items, a->capacity);
                continue;
            }
            s = array_sync_to_device(a, g->stream);
        }
        else if (r->type == VX_TYPE_PYRAMID)
            for (Image *lv : static_cast<Pyramid *>(r)->level) if (!s) s = image_sync_to_device(lv, g->stream);
        if (s) return s;
    }
    g->state = VX_GRAPH_STATE_RUNNING;
    cudaEventRecord(g->ev0, g->stream);
    int rc = 0;
    if (g->cexec) {
        if (cudaGraphLaunch(g->cexec, g->stream) != cudaSuccess) rc = -1;
    } else {
        for (Step &s : g->steps) { rc = s.launch(g->stream); if (rc) break; }
    }
    cudaEventRecord(g->ev1, g->stream);
    for (Image *img : g->streamed_in) img->dev_valid = true;
    for (Array *a : g->staged_in) a->dev_valid = true;
    // outputs are now current on the device only (and in the application's buffer when
    // the CUDA graph downloads them)
    for (Ref *r : g->outputs) {
        if (r->type == VX_TYPE_IMAGE) {
            Image *root = IMG(r)->parent ? IMG(r)->parent : IMG(r);
            root->dev_valid = true;
            root->host_valid = std::find(g->streamed_out.begin(), g->streamed_out.end(), root) != g->streamed_out.end();
        } else if (r->type == VX_TYPE_ARRAY) {
            static_cast<Array *>(r)->dev_valid = true; static_cast<Array *>(r)->host_valid = false;
        } else if (r->type == VX_TYPE_SCALAR) {
            static_cast<Scalar *>(r)->dev_newer = true;
        } else if (r->type == VX_TYPE_DISTRIBUTION) {
            static_cast<Distribution *>(r)->dev_newer = true;
        } else if (r->type == VX_TYPE_PYRAMID) {
            for (Image *lv : static_cast<Pyramid *>(r)->level) { lv->dev_valid = true; lv->host_valid = false; }
        }
    }
    if (rc) {
        g->state = VX_GRAPH_STATE_ABANDONED;
        log_error(g, VX_FAILURE, "ERROR: vxProcessGraph: launch failed (%d)\n", rc);
        return VX_FAILURE;
    }
    g->scheduled = true;
    if (!wait) return VX_SUCCESS;
    vx_status st = graph_wait(g);
    const uint64_t t1 = now_ns();
    vx_perf_t &p = g->perf;
    p.tmp = t1 - t0; p.beg = t0; p.end = t1; p.sum += p.tmp; p.num++;
    p.avg = p.sum / p.num;
    p.min = p.num == 1 ? p.tmp : std::min(p.min, p.tmp);
    p.max = std::max(p.max, p.tmp);
    return st;
}

vx_status graph_wait(Graph *g)
{
    if (!g->scheduled) return VX_FAILURE;
    g->scheduled = false;
    cudaError_t e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) {
        g->state = VX_GRAPH_STATE_ABANDONED;
        log_error(g, VX_FAILURE, "ERROR: graph execution failed: %s\n", cudaGetErrorString(e));
        return VX_FAILURE;
    }
    cudaEventElapsedTime(&g->gpu_ms_last, g->ev0, g->ev1);
    g->gpu_ns_total += (double)g->gpu_ms_last * 1e6;
    g->gpu_runs++;
    // host-imported output images the CUDA graph did not download (pageable buffers, the
    // serial or uncaptured forms): copy them back, so the application's buffers are current
    for (Ref *r : g->outputs) {
        if (r->type != VX_TYPE_IMAGE) continue;
        Image *root = IMG(r)->parent ? IMG(r)->parent : IMG(r);
        if (root->import_type == VX_MEMORY_TYPE_HOST && !root->host_valid && image_sync_to_host(root)) {
            g->state = VX_GRAPH_STATE_ABANDONED;
            log_error(g, VX_FAILURE, "ERROR: graph output copy to the application's buffer failed\n");
            return VX_FAILURE;
        }
    }
    // arrays the CUDA graph downloaded: their host buffers and counts are current
    for (size_t i = 0; i < g->staged_out.size(); i++) {
        Array *a = g->staged_out[i];
        a->num_items = std::min((vx_size)g->io_slots_host[g->staged_in.size() + i], a->capacity);
        a->host_valid = true;
    }
    // kernels that detect a failure (bounded walks, candidate overflow) set status bits
    if (g->status_host && *(volatile uint32_t *)g->status_host) {
        const uint32_t st = *g->status_host;
        *g->status_host = 0;
        g->state = VX_GRAPH_STATE_ABANDONED;
        log_error(g, VX_FAILURE, "ERROR: graph execution reported device status 0x%x\n", st);
        return VX_FAILURE;
    }
    g->state = VX_GRAPH_STATE_COMPLETED;
    // vxRegisterAutoAging: age after every completed execution
    for (Delay *d : g->auto_age) delay_age(d);
    return VX_SUCCESS;
}

}  // namespace agovx

// ====================================================================================
// Public API
// ====================================================================================
template <class T> static T *as(void *h) { return static_cast<T *>(static_cast<Ref *>(h)); }
#define CHECK_REF(h, T) if (!is_valid(h, T)) return VX_ERROR_INVALID_REFERENCE

namespace agovx {
Node *graph_add_node(Graph *g, vx_enum kernel, const std::vector<Ref *> &params)
{
    Node *n = new Node();
    n->type = VX_TYPE_NODE;
    n->scope = g;
    n->kernel = kernel;
    n->params = params;
    for (Ref *r : n->params) retain_internal(r);
    add_ref(g->ctx, n);
    g->nodes.push_back(n);
    graph_invalidate(g);
    return n;
}
}  // namespace agovx

extern "C" {

vx_graph vxCreateGraph(vx_context context)
{
    if (!is_valid(context, VX_TYPE_CONTEXT)) return nullptr;
    Graph *g = new Graph();
    g->type = VX_TYPE_GRAPH;
    add_ref(as<Context>(context), g);
    if (const char *f = getenv("AGO_B200_OPTIMIZER_FLAGS")) g->optimizer_flags = (uint32_t)strtoul(f, nullptr, 0);
    return (vx_graph)g;
}

vx_status vxReleaseGraph(vx_graph *graph)
{
    if (!graph || !is_valid(*graph, VX_TYPE_GRAPH)) return VX_ERROR_INVALID_REFERENCE;
    Graph *g = as<Graph>(*graph);
    if (g->scheduled) graph_wait(g);
    *graph = nullptr;
    g->ext_count = 0;
    g->released = true;
    if (g->int_count == 0) destroy_ref(g);   // its nodes, plans and lowered data go with it
    return VX_SUCCESS;
}

vx_status vxVerifyGraph(vx_graph graph)
{
    CHECK_REF(graph, VX_TYPE_GRAPH);
    return graph_verify(as<Graph>(graph));
}

vx_status vxProcessGraph(vx_graph graph)
{
    CHECK_REF(graph, VX_TYPE_GRAPH);
    return graph_process(as<Graph>(graph), true);
}

vx_status vxScheduleGraph(vx_graph graph)
{
    CHECK_REF(graph, VX_TYPE_GRAPH);
    Graph *g = as<Graph>(graph);
    if (g->scheduled) return VX_ERROR_GRAPH_SCHEDULED;
    return graph_process(g, false);
}

vx_status vxWaitGraph(vx_graph graph)
{
    CHECK_REF(graph, VX_TYPE_GRAPH);
    return graph_wait(as<Graph>(graph));
}

vx_status vxQueryGraph(vx_graph graph, vx_enum attribute, void *ptr, vx_size size)
{
    CHECK_REF(graph, VX_TYPE_GRAPH);
    Graph *g = as<Graph>(graph);
    switch (attribute) {
    case VX_GRAPH_NUMNODES: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint32 *)ptr = (vx_uint32)g->nodes.size(); return VX_SUCCESS;
    case VX_GRAPH_PERFORMANCE: if (size != sizeof(vx_perf_t)) return VX_ERROR_INVALID_PARAMETERS; *(vx_perf_t *)ptr = g->perf; return VX_SUCCESS;
    case VX_GRAPH_NUMPARAMETERS: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint32 *)ptr = 0; return VX_SUCCESS;
    case VX_GRAPH_STATE: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_enum *)ptr = g->state; return VX_SUCCESS;
    case VX_GRAPH_ATTRIBUTE_AMD_OPTIMIZER_FLAGS: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint32 *)ptr = g->optimizer_flags; return VX_SUCCESS;
    case VX_GRAPH_ATTRIBUTE_AMD_AFFINITY:
        if (size != sizeof(AgoTargetAffinityInfo)) return VX_ERROR_INVALID_PARAMETERS;
        memset(ptr, 0, size); ((AgoTargetAffinityInfo *)ptr)->device_type = AGO_TARGET_AFFINITY_GPU; return VX_SUCCESS;
    case VX_GRAPH_ATTRIBUTE_AMD_PERFORMANCE_INTERNAL_LAST: case VX_GRAPH_ATTRIBUTE_AMD_PERFORMANCE_INTERNAL_AVG: {
        // vx_api.cpp:3106: AgoGraphPerfInternalInfo in nanoseconds; kernel_wait is the device
        // time of the launch (CUDA events around the captured graph), last or averaged; the
        // host<->device copies happen inside that launch, so the buffer times stay 0
        if (size != sizeof(AgoGraphPerfInternalInfo) || !ptr) return VX_ERROR_INVALID_PARAMETERS;
        AgoGraphPerfInternalInfo p{};
        if (attribute == VX_GRAPH_ATTRIBUTE_AMD_PERFORMANCE_INTERNAL_LAST) p.kernel_wait = (vx_uint64)(g->gpu_ms_last * 1e6);
        else if (g->gpu_runs) p.kernel_wait = (vx_uint64)(g->gpu_ns_total / (double)g->gpu_runs);
        *(AgoGraphPerfInternalInfo *)ptr = p; return VX_SUCCESS;
    }
    case VX_GRAPH_ATTRIBUTE_AMD_PERFORMANCE_INTERNAL_PROFILE: {
        // ago_interface.cpp:2740 layout: a header and one line per timed object; the nodes of
        // this target run inside one captured CUDA graph, so the lines are the graph's host
        // time (vxProcessGraph) and its device time (CUDA events around the launch)
        const char *file = (const char *)ptr;
        FILE *fp = (!file || !strcmp(file, "stdout")) ? stdout : fopen(file, "w");
        if (!fp) return VX_FAILURE;
        fprintf(fp, " COUNT,tmp(ms),avg(ms),min(ms),max(ms),DEV,KERNEL\n");
        if (g->perf.num > 0)
            fprintf(fp, "%6d,%7.3f,%7.3f,%7.3f,%7.3f,GPU,GRAPH\n", (int)g->perf.num, g->perf.tmp * 1e-6, g->perf.avg * 1e-6,
                    g->perf.min * 1e-6, g->perf.max * 1e-6);
        if (g->gpu_runs > 0)
            fprintf(fp, "%6d,%7.3f,%7.3f,      -,      -,GPU,GRAPH(device)\n", (int)g->gpu_runs, (double)g->gpu_ms_last,
                    g->gpu_ns_total * 1e-6 / (double)g->gpu_runs);
        fflush(fp);
        if (fp != stdout) fclose(fp);
        return VX_SUCCESS;
    }
    case VX_GRAPH_ATTRIBUTE_AMD_EXPORT_TO_TEXT: {
        // the verified plan as text: one line per step ("kernel nodes...")
        if (!ptr || size == 0) return VX_ERROR_INVALID_PARAMETERS;
        snprintf((char *)ptr, size, "%s", g->plan_text.c_str());
        return VX_SUCCESS;
    }
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxSetGraphAttribute(vx_graph graph, vx_enum attribute, const void *ptr, vx_size size)
{
    CHECK_REF(graph, VX_TYPE_GRAPH);
    Graph *g = as<Graph>(graph);
    switch (attribute) {
    case VX_GRAPH_ATTRIBUTE_AMD_OPTIMIZER_FLAGS:
        if (size != 4) return VX_ERROR_INVALID_PARAMETERS;
        g->optimizer_flags = *(const vx_uint32 *)ptr; graph_invalidate(g); return VX_SUCCESS;
    case VX_GRAPH_ATTRIBUTE_AMD_AFFINITY:
        if (size != sizeof(AgoTargetAffinityInfo)) return VX_ERROR_INVALID_PARAMETERS;
        g->affinity = ((const AgoTargetAffinityInfo *)ptr)->device_type;
        return VX_SUCCESS;   // every node runs on the GPU target; CPU affinity is accepted and ignored
    case VX_GRAPH_ATTRIBUTE_AMD_IMPORT_FROM_TEXT: {     // vx_api.cpp:3183
        if (size != sizeof(AgoGraphImportInfo) || !ptr) return VX_ERROR_INVALID_PARAMETERS;
        std::lock_guard<std::recursive_mutex> lk(g->lock);
        vx_status s = graph_import_text(g, (const AgoGraphImportInfo *)ptr);
        graph_invalidate(g);
        return s ? VX_FAILURE : VX_SUCCESS;
    }
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_bool vxIsGraphVerified(vx_graph graph)
{
    return is_valid(graph, VX_TYPE_GRAPH) && as<Graph>(graph)->verified ? vx_true_e : vx_false_e;
}

vx_status vxQueryNode(vx_node node, vx_enum attribute, void *ptr, vx_size size)
{
    CHECK_REF(node, VX_TYPE_NODE);
    Node *n = as<Node>(node);
    switch (attribute) {
    case VX_NODE_STATUS: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_status *)ptr = n->status; return VX_SUCCESS;
    case VX_NODE_PERFORMANCE: if (size != sizeof(vx_perf_t)) return VX_ERROR_INVALID_PARAMETERS; *(vx_perf_t *)ptr = n->perf; return VX_SUCCESS;
    case VX_NODE_BORDER: if (size != sizeof(vx_border_t)) return VX_ERROR_INVALID_PARAMETERS; *(vx_border_t *)ptr = n->border; return VX_SUCCESS;
    case VX_NODE_PARAMETERS: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint32 *)ptr = (vx_uint32)n->params.size(); return VX_SUCCESS;
    case VX_NODE_LOCAL_DATA_SIZE: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = n->local_size; return VX_SUCCESS;
    case VX_NODE_LOCAL_DATA_PTR: if (size != sizeof(void *)) return VX_ERROR_INVALID_PARAMETERS; *(void **)ptr = n->local_ptr; return VX_SUCCESS;
    case VX_NODE_ATTRIBUTE_AMD_AFFINITY:
        if (size != sizeof(AgoTargetAffinityInfo)) return VX_ERROR_INVALID_PARAMETERS;
        memset(ptr, 0, size); ((AgoTargetAffinityInfo *)ptr)->device_type = AGO_TARGET_AFFINITY_GPU; return VX_SUCCESS;
    case VX_NODE_ATTRIBUTE_AMD_HIP_STREAM: {
        // the CUDA stream the node's graph launches on (cudaStream_t)
        if (size != sizeof(void *)) return VX_ERROR_INVALID_PARAMETERS;
        Graph *g = n->scope;
        *(void **)ptr = g ? (void *)g->stream : nullptr; return VX_SUCCESS;
    }
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxSetNodeAttribute(vx_node node, vx_enum attribute, const void *ptr, vx_size size)
{
    CHECK_REF(node, VX_TYPE_NODE);
    Node *n = as<Node>(node);
    switch (attribute) {
    case VX_NODE_BORDER:
        if (size != sizeof(vx_border_t)) return VX_ERROR_INVALID_PARAMETERS;
        n->border = *(const vx_border_t *)ptr;
        if (n->scope) graph_invalidate(n->scope);
        return VX_SUCCESS;
    case VX_NODE_ATTRIBUTE_AMD_AFFINITY:
        if (size != sizeof(AgoTargetAffinityInfo)) return VX_ERROR_INVALID_PARAMETERS;
        n->affinity = ((const AgoTargetAffinityInfo *)ptr)->device_type;
        return VX_SUCCESS;
    // user-kernel node local data, settable when the kernel declares no local data size
    // (vx_types.h VX_NODE_LOCAL_DATA_SIZE / _PTR)
    case VX_NODE_LOCAL_DATA_SIZE:
        if (size != sizeof(vx_size) || !n->ukernel || n->ukernel->local_size) return VX_ERROR_NOT_SUPPORTED;
        n->local_size = *(const vx_size *)ptr;
        return VX_SUCCESS;
    case VX_NODE_LOCAL_DATA_PTR:
        if (size != sizeof(void *) || !n->ukernel || n->ukernel->local_size) return VX_ERROR_NOT_SUPPORTED;
        if (n->local_owned) { free(n->local_ptr); n->local_owned = false; }
        n->local_ptr = *(void *const *)ptr;
        return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxReleaseNode(vx_node *node)
{
    if (!node || !is_valid(*node, VX_TYPE_NODE)) return VX_ERROR_INVALID_REFERENCE;
    as<Node>(*node)->ext_count = 0;
    as<Node>(*node)->released = true;
    as<Node>(*node)->int_count = 1;     // the graph keeps it
    *node = nullptr;
    return VX_SUCCESS;
}

vx_status vxRemoveNode(vx_node *node)
{
    if (!node || !is_valid(*node, VX_TYPE_NODE)) return VX_ERROR_INVALID_REFERENCE;
    Node *n = as<Node>(*node);
    n->removed = true;
    if (n->scope) graph_invalidate(n->scope);
    *node = nullptr;
    return VX_SUCCESS;
}

vx_status vxSetNodeTarget(vx_node node, vx_enum target_enum, const char *target_string)
{
    CHECK_REF(node, VX_TYPE_NODE);
    if (target_enum == VX_TARGET_ANY) return VX_SUCCESS;
    if (target_enum == VX_TARGET_STRING && target_string) {
        std::string t(target_string);
        for (auto &c : t) c = (char)toupper(c);
        if (t == "GPU" || t == "ANY" || t == "CUDA") return VX_SUCCESS;
        return VX_ERROR_NOT_SUPPORTED;   // no CPU target on this implementation
    }
    return VX_ERROR_NOT_SUPPORTED;
}

// ---------------------------------------------------------------- node factories
static vx_node make_node(vx_graph graph, vx_enum kernel, std::initializer_list<Ref *> params)
{
    if (!is_valid(graph, VX_TYPE_GRAPH)) return nullptr;
    Graph *g = as<Graph>(graph);
    Node *n = new Node();
    n->type = VX_TYPE_NODE;
    n->scope = g;
    n->kernel = kernel;
    n->params.assign(params.begin(), params.end());
    for (Ref *r : n->params) retain_internal(r);
    add_ref(g->ctx, n);
    g->nodes.push_back(n);
    graph_invalidate(g);
    return (vx_node)n;
}


static Ref *scalar_of(vx_graph graph, vx_enum type, const void *v)
{
    if (!is_valid(graph, VX_TYPE_GRAPH)) return nullptr;
    Scalar *s = make_scalar(as<Graph>(graph)->ctx, as<Graph>(graph), type, v);
    s->ext_count = 0;
    s->int_count = 1;
    return s;
}

#define R(x) static_cast<Ref *>(static_cast<void *>(x))

vx_node vxColorConvertNode(vx_graph graph, vx_image input, vx_image output)
{ return make_node(graph, VX_KERNEL_COLOR_CONVERT, {R(input), R(output)}); }

vx_node vxChannelExtractNode(vx_graph graph, vx_image input, vx_enum channel, vx_image output)
{ return make_node(graph, VX_KERNEL_CHANNEL_EXTRACT, {R(input), scalar_of(graph, VX_TYPE_ENUM, &channel), R(output)}); }

vx_node vxSobel3x3Node(vx_graph graph, vx_image input, vx_image output_x, vx_image output_y)
{ return make_node(graph, VX_KERNEL_SOBEL_3x3, {R(input), R(output_x), R(output_y)}); }

vx_node vxMagnitudeNode(vx_graph graph, vx_image grad_x, vx_image grad_y, vx_image mag)
{ return make_node(graph, VX_KERNEL_MAGNITUDE, {R(grad_x), R(grad_y), R(mag)}); }

vx_node vxScaleImageNode(vx_graph graph, vx_image src, vx_image dst, vx_enum type)
{ return make_node(graph, VX_KERNEL_SCALE_IMAGE, {R(src), R(dst), scalar_of(graph, VX_TYPE_ENUM, &type)}); }

vx_node vxThresholdNode(vx_graph graph, vx_image input, vx_threshold thresh, vx_image output)
{ return make_node(graph, VX_KERNEL_THRESHOLD, {R(input), R(thresh), R(output)}); }

vx_node vxGaussian3x3Node(vx_graph graph, vx_image input, vx_image output)
{ return make_node(graph, VX_KERNEL_GAUSSIAN_3x3, {R(input), R(output)}); }

vx_node vxGaussianPyramidNode(vx_graph graph, vx_image input, vx_pyramid gaussian)
{ return make_node(graph, VX_KERNEL_GAUSSIAN_PYRAMID, {R(input), R(gaussian)}); }

vx_node vxConvertDepthNode(vx_graph graph, vx_image input, vx_image output, vx_enum policy, vx_scalar shift)
{ return make_node(graph, VX_KERNEL_CONVERTDEPTH, {R(input), R(output), scalar_of(graph, VX_TYPE_ENUM, &policy), R(shift)}); }

vx_node vxCannyEdgeDetectorNode(vx_graph graph, vx_image input, vx_threshold hyst, vx_int32 gradient_size,
                                vx_enum norm_type, vx_image output)
{
    return make_node(graph, VX_KERNEL_CANNY_EDGE_DETECTOR,
                     {R(input), R(hyst), scalar_of(graph, VX_TYPE_INT32, &gradient_size), scalar_of(graph, VX_TYPE_ENUM, &norm_type), R(output)});
}

vx_node vxWarpAffineNode(vx_graph graph, vx_image input, vx_matrix matrix, vx_enum type, vx_image output)
{ return make_node(graph, VX_KERNEL_WARP_AFFINE, {R(input), R(matrix), scalar_of(graph, VX_TYPE_ENUM, &type), R(output)}); }

vx_node vxWarpPerspectiveNode(vx_graph graph, vx_image input, vx_matrix matrix, vx_enum type, vx_image output)
{ return make_node(graph, VX_KERNEL_WARP_PERSPECTIVE, {R(input), R(matrix), scalar_of(graph, VX_TYPE_ENUM, &type), R(output)}); }

vx_node vxHarrisCornersNode(vx_graph graph, vx_image input, vx_scalar strength_thresh, vx_scalar min_distance,
                            vx_scalar sensitivity, vx_int32 gradient_size, vx_int32 block_size, vx_array corners,
                            vx_scalar num_corners)
{
    return make_node(graph, VX_KERNEL_HARRIS_CORNERS,
                     {R(input), R(strength_thresh), R(min_distance), R(sensitivity), scalar_of(graph, VX_TYPE_INT32, &gradient_size),
                      scalar_of(graph, VX_TYPE_INT32, &block_size), R(corners), R(num_corners)});
}

vx_node vxFastCornersNode(vx_graph graph, vx_image input, vx_scalar strength_thresh, vx_bool nonmax_suppression,
                          vx_array corners, vx_scalar num_corners)
{
    return make_node(graph, VX_KERNEL_FAST_CORNERS,
                     {R(input), R(strength_thresh), scalar_of(graph, VX_TYPE_BOOL, &nonmax_suppression), R(corners), R(num_corners)});
}

vx_node vxOpticalFlowPyrLKNode(vx_graph graph, vx_pyramid old_images, vx_pyramid new_images, vx_array old_points,
                               vx_array new_points_estimates, vx_array new_points, vx_enum termination, vx_scalar epsilon,
                               vx_scalar num_iterations, vx_scalar use_initial_estimate, vx_size window_dimension)
{
    return make_node(graph, VX_KERNEL_OPTICAL_FLOW_PYR_LK,
                     {R(old_images), R(new_images), R(old_points), R(new_points_estimates), R(new_points),
                      scalar_of(graph, VX_TYPE_ENUM, &termination), R(epsilon), R(num_iterations), R(use_initial_estimate),
                      scalar_of(graph, VX_TYPE_SIZE, &window_dimension)});
}

vx_node vxRemapNode(vx_graph graph, vx_image input, vx_remap table, vx_enum policy, vx_image output)
{ return make_node(graph, VX_KERNEL_REMAP, {R(input), R(table), scalar_of(graph, VX_TYPE_ENUM, &policy), R(output)}); }

vx_node vxHalfScaleGaussianNode(vx_graph graph, vx_image input, vx_image output, vx_int32 kernel_size)
{ return make_node(graph, VX_KERNEL_HALFSCALE_GAUSSIAN, {R(input), R(output), scalar_of(graph, VX_TYPE_INT32, &kernel_size)}); }

vx_node vxBox3x3Node(vx_graph graph, vx_image input, vx_image output)
{ return make_node(graph, VX_KERNEL_BOX_3x3, {R(input), R(output)}); }

vx_node vxMedian3x3Node(vx_graph graph, vx_image input, vx_image output)
{ return make_node(graph, VX_KERNEL_MEDIAN_3x3, {R(input), R(output)}); }

vx_node vxDilate3x3Node(vx_graph graph, vx_image input, vx_image output)
{ return make_node(graph, VX_KERNEL_DILATE_3x3, {R(input), R(output)}); }

vx_node vxErode3x3Node(vx_graph graph, vx_image input, vx_image output)
{ return make_node(graph, VX_KERNEL_ERODE_3x3, {R(input), R(output)}); }

vx_node vxAbsDiffNode(vx_graph graph, vx_image in1, vx_image in2, vx_image out)
{ return make_node(graph, VX_KERNEL_ABSDIFF, {R(in1), R(in2), R(out)}); }

vx_node vxAddNode(vx_graph graph, vx_image in1, vx_image in2, vx_enum policy, vx_image out)
{ return make_node(graph, VX_KERNEL_ADD, {R(in1), R(in2), scalar_of(graph, VX_TYPE_ENUM, &policy), R(out)}); }

vx_node vxSubtractNode(vx_graph graph, vx_image in1, vx_image in2, vx_enum policy, vx_image out)
{ return make_node(graph, VX_KERNEL_SUBTRACT, {R(in1), R(in2), scalar_of(graph, VX_TYPE_ENUM, &policy), R(out)}); }

vx_node vxAndNode(vx_graph graph, vx_image in1, vx_image in2, vx_image out)
{ return make_node(graph, VX_KERNEL_AND, {R(in1), R(in2), R(out)}); }

vx_node vxOrNode(vx_graph graph, vx_image in1, vx_image in2, vx_image out)
{ return make_node(graph, VX_KERNEL_OR, {R(in1), R(in2), R(out)}); }

vx_node vxXorNode(vx_graph graph, vx_image in1, vx_image in2, vx_image out)
{ return make_node(graph, VX_KERNEL_XOR, {R(in1), R(in2), R(out)}); }

vx_node vxNotNode(vx_graph graph, vx_image input, vx_image output)
{ return make_node(graph, VX_KERNEL_NOT, {R(input), R(output)}); }

vx_node vxTableLookupNode(vx_graph graph, vx_image input, vx_lut lut, vx_image output)
{ return make_node(graph, VX_KERNEL_TABLE_LOOKUP, {R(input), R(lut), R(output)}); }

vx_node vxIntegralImageNode(vx_graph graph, vx_image input, vx_image output)
{ return make_node(graph, VX_KERNEL_INTEGRAL_IMAGE, {R(input), R(output)}); }

vx_node vxHistogramNode(vx_graph graph, vx_image input, vx_distribution distribution)
{ return make_node(graph, VX_KERNEL_HISTOGRAM, {R(input), R(distribution)}); }

vx_node vxChannelCombineNode(vx_graph graph, vx_image plane0, vx_image plane1, vx_image plane2, vx_image plane3,
                             vx_image output)
{ return make_node(graph, VX_KERNEL_CHANNEL_COMBINE, {R(plane0), R(plane1), R(plane2), R(plane3), R(output)}); }

vx_node vxConvolveNode(vx_graph graph, vx_image input, vx_convolution conv, vx_image output)
{ return make_node(graph, VX_KERNEL_CUSTOM_CONVOLUTION, {R(input), R(conv), R(output)}); }

}  // extern "C"
