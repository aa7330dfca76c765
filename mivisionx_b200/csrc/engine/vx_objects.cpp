// vx_objects.cpp -- OpenVX context and data objects (images, scalars, thresholds,
// matrices, arrays, pyramids, remaps) of the B200 engine.  Public semantics follow the
// reference API layer (amd_openvx/openvx/api/vx_api.cpp); storage is device-first.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>

#include "vx_internal.h"

using namespace agovx;

namespace agovx {

uint32_t align_up(uint32_t v, uint32_t a) { return (v + a - 1) / a * a; }

bool is_valid(const void *r, vx_enum type)
{
    if (!is_ref(r)) return false;
    const Ref *x = static_cast<const Ref *>(r);
    return (type == VX_TYPE_REFERENCE || x->type == type) && !(x->released && x->int_count == 0);
}

void log_error(Ref *ref, vx_status st, const char *fmt, ...)
{
    char buf[VX_MAX_LOG_MESSAGE_LEN];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    Context *ctx = ref ? (ref->type == VX_TYPE_CONTEXT ? static_cast<Context *>(ref) : ref->ctx) : nullptr;
    if (ctx && ctx->log_cb) {
        std::unique_lock<std::mutex> lk(ctx->log_mutex, std::defer_lock);
        if (!ctx->log_reentrant) lk.lock();
        ctx->log_cb((vx_context)ctx, (vx_reference)ref, st, buf);
    } else if (getenv("AGO_B200_VERBOSE")) {
        fprintf(stderr, "%s", buf);
    }
}

vx_size type_size(vx_enum t)
{
    switch (t) {
    case VX_TYPE_CHAR: case VX_TYPE_INT8: case VX_TYPE_UINT8: return 1;
    case VX_TYPE_INT16: case VX_TYPE_UINT16: return 2;
    case VX_TYPE_INT32: case VX_TYPE_UINT32: case VX_TYPE_FLOAT32: case VX_TYPE_ENUM: case VX_TYPE_DF_IMAGE:
    case VX_TYPE_BOOL: return 4;
    case VX_TYPE_INT64: case VX_TYPE_UINT64: case VX_TYPE_FLOAT64: case VX_TYPE_SIZE: return 8;
    case VX_TYPE_RECTANGLE: return sizeof(vx_rectangle_t);
    case VX_TYPE_KEYPOINT: return sizeof(vx_keypoint_t);
    case VX_TYPE_COORDINATES2D: return sizeof(vx_coordinates2d_t);
    case VX_TYPE_COORDINATES3D: return 12;
    case VX_TYPE_COORDINATES2DF: return sizeof(vx_coordinates2df_t);
    default: return 0;
    }
}

// Plane geometry of each supported format (ago/ago_util.cpp agoGetImageComponentsAndPlanes).
int format_planes(vx_df_image f, uint32_t w, uint32_t h, Plane *pl)
{
    auto set = [&](int i, uint32_t pw, uint32_t ph, uint32_t bpp) {
        pl[i].width = pw; pl[i].height = ph; pl[i].bpp = bpp;
    };
    const uint32_t w2 = (w + 1) >> 1, h2 = (h + 1) >> 1;
    switch (f) {
    case VX_DF_IMAGE_U8: set(0, w, h, 1); return 1;
    case VX_DF_IMAGE_U16: case VX_DF_IMAGE_S16: set(0, w, h, 2); return 1;
    case VX_DF_IMAGE_U32: case VX_DF_IMAGE_S32: case VX_DF_IMAGE_F32_AMD: set(0, w, h, 4); return 1;
    case VX_DF_IMAGE('F', '3', '3', '2'): set(0, w, h, 12); return 1;   // AMD F32x3 (Harris HG3)
    case VX_DF_IMAGE_RGB: set(0, w, h, 3); return 1;
    case VX_DF_IMAGE_RGBX: set(0, w, h, 4); return 1;
    case VX_DF_IMAGE_UYVY: case VX_DF_IMAGE_YUYV: set(0, w, h, 2); return 1;
    case VX_DF_IMAGE_NV12: case VX_DF_IMAGE_NV21: set(0, w, h, 1); set(1, w2, h2, 2); return 2;
    case VX_DF_IMAGE_IYUV: set(0, w, h, 1); set(1, w2, h2, 1); set(2, w2, h2, 1); return 3;
    case VX_DF_IMAGE_YUV4: set(0, w, h, 1); set(1, w, h, 1); set(2, w, h, 1); return 3;
    default: return 0;
    }
}

void add_ref(Context *ctx, Ref *r)
{
    r->ctx = ctx;
    if (ctx) ctx->refs.push_back(r);
}

// Lifetime: an object dies when its last application reference and its last internal one
// (a node parameter, a multi-plane parent, a pyramid, a delay, a graph's lowering) are both
// gone, and its host and device storage go with it -- agoReleaseData (ago/ago_util.cpp:2771)
// frees AGO's objects the same way.
void retain_internal(Ref *r) { if (r) r->int_count++; }

void release_internal(Ref *r)
{
    if (!r || r->int_count <= 0) return;
    if (--r->int_count == 0 && r->ext_count == 0) destroy_ref(r);
}

void graph_own(Graph *g, Ref *r)
{
    retain_internal(r);
    g->owned_virtual.push_back(r);
}

void graph_release_owned(Graph *g)
{
    std::vector<Ref *> owned;
    owned.swap(g->owned_virtual);
    for (Ref *r : owned) release_internal(r);
}

static void graph_destroy_contents(Graph *g)
{
    if (g->scheduled) graph_wait(g);
    if (g->stream) cudaStreamSynchronize(g->stream);
    user_nodes_deinit(g);
    graph_invalidate(g);
    g->lnodes.clear();
    g->replaced.clear();
    // nodes belong to their graph: they go with it even if the application kept a handle
    std::vector<Node *> nodes;
    nodes.swap(g->nodes);
    for (Node *n : nodes) destroy_ref(n);
    graph_release_owned(g);
    std::vector<Delay *> aged;
    aged.swap(g->auto_age);
    for (Delay *d : aged) release_internal(d);
    // virtual data the application still holds outlives its graph's scope
    for (Ref *r : g->ctx->refs) if (r->scope == g) r->scope = nullptr;
}

void destroy_ref(Ref *r)
{
    if (!is_ref(r) || r->type == VX_TYPE_CONTEXT) return;
    Context *c = r->ctx;
    if (c && c->tearing_down) return;
    r->magic = 0;
    if (c) {
        auto it = std::find(c->refs.begin(), c->refs.end(), r);
        if (it != c->refs.end()) c->refs.erase(it);
    }
    switch (r->type) {
    case VX_TYPE_GRAPH: graph_destroy_contents(static_cast<Graph *>(r)); break;
    case VX_TYPE_NODE: {
        std::vector<Ref *> params;
        params.swap(static_cast<Node *>(r)->params);
        for (Ref *p : params) release_internal(p);
        break;
    }
    case VX_TYPE_IMAGE: {
        Image *img = static_cast<Image *>(r);
        // plane images share the parent's storage: they cannot outlive it
        std::vector<Image *> children;
        children.swap(img->children);
        for (Image *ch : children) { ch->parent = nullptr; ch->ext_count = ch->int_count = 0; destroy_ref(ch); }
        if (img->roi_view && img->parent) {
            auto &v = img->parent->views;
            v.erase(std::remove(v.begin(), v.end(), img), v.end());
        }
        if (img->view_of) { Image *p = img->view_of; img->view_of = nullptr; release_internal(p); }
        break;
    }
    case VX_TYPE_PYRAMID: {
        std::vector<Image *> levels;
        levels.swap(static_cast<Pyramid *>(r)->level);
        for (Image *lv : levels) release_internal(lv);
        break;
    }
    case VX_TYPE_DELAY: {
        std::vector<Ref *> slots;
        slots.swap(static_cast<Delay *>(r)->slots);
        for (Ref *sl : slots) release_internal(sl);
        break;
    }
    default: break;
    }
    delete r;
}

// ---------------------------------------------------------------- images
Image::~Image()
{
    for (int i = 0; i < num_planes; i++) {
        if (planes[i].dev_owned && planes[i].dev) cudaFree(planes[i].dev);
        if (planes[i].host_owned && planes[i].host) cudaFreeHost(planes[i].host);
    }
}

// Planes of multi-plane images are also addressable as single-plane images (AGO's
// "children", ago/ago_util.cpp:1095): lowered kernels read/write them directly.
void image_init_planes(Image *img)
{
    const uint32_t w = img->width, h = img->height;
    const vx_df_image fmt = img->format;
    img->num_planes = (fmt == VX_DF_IMAGE_VIRT || !w || !h) ? 0 : format_planes(fmt, w, h, img->planes);
    if (img->num_planes > 1 && img->children.empty()) {
        for (int i = 0; i < img->num_planes; i++) {
            const Plane &p = img->planes[i];
            Image *c = new Image();
            c->type = VX_TYPE_IMAGE;
            c->scope = img->scope;
            c->is_virtual = img->is_virtual;
            c->width = p.width; c->height = p.height;
            c->format = p.bpp == 1 ? VX_DF_IMAGE_U8 : VX_DF_IMAGE_U16;
            c->num_planes = 1;
            c->planes[0] = p;
            c->valid = vx_rectangle_t{0, 0, p.width, p.height};
            c->parent = img;
            c->ext_count = 0;
            c->int_count = 1;
            add_ref(img->ctx, c);
            img->children.push_back(c);
        }
    }
}

Image *make_image(Context *ctx, Graph *scope, uint32_t w, uint32_t h, vx_df_image fmt, bool virt)
{
    Image *img = new Image();
    img->type = VX_TYPE_IMAGE;
    img->scope = scope;
    img->is_virtual = virt;
    img->width = w; img->height = h; img->format = fmt;
    img->valid = vx_rectangle_t{0, 0, w, h};
    add_ref(ctx, img);
    image_init_planes(img);
    return img;
}

// Plane images (AGO children) alias the parent's planes; ROI views alias a window of plane 0.
// Called whenever the parent's storage moves (allocation, host mirror, handle swap, ageing).
void image_refresh_views(Image *root)
{
    for (size_t c = 0; c < root->children.size(); c++) {
        Plane &cp = root->children[c]->planes[0];
        const Plane &p = root->planes[c];
        cp.dev = p.dev; cp.dev_stride = p.dev_stride;
        cp.host = p.host; cp.host_stride = p.host_stride;
        cp.dev_owned = cp.host_owned = false;
    }
    const Plane &p = root->planes[0];
    for (Image *v : root->views) {
        Plane &vp = v->planes[0];
        const size_t off_dev = (size_t)v->view_y * p.dev_stride + (size_t)v->view_x * p.bpp;
        const size_t off_host = (size_t)v->view_y * p.host_stride + (size_t)v->view_x * p.bpp;
        vp.bpp = p.bpp;
        vp.dev = p.dev ? p.dev + off_dev : nullptr; vp.dev_stride = p.dev_stride;
        vp.host = p.host ? p.host + off_host : nullptr; vp.host_stride = p.host_stride;
        vp.dev_owned = vp.host_owned = false;
    }
}

// every CUDA call is made on the context's device (VX_CONTEXT_ATTRIBUTE_AMD_HIP_DEVICE)
static void use_device(Ref *r)
{
    if (r && r->ctx) cudaSetDevice(r->ctx->device);
}

vx_status image_alloc_device(Image *img)
{
    use_device(img);
    if (img->parent) return image_alloc_device(img->parent);
    if (!img->num_planes) return VX_ERROR_INVALID_FORMAT;
    for (int i = 0; i < img->num_planes; i++) {
        Plane &p = img->planes[i];
        if (p.dev) continue;
        p.dev_stride = align_up(p.width * p.bpp, 64);
        void *d = nullptr;
        if (cudaMalloc(&d, p.dev_bytes() + 256) != cudaSuccess) {
            log_error(img, VX_ERROR_NO_MEMORY, "ERROR: device allocation of %zu bytes failed\n", p.dev_bytes());
            return VX_ERROR_NO_MEMORY;
        }
        cudaMemset(d, 0, p.dev_bytes() + 256);
        p.dev = (uint8_t *)d;
        p.dev_owned = true;
        if (!p.host_stride) p.host_stride = p.dev_stride;
    }
    image_refresh_views(img);
    if (img->uniform || (!img->dev_valid && !img->host_valid)) {
        // uniform images and fresh images: materialise on the host and upload
        if (img->uniform) {
            for (int i = 0; i < img->num_planes; i++) {
                Plane &p = img->planes[i];
                std::vector<uint8_t> row(p.dev_stride, 0);
                for (uint32_t x = 0; x < p.width; x++) {
                    for (uint32_t b = 0; b < p.bpp; b++) {
                        uint8_t v;
                        if (img->format == VX_DF_IMAGE_U8) v = img->uniform_value.U8;
                        else if (p.bpp <= 4 && img->num_planes == 1) v = img->uniform_value.reserved[b];
                        else v = img->uniform_value.YUV[i];
                        row[x * p.bpp + b] = v;
                    }
                }
                for (uint32_t y = 0; y < p.height; y++)
                    cudaMemcpy(p.dev + (size_t)y * p.dev_stride, row.data(), p.dev_stride, cudaMemcpyHostToDevice);
            }
        }
        img->dev_valid = true;
    }
    return VX_SUCCESS;
}

static vx_status ensure_host(Image *img)
{
    Image *root = img->parent ? img->parent : img;
    for (int i = 0; i < root->num_planes; i++) {
        Plane &p = root->planes[i];
        if (p.host) continue;
        if (!p.host_stride) p.host_stride = p.dev_stride ? p.dev_stride : align_up(p.width * p.bpp, 64);
        void *h = nullptr;
        if (cudaMallocHost(&h, p.host_bytes() + 64) != cudaSuccess) return VX_ERROR_NO_MEMORY;
        memset(h, 0, p.host_bytes() + 64);
        p.host = (uint8_t *)h;
        p.host_owned = true;
    }
    image_refresh_views(root);
    return VX_SUCCESS;
}

vx_status image_sync_to_device(Image *img, cudaStream_t s)
{
    use_device(img);
    Image *root = img->parent ? img->parent : img;
    vx_status st = image_alloc_device(root);
    if (st) return st;
    if (root->dev_valid && root->import_type != VX_MEMORY_TYPE_HOST) return VX_SUCCESS;
    if (!root->host_valid) { root->dev_valid = true; return VX_SUCCESS; }
    for (int i = 0; i < root->num_planes; i++) {
        Plane &p = root->planes[i];
        if (cudaMemcpy2DAsync(p.dev, p.dev_stride, p.host, p.host_stride, (size_t)p.width * p.bpp, p.height,
                              cudaMemcpyHostToDevice, s) != cudaSuccess)
            return VX_FAILURE;
    }
    root->dev_valid = true;
    return VX_SUCCESS;
}

vx_status image_sync_to_host(Image *img)
{
    use_device(img);
    Image *root = img->parent ? img->parent : img;
    vx_status st = ensure_host(root);
    if (st) return st;
    if (root->host_valid) return VX_SUCCESS;
    if (root->dev_valid) {
        for (int i = 0; i < root->num_planes; i++) {
            Plane &p = root->planes[i];
            if (cudaMemcpy2D(p.host, p.host_stride, p.dev, p.dev_stride, (size_t)p.width * p.bpp, p.height,
                             cudaMemcpyDeviceToHost) != cudaSuccess)
                return VX_FAILURE;
        }
    }
    root->host_valid = true;
    return VX_SUCCESS;
}

static void mark_written_on_host(Image *img)
{
    Image *root = img->parent ? img->parent : img;
    root->host_valid = true;
    root->dev_valid = false;
}

static void mark_written_on_device(Image *img)
{
    Image *root = img->parent ? img->parent : img;
    root->dev_valid = true;
    root->host_valid = false;
}

// ---------------------------------------------------------------- arrays / scalars
Array::~Array()
{
    if (host_mapped) cudaHostUnregister(host.data());
    if (dev) cudaFree(dev);
    if (dev_count) cudaFree(dev_count);
}

Scalar::~Scalar() { if (dev) cudaFree(dev); }

Array *make_array(Context *ctx, Graph *scope, vx_enum item_type, vx_size capacity, bool virt)
{
    Array *a = new Array();
    a->type = VX_TYPE_ARRAY;
    a->scope = scope;
    a->is_virtual = virt;
    a->item_type = item_type;
    a->item_size = type_size(item_type);
    // user structs (vxRegisterUserStruct): enums from 0x100 in registration order
    if (!a->item_size && ctx && item_type >= 0x100 && (size_t)(item_type - 0x100) < ctx->user_structs.size())
        a->item_size = ctx->user_structs[(size_t)(item_type - 0x100)];
    a->capacity = capacity;
    add_ref(ctx, a);
    return a;
}

vx_status array_alloc_device(Array *a)
{
    use_device(a);
    if (a->dev) return VX_SUCCESS;
    if (!a->item_size || !a->capacity) return VX_ERROR_INVALID_PARAMETERS;
    if (cudaMalloc((void **)&a->dev, a->item_size * a->capacity + 64) != cudaSuccess) return VX_ERROR_NO_MEMORY;
    // zeroed like AGO's buffers (agoAllocMemory uses calloc): fields a kernel leaves alone read 0
    cudaMemset(a->dev, 0, a->item_size * a->capacity + 64);
    if (cudaMalloc((void **)&a->dev_count, 16) != cudaSuccess) return VX_ERROR_NO_MEMORY;
    cudaMemset(a->dev_count, 0, 16);
    return VX_SUCCESS;
}

vx_status array_sync_to_device(Array *a, cudaStream_t s)
{
    vx_status st = array_alloc_device(a);
    if (st) return st;
    if (a->dev_valid) return VX_SUCCESS;
    uint32_t n = (uint32_t)a->num_items;
    if (n && cudaMemcpyAsync(a->dev, a->host.data(), n * a->item_size, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return VX_FAILURE;
    // the count word is copied from a host value that outlives the async copy
    static thread_local uint32_t staged[64];
    static thread_local int slot = 0;
    uint32_t *src = &staged[slot++ & 63];
    *src = n;
    if (cudaMemcpyAsync(a->dev_count, src, 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return VX_FAILURE;
    cudaStreamSynchronize(s);
    a->dev_valid = true;
    return VX_SUCCESS;
}

vx_status array_sync_to_host(Array *a)
{
    if (a->host_valid) return VX_SUCCESS;
    if (a->host.size() < a->capacity * a->item_size) a->host.resize(a->capacity * a->item_size);
    if (a->dev_valid && a->dev) {
        uint32_t n = 0;
        if (cudaMemcpy(&n, a->dev_count, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return VX_FAILURE;
        a->num_items = n < a->capacity ? n : a->capacity;
        if (a->num_items &&
            cudaMemcpy(a->host.data(), a->dev, a->num_items * a->item_size, cudaMemcpyDeviceToHost) != cudaSuccess)
            return VX_FAILURE;
    }
    a->host_valid = true;
    return VX_SUCCESS;
}

Scalar *make_scalar(Context *ctx, Graph *scope, vx_enum type, const void *ptr)
{
    Scalar *s = new Scalar();
    s->type = VX_TYPE_SCALAR;
    s->scope = scope;
    s->data_type = type;
    if (ptr) memcpy(s->v.raw, ptr, type_size(type) ? type_size(type) : 4);
    add_ref(ctx, s);
    return s;
}

vx_status scalar_alloc_device(Scalar *s)
{
    use_device(s);
    if (s->dev) return VX_SUCCESS;
    if (cudaMalloc((void **)&s->dev, 16) != cudaSuccess) return VX_ERROR_NO_MEMORY;
    cudaMemset(s->dev, 0, 16);
    return VX_SUCCESS;
}

vx_status scalar_sync_to_host(Scalar *s)
{
    if (!s->dev_newer || !s->dev) return VX_SUCCESS;
    uint32_t v = 0;
    if (cudaMemcpy(&v, s->dev, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return VX_FAILURE;
    if (s->data_type == VX_TYPE_SIZE) s->v.sz = v;
    else s->v.u32 = v;
    s->dev_newer = false;
    return VX_SUCCESS;
}

void graph_plan_cache_clear(Graph *g);

Graph::~Graph()
{
    graph_plan_cache_clear(this);
    if (cexec) cudaGraphExecDestroy(cexec);
    if (cgraph) cudaGraphDestroy(cgraph);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (cudaEvent_t e : cap_events) cudaEventDestroy(e);
    for (cudaStream_t s : lanes) cudaStreamDestroy(s);
    if (stream) cudaStreamDestroy(stream);
    for (void *p : dev_scratch) cudaFree(p);
    if (status_host) cudaFreeHost(status_host);
    if (io_slots_host) cudaFreeHost(io_slots_host);
}

}  // namespace agovx

// ====================================================================================
// Public API
// ====================================================================================
template <class T> static T *as(void *h) { return static_cast<T *>(static_cast<Ref *>(h)); }
#define CHECK_REF(h, T) if (!is_valid(h, T)) return VX_ERROR_INVALID_REFERENCE

extern "C" {

vx_context vxCreateContext(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return nullptr;   // no CPU fallback
    Context *c = new Context();
    c->type = VX_TYPE_CONTEXT;
    c->ctx = c;
    cudaGetDevice(&c->device);
    const char *t = getenv("AGO_DEFAULT_TARGET");
    if (t && (!strcmp(t, "CPU") || !strcmp(t, "cpu")))
        log_error(c, VX_SUCCESS, "WARNING: AGO_DEFAULT_TARGET=CPU ignored: this target executes on the GPU only\n");
    return (vx_context)c;
}

vx_status vxReleaseContext(vx_context *context)
{
    if (!context || !is_valid(*context, VX_TYPE_CONTEXT)) return VX_ERROR_INVALID_REFERENCE;
    Context *c = as<Context>(*context);
    cudaDeviceSynchronize();
    c->tearing_down = true;
    std::vector<Ref *> graphs, others;
    for (Ref *r : c->refs) (r->type == VX_TYPE_GRAPH ? graphs : others).push_back(r);
    c->refs.clear();
    // user kernels' deinitialize callbacks run while every object still exists
    for (Ref *r : graphs) user_nodes_deinit(static_cast<Graph *>(r));
    // graphs first: their plans and captured CUDA graphs name the other objects' storage
    for (Ref *r : graphs) { r->magic = 0; delete r; }
    for (Ref *r : others) { r->magic = 0; delete r; }
    c->magic = 0;
    delete c;
    *context = nullptr;
    return VX_SUCCESS;
}

vx_context vxGetContext(vx_reference reference)
{
    if (!is_ref(reference)) return nullptr;
    return (vx_context)as<Ref>(reference)->ctx;
}

vx_status vxGetStatus(vx_reference reference)
{
    if (!reference) return VX_ERROR_NO_RESOURCES;
    return is_ref(reference) ? VX_SUCCESS : VX_ERROR_INVALID_REFERENCE;
}

vx_status vxQueryContext(vx_context context, vx_enum attribute, void *ptr, vx_size size)
{
    CHECK_REF(context, VX_TYPE_CONTEXT);
    Context *c = as<Context>(context);
    switch (attribute) {
    case VX_CONTEXT_VENDOR_ID: if (size != 2) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint16 *)ptr = VX_ID_AMD; return VX_SUCCESS;
    case VX_CONTEXT_VERSION: if (size != 2) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint16 *)ptr = (1 << 8) | 3; return VX_SUCCESS;
    case VX_CONTEXT_REFERENCES: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint32 *)ptr = (vx_uint32)c->refs.size(); return VX_SUCCESS;
    case VX_CONTEXT_IMPLEMENTATION:
        if (size < 8) return VX_ERROR_INVALID_PARAMETERS;
        snprintf((char *)ptr, size, "AMD OpenVX (B200 sm_100a target)");
        return VX_SUCCESS;
    case VX_CONTEXT_ATTRIBUTE_AMD_HIP_DEVICE: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(int *)ptr = c->device; return VX_SUCCESS;
    case VX_CONTEXT_ATTRIBUTE_AMD_AFFINITY:
        if (size != sizeof(AgoTargetAffinityInfo)) return VX_ERROR_INVALID_PARAMETERS;
        memset(ptr, 0, size); ((AgoTargetAffinityInfo *)ptr)->device_type = c->affinity; return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxSetContextAttribute(vx_context context, vx_enum attribute, const void *ptr, vx_size size)
{
    CHECK_REF(context, VX_TYPE_CONTEXT);
    Context *c = as<Context>(context);
    switch (attribute) {
    case VX_CONTEXT_IMMEDIATE_BORDER:
        if (size != sizeof(vx_border_t)) return VX_ERROR_INVALID_PARAMETERS;
        c->immediate_border = *(const vx_border_t *)ptr; return VX_SUCCESS;
    case VX_CONTEXT_ATTRIBUTE_AMD_HIP_DEVICE:
        if (size != 4) return VX_ERROR_INVALID_PARAMETERS;
        if (cudaSetDevice(*(const int *)ptr) != cudaSuccess) return VX_ERROR_INVALID_VALUE;
        c->device = *(const int *)ptr; return VX_SUCCESS;
    case VX_CONTEXT_ATTRIBUTE_AMD_AFFINITY:
        if (size != sizeof(AgoTargetAffinityInfo)) return VX_ERROR_INVALID_PARAMETERS;
        c->affinity = ((const AgoTargetAffinityInfo *)ptr)->device_type; return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxDirective(vx_reference reference, vx_enum directive)
{
    if (!is_ref(reference)) return VX_ERROR_INVALID_REFERENCE;
    Ref *r = as<Ref>(reference);
    switch (directive) {
    case VX_DIRECTIVE_DISABLE_LOGGING: case VX_DIRECTIVE_ENABLE_LOGGING:
    case VX_DIRECTIVE_ENABLE_PERFORMANCE: case VX_DIRECTIVE_DISABLE_PERFORMANCE:
    case VX_DIRECTIVE_AMD_ENABLE_PROFILE_CAPTURE: case VX_DIRECTIVE_AMD_DISABLE_PROFILE_CAPTURE:
    case VX_DIRECTIVE_AMD_DISABLE_GPU_FLUSH: case VX_DIRECTIVE_AMD_READ_ONLY:
        return VX_SUCCESS;
    case VX_DIRECTIVE_AMD_COPY_TO_HIPMEM:
        if (r->type == VX_TYPE_IMAGE) { vx_status s = image_sync_to_device(as<Image>(r), 0); cudaDeviceSynchronize(); return s; }
        if (r->type == VX_TYPE_ARRAY) return array_sync_to_device(as<Array>(r), 0);
        return VX_ERROR_NOT_SUPPORTED;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxQueryReference(vx_reference ref, vx_enum attribute, void *ptr, vx_size size)
{
    if (!is_ref(ref)) return VX_ERROR_INVALID_REFERENCE;
    Ref *r = as<Ref>(ref);
    switch (attribute) {
    case VX_REFERENCE_COUNT: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint32 *)ptr = r->ext_count; return VX_SUCCESS;
    case VX_REFERENCE_TYPE: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_enum *)ptr = r->type; return VX_SUCCESS;
    case VX_REFERENCE_NAME: if (size != sizeof(char *)) return VX_ERROR_INVALID_PARAMETERS; *(const char **)ptr = r->name.c_str(); return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

static vx_status release_ref(Ref *r)
{
    if (!is_ref(r) || r->ext_count <= 0) return VX_ERROR_INVALID_REFERENCE;
    r->ext_count--;
    if (r->ext_count == 0) {
        r->released = true;
        // a plane handed out by vxCreateImageFromChannel stays with its parent but stops
        // holding it; the parent may then go, and takes its planes with it
        Image *hold = nullptr;
        if (r->type == VX_TYPE_IMAGE && !static_cast<Image *>(r)->roi_view) {
            hold = static_cast<Image *>(r)->view_of;
            static_cast<Image *>(r)->view_of = nullptr;
        }
        if (r->int_count == 0) destroy_ref(r);
        if (hold) release_internal(hold);
    }
    return VX_SUCCESS;
}

vx_status vxReleaseReference(vx_reference *ref_ptr)
{
    if (!ref_ptr || !is_ref(*ref_ptr)) return VX_ERROR_INVALID_REFERENCE;
    vx_status s = release_ref(as<Ref>(*ref_ptr));
    if (!s) *ref_ptr = nullptr;
    return s;
}

vx_status vxRetainReference(vx_reference ref)
{
    if (!is_ref(ref)) return VX_ERROR_INVALID_REFERENCE;
    as<Ref>(ref)->ext_count++;
    as<Ref>(ref)->released = false;
    return VX_SUCCESS;
}

vx_status vxSetReferenceName(vx_reference ref, const vx_char *name)
{
    if (!is_ref(ref)) return VX_ERROR_INVALID_REFERENCE;
    as<Ref>(ref)->name = name ? name : "";
    return VX_SUCCESS;
}

void vxRegisterLogCallback(vx_context context, vx_log_callback_f callback, vx_bool reentrant)
{
    if (!is_valid(context, VX_TYPE_CONTEXT)) return;
    as<Context>(context)->log_cb = callback;
    as<Context>(context)->log_reentrant = reentrant != 0;
}

void vxAddLogEntry(vx_reference ref, vx_status status, const char *message, ...)
{
    if (!is_ref(ref) || !message) return;
    char buf[VX_MAX_LOG_MESSAGE_LEN];
    va_list ap;
    va_start(ap, message);
    vsnprintf(buf, sizeof(buf), message, ap);
    va_end(ap);
    log_error(as<Ref>(ref), status, "%s", buf);
}

// ---------------------------------------------------------------- images
vx_image vxCreateImage(vx_context context, vx_uint32 width, vx_uint32 height, vx_df_image color)
{
    if (!is_valid(context, VX_TYPE_CONTEXT)) return nullptr;
    Plane tmp[3];
    if (!width || !height || !format_planes(color, width, height, tmp)) return nullptr;
    Image *img = make_image(as<Context>(context), nullptr, width, height, color, false);
    if (image_alloc_device(img)) return nullptr;
    return (vx_image)img;
}

vx_image vxCreateVirtualImage(vx_graph graph, vx_uint32 width, vx_uint32 height, vx_df_image color)
{
    if (!is_valid(graph, VX_TYPE_GRAPH)) return nullptr;
    Graph *g = as<Graph>(graph);
    Image *img = make_image(g->ctx, g, width, height, color, true);
    return (vx_image)img;
}

vx_image vxCreateUniformImage(vx_context context, vx_uint32 width, vx_uint32 height, vx_df_image color,
                              const vx_pixel_value_t *value)
{
    if (!is_valid(context, VX_TYPE_CONTEXT) || !value) return nullptr;
    Plane tmp[3];
    if (!width || !height || !format_planes(color, width, height, tmp)) return nullptr;
    Image *img = make_image(as<Context>(context), nullptr, width, height, color, false);
    img->uniform = true;
    img->uniform_value = *value;
    if (image_alloc_device(img)) return nullptr;
    return (vx_image)img;
}

// Device memory imported from the application must have the layout of the engine's own
// planes: the kernels read and write rows with word and 16-byte vector accesses (and
// cp.async copies), which need aligned rows; a misaligned plane is refused here instead of
// faulting on the GPU.
static bool device_layout_ok(const void *p, uint32_t stride)
{
    return ((uintptr_t)p % 256) == 0 && (stride % 64) == 0;
}

vx_image vxCreateImageFromHandle(vx_context context, vx_df_image color, const vx_imagepatch_addressing_t addrs[],
                                 void *const ptrs[], vx_enum memory_type)
{
    if (!is_valid(context, VX_TYPE_CONTEXT) || !addrs || !ptrs) return nullptr;
    if (memory_type != VX_MEMORY_TYPE_HOST && memory_type != VX_MEMORY_TYPE_HIP) return nullptr;
    Plane tmp[3];
    uint32_t w = addrs[0].dim_x, h = addrs[0].dim_y;
    int np = format_planes(color, w, h, tmp);
    if (!np) return nullptr;
    for (int i = 0; i < np; i++) {
        if ((uint32_t)addrs[i].stride_x != tmp[i].bpp || !ptrs[i]) return nullptr;   // packed pixels only
        if ((uint64_t)addrs[i].stride_y < (uint64_t)tmp[i].width * tmp[i].bpp) return nullptr;
        if (memory_type == VX_MEMORY_TYPE_HIP && !device_layout_ok(ptrs[i], (uint32_t)addrs[i].stride_y)) return nullptr;
    }
    Image *img = make_image(as<Context>(context), nullptr, w, h, color, false);
    img->import_type = memory_type;
    for (int i = 0; i < np; i++) {
        Plane &p = img->planes[i];
        if (memory_type == VX_MEMORY_TYPE_HOST) {
            p.host = (uint8_t *)ptrs[i]; p.host_stride = (uint32_t)addrs[i].stride_y; p.host_owned = false;
        } else {
            p.dev = (uint8_t *)ptrs[i]; p.dev_stride = (uint32_t)addrs[i].stride_y; p.dev_owned = false;
        }
    }
    if (memory_type == VX_MEMORY_TYPE_HOST) img->host_valid = true;
    else img->dev_valid = true;
    return (vx_image)img;
}

vx_status vxSwapImageHandle(vx_image image, void *const new_ptrs[], void *prev_ptrs[], vx_size num_planes)
{
    CHECK_REF(image, VX_TYPE_IMAGE);
    Image *img = as<Image>(image);
    if (img->import_type == VX_MEMORY_TYPE_NONE || (int)num_planes != img->num_planes) return VX_ERROR_INVALID_PARAMETERS;
    if (new_ptrs && img->import_type == VX_MEMORY_TYPE_HIP)
        for (int i = 0; i < img->num_planes; i++)
            if (new_ptrs[i] && !device_layout_ok(new_ptrs[i], img->planes[i].dev_stride)) return VX_ERROR_INVALID_PARAMETERS;
    for (int i = 0; i < img->num_planes; i++) {
        uint8_t *&slot = img->import_type == VX_MEMORY_TYPE_HOST ? img->planes[i].host : img->planes[i].dev;
        if (prev_ptrs) prev_ptrs[i] = slot;
        if (new_ptrs) slot = (uint8_t *)new_ptrs[i];
    }
    image_refresh_views(img);
    if (img->import_type == VX_MEMORY_TYPE_HOST) { img->host_valid = new_ptrs != nullptr; img->dev_valid = false; }
    else img->dev_valid = new_ptrs != nullptr;
    // pointers are baked into captured launches: graphs using this image re-capture
    for (Ref *r : img->ctx->refs) if (r->type == VX_TYPE_GRAPH && r->magic == kMagic) static_cast<Graph *>(r)->param_signature ^= 1;
    return VX_SUCCESS;
}

vx_status vxQueryImage(vx_image image, vx_enum attribute, void *ptr, vx_size size)
{
    CHECK_REF(image, VX_TYPE_IMAGE);
    Image *img = as<Image>(image);
    switch (attribute) {
    case VX_IMAGE_WIDTH: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint32 *)ptr = img->width; return VX_SUCCESS;
    case VX_IMAGE_HEIGHT: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint32 *)ptr = img->height; return VX_SUCCESS;
    case VX_IMAGE_FORMAT: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_df_image *)ptr = img->format; return VX_SUCCESS;
    case VX_IMAGE_PLANES: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = img->num_planes; return VX_SUCCESS;
    case VX_IMAGE_SPACE: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_enum *)ptr = img->color_space; return VX_SUCCESS;
    case VX_IMAGE_RANGE: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_enum *)ptr = img->color_range; return VX_SUCCESS;
    case VX_IMAGE_SIZE: {
        if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS;
        vx_size s = 0;
        for (int i = 0; i < img->num_planes; i++) s += (vx_size)img->planes[i].width * img->planes[i].bpp * img->planes[i].height;
        *(vx_size *)ptr = s; return VX_SUCCESS;
    }
    case VX_IMAGE_MEMORY_TYPE: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_enum *)ptr = img->import_type; return VX_SUCCESS;
    case VX_IMAGE_IS_UNIFORM: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_bool *)ptr = img->uniform; return VX_SUCCESS;
    case VX_IMAGE_UNIFORM_VALUE: if (size != sizeof(vx_pixel_value_t)) return VX_ERROR_INVALID_PARAMETERS; *(vx_pixel_value_t *)ptr = img->uniform_value; return VX_SUCCESS;
    case VX_IMAGE_ATTRIBUTE_AMD_HIP_BUFFER:
        if (size != sizeof(void *)) return VX_ERROR_INVALID_PARAMETERS;
        if (!img->ctx->in_user_kernel) {           // inside a user kernel the stream orders the data
            if (image_sync_to_device(img, 0)) return VX_FAILURE;
            cudaDeviceSynchronize();
        } else if (image_alloc_device(img->parent ? img->parent : img)) {
            return VX_ERROR_NO_MEMORY;
        }
        *(void **)ptr = img->planes[0].dev; return VX_SUCCESS;
    case VX_IMAGE_ATTRIBUTE_AMD_GPU_BUFFER_OFFSET:     // plane 0 starts at the buffer
        if (size != sizeof(vx_uint32)) return VX_ERROR_INVALID_PARAMETERS;
        *(vx_uint32 *)ptr = 0; return VX_SUCCESS;
    case VX_IMAGE_ATTRIBUTE_AMD_GPU_BUFFER_STRIDE:     // device row pitch of plane 0, bytes
        if (size != sizeof(vx_uint32)) return VX_ERROR_INVALID_PARAMETERS;
        if (image_alloc_device(img->parent ? img->parent : img)) return VX_ERROR_NO_MEMORY;
        *(vx_uint32 *)ptr = img->planes[0].dev_stride; return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxReleaseImage(vx_image *image)
{
    if (!image || !is_valid(*image, VX_TYPE_IMAGE)) return VX_ERROR_INVALID_REFERENCE;
    vx_status s = release_ref(as<Ref>(*image));
    if (!s) *image = nullptr;
    return s;
}

static bool plane_rect(Image *img, uint32_t plane, const vx_rectangle_t *r, uint32_t &x0, uint32_t &y0, uint32_t &x1, uint32_t &y1)
{
    if (plane >= (uint32_t)img->num_planes || !r) return false;
    if (r->start_x >= r->end_x || r->start_y >= r->end_y || r->end_x > img->width || r->end_y > img->height) return false;
    const Plane &p = img->planes[plane];
    const uint32_t sx = img->width / p.width, sy = img->height / p.height;   // 1 or 2
    x0 = r->start_x / sx; y0 = r->start_y / sy;
    x1 = (r->end_x + sx - 1) / sx; y1 = (r->end_y + sy - 1) / sy;
    return true;
}

vx_status vxCopyImagePatch(vx_image image, const vx_rectangle_t *image_rect, vx_uint32 image_plane_index,
                           const vx_imagepatch_addressing_t *user_addr, void *user_ptr, vx_enum usage, vx_enum user_mem_type)
{
    CHECK_REF(image, VX_TYPE_IMAGE);
    Image *img = as<Image>(image);
    if ((img->is_virtual && !img->ctx->in_user_kernel) || !user_addr || !user_ptr) return VX_ERROR_INVALID_PARAMETERS;
    use_device(img);
    if (usage != VX_READ_ONLY && usage != VX_WRITE_ONLY) return VX_ERROR_INVALID_PARAMETERS;
    uint32_t x0, y0, x1, y1;
    if (!plane_rect(img, image_plane_index, image_rect, x0, y0, x1, y1)) return VX_ERROR_INVALID_PARAMETERS;
    Image *root = img->parent ? img->parent : img;
    if (image_alloc_device(root)) return VX_ERROR_NO_MEMORY;
    Plane &p = img->planes[image_plane_index];
    const size_t row_bytes = (size_t)(x1 - x0) * p.bpp;
    const bool packed = (uint32_t)user_addr->stride_x == p.bpp;
    const cudaMemcpyKind kind_in = user_mem_type == VX_MEMORY_TYPE_HIP ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind kind_out = user_mem_type == VX_MEMORY_TYPE_HIP ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (!packed) return VX_ERROR_NOT_SUPPORTED;
    if (usage == VX_WRITE_ONLY) {
        const bool whole = x0 == 0 && y0 == 0 && x1 == p.width && y1 == p.height && root->num_planes == 1;
        if (!whole) { vx_status s = image_sync_to_device(root, 0); if (s) return s; cudaDeviceSynchronize(); }
        else if (image_alloc_device(root)) return VX_ERROR_NO_MEMORY;
        if (cudaMemcpy2D(p.dev + (size_t)y0 * p.dev_stride + (size_t)x0 * p.bpp, p.dev_stride, user_ptr,
                         (size_t)user_addr->stride_y, row_bytes, y1 - y0, kind_in) != cudaSuccess)
            return VX_FAILURE;
        if (root->import_type == VX_MEMORY_TYPE_HOST) {
            // keep the application's own buffer authoritative
            for (uint32_t y = y0; y < y1; y++)
                memcpy(p.host + (size_t)y * p.host_stride + (size_t)x0 * p.bpp,
                       (uint8_t *)user_ptr + (size_t)(y - y0) * user_addr->stride_y, row_bytes);
        }
        mark_written_on_device(root);
        if (root->import_type == VX_MEMORY_TYPE_HOST) root->host_valid = true;
    } else {
        if (root->host_valid && p.host && !root->dev_valid) {
            for (uint32_t y = y0; y < y1; y++)
                memcpy((uint8_t *)user_ptr + (size_t)(y - y0) * user_addr->stride_y,
                       p.host + (size_t)y * p.host_stride + (size_t)x0 * p.bpp, row_bytes);
            return VX_SUCCESS;
        }
        vx_status s = image_sync_to_device(root, 0);
        if (s) return s;
        cudaDeviceSynchronize();
        if (cudaMemcpy2D(user_ptr, (size_t)user_addr->stride_y, p.dev + (size_t)y0 * p.dev_stride + (size_t)x0 * p.bpp,
                         p.dev_stride, row_bytes, y1 - y0, kind_out) != cudaSuccess)
            return VX_FAILURE;
    }
    return VX_SUCCESS;
}

vx_status vxMapImagePatch(vx_image image, const vx_rectangle_t *rect, vx_uint32 plane_index, vx_map_id *map_id,
                          vx_imagepatch_addressing_t *addr, void **ptr, vx_enum usage, vx_enum mem_type, vx_uint32 flags)
{
    (void)flags;
    CHECK_REF(image, VX_TYPE_IMAGE);
    Image *img = as<Image>(image);
    if ((img->is_virtual && !img->ctx->in_user_kernel) || !map_id || !addr || !ptr) return VX_ERROR_INVALID_PARAMETERS;
    if (mem_type != VX_MEMORY_TYPE_HOST) return VX_ERROR_NOT_SUPPORTED;
    vx_rectangle_t full{0, 0, img->width, img->height};
    if (!rect) rect = &full;
    uint32_t x0, y0, x1, y1;
    if (!plane_rect(img, plane_index, rect, x0, y0, x1, y1)) return VX_ERROR_INVALID_PARAMETERS;
    vx_status s = image_sync_to_host(img);
    if (s) return s;
    Plane &p = img->planes[plane_index];
    uint8_t *base = p.host + (size_t)y0 * p.host_stride + (size_t)x0 * p.bpp;
    memset(addr, 0, sizeof(*addr));
    // dim_x / dim_y count the patch in image (plane 0) pixels; scale_x / scale_y shrink them to
    // the plane's elements and step_x / step_y are the image pixels per element, as
    // vx_api.cpp:2159-2164 reports a subsampled plane
    addr->dim_x = rect->end_x - rect->start_x; addr->dim_y = rect->end_y - rect->start_y;
    addr->stride_x = (vx_int32)p.bpp; addr->stride_y = (vx_int32)p.host_stride;
    const uint32_t sx = p.width < img->width ? 2 : 1, sy = p.height < img->height ? 2 : 1;
    addr->scale_x = VX_SCALE_UNITY / sx; addr->scale_y = VX_SCALE_UNITY / sy;
    addr->step_x = sx; addr->step_y = sy;
    *ptr = base;
    vx_map_id id = img->next_map++;
    img->maps[id] = MapInfo{plane_index, *rect, usage, base};
    *map_id = id;
    return VX_SUCCESS;
}

vx_status vxUnmapImagePatch(vx_image image, vx_map_id map_id)
{
    CHECK_REF(image, VX_TYPE_IMAGE);
    Image *img = as<Image>(image);
    auto it = img->maps.find(map_id);
    if (it == img->maps.end()) return VX_ERROR_INVALID_PARAMETERS;
    if (it->second.usage != VX_READ_ONLY) mark_written_on_host(img);
    img->maps.erase(it);
    return VX_SUCCESS;
}

vx_status vxGetValidRegionImage(vx_image image, vx_rectangle_t *rect)
{
    CHECK_REF(image, VX_TYPE_IMAGE);
    if (!rect) return VX_ERROR_INVALID_PARAMETERS;
    *rect = as<Image>(image)->valid;
    return VX_SUCCESS;
}

vx_status vxSetImageValidRectangle(vx_image image, const vx_rectangle_t *rect)
{
    CHECK_REF(image, VX_TYPE_IMAGE);
    Image *img = as<Image>(image);
    if (!rect) { img->valid = vx_rectangle_t{0, 0, img->width, img->height}; return VX_SUCCESS; }
    if (rect->start_x > rect->end_x || rect->start_y > rect->end_y || rect->end_x > img->width || rect->end_y > img->height)
        return VX_ERROR_INVALID_PARAMETERS;
    img->valid = *rect;
    for (Ref *r : img->ctx->refs) if (r->type == VX_TYPE_GRAPH && r->magic == kMagic) static_cast<Graph *>(r)->param_signature ^= 2;
    return VX_SUCCESS;
}

// ---------------------------------------------------------------- scalars
vx_scalar vxCreateScalar(vx_context context, vx_enum data_type, const void *ptr)
{
    if (!is_valid(context, VX_TYPE_CONTEXT) || !type_size(data_type)) return nullptr;
    return (vx_scalar)make_scalar(as<Context>(context), nullptr, data_type, ptr);
}

vx_status vxReleaseScalar(vx_scalar *scalar)
{
    if (!scalar || !is_valid(*scalar, VX_TYPE_SCALAR)) return VX_ERROR_INVALID_REFERENCE;
    vx_status s = release_ref(as<Ref>(*scalar));
    if (!s) *scalar = nullptr;
    return s;
}

vx_status vxQueryScalar(vx_scalar scalar, vx_enum attribute, void *ptr, vx_size size)
{
    CHECK_REF(scalar, VX_TYPE_SCALAR);
    if (attribute != VX_SCALAR_TYPE || size != 4) return VX_ERROR_INVALID_PARAMETERS;
    *(vx_enum *)ptr = as<Scalar>(scalar)->data_type;
    return VX_SUCCESS;
}

vx_status vxCopyScalar(vx_scalar scalar, void *user_ptr, vx_enum usage, vx_enum user_mem_type)
{
    CHECK_REF(scalar, VX_TYPE_SCALAR);
    Scalar *s = as<Scalar>(scalar);
    if (!user_ptr || user_mem_type != VX_MEMORY_TYPE_HOST) return VX_ERROR_INVALID_PARAMETERS;
    const vx_size n = type_size(s->data_type);
    if (usage == VX_READ_ONLY) {
        if (scalar_sync_to_host(s)) return VX_FAILURE;
        memcpy(user_ptr, s->v.raw, n);
    } else if (usage == VX_WRITE_ONLY) {
        if (memcmp(s->v.raw, user_ptr, n)) { memcpy(s->v.raw, user_ptr, n); s->version++; }
        s->dev_newer = false;
    } else return VX_ERROR_INVALID_PARAMETERS;
    return VX_SUCCESS;
}

// ---------------------------------------------------------------- thresholds
static vx_threshold new_threshold(Context *c, vx_enum type, vx_enum data_type, vx_df_image in, vx_df_image out)
{
    Threshold *t = new Threshold();
    t->type = VX_TYPE_THRESHOLD;
    t->thresh_type = type; t->data_type = data_type; t->input_format = in; t->output_format = out;
    // AGO defaults (ago/ago_internal.h:184-185): true 255, false 0
    t->true_value.U8 = 255; t->false_value.U8 = 0;
    if (out == VX_DF_IMAGE_S16) { t->true_value.S16 = -1; t->false_value.S16 = 0; }
    add_ref(c, t);
    return (vx_threshold)t;
}

vx_threshold vxCreateThreshold(vx_context c, vx_enum thresh_type, vx_enum data_type)
{
    if (!is_valid(c, VX_TYPE_CONTEXT)) return nullptr;
    if (thresh_type != VX_THRESHOLD_TYPE_BINARY && thresh_type != VX_THRESHOLD_TYPE_RANGE) return nullptr;
    vx_df_image in = data_type == VX_TYPE_INT16 ? VX_DF_IMAGE_S16 : VX_DF_IMAGE_U8;
    return new_threshold(as<Context>(c), thresh_type, data_type, in, VX_DF_IMAGE_U8);
}

vx_threshold vxCreateThresholdForImage(vx_context context, vx_enum thresh_type, vx_df_image input_format, vx_df_image output_format)
{
    if (!is_valid(context, VX_TYPE_CONTEXT)) return nullptr;
    if (thresh_type != VX_THRESHOLD_TYPE_BINARY && thresh_type != VX_THRESHOLD_TYPE_RANGE) return nullptr;
    vx_enum dt = input_format == VX_DF_IMAGE_S16 ? VX_TYPE_INT16 : input_format == VX_DF_IMAGE_U16 ? VX_TYPE_UINT16 : VX_TYPE_UINT8;
    return new_threshold(as<Context>(context), thresh_type, dt, input_format, output_format);
}

vx_status vxReleaseThreshold(vx_threshold *thresh)
{
    if (!thresh || !is_valid(*thresh, VX_TYPE_THRESHOLD)) return VX_ERROR_INVALID_REFERENCE;
    vx_status s = release_ref(as<Ref>(*thresh));
    if (!s) *thresh = nullptr;
    return s;
}

// The reference keeps the whole 32-bit value whatever the data type (vx_api.cpp:6328 copies
// the pixel union); kernels read the view they need (U8 = low byte, Canny the 32-bit one).
static void set_pixel_int(vx_pixel_value_t &v, int32_t x, vx_enum)
{
    memset(&v, 0, sizeof(v));
    v.S32 = x;
}

static int32_t get_pixel_int(const vx_pixel_value_t &v, vx_enum dt)
{
    if (dt == VX_TYPE_INT16) return v.S16;
    if (dt == VX_TYPE_UINT16) return v.U16;
    if (dt == VX_TYPE_UINT8) return v.U8;
    return v.S32;
}

vx_status vxSetThresholdAttribute(vx_threshold thresh, vx_enum attribute, const void *ptr, vx_size size)
{
    CHECK_REF(thresh, VX_TYPE_THRESHOLD);
    Threshold *t = as<Threshold>(thresh);
    if (!ptr || size != 4) return VX_ERROR_INVALID_PARAMETERS;
    const int32_t v = *(const int32_t *)ptr;
    switch (attribute) {
    case VX_THRESHOLD_THRESHOLD_VALUE: set_pixel_int(t->value, v, t->data_type); break;
    case VX_THRESHOLD_THRESHOLD_LOWER: set_pixel_int(t->lower, v, t->data_type); break;
    case VX_THRESHOLD_THRESHOLD_UPPER: set_pixel_int(t->upper, v, t->data_type); break;
    case VX_THRESHOLD_TRUE_VALUE: set_pixel_int(t->true_value, v, VX_TYPE_UINT8); break;
    case VX_THRESHOLD_FALSE_VALUE: set_pixel_int(t->false_value, v, VX_TYPE_UINT8); break;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
    t->version++;
    return VX_SUCCESS;
}

vx_status vxQueryThreshold(vx_threshold thresh, vx_enum attribute, void *ptr, vx_size size)
{
    CHECK_REF(thresh, VX_TYPE_THRESHOLD);
    Threshold *t = as<Threshold>(thresh);
    if (!ptr || size != 4) return VX_ERROR_INVALID_PARAMETERS;
    switch (attribute) {
    case VX_THRESHOLD_TYPE: *(vx_enum *)ptr = t->thresh_type; return VX_SUCCESS;
    case VX_THRESHOLD_DATA_TYPE: *(vx_enum *)ptr = t->data_type; return VX_SUCCESS;
    case VX_THRESHOLD_INPUT_FORMAT: *(vx_df_image *)ptr = t->input_format; return VX_SUCCESS;
    case VX_THRESHOLD_OUTPUT_FORMAT: *(vx_df_image *)ptr = t->output_format; return VX_SUCCESS;
    case VX_THRESHOLD_THRESHOLD_VALUE: *(int32_t *)ptr = get_pixel_int(t->value, t->data_type); return VX_SUCCESS;
    case VX_THRESHOLD_THRESHOLD_LOWER: *(int32_t *)ptr = get_pixel_int(t->lower, t->data_type); return VX_SUCCESS;
    case VX_THRESHOLD_THRESHOLD_UPPER: *(int32_t *)ptr = get_pixel_int(t->upper, t->data_type); return VX_SUCCESS;
    case VX_THRESHOLD_TRUE_VALUE: *(int32_t *)ptr = t->true_value.U8; return VX_SUCCESS;
    case VX_THRESHOLD_FALSE_VALUE: *(int32_t *)ptr = t->false_value.U8; return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxCopyThresholdValue(vx_threshold thresh, vx_pixel_value_t *value_ptr, vx_enum usage, vx_enum user_mem_type)
{
    CHECK_REF(thresh, VX_TYPE_THRESHOLD);
    Threshold *t = as<Threshold>(thresh);
    if (!value_ptr || user_mem_type != VX_MEMORY_TYPE_HOST || t->thresh_type != VX_THRESHOLD_TYPE_BINARY) return VX_ERROR_INVALID_PARAMETERS;
    if (usage == VX_READ_ONLY) *value_ptr = t->value;
    else { t->value = *value_ptr; t->version++; }
    return VX_SUCCESS;
}

vx_status vxCopyThresholdRange(vx_threshold thresh, vx_pixel_value_t *lower_value_ptr, vx_pixel_value_t *upper_value_ptr,
                               vx_enum usage, vx_enum user_mem_type)
{
    CHECK_REF(thresh, VX_TYPE_THRESHOLD);
    Threshold *t = as<Threshold>(thresh);
    if (!lower_value_ptr || !upper_value_ptr || user_mem_type != VX_MEMORY_TYPE_HOST || t->thresh_type != VX_THRESHOLD_TYPE_RANGE)
        return VX_ERROR_INVALID_PARAMETERS;
    if (usage == VX_READ_ONLY) { *lower_value_ptr = t->lower; *upper_value_ptr = t->upper; }
    else { t->lower = *lower_value_ptr; t->upper = *upper_value_ptr; t->version++; }
    return VX_SUCCESS;
}

// ---------------------------------------------------------------- node state
void *Node::node_state(int slot, size_t bytes)
{
    if (state[slot] && state_bytes[slot] == bytes) return state[slot];
    if (state[slot]) cudaFree(state[slot]);
    state[slot] = nullptr;
    state_bytes[slot] = 0;
    if (cudaMalloc(&state[slot], bytes) != cudaSuccess) return nullptr;
    cudaMemset(state[slot], 0, bytes);
    state_bytes[slot] = bytes;
    return state[slot];
}

Node::~Node()
{
    for (void *p : state) if (p) cudaFree(p);
    if (local_owned) free(local_ptr);
}

// ---------------------------------------------------------------- distributions
// vx_api.cpp vxCreateDistribution ("distribution:<bins>,<offset>,<range>", ago_util.cpp:1459)
Distribution::~Distribution() { if (dev) cudaFree(dev); }

static Distribution *make_distribution(Context *c, Graph *scope, vx_size bins, vx_int32 offset, vx_uint32 range)
{
    if (!bins || !range || bins > range) return nullptr;
    Distribution *d = new Distribution();
    d->type = VX_TYPE_DISTRIBUTION;
    d->scope = scope;
    d->is_virtual = scope != nullptr;
    d->bins = bins; d->offset = offset; d->range = range;
    d->window = (vx_uint32)((range + bins - 1) / bins);
    d->host.assign(bins, 0);
    add_ref(c, d);
    return d;
}

vx_status distribution_sync_to_host(Distribution *d)
{
    if (!d->dev_newer || !d->dev) return VX_SUCCESS;
    if (cudaMemcpy(d->host.data(), d->dev, d->bins * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return VX_FAILURE;
    d->dev_newer = false;
    return VX_SUCCESS;
}

vx_distribution vxCreateDistribution(vx_context context, vx_size numBins, vx_int32 offset, vx_uint32 range)
{
    if (!is_valid(context, VX_TYPE_CONTEXT)) return nullptr;
    return (vx_distribution)make_distribution(as<Context>(context), nullptr, numBins, offset, range);
}

vx_distribution vxCreateVirtualDistribution(vx_graph graph, vx_size numBins, vx_int32 offset, vx_uint32 range)
{
    if (!is_valid(graph, VX_TYPE_GRAPH)) return nullptr;
    return (vx_distribution)make_distribution(as<Graph>(graph)->ctx, as<Graph>(graph), numBins, offset, range);
}

vx_status vxReleaseDistribution(vx_distribution *distribution)
{
    if (!distribution || !is_valid(*distribution, VX_TYPE_DISTRIBUTION)) return VX_ERROR_INVALID_REFERENCE;
    vx_status s = release_ref(as<Ref>(*distribution));
    if (!s) *distribution = nullptr;
    return s;
}

vx_status vxQueryDistribution(vx_distribution distribution, vx_enum attribute, void *ptr, vx_size size)
{
    CHECK_REF(distribution, VX_TYPE_DISTRIBUTION);
    Distribution *d = as<Distribution>(distribution);
    if (!ptr) return VX_ERROR_INVALID_PARAMETERS;
    switch (attribute) {
    case VX_DISTRIBUTION_DIMENSIONS: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = 1; return VX_SUCCESS;
    case VX_DISTRIBUTION_OFFSET: if (size != sizeof(vx_int32)) return VX_ERROR_INVALID_PARAMETERS; *(vx_int32 *)ptr = d->offset; return VX_SUCCESS;
    case VX_DISTRIBUTION_RANGE: if (size != sizeof(vx_uint32)) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint32 *)ptr = d->range; return VX_SUCCESS;
    case VX_DISTRIBUTION_BINS: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = d->bins; return VX_SUCCESS;
    case VX_DISTRIBUTION_WINDOW: if (size != sizeof(vx_uint32)) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint32 *)ptr = d->window; return VX_SUCCESS;
    case VX_DISTRIBUTION_SIZE: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = d->bins * 4; return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxCopyDistribution(vx_distribution distribution, void *user_ptr, vx_enum usage, vx_enum user_mem_type)
{
    CHECK_REF(distribution, VX_TYPE_DISTRIBUTION);
    Distribution *d = as<Distribution>(distribution);
    if (!user_ptr || user_mem_type != VX_MEMORY_TYPE_HOST) return VX_ERROR_INVALID_PARAMETERS;
    if (usage == VX_READ_ONLY) {
        if (distribution_sync_to_host(d)) return VX_FAILURE;
        memcpy(user_ptr, d->host.data(), d->bins * 4);
    } else if (usage == VX_WRITE_ONLY) {
        memcpy(d->host.data(), user_ptr, d->bins * 4);
        d->dev_newer = false;
    } else {
        return VX_ERROR_INVALID_PARAMETERS;
    }
    return VX_SUCCESS;
}

vx_status vxMapDistribution(vx_distribution distribution, vx_map_id *map_id, void **ptr, vx_enum usage, vx_enum mem_type,
                            vx_uint32 flags)
{
    (void)flags;
    CHECK_REF(distribution, VX_TYPE_DISTRIBUTION);
    Distribution *d = as<Distribution>(distribution);
    if (!map_id || !ptr || mem_type != VX_MEMORY_TYPE_HOST) return VX_ERROR_INVALID_PARAMETERS;
    if (distribution_sync_to_host(d)) return VX_FAILURE;
    *ptr = d->host.data();
    vx_map_id id = d->next_map++;
    d->maps[id] = usage;
    *map_id = id;
    return VX_SUCCESS;
}

vx_status vxUnmapDistribution(vx_distribution distribution, vx_map_id map_id)
{
    CHECK_REF(distribution, VX_TYPE_DISTRIBUTION);
    Distribution *d = as<Distribution>(distribution);
    auto it = d->maps.find(map_id);
    if (it == d->maps.end()) return VX_ERROR_INVALID_PARAMETERS;
    d->maps.erase(it);
    return VX_SUCCESS;
}

// ---------------------------------------------------------------- LUTs
// vx_api.cpp:4859-5200 (data description "lut:<type>,<count>", ago_util.cpp:1476: offset 0
// for UINT8, count / 2 for INT16)
static Lut *make_lut(Context *c, Graph *scope, vx_enum data_type, vx_size count)
{
    if ((data_type != VX_TYPE_UINT8 && data_type != VX_TYPE_INT16) || !count) return nullptr;
    if ((data_type == VX_TYPE_UINT8 && count > 256) || (data_type == VX_TYPE_INT16 && count > 65536)) return nullptr;
    Lut *l = new Lut();
    l->type = VX_TYPE_LUT;
    l->scope = scope;
    l->is_virtual = scope != nullptr;
    l->data_type = data_type; l->count = count;
    l->offset = data_type == VX_TYPE_INT16 ? (uint32_t)(count / 2) : 0;
    l->data.assign(count * type_size(data_type), 0);
    add_ref(c, l);
    return l;
}

vx_lut vxCreateLUT(vx_context context, vx_enum data_type, vx_size count)
{
    if (!is_valid(context, VX_TYPE_CONTEXT)) return nullptr;
    return (vx_lut)make_lut(as<Context>(context), nullptr, data_type, count);
}

vx_lut vxCreateVirtualLUT(vx_graph graph, vx_enum data_type, vx_size count)
{
    if (!is_valid(graph, VX_TYPE_GRAPH)) return nullptr;
    return (vx_lut)make_lut(as<Graph>(graph)->ctx, as<Graph>(graph), data_type, count);
}

vx_status vxReleaseLUT(vx_lut *lut)
{
    if (!lut || !is_valid(*lut, VX_TYPE_LUT)) return VX_ERROR_INVALID_REFERENCE;
    vx_status s = release_ref(as<Ref>(*lut));
    if (!s) *lut = nullptr;
    return s;
}

vx_status vxQueryLUT(vx_lut lut, vx_enum attribute, void *ptr, vx_size size)
{
    CHECK_REF(lut, VX_TYPE_LUT);
    Lut *l = as<Lut>(lut);
    if (!ptr) return VX_ERROR_INVALID_PARAMETERS;
    switch (attribute) {
    case VX_LUT_TYPE: if (size != sizeof(vx_enum)) return VX_ERROR_INVALID_PARAMETERS; *(vx_enum *)ptr = l->data_type; return VX_SUCCESS;
    case VX_LUT_COUNT: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = l->count; return VX_SUCCESS;
    case VX_LUT_SIZE: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = l->data.size(); return VX_SUCCESS;
    case VX_LUT_OFFSET: if (size != sizeof(vx_uint32)) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint32 *)ptr = l->offset; return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxCopyLUT(vx_lut lut, void *user_ptr, vx_enum usage, vx_enum user_mem_type)
{
    CHECK_REF(lut, VX_TYPE_LUT);
    Lut *l = as<Lut>(lut);
    if (!user_ptr || user_mem_type != VX_MEMORY_TYPE_HOST) return VX_ERROR_INVALID_PARAMETERS;
    if (usage == VX_READ_ONLY) memcpy(user_ptr, l->data.data(), l->data.size());
    else if (usage == VX_WRITE_ONLY) { memcpy(l->data.data(), user_ptr, l->data.size()); l->version++; }
    else return VX_ERROR_INVALID_PARAMETERS;
    return VX_SUCCESS;
}

vx_status vxMapLUT(vx_lut lut, vx_map_id *map_id, void **ptr, vx_enum usage, vx_enum mem_type, vx_uint32 flags)
{
    (void)flags;
    CHECK_REF(lut, VX_TYPE_LUT);
    Lut *l = as<Lut>(lut);
    if (!map_id || !ptr || mem_type != VX_MEMORY_TYPE_HOST) return VX_ERROR_INVALID_PARAMETERS;
    if (usage != VX_READ_ONLY && usage != VX_WRITE_ONLY && usage != VX_READ_AND_WRITE) return VX_ERROR_INVALID_PARAMETERS;
    *ptr = l->data.data();
    vx_map_id id = l->next_map++;
    l->maps[id] = usage;
    *map_id = id;
    return VX_SUCCESS;
}

vx_status vxUnmapLUT(vx_lut lut, vx_map_id map_id)
{
    CHECK_REF(lut, VX_TYPE_LUT);
    Lut *l = as<Lut>(lut);
    auto it = l->maps.find(map_id);
    if (it == l->maps.end()) return VX_ERROR_INVALID_PARAMETERS;
    if (it->second != VX_READ_ONLY) l->version++;
    l->maps.erase(it);
    return VX_SUCCESS;
}

// ---------------------------------------------------------------- matrices
vx_matrix vxCreateMatrix(vx_context c, vx_enum data_type, vx_size columns, vx_size rows)
{
    if (!is_valid(c, VX_TYPE_CONTEXT) || !columns || !rows) return nullptr;
    if (data_type != VX_TYPE_FLOAT32 && data_type != VX_TYPE_INT32 && data_type != VX_TYPE_UINT8) return nullptr;
    Matrix *m = new Matrix();
    m->type = VX_TYPE_MATRIX;
    m->data_type = data_type; m->columns = columns; m->rows = rows;
    m->data.assign(columns * rows * type_size(data_type), 0);
    add_ref(as<Context>(c), m);
    return (vx_matrix)m;
}

vx_status vxReleaseMatrix(vx_matrix *mat)
{
    if (!mat || !is_valid(*mat, VX_TYPE_MATRIX)) return VX_ERROR_INVALID_REFERENCE;
    vx_status s = release_ref(as<Ref>(*mat));
    if (!s) *mat = nullptr;
    return s;
}

vx_status vxQueryMatrix(vx_matrix mat, vx_enum attribute, void *ptr, vx_size size)
{
    CHECK_REF(mat, VX_TYPE_MATRIX);
    Matrix *m = as<Matrix>(mat);
    switch (attribute) {
    case VX_MATRIX_TYPE: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_enum *)ptr = m->data_type; return VX_SUCCESS;
    case VX_MATRIX_ROWS: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = m->rows; return VX_SUCCESS;
    case VX_MATRIX_COLUMNS: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = m->columns; return VX_SUCCESS;
    case VX_MATRIX_SIZE: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = m->data.size(); return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxCopyMatrix(vx_matrix matrix, void *user_ptr, vx_enum usage, vx_enum user_mem_type)
{
    CHECK_REF(matrix, VX_TYPE_MATRIX);
    Matrix *m = as<Matrix>(matrix);
    if (!user_ptr || user_mem_type != VX_MEMORY_TYPE_HOST) return VX_ERROR_INVALID_PARAMETERS;
    if (usage == VX_READ_ONLY) memcpy(user_ptr, m->data.data(), m->data.size());
    else if (usage == VX_WRITE_ONLY) { memcpy(m->data.data(), user_ptr, m->data.size()); m->version++; }
    else return VX_ERROR_INVALID_PARAMETERS;
    return VX_SUCCESS;
}

// ---------------------------------------------------------------- arrays
vx_array vxCreateArray(vx_context context, vx_enum item_type, vx_size capacity)
{
    if (!is_valid(context, VX_TYPE_CONTEXT) || !capacity) return nullptr;
    Array *a = make_array(as<Context>(context), nullptr, item_type, capacity, false);
    if (!a->item_size) { destroy_ref(a); return nullptr; }
    a->host.assign(a->capacity * a->item_size, 0);
    return (vx_array)a;
}

vx_array vxCreateVirtualArray(vx_graph graph, vx_enum item_type, vx_size capacity)
{
    if (!is_valid(graph, VX_TYPE_GRAPH)) return nullptr;
    Graph *g = as<Graph>(graph);
    Array *a = make_array(g->ctx, g, item_type, capacity, true);
    return (vx_array)a;
}

vx_status vxReleaseArray(vx_array *arr)
{
    if (!arr || !is_valid(*arr, VX_TYPE_ARRAY)) return VX_ERROR_INVALID_REFERENCE;
    vx_status s = release_ref(as<Ref>(*arr));
    if (!s) *arr = nullptr;
    return s;
}

vx_status vxQueryArray(vx_array arr, vx_enum attribute, void *ptr, vx_size size)
{
    CHECK_REF(arr, VX_TYPE_ARRAY);
    Array *a = as<Array>(arr);
    switch (attribute) {
    case VX_ARRAY_ITEMTYPE: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_enum *)ptr = a->item_type; return VX_SUCCESS;
    case VX_ARRAY_NUMITEMS:
        if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS;
        if (array_sync_to_host(a)) return VX_FAILURE;
        *(vx_size *)ptr = a->num_items; return VX_SUCCESS;
    case VX_ARRAY_CAPACITY: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = a->capacity; return VX_SUCCESS;
    case VX_ARRAY_ITEMSIZE: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = a->item_size; return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxAddArrayItems(vx_array arr, vx_size count, const void *ptr, vx_size stride)
{
    CHECK_REF(arr, VX_TYPE_ARRAY);
    Array *a = as<Array>(arr);
    if (!ptr || stride < a->item_size) return VX_ERROR_INVALID_PARAMETERS;
    if (array_sync_to_host(a)) return VX_FAILURE;
    if (a->num_items + count > a->capacity) return VX_FAILURE;
    if (a->host.size() < a->capacity * a->item_size) a->host.resize(a->capacity * a->item_size);
    for (vx_size i = 0; i < count; i++)
        memcpy(&a->host[(a->num_items + i) * a->item_size], (const uint8_t *)ptr + i * stride, a->item_size);
    a->num_items += count;
    a->dev_valid = false;
    return VX_SUCCESS;
}

vx_status vxTruncateArray(vx_array arr, vx_size new_num_items)
{
    CHECK_REF(arr, VX_TYPE_ARRAY);
    Array *a = as<Array>(arr);
    if (array_sync_to_host(a)) return VX_FAILURE;
    if (new_num_items > a->num_items) return VX_ERROR_INVALID_PARAMETERS;
    a->num_items = new_num_items;
    a->dev_valid = false;
    return VX_SUCCESS;
}

vx_status vxCopyArrayRange(vx_array array, vx_size range_start, vx_size range_end, vx_size user_stride, void *user_ptr,
                           vx_enum usage, vx_enum user_mem_type)
{
    CHECK_REF(array, VX_TYPE_ARRAY);
    Array *a = as<Array>(array);
    if (!user_ptr || user_mem_type != VX_MEMORY_TYPE_HOST || user_stride < a->item_size) return VX_ERROR_INVALID_PARAMETERS;
    if (array_sync_to_host(a)) return VX_FAILURE;
    if (range_start >= range_end || range_end > a->num_items) return VX_ERROR_INVALID_PARAMETERS;
    for (vx_size i = range_start; i < range_end; i++) {
        uint8_t *u = (uint8_t *)user_ptr + (i - range_start) * user_stride;
        if (usage == VX_READ_ONLY) memcpy(u, &a->host[i * a->item_size], a->item_size);
        else memcpy(&a->host[i * a->item_size], u, a->item_size);
    }
    if (usage != VX_READ_ONLY) a->dev_valid = false;
    return VX_SUCCESS;
}

vx_status vxMapArrayRange(vx_array array, vx_size range_start, vx_size range_end, vx_map_id *map_id, vx_size *stride,
                          void **ptr, vx_enum usage, vx_enum mem_type, vx_uint32 flags)
{
    (void)flags;
    CHECK_REF(array, VX_TYPE_ARRAY);
    Array *a = as<Array>(array);
    if (!map_id || !stride || !ptr || mem_type != VX_MEMORY_TYPE_HOST) return VX_ERROR_INVALID_PARAMETERS;
    if (array_sync_to_host(a)) return VX_FAILURE;
    if (range_start >= range_end || range_end > a->num_items) return VX_ERROR_INVALID_PARAMETERS;
    *stride = a->item_size;
    *ptr = &a->host[range_start * a->item_size];
    vx_map_id id = a->next_map++;
    a->maps[id] = {range_start, usage};
    *map_id = id;
    return VX_SUCCESS;
}

vx_status vxUnmapArrayRange(vx_array array, vx_map_id map_id)
{
    CHECK_REF(array, VX_TYPE_ARRAY);
    Array *a = as<Array>(array);
    auto it = a->maps.find(map_id);
    if (it == a->maps.end()) return VX_ERROR_INVALID_PARAMETERS;
    if (it->second.second != VX_READ_ONLY) a->dev_valid = false;
    a->maps.erase(it);
    return VX_SUCCESS;
}

// ---------------------------------------------------------------- pyramids
static Pyramid *make_pyramid(Context *c, Graph *scope, vx_size levels, vx_float32 scale, uint32_t w, uint32_t h,
                             vx_df_image format, bool virt)
{
    Pyramid *p = new Pyramid();
    p->type = VX_TYPE_PYRAMID;
    p->scope = scope;
    p->is_virtual = virt;
    p->levels = levels; p->scale = scale; p->width = w; p->height = h; p->format = format;
    add_ref(c, p);
    // level sizes: ceilf(scale * previous) (ago/ago_util.cpp:1331-1332)
    for (vx_size l = 0, lw = w, lh = h; l < levels; l++) {
        Image *img = make_image(c, scope, (uint32_t)lw, (uint32_t)lh, format, virt);
        img->int_count++;
        img->ext_count = 0;
        p->level.push_back(img);
        lw = (vx_size)ceilf(scale * (float)lw);
        lh = (vx_size)ceilf(scale * (float)lh);
    }
    return p;
}

vx_pyramid vxCreatePyramid(vx_context context, vx_size levels, vx_float32 scale, vx_uint32 width, vx_uint32 height, vx_df_image format)
{
    if (!is_valid(context, VX_TYPE_CONTEXT) || !levels || !width || !height) return nullptr;
    if (scale != VX_SCALE_PYRAMID_HALF) return nullptr;   // ORB scale is out of scope for this target
    Pyramid *p = make_pyramid(as<Context>(context), nullptr, levels, scale, width, height, format, false);
    for (Image *img : p->level) if (image_alloc_device(img)) return nullptr;
    return (vx_pyramid)p;
}

vx_pyramid vxCreateVirtualPyramid(vx_graph graph, vx_size levels, vx_float32 scale, vx_uint32 width, vx_uint32 height, vx_df_image format)
{
    if (!is_valid(graph, VX_TYPE_GRAPH) || !levels || !width || !height) return nullptr;
    if (scale != VX_SCALE_PYRAMID_HALF) return nullptr;
    Graph *g = as<Graph>(graph);
    return (vx_pyramid)make_pyramid(g->ctx, g, levels, scale, width, height, format, true);
}

vx_image vxGetPyramidLevel(vx_pyramid pyr, vx_uint32 index)
{
    if (!is_valid(pyr, VX_TYPE_PYRAMID)) return nullptr;
    Pyramid *p = as<Pyramid>(pyr);
    if (index >= p->levels) return nullptr;
    p->level[index]->ext_count++;
    p->level[index]->released = false;
    return (vx_image)p->level[index];
}

vx_status vxQueryPyramid(vx_pyramid pyr, vx_enum attribute, void *ptr, vx_size size)
{
    CHECK_REF(pyr, VX_TYPE_PYRAMID);
    Pyramid *p = as<Pyramid>(pyr);
    switch (attribute) {
    case VX_PYRAMID_LEVELS: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = p->levels; return VX_SUCCESS;
    case VX_PYRAMID_SCALE: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_float32 *)ptr = p->scale; return VX_SUCCESS;
    case VX_PYRAMID_WIDTH: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint32 *)ptr = p->width; return VX_SUCCESS;
    case VX_PYRAMID_HEIGHT: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint32 *)ptr = p->height; return VX_SUCCESS;
    case VX_PYRAMID_FORMAT: if (size != 4) return VX_ERROR_INVALID_PARAMETERS; *(vx_df_image *)ptr = p->format; return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxReleasePyramid(vx_pyramid *pyr)
{
    if (!pyr || !is_valid(*pyr, VX_TYPE_PYRAMID)) return VX_ERROR_INVALID_REFERENCE;
    vx_status s = release_ref(as<Ref>(*pyr));
    if (!s) *pyr = nullptr;
    return s;
}

// ---------------------------------------------------------------- remaps
vx_remap vxCreateRemap(vx_context context, vx_uint32 src_width, vx_uint32 src_height, vx_uint32 dst_width, vx_uint32 dst_height)
{
    if (!is_valid(context, VX_TYPE_CONTEXT) || !src_width || !src_height || !dst_width || !dst_height) return nullptr;
    Remap *r = new Remap();
    r->type = VX_TYPE_REMAP;
    r->src_width = src_width; r->src_height = src_height; r->dst_width = dst_width; r->dst_height = dst_height;
    r->table.assign((size_t)dst_width * dst_height, vx_coordinates2df_t{0.f, 0.f});
    add_ref(as<Context>(context), r);
    return (vx_remap)r;
}

vx_status vxReleaseRemap(vx_remap *table)
{
    if (!table || !is_valid(*table, VX_TYPE_REMAP)) return VX_ERROR_INVALID_REFERENCE;
    vx_status s = release_ref(as<Ref>(*table));
    if (!s) *table = nullptr;
    return s;
}

vx_status vxSetRemapPoint(vx_remap table, vx_uint32 dst_x, vx_uint32 dst_y, vx_float32 src_x, vx_float32 src_y)
{
    CHECK_REF(table, VX_TYPE_REMAP);
    Remap *r = as<Remap>(table);
    if (dst_x >= r->dst_width || dst_y >= r->dst_height) return VX_ERROR_INVALID_PARAMETERS;
    r->table[(size_t)dst_y * r->dst_width + dst_x] = vx_coordinates2df_t{src_x, src_y};
    r->version++;
    return VX_SUCCESS;
}

vx_status vxCopyRemapPatch(vx_remap remap, const vx_rectangle_t *rect, vx_size user_stride_y, void *user_ptr,
                           vx_enum user_coordinate_type, vx_enum usage, vx_enum user_mem_type)
{
    CHECK_REF(remap, VX_TYPE_REMAP);
    Remap *r = as<Remap>(remap);
    if (!rect || !user_ptr || user_coordinate_type != VX_TYPE_COORDINATES2DF || user_mem_type != VX_MEMORY_TYPE_HOST)
        return VX_ERROR_INVALID_PARAMETERS;
    if (rect->end_x > r->dst_width || rect->end_y > r->dst_height || rect->start_x >= rect->end_x || rect->start_y >= rect->end_y)
        return VX_ERROR_INVALID_PARAMETERS;
    for (uint32_t y = rect->start_y; y < rect->end_y; y++) {
        uint8_t *u = (uint8_t *)user_ptr + (size_t)(y - rect->start_y) * user_stride_y;
        vx_coordinates2df_t *t = &r->table[(size_t)y * r->dst_width + rect->start_x];
        size_t n = (rect->end_x - rect->start_x) * sizeof(vx_coordinates2df_t);
        if (usage == VX_READ_ONLY) memcpy(u, t, n);
        else memcpy(t, u, n);
    }
    if (usage != VX_READ_ONLY) r->version++;
    return VX_SUCCESS;
}

vx_status vxQueryRemap(vx_remap table, vx_enum attribute, void *ptr, vx_size size)
{
    CHECK_REF(table, VX_TYPE_REMAP);
    Remap *r = as<Remap>(table);
    if (size != 4) return VX_ERROR_INVALID_PARAMETERS;
    switch (attribute) {
    case VX_REMAP_SOURCE_WIDTH: *(vx_uint32 *)ptr = r->src_width; return VX_SUCCESS;
    case VX_REMAP_SOURCE_HEIGHT: *(vx_uint32 *)ptr = r->src_height; return VX_SUCCESS;
    case VX_REMAP_DESTINATION_WIDTH: *(vx_uint32 *)ptr = r->dst_width; return VX_SUCCESS;
    case VX_REMAP_DESTINATION_HEIGHT: *(vx_uint32 *)ptr = r->dst_height; return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

}  // extern "C"

// ---------------------------------------------------------------- delays
// vx_api.cpp vxCreateDelay / vxAgeDelay (ago_interface.cpp agoAgeDelay)
namespace agovx {

static void swap_image_storage(Image *a, Image *b)
{
    std::swap(a->planes, b->planes);
    std::swap(a->host_valid, b->host_valid);
    std::swap(a->dev_valid, b->dev_valid);
    std::swap(a->valid, b->valid);
    for (Image *img : {a, b}) {
        image_refresh_views(img);
        for (Image *c : img->children) { c->dev_valid = img->dev_valid; c->host_valid = img->host_valid; }
    }
}

static void swap_storage(Ref *a, Ref *b)
{
    switch (a->type) {
    case VX_TYPE_IMAGE: swap_image_storage(IMG(a), IMG(b)); break;
    case VX_TYPE_PYRAMID: {
        Pyramid *x = static_cast<Pyramid *>(a), *y = static_cast<Pyramid *>(b);
        for (size_t l = 0; l < x->level.size(); l++) swap_image_storage(x->level[l], y->level[l]);
        break;
    }
    case VX_TYPE_ARRAY: {
        Array *x = static_cast<Array *>(a), *y = static_cast<Array *>(b);
        std::swap(x->dev, y->dev);
        std::swap(x->dev_count, y->dev_count);
        std::swap(x->host, y->host);
        std::swap(x->num_items, y->num_items);
        std::swap(x->host_valid, y->host_valid);
        std::swap(x->dev_valid, y->dev_valid);
        std::swap(x->host_mapped, y->host_mapped);
        break;
    }
    case VX_TYPE_SCALAR: {
        Scalar *x = static_cast<Scalar *>(a), *y = static_cast<Scalar *>(b);
        std::swap(x->v, y->v);
        std::swap(x->dev, y->dev);
        std::swap(x->dev_newer, y->dev_newer);
        x->version++; y->version++;
        break;
    }
    default: break;
    }
}

vx_status delay_age(Delay *d)
{
    // the data at index 0 moves to -1, ..., and the oldest slot's storage becomes index 0
    for (size_t k = d->slots.size() - 1; k > 0; k--) swap_storage(d->slots[k], d->slots[k - 1]);
    return VX_SUCCESS;
}

}  // namespace agovx

extern "C" {

vx_delay vxCreateDelay(vx_context context, vx_reference exemplar, vx_size num_slots)
{
    if (!is_valid(context, VX_TYPE_CONTEXT) || !is_ref(exemplar) || num_slots < 1) return nullptr;
    Context *c = as<Context>(context);
    Ref *ex = as<Ref>(exemplar);
    Delay *d = new Delay();
    d->type = VX_TYPE_DELAY;
    d->item_type = ex->type;
    for (vx_size k = 0; k < num_slots; k++) {
        Ref *r = nullptr;
        switch (ex->type) {
        case VX_TYPE_IMAGE: {
            Image *e = IMG(ex);
            if (!e->width || !e->height || e->format == VX_DF_IMAGE_VIRT) break;
            r = make_image(c, nullptr, e->width, e->height, e->format, false);
            break;
        }
        case VX_TYPE_PYRAMID: {
            Pyramid *e = static_cast<Pyramid *>(ex);
            r = make_pyramid(c, nullptr, e->levels, e->scale, e->width, e->height, e->format, false);
            break;
        }
        case VX_TYPE_ARRAY: {
            Array *e = static_cast<Array *>(ex);
            if (e->item_type == VX_TYPE_INVALID) break;
            Array *a = make_array(c, nullptr, e->item_type, e->capacity, false);
            a->host.assign(a->capacity * a->item_size, 0);
            r = a;
            break;
        }
        case VX_TYPE_SCALAR: {
            Scalar *e = static_cast<Scalar *>(ex);
            r = make_scalar(c, nullptr, e->data_type, e->v.raw);
            break;
        }
        default: break;
        }
        if (!r) { for (Ref *s : d->slots) release_ref(s); delete d; return nullptr; }
        r->ext_count = 0;
        r->int_count = 1;          // held by the delay
        d->slots.push_back(r);
    }
    add_ref(c, d);
    return (vx_delay)d;
}

vx_status vxReleaseDelay(vx_delay *delay)
{
    if (!delay || !is_valid(*delay, VX_TYPE_DELAY)) return VX_ERROR_INVALID_REFERENCE;
    vx_status s = release_ref(as<Ref>(*delay));
    if (!s) *delay = nullptr;
    return s;
}

vx_status vxQueryDelay(vx_delay delay, vx_enum attribute, void *ptr, vx_size size)
{
    CHECK_REF(delay, VX_TYPE_DELAY);
    Delay *d = as<Delay>(delay);
    if (!ptr) return VX_ERROR_INVALID_PARAMETERS;
    switch (attribute) {
    case VX_DELAY_TYPE: if (size != sizeof(vx_enum)) return VX_ERROR_INVALID_PARAMETERS; *(vx_enum *)ptr = d->item_type; return VX_SUCCESS;
    case VX_DELAY_SLOTS: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = d->slots.size(); return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_reference vxGetReferenceFromDelay(vx_delay delay, vx_int32 index)
{
    if (!is_valid(delay, VX_TYPE_DELAY)) return nullptr;
    Delay *d = as<Delay>(delay);
    if (index > 0 || -index >= (vx_int32)d->slots.size()) return nullptr;
    return (vx_reference)d->slots[-index];
}

vx_status vxAgeDelay(vx_delay delay)
{
    CHECK_REF(delay, VX_TYPE_DELAY);
    return delay_age(as<Delay>(delay));
}

vx_status vxRegisterAutoAging(vx_graph graph, vx_delay delay)
{
    CHECK_REF(graph, VX_TYPE_GRAPH);
    CHECK_REF(delay, VX_TYPE_DELAY);
    Graph *g = as<Graph>(graph);
    if (std::find(g->auto_age.begin(), g->auto_age.end(), as<Delay>(delay)) == g->auto_age.end()) {
        g->auto_age.push_back(as<Delay>(delay));
        retain_internal(as<Delay>(delay));
    }
    return VX_SUCCESS;
}

}  // extern "C"
