// vx_compat.cpp -- the rest of the OpenVX / AMD API surface an application such as runvx
// links against (utilities/runvx): image views (vxCreateImageFromROI, vxCreateImageFromChannel),
// image attributes and format descriptions, the OpenVX 1.0 access/commit calls of
// VX/vx_compatibility.h, convolution objects, user structs, reference names, and tensor entry
// points that report "not supported" (tensors are not part of this target's vision path).
//
// Access/commit follow vx_api.cpp: with *ptr == NULL the implementation lends its own host
// buffer (the same buffer vxMap* hands out, so commit is an unmap); with a caller buffer the
// data is copied in at access (read usages) and out at commit (write usages).
#include <cstdio>
#include <cstring>
#include <map>

#include "vx_internal.h"

using namespace agovx;

namespace agovx {
vx_size type_size(vx_enum t);

namespace {

template <class T> T *as(void *h) { return static_cast<T *>(static_cast<Ref *>(h)); }

// Outstanding legacy accesses, per object: the pointer the application got (or gave) and
// what commit must do with it.
struct Access { vx_map_id map = 0; vx_enum usage = 0; bool lent = false; vx_size start = 0, stride = 0;
                vx_imagepatch_addressing_t addr{}; vx_rectangle_t rect{}; uint32_t plane = 0; };
std::mutex g_access_mu;
std::map<std::pair<const Ref *, const void *>, Access> g_access;

bool take_access(const Ref *r, const void *p, Access &a)
{
    std::lock_guard<std::mutex> lk(g_access_mu);
    auto it = g_access.find({r, p});
    if (it == g_access.end()) return false;
    a = it->second;
    g_access.erase(it);
    return true;
}

void put_access(const Ref *r, const void *p, const Access &a)
{
    std::lock_guard<std::mutex> lk(g_access_mu);
    g_access[{r, p}] = a;
}

bool reads(vx_enum usage) { return usage == VX_READ_ONLY || usage == VX_READ_AND_WRITE; }
bool writes(vx_enum usage) { return usage == VX_WRITE_ONLY || usage == VX_READ_AND_WRITE; }

struct FormatInfo { vx_df_image format; vx_size components, planes, bits_num, bits_denom; };

// Components, planes and pixel size of every format this target stores (for a multi-plane
// format the pixel size counts all planes: 12 bits for 4:2:0, 24 for 4:4:4).
const FormatInfo kFormats[] = {
    {VX_DF_IMAGE_U8, 1, 1, 8, 1},     {VX_DF_IMAGE_U16, 1, 1, 16, 1},   {VX_DF_IMAGE_S16, 1, 1, 16, 1},
    {VX_DF_IMAGE_U32, 1, 1, 32, 1},   {VX_DF_IMAGE_S32, 1, 1, 32, 1},   {VX_DF_IMAGE_F32_AMD, 1, 1, 32, 1},
    {VX_DF_IMAGE_RGB, 3, 1, 24, 1},   {VX_DF_IMAGE_RGBX, 4, 1, 32, 1},  {VX_DF_IMAGE_UYVY, 3, 1, 16, 1},
    {VX_DF_IMAGE_YUYV, 3, 1, 16, 1},  {VX_DF_IMAGE_NV12, 3, 2, 12, 1},  {VX_DF_IMAGE_NV21, 3, 2, 12, 1},
    {VX_DF_IMAGE_IYUV, 3, 3, 12, 1},  {VX_DF_IMAGE_YUV4, 3, 3, 24, 1},
};

}  // namespace

// Convolutions (vx_api.cpp vxCreateConvolution): odd sizes from 3 to 9 (AGO's limit for
// custom convolution), coefficients zero and scale 1 until the application sets them.
constexpr vx_size kMaxConvolutionDim = 9;

}  // namespace agovx

#define CHECK_REF(h, T) if (!is_valid(h, T)) return VX_ERROR_INVALID_REFERENCE

extern "C" {

// ------------------------------------------------------------------ image views
vx_image vxCreateImageFromROI(vx_image img, const vx_rectangle_t *rect)
{
    if (!is_valid(img, VX_TYPE_IMAGE) || !rect) return nullptr;
    Image *src = as<Image>(img);
    if (src->num_planes != 1 || src->is_virtual) return nullptr;           // single-plane images
    if (rect->start_x >= rect->end_x || rect->start_y >= rect->end_y || rect->end_x > src->width || rect->end_y > src->height)
        return nullptr;
    Image *root = src->roi_view ? src->parent : src;
    Image *v = make_image(src->ctx, nullptr, rect->end_x - rect->start_x, rect->end_y - rect->start_y, src->format, false);
    v->roi_view = true;
    v->parent = root;
    v->view_x = rect->start_x + (src->roi_view ? src->view_x : 0);
    v->view_y = rect->start_y + (src->roi_view ? src->view_y : 0);
    v->color_space = src->color_space;
    v->color_range = src->color_range;
    // the view's valid region is the parent's, clipped to the window and in window coordinates
    const vx_rectangle_t &pv = src->valid;
    auto clip = [](int64_t a, int64_t lo, int64_t hi) { return (vx_uint32)(a < lo ? lo : a > hi ? hi : a); };
    v->valid.start_x = clip((int64_t)pv.start_x - rect->start_x, 0, v->width);
    v->valid.start_y = clip((int64_t)pv.start_y - rect->start_y, 0, v->height);
    v->valid.end_x = clip((int64_t)pv.end_x - rect->start_x, v->valid.start_x, v->width);
    v->valid.end_y = clip((int64_t)pv.end_y - rect->start_y, v->valid.start_y, v->height);
    v->view_of = root;
    retain_internal(root);
    root->views.push_back(v);
    image_refresh_views(root);
    return (vx_image)v;
}

vx_image vxCreateImageFromChannel(vx_image img, vx_enum channel)
{
    if (!is_valid(img, VX_TYPE_IMAGE)) return nullptr;
    Image *src = as<Image>(img);
    int plane = -1;
    switch (src->format) {
    case VX_DF_IMAGE_IYUV: case VX_DF_IMAGE_YUV4:
        plane = channel == VX_CHANNEL_Y ? 0 : channel == VX_CHANNEL_U ? 1 : channel == VX_CHANNEL_V ? 2 : -1;
        break;
    case VX_DF_IMAGE_NV12: case VX_DF_IMAGE_NV21:
        plane = channel == VX_CHANNEL_Y ? 0 : -1;
        break;
    default: break;
    }
    if (plane < 0 || plane >= (int)src->children.size()) return nullptr;
    Image *c = src->children[plane];
    if (c->ext_count++ == 0) {        // the application's handle keeps the parent alive
        c->released = false;
        c->view_of = src;
        retain_internal(src);
    }
    return (vx_image)c;
}

vx_status vxSetImageAttribute(vx_image image, vx_enum attribute, const void *ptr, vx_size size)
{
    CHECK_REF(image, VX_TYPE_IMAGE);
    Image *img = as<Image>(image);
    if (!ptr || size != sizeof(vx_enum)) return VX_ERROR_INVALID_PARAMETERS;
    switch (attribute) {
    case VX_IMAGE_SPACE: img->color_space = *(const vx_enum *)ptr; return VX_SUCCESS;
    case VX_IMAGE_RANGE: img->color_range = *(const vx_enum *)ptr; return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

// x and y count image (plane 0) pixels; a plane subsampled by 2 has scale VX_SCALE_UNITY / 2,
// so (scale * x) / VX_SCALE_UNITY is its element (vx_api.cpp:27-36, vxComputePatchOffset).
void *vxFormatImagePatchAddress2d(void *ptr, vx_uint32 x, vx_uint32 y, const vx_imagepatch_addressing_t *addr)
{
    if (!ptr || !addr || x >= addr->dim_x || y >= addr->dim_y) return nullptr;
    const vx_size ox = (vx_size)addr->scale_x * x / VX_SCALE_UNITY, oy = (vx_size)addr->scale_y * y / VX_SCALE_UNITY;
    return (uint8_t *)ptr + (vx_int64)oy * addr->stride_y + (vx_int64)ox * addr->stride_x;
}

vx_status vxGetContextImageFormatDescription(vx_context context, vx_df_image format, AgoImageFormatDescription *desc)
{
    CHECK_REF(context, VX_TYPE_CONTEXT);
    if (!desc) return VX_ERROR_INVALID_PARAMETERS;
    for (const FormatInfo &f : kFormats)
        if (f.format == format) {
            desc->components = f.components;
            desc->planes = f.planes;
            desc->pixelSizeInBitsNum = f.bits_num;
            desc->pixelSizeInBitsDenom = f.bits_denom;
            desc->colorSpace = VX_COLOR_SPACE_BT709;
            desc->channelRange = VX_CHANNEL_RANGE_FULL;
            return VX_SUCCESS;
        }
    return VX_ERROR_INVALID_FORMAT;
}

// ------------------------------------------------------------------ access / commit
vx_status vxAccessImagePatch(vx_image image, const vx_rectangle_t *rect, vx_uint32 plane_index,
                             vx_imagepatch_addressing_t *addr, void **ptr, vx_enum usage)
{
    CHECK_REF(image, VX_TYPE_IMAGE);
    if (!addr || !ptr || !rect) return VX_ERROR_INVALID_PARAMETERS;
    Access a;
    a.usage = usage; a.rect = *rect; a.plane = plane_index;
    if (!*ptr) {
        vx_status s = vxMapImagePatch(image, rect, plane_index, &a.map, addr, ptr, usage, VX_MEMORY_TYPE_HOST, 0);
        if (s) return s;
        a.lent = true;
    } else {
        Image *img = as<Image>(image);
        if (plane_index >= (vx_uint32)img->num_planes) return VX_ERROR_INVALID_PARAMETERS;
        if (!addr->stride_x) {        // the caller's buffer in the image's own packing
            const Plane &p = img->planes[plane_index];
            const uint32_t sx = img->width / p.width, sy = img->height / p.height;
            addr->dim_x = rect->end_x - rect->start_x;     // image pixels; the plane holds dim / scale
            addr->dim_y = rect->end_y - rect->start_y;
            addr->stride_x = (vx_int32)p.bpp;
            addr->stride_y = (vx_int32)(((addr->dim_x + sx - 1) / sx) * p.bpp);
            addr->scale_x = VX_SCALE_UNITY / sx; addr->scale_y = VX_SCALE_UNITY / sy;
            addr->step_x = sx; addr->step_y = sy;
        }
        if (reads(usage)) {
            vx_status s = vxCopyImagePatch(image, rect, plane_index, addr, *ptr, VX_READ_ONLY, VX_MEMORY_TYPE_HOST);
            if (s) return s;
        }
        a.addr = *addr;
    }
    put_access(as<Ref>(image), *ptr, a);
    return VX_SUCCESS;
}

vx_status vxCommitImagePatch(vx_image image, const vx_rectangle_t *rect, vx_uint32 plane_index,
                             const vx_imagepatch_addressing_t *addr, const void *ptr)
{
    CHECK_REF(image, VX_TYPE_IMAGE);
    Access a;
    if (!ptr || !take_access(as<Ref>(image), ptr, a)) return VX_ERROR_INVALID_PARAMETERS;
    if (a.lent) return vxUnmapImagePatch(image, a.map);
    // a zero-area rectangle commits nothing (vx_compatibility.h)
    const bool area = rect && rect->end_x > rect->start_x && rect->end_y > rect->start_y;
    if (!writes(a.usage) || !area) return VX_SUCCESS;
    vx_imagepatch_addressing_t ad = addr ? *addr : a.addr;
    return vxCopyImagePatch(image, rect, plane_index, &ad, const_cast<void *>(ptr), VX_WRITE_ONLY, VX_MEMORY_TYPE_HOST);
}

vx_status vxAccessArrayRange(vx_array arr, vx_size start, vx_size end, vx_size *stride, void **ptr, vx_enum usage)
{
    CHECK_REF(arr, VX_TYPE_ARRAY);
    if (!stride || !ptr) return VX_ERROR_INVALID_PARAMETERS;
    Access a;
    a.usage = usage; a.start = start;
    if (!*ptr) {
        vx_status s = vxMapArrayRange(arr, start, end, &a.map, stride, ptr, usage, VX_MEMORY_TYPE_HOST, 0);
        if (s) return s;
        a.lent = true;
    } else {
        if (!*stride) *stride = as<Array>(arr)->item_size;
        if (reads(usage)) {
            vx_status s = vxCopyArrayRange(arr, start, end, *stride, *ptr, VX_READ_ONLY, VX_MEMORY_TYPE_HOST);
            if (s) return s;
        }
        a.stride = *stride;
    }
    put_access(as<Ref>(arr), *ptr, a);
    return VX_SUCCESS;
}

vx_status vxCommitArrayRange(vx_array arr, vx_size start, vx_size end, const void *ptr)
{
    CHECK_REF(arr, VX_TYPE_ARRAY);
    Access a;
    if (!ptr || !take_access(as<Ref>(arr), ptr, a)) return VX_ERROR_INVALID_PARAMETERS;
    if (a.lent) return vxUnmapArrayRange(arr, a.map);
    if (!writes(a.usage) || end <= start) return VX_SUCCESS;
    return vxCopyArrayRange(arr, start, end, a.stride, const_cast<void *>(ptr), VX_WRITE_ONLY, VX_MEMORY_TYPE_HOST);
}

vx_status vxAccessDistribution(vx_distribution distribution, void **ptr, vx_enum usage)
{
    CHECK_REF(distribution, VX_TYPE_DISTRIBUTION);
    if (!ptr) return VX_ERROR_INVALID_PARAMETERS;
    Access a;
    a.usage = usage;
    if (!*ptr) {
        vx_status s = vxMapDistribution(distribution, &a.map, ptr, usage, VX_MEMORY_TYPE_HOST, 0);
        if (s) return s;
        a.lent = true;
    } else if (reads(usage)) {
        vx_status s = vxCopyDistribution(distribution, *ptr, VX_READ_ONLY, VX_MEMORY_TYPE_HOST);
        if (s) return s;
    }
    put_access(as<Ref>(distribution), *ptr, a);
    return VX_SUCCESS;
}

vx_status vxCommitDistribution(vx_distribution distribution, const void *ptr)
{
    CHECK_REF(distribution, VX_TYPE_DISTRIBUTION);
    Access a;
    if (!ptr || !take_access(as<Ref>(distribution), ptr, a)) return VX_ERROR_INVALID_PARAMETERS;
    if (a.lent) return vxUnmapDistribution(distribution, a.map);
    if (!writes(a.usage)) return VX_SUCCESS;
    return vxCopyDistribution(distribution, const_cast<void *>(ptr), VX_WRITE_ONLY, VX_MEMORY_TYPE_HOST);
}

vx_status vxAccessLUT(vx_lut lut, void **ptr, vx_enum usage)
{
    CHECK_REF(lut, VX_TYPE_LUT);
    if (!ptr) return VX_ERROR_INVALID_PARAMETERS;
    Access a;
    a.usage = usage;
    if (!*ptr) {
        vx_status s = vxMapLUT(lut, &a.map, ptr, usage, VX_MEMORY_TYPE_HOST, 0);
        if (s) return s;
        a.lent = true;
    } else if (reads(usage)) {
        vx_status s = vxCopyLUT(lut, *ptr, VX_READ_ONLY, VX_MEMORY_TYPE_HOST);
        if (s) return s;
    }
    put_access(as<Ref>(lut), *ptr, a);
    return VX_SUCCESS;
}

vx_status vxCommitLUT(vx_lut lut, const void *ptr)
{
    CHECK_REF(lut, VX_TYPE_LUT);
    Access a;
    if (!ptr || !take_access(as<Ref>(lut), ptr, a)) return VX_ERROR_INVALID_PARAMETERS;
    if (a.lent) return vxUnmapLUT(lut, a.map);
    if (!writes(a.usage)) return VX_SUCCESS;
    return vxCopyLUT(lut, const_cast<void *>(ptr), VX_WRITE_ONLY, VX_MEMORY_TYPE_HOST);
}

// ------------------------------------------------------------------ value objects
vx_status vxReadMatrix(vx_matrix mat, void *array)
{ return vxCopyMatrix(mat, array, VX_READ_ONLY, VX_MEMORY_TYPE_HOST); }

vx_status vxWriteMatrix(vx_matrix mat, const void *array)
{ return vxCopyMatrix(mat, const_cast<void *>(array), VX_WRITE_ONLY, VX_MEMORY_TYPE_HOST); }

vx_status vxReadScalarValue(vx_scalar ref, void *ptr)
{ return vxCopyScalar(ref, ptr, VX_READ_ONLY, VX_MEMORY_TYPE_HOST); }

vx_status vxWriteScalarValue(vx_scalar ref, const void *ptr)
{ return vxCopyScalar(ref, const_cast<void *>(ptr), VX_WRITE_ONLY, VX_MEMORY_TYPE_HOST); }

vx_status vxGetRemapPoint(vx_remap table, vx_uint32 dst_x, vx_uint32 dst_y, vx_float32 *src_x, vx_float32 *src_y)
{
    CHECK_REF(table, VX_TYPE_REMAP);
    Remap *r = as<Remap>(table);
    if (!src_x || !src_y || dst_x >= r->dst_width || dst_y >= r->dst_height) return VX_ERROR_INVALID_PARAMETERS;
    const vx_coordinates2df_t &c = r->table[(size_t)dst_y * r->dst_width + dst_x];
    *src_x = c.x;
    *src_y = c.y;
    return VX_SUCCESS;
}

vx_status vxGetReferenceName(vx_reference ref, vx_char name[], vx_size size)
{
    if (!is_ref(ref)) return VX_ERROR_INVALID_REFERENCE;
    if (!name || !size) return VX_ERROR_INVALID_PARAMETERS;
    snprintf(name, size, "%s", as<Ref>(ref)->name.c_str());
    return VX_SUCCESS;
}

// vx_api.cpp:523: user struct enums count up from VX_TYPE_USER_STRUCT_START (0x100);
// arrays of them take the registered item size.
vx_enum vxRegisterUserStruct(vx_context context, vx_size size)
{
    if (!is_valid(context, VX_TYPE_CONTEXT) || !size) return VX_TYPE_INVALID;
    Context *c = as<Context>(context);
    c->user_structs.push_back(size);
    return (vx_enum)(0x100 + c->user_structs.size() - 1);
}

// ------------------------------------------------------------------ convolutions
vx_convolution vxCreateConvolution(vx_context context, vx_size columns, vx_size rows)
{
    if (!is_valid(context, VX_TYPE_CONTEXT)) return nullptr;
    if (columns < 3 || rows < 3 || columns > kMaxConvolutionDim || rows > kMaxConvolutionDim || !(columns & 1) || !(rows & 1))
        return nullptr;
    Convolution *cv = new Convolution();
    cv->type = VX_TYPE_CONVOLUTION;
    cv->columns = columns;
    cv->rows = rows;
    cv->coeffs.assign(columns * rows, 0);
    add_ref(as<Context>(context), cv);
    return (vx_convolution)cv;
}

vx_status vxReleaseConvolution(vx_convolution *conv)
{
    if (!conv || !is_valid(*conv, VX_TYPE_CONVOLUTION)) return VX_ERROR_INVALID_REFERENCE;
    return vxReleaseReference((vx_reference *)conv);
}

vx_status vxQueryConvolution(vx_convolution conv, vx_enum attribute, void *ptr, vx_size size)
{
    CHECK_REF(conv, VX_TYPE_CONVOLUTION);
    Convolution *cv = as<Convolution>(conv);
    if (!ptr) return VX_ERROR_INVALID_PARAMETERS;
    switch (attribute) {
    case VX_CONVOLUTION_ROWS: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = cv->rows; return VX_SUCCESS;
    case VX_CONVOLUTION_COLUMNS: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = cv->columns; return VX_SUCCESS;
    case VX_CONVOLUTION_SCALE: if (size != sizeof(vx_uint32)) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint32 *)ptr = cv->scale; return VX_SUCCESS;
    case VX_CONVOLUTION_SIZE:
        if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS;
        *(vx_size *)ptr = cv->coeffs.size() * sizeof(vx_int16); return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxSetConvolutionAttribute(vx_convolution conv, vx_enum attribute, const void *ptr, vx_size size)
{
    CHECK_REF(conv, VX_TYPE_CONVOLUTION);
    Convolution *cv = as<Convolution>(conv);
    if (!ptr) return VX_ERROR_INVALID_PARAMETERS;
    if (attribute != VX_CONVOLUTION_SCALE) return VX_ERROR_NOT_SUPPORTED;
    if (size != sizeof(vx_uint32)) return VX_ERROR_INVALID_PARAMETERS;
    const vx_uint32 s = *(const vx_uint32 *)ptr;
    if (!s || (s & (s - 1)) || s > (1u << 31)) return VX_ERROR_INVALID_VALUE;   // a power of two
    cv->scale = s;
    cv->version++;
    return VX_SUCCESS;
}

vx_status vxCopyConvolutionCoefficients(vx_convolution conv, void *user_ptr, vx_enum usage, vx_enum user_mem_type)
{
    CHECK_REF(conv, VX_TYPE_CONVOLUTION);
    Convolution *cv = as<Convolution>(conv);
    if (!user_ptr || user_mem_type != VX_MEMORY_TYPE_HOST) return VX_ERROR_INVALID_PARAMETERS;
    const size_t bytes = cv->coeffs.size() * sizeof(vx_int16);
    if (usage == VX_READ_ONLY) memcpy(user_ptr, cv->coeffs.data(), bytes);
    else if (usage == VX_WRITE_ONLY) { memcpy(cv->coeffs.data(), user_ptr, bytes); cv->version++; }
    else return VX_ERROR_INVALID_PARAMETERS;
    return VX_SUCCESS;
}

vx_status vxReadConvolutionCoefficients(vx_convolution conv, vx_int16 *array)
{ return vxCopyConvolutionCoefficients(conv, array, VX_READ_ONLY, VX_MEMORY_TYPE_HOST); }

vx_status vxWriteConvolutionCoefficients(vx_convolution conv, const vx_int16 *array)
{ return vxCopyConvolutionCoefficients(conv, const_cast<vx_int16 *>(array), VX_WRITE_ONLY, VX_MEMORY_TYPE_HOST); }

// ------------------------------------------------------------------ tensors (not supported)
vx_tensor vxCreateTensor(vx_context, vx_size, const vx_size *, vx_enum, vx_int8) { return nullptr; }
vx_tensor vxCreateVirtualTensor(vx_graph, vx_size, const vx_size *, vx_enum, vx_int8) { return nullptr; }
vx_tensor vxCreateTensorFromView(vx_tensor, vx_size, const vx_size *, const vx_size *) { return nullptr; }
vx_tensor vxCreateTensorFromHandle(vx_context, vx_size, const vx_size *, vx_enum, vx_int8, const vx_size *, void *, vx_enum)
{ return nullptr; }
vx_status vxQueryTensor(vx_tensor, vx_enum, void *, vx_size) { return VX_ERROR_NOT_SUPPORTED; }
vx_status vxReleaseTensor(vx_tensor *) { return VX_ERROR_NOT_SUPPORTED; }
vx_status vxSwapTensorHandle(vx_tensor, void *, void **) { return VX_ERROR_NOT_SUPPORTED; }
vx_status vxCopyTensorPatch(vx_tensor, vx_size, const vx_size *, const vx_size *, const vx_size *, void *, vx_enum, vx_enum)
{ return VX_ERROR_NOT_SUPPORTED; }
vx_status vxMapTensorPatch(vx_tensor, vx_size, const vx_size *, const vx_size *, vx_map_id *, vx_size *, void **, vx_enum, vx_enum)
{ return VX_ERROR_NOT_SUPPORTED; }
vx_status vxUnmapTensorPatch(vx_tensor, const vx_map_id) { return VX_ERROR_NOT_SUPPORTED; }

}  // extern "C"
