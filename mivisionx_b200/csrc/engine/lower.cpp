// lower.cpp -- node validation (output meta inference), lowering of OpenVX nodes to AGO
// low-level kernels, AGO's node-merge / copy-removal rules and valid-rectangle propagation.
//
// The lowering reproduces the reference's "divide" step (ago/ago_drama_divide.cpp) and the
// subset of its merge rule book (ago/ago_drama_remove.cpp:38-) that fires for the kernels
// of this target, because the merged kernels round differently from the unmerged ones
// (e.g. SobelMagnitude vs Sobel+Magnitude) and parity is defined on the merged graph.
#include <algorithm>
#include <cmath>
#include <set>

#include "vx_internal.h"

namespace agovx {

static const char *kLKNames[] = {
    "INVALID",
    "Gaussian_U8_U8_3x3", "Sobel_S16_U8_3x3_GX", "Sobel_S16_U8_3x3_GY", "Sobel_S16S16_U8_3x3_GXY",
    "Magnitude_S16_S16S16", "SobelMagnitude_S16_U8_3x3", "ColorDepth_U8_S16_Sat", "ColorDepth_U8_S16_Wrap",
    "ColorDepth_S16_U8", "Threshold_U8_U8_Binary", "ChannelCopy_U8_U8",
    "CannySobel_U16_U8_3x3_L1NORM", "CannySobel_U16_U8_3x3_L2NORM", "CannySuppThreshold_U8XY_U16_3x3",
    "CannyEdgeTrace_U8_U8XY",
    "HarrisSobel_HG3_U8_3x3", "HarrisScore_HVC_HG3_3x3", "NonMaxSupp_XY_ANY_3x3", "HarrisMergeSortAndPick_XY_XYS",
    "ColorConvert_Y_RGB", "ColorConvert_UV12_RGB", "ColorConvert_IU_RGB", "ColorConvert_IV_RGB",
    "ColorConvert_NV12_RGB", "ColorConvert_IYUV_RGB",
    "ScaleImage_U8_U8_Nearest", "ScaleImage_U8_U8_Bilinear", "ScaleImage_U8_U8_Area",
    "WarpAffine_U8_U8_Nearest", "WarpAffine_U8_U8_Nearest_Constant", "WarpAffine_U8_U8_Bilinear",
    "WarpAffine_U8_U8_Bilinear_Constant", "WarpPerspective_U8_U8_Nearest_Constant",
    "WarpPerspective_U8_U8_Bilinear_Constant", "Remap_U8_U8_Nearest_Constant", "Remap_U8_U8_Bilinear_Constant",
    "ScaleGaussianHalf_U8_U8_5x5", "OpticalFlowPyrLK_XY_XY",
    "WarpPerspective_U8_U8_Nearest", "WarpPerspective_U8_U8_Bilinear", "Remap_U8_U8_Nearest", "Remap_U8_U8_Bilinear",
    "Box_U8_U8_3x3", "Dilate_U8_U8_3x3", "Erode_U8_U8_3x3", "Median_U8_U8_3x3",
    "AbsDiff_U8_U8U8", "AbsDiff_S16_S16S16_Sat",
    "Add_U8_U8U8_Wrap", "Add_U8_U8U8_Sat", "Add_S16_U8U8", "Add_S16_S16U8_Wrap", "Add_S16_S16U8_Sat",
    "Add_S16_S16S16_Wrap", "Add_S16_S16S16_Sat",
    "Sub_U8_U8U8_Wrap", "Sub_U8_U8U8_Sat", "Sub_S16_U8U8", "Sub_S16_S16U8_Wrap", "Sub_S16_S16U8_Sat",
    "Sub_S16_U8S16_Wrap", "Sub_S16_U8S16_Sat", "Sub_S16_S16S16_Wrap", "Sub_S16_S16S16_Sat",
    "And_U8_U8U8", "Or_U8_U8U8", "Xor_U8_U8U8", "Not_U8_U8", "Threshold_U8_U8_Range",
    "ChannelExtract_U8_U16_Pos0", "ChannelExtract_U8_U16_Pos1", "ChannelExtract_U8_U24_Pos0", "ChannelExtract_U8_U24_Pos1",
    "ChannelExtract_U8_U24_Pos2", "ChannelExtract_U8_U32_Pos0", "ChannelExtract_U8_U32_Pos1", "ChannelExtract_U8_U32_Pos2",
    "ChannelExtract_U8_U32_Pos3", "ChannelCombine_U16_U8U8", "ChannelCombine_U24_U8U8U8_RGB",
    "ChannelCombine_U32_U8U8U8_UYVY", "ChannelCombine_U32_U8U8U8_YUYV", "ChannelCombine_U32_U8U8U8U8_RGBX",
    "Lut_U8_U8", "Lut_S16_S16", "IntegralImage_U32_U8", "Histogram_DATA_U8",
    "CannySobel_U16_U8_5x5_L1NORM", "CannySobel_U16_U8_5x5_L2NORM", "CannySobel_U16_U8_7x7_L1NORM",
    "CannySobel_U16_U8_7x7_L2NORM", "CannySuppThreshold_U8XY_U16_7x7",
    "Convolve_U8_U8", "Convolve_S16_U8",
    "HarrisSobel_HG3_U8_5x5", "HarrisSobel_HG3_U8_7x7", "HarrisScore_HVC_HG3_5x5", "HarrisScore_HVC_HG3_7x7",
    "FastCorners_XY_U8_Supression", "FastCorners_XY_U8_NoSupression",
    "UserKernel",
};
static_assert(sizeof(kLKNames) / sizeof(kLKNames[0]) == (size_t)LK::COUNT, "kernel name table");

const char *lk_name(LK k) { return kLKNames[(int)k]; }

// ------------------------------------------------------------------------------------
// meta inference (the role of the kernels' `validate` command in AGO)
// ------------------------------------------------------------------------------------
void image_init_planes(Image *img);

static vx_status set_meta(Image *out, uint32_t w, uint32_t h, vx_df_image f)
{
    if (out->num_planes == 0) {
        if (!out->is_virtual) return VX_ERROR_INVALID_PARAMETERS;
        out->width = out->width ? out->width : w;
        out->height = out->height ? out->height : h;
        out->format = out->format != VX_DF_IMAGE_VIRT ? out->format : f;
        image_init_planes(out);
        if (!out->num_planes) return VX_ERROR_INVALID_FORMAT;
        out->valid = vx_rectangle_t{0, 0, out->width, out->height};
    }
    if (out->format != f) return VX_ERROR_INVALID_FORMAT;
    if (out->width != w || out->height != h) return VX_ERROR_INVALID_DIMENSION;
    return VX_SUCCESS;
}

// agoChannelEnum2Index: R / Y / channel 0 -> 0, G / U / 1 -> 1, B / V / 2 -> 2, A / 3 -> 3
static int channel_index(vx_enum ch)
{
    switch (ch) {
    case VX_CHANNEL_0: case VX_CHANNEL_R: case VX_CHANNEL_Y: return 0;
    case VX_CHANNEL_1: case VX_CHANNEL_G: case VX_CHANNEL_U: return 1;
    case VX_CHANNEL_2: case VX_CHANNEL_B: case VX_CHANNEL_V: return 2;
    case VX_CHANNEL_3: case VX_CHANNEL_A: return 3;
    default: return -1;
    }
}

static bool fmt_is(Ref *r, vx_df_image f) { return r && r->type == VX_TYPE_IMAGE && IMG(r)->format == f && IMG(r)->num_planes; }

vx_status check_node_params(Node *n);   // vx_kernels.cpp: required parameters present, types as declared

// A user kernel's node: its validator describes each output in a vx_meta_format (types as
// declared by default); virtual outputs take the described format and size, others must match
// (ago_interface.cpp:1275-1380).
static vx_status validate_user_node(Node *n)
{
    Kernel *k = n->ukernel;
    const size_t np = n->params.size();
    std::vector<MetaFormat> metas(np);
    std::vector<vx_meta_format> mp(np);
    for (size_t i = 0; i < np; i++) {
        if (k->uparams[i].dir == VX_OUTPUT && k->uparams[i].type != VX_TYPE_REFERENCE) metas[i].type = k->uparams[i].type;
        mp[i] = reinterpret_cast<vx_meta_format>(&metas[i]);
    }
    const vx_status s = k->validate((vx_node)n, (const vx_reference *)n->params.data(), (vx_uint32)np, mp.data());
    if (s) {
        log_error(n, s, "ERROR: vxVerifyGraph: kernel %s: kernel_validate failed (%d)\n", k->kname.c_str(), s);
        return s;
    }
    for (size_t i = 0; i < np; i++) {
        Ref *r = n->params[i];
        if (!r || k->uparams[i].dir != VX_OUTPUT) continue;
        const MetaFormat &m = metas[i];
        if (m.type && m.type != r->type) return VX_ERROR_INVALID_TYPE;
        if (r->type == VX_TYPE_IMAGE) {
            Image *o = IMG(r);
            if (o->num_planes == 0) {
                if (!o->is_virtual) return VX_ERROR_INVALID_PARAMETERS;
                if (!o->width) o->width = m.width;
                if (!o->height) o->height = m.height;
                if (o->format == VX_DF_IMAGE_VIRT) o->format = m.format;
                image_init_planes(o);
                if (!o->num_planes) return VX_ERROR_INVALID_FORMAT;
            }
            if (m.format && o->format != m.format) return VX_ERROR_INVALID_FORMAT;
            if ((m.width && o->width != m.width) || (m.height && o->height != m.height)) return VX_ERROR_INVALID_DIMENSION;
        } else if (r->type == VX_TYPE_ARRAY) {
            Array *a = static_cast<Array *>(r);
            if (a->item_type == VX_TYPE_INVALID && a->is_virtual && m.item_type) {
                a->item_type = m.item_type;
                a->item_size = type_size(m.item_type);
            }
            if (m.item_type && a->item_type != m.item_type) return VX_ERROR_INVALID_TYPE;
            if (a->is_virtual && !a->capacity) a->capacity = m.capacity;
            if (m.capacity && a->capacity < m.capacity) return VX_ERROR_INVALID_DIMENSION;
        } else if (r->type == VX_TYPE_SCALAR) {
            if (m.scalar_type && static_cast<Scalar *>(r)->data_type != m.scalar_type) return VX_ERROR_INVALID_TYPE;
        }
    }
    return VX_SUCCESS;
}

vx_status validate_node(Graph *g, Node *n)
{
    (void)g;
    if (vx_status s = check_node_params(n)) return s;
    if (n->ukernel) return validate_user_node(n);
    for (Ref *r : n->params)
        if (r && r->type == VX_TYPE_IMAGE && IMG(r)->roi_view) {
            // the kernels address whole aligned rows of their planes; a window into another
            // image's rows is for the application's copies and maps, not for graph nodes
            log_error(n, VX_ERROR_NOT_SUPPORTED, "ERROR: vxVerifyGraph: ROI views (vxCreateImageFromROI) cannot be node parameters on this target\n");
            return VX_ERROR_NOT_SUPPORTED;
        }
    auto &p = n->params;
    auto img = [&](int i) { return i < (int)p.size() && p[i] && p[i]->type == VX_TYPE_IMAGE ? IMG(p[i]) : nullptr; };
    switch (n->kernel) {
    case VX_KERNEL_GAUSSIAN_3x3:
        if (!fmt_is(p[0], VX_DF_IMAGE_U8)) return VX_ERROR_INVALID_FORMAT;
        return set_meta(img(1), img(0)->width, img(0)->height, VX_DF_IMAGE_U8);
    case VX_KERNEL_SOBEL_3x3: {
        if (!fmt_is(p[0], VX_DF_IMAGE_U8)) return VX_ERROR_INVALID_FORMAT;
        if (!p[1] && !p[2]) return VX_ERROR_INVALID_PARAMETERS;
        for (int i = 1; i <= 2; i++)
            if (img(i)) { vx_status s = set_meta(img(i), img(0)->width, img(0)->height, VX_DF_IMAGE_S16); if (s) return s; }
        return VX_SUCCESS;
    }
    case VX_KERNEL_MAGNITUDE:
        if (!fmt_is(p[0], VX_DF_IMAGE_S16) || !fmt_is(p[1], VX_DF_IMAGE_S16)) return VX_ERROR_INVALID_FORMAT;
        if (img(0)->width != img(1)->width || img(0)->height != img(1)->height) return VX_ERROR_INVALID_DIMENSION;
        return set_meta(img(2), img(0)->width, img(0)->height, VX_DF_IMAGE_S16);
    case VX_KERNEL_CONVERTDEPTH: {
        Image *i0 = img(0), *o = img(1);
        if (!i0 || !i0->num_planes || !o) return VX_ERROR_INVALID_PARAMETERS;
        vx_df_image of = o->format;
        if (of == VX_DF_IMAGE_VIRT) return VX_ERROR_INVALID_FORMAT;
        if (!((i0->format == VX_DF_IMAGE_S16 && of == VX_DF_IMAGE_U8) || (i0->format == VX_DF_IMAGE_U8 && of == VX_DF_IMAGE_S16)))
            return VX_ERROR_INVALID_FORMAT;
        return set_meta(o, i0->width, i0->height, of);
    }
    case VX_KERNEL_THRESHOLD: {
        if (!fmt_is(p[0], VX_DF_IMAGE_U8) || !is_valid(p[1], VX_TYPE_THRESHOLD)) return VX_ERROR_INVALID_PARAMETERS;
        Threshold *t = static_cast<Threshold *>(p[1]);
        if (t->thresh_type != VX_THRESHOLD_TYPE_BINARY && t->thresh_type != VX_THRESHOLD_TYPE_RANGE) return VX_ERROR_NOT_SUPPORTED;
        return set_meta(img(2), img(0)->width, img(0)->height, VX_DF_IMAGE_U8);
    }
    // ago_kernel_api.cpp ovxKernel_Box3x3 (:1052) and the Median / Dilate / Erode validators
    case VX_KERNEL_BOX_3x3: case VX_KERNEL_MEDIAN_3x3: case VX_KERNEL_DILATE_3x3: case VX_KERNEL_ERODE_3x3:
    case VX_KERNEL_NOT:
        if (!fmt_is(p[0], VX_DF_IMAGE_U8)) return VX_ERROR_INVALID_FORMAT;
        return set_meta(img(1), img(0)->width, img(0)->height, VX_DF_IMAGE_U8);
    case VX_KERNEL_AND: case VX_KERNEL_OR: case VX_KERNEL_XOR:      // ovxKernel_And (:1473)
    case VX_KERNEL_ABSDIFF: {                                       // ovxKernel_AbsDiff (:782)
        Image *a = img(0), *b = img(1);
        const vx_df_image f = a && a->num_planes ? a->format : VX_DF_IMAGE_VIRT;
        const bool ok = n->kernel == VX_KERNEL_ABSDIFF ? (f == VX_DF_IMAGE_U8 || f == VX_DF_IMAGE_S16) : f == VX_DF_IMAGE_U8;
        if (!ok || !fmt_is(b, f)) return VX_ERROR_INVALID_FORMAT;
        if (a->width != b->width || a->height != b->height) return VX_ERROR_INVALID_DIMENSION;
        return set_meta(img(2), a->width, a->height, f);
    }
    case VX_KERNEL_ADD: case VX_KERNEL_SUBTRACT: {                  // ovxKernel_Add (:1681), _Subtract (:1729)
        Image *a = img(0), *b = img(1), *o = img(3);
        auto u8s16 = [](Image *i) { return i && i->num_planes && (i->format == VX_DF_IMAGE_U8 || i->format == VX_DF_IMAGE_S16); };
        if (!u8s16(a) || !u8s16(b) || !o) return VX_ERROR_INVALID_FORMAT;
        if (a->width != b->width || a->height != b->height) return VX_ERROR_INVALID_DIMENSION;
        if (!is_valid(p[2], VX_TYPE_SCALAR) || static_cast<Scalar *>(p[2])->data_type != VX_TYPE_ENUM) return VX_ERROR_INVALID_TYPE;
        const vx_enum pol = sc_enum(p[2]);
        if (pol != VX_CONVERT_POLICY_WRAP && pol != VX_CONVERT_POLICY_SATURATE) return VX_ERROR_INVALID_VALUE;
        // U8 only when both inputs and the output are U8; a virtual output of unset format is S16
        const vx_df_image f = a->format == VX_DF_IMAGE_U8 && b->format == VX_DF_IMAGE_U8 && o->format == VX_DF_IMAGE_U8
                                  ? VX_DF_IMAGE_U8 : VX_DF_IMAGE_S16;
        return set_meta(o, a->width, a->height, f);
    }
    case VX_KERNEL_CANNY_EDGE_DETECTOR: {
        if (!fmt_is(p[0], VX_DF_IMAGE_U8) || !is_valid(p[1], VX_TYPE_THRESHOLD)) return VX_ERROR_INVALID_PARAMETERS;
        if (static_cast<Threshold *>(p[1])->thresh_type != VX_THRESHOLD_TYPE_RANGE) return VX_ERROR_INVALID_TYPE;
        const int gs = sc_i32(p[2]);
        if (gs != 3 && gs != 5 && gs != 7) return VX_ERROR_INVALID_VALUE;
        if (sc_enum(p[3]) != VX_NORM_L1 && sc_enum(p[3]) != VX_NORM_L2) return VX_ERROR_INVALID_VALUE;
        return set_meta(img(4), img(0)->width, img(0)->height, VX_DF_IMAGE_U8);
    }
    case VX_KERNEL_HARRIS_CORNERS: {
        if (!fmt_is(p[0], VX_DF_IMAGE_U8)) return VX_ERROR_INVALID_FORMAT;
        for (int i : {4, 5}) {                             // gradient and block sizes (ago_drama_divide.cpp:1748, :1764)
            const int32_t v = sc_i32(p[i]);
            if (v != 3 && v != 5 && v != 7) return VX_ERROR_INVALID_VALUE;
        }
        if (!is_valid(p[6], VX_TYPE_ARRAY)) return VX_ERROR_INVALID_PARAMETERS;
        Array *a = static_cast<Array *>(p[6]);
        if (a->item_type == VX_TYPE_INVALID && a->is_virtual) { a->item_type = VX_TYPE_KEYPOINT; a->item_size = sizeof(vx_keypoint_t); }
        if (a->item_type != VX_TYPE_KEYPOINT) return VX_ERROR_INVALID_TYPE;
        if (!a->capacity) return VX_ERROR_INVALID_DIMENSION;
        return VX_SUCCESS;
    }
    case VX_KERNEL_FAST_CORNERS: {                     // agoKernel_FastCorners_XY_U8_* validate (ago_kernel_api.cpp:16606)
        if (!fmt_is(p[0], VX_DF_IMAGE_U8)) return VX_ERROR_INVALID_FORMAT;
        if (img(0)->width < 7 || img(0)->height < 7) return VX_ERROR_INVALID_DIMENSION;
        if (!is_valid(p[1], VX_TYPE_SCALAR) || static_cast<Scalar *>(p[1])->data_type != VX_TYPE_FLOAT32) return VX_ERROR_INVALID_TYPE;
        if (!is_valid(p[2], VX_TYPE_SCALAR)) return VX_ERROR_INVALID_PARAMETERS;
        if (!is_valid(p[3], VX_TYPE_ARRAY)) return VX_ERROR_INVALID_PARAMETERS;
        Array *a = static_cast<Array *>(p[3]);
        if (a->item_type == VX_TYPE_INVALID && a->is_virtual) { a->item_type = VX_TYPE_KEYPOINT; a->item_size = sizeof(vx_keypoint_t); }
        if (a->item_type != VX_TYPE_KEYPOINT) return VX_ERROR_INVALID_TYPE;
        if (!a->capacity) return VX_ERROR_INVALID_DIMENSION;
        return VX_SUCCESS;
    }
    case VX_KERNEL_COLOR_CONVERT: {
        Image *i0 = img(0), *o = img(1);
        if (!i0 || !i0->num_planes || !o || o->format == VX_DF_IMAGE_VIRT) return VX_ERROR_INVALID_FORMAT;
        if (i0->format != VX_DF_IMAGE_RGB) return VX_ERROR_NOT_SUPPORTED;
        if (o->format != VX_DF_IMAGE_NV12 && o->format != VX_DF_IMAGE_IYUV) return VX_ERROR_NOT_SUPPORTED;
        return set_meta(o, i0->width, i0->height, o->format);
    }
    case VX_KERNEL_CHANNEL_EXTRACT: {                   // ovxKernel_ChannelExtract (ago_kernel_api.cpp)
        Image *i0 = img(0), *o = img(2);
        if (!i0 || !i0->num_planes) return VX_ERROR_INVALID_PARAMETERS;
        const vx_df_image f = i0->format;
        if (f != VX_DF_IMAGE_RGB && f != VX_DF_IMAGE_RGBX && f != VX_DF_IMAGE_NV12 && f != VX_DF_IMAGE_NV21 &&
            f != VX_DF_IMAGE_IYUV && f != VX_DF_IMAGE_YUYV && f != VX_DF_IMAGE_UYVY && f != VX_DF_IMAGE_YUV4)
            return VX_ERROR_INVALID_FORMAT;
        if ((i0->width & 1) || (i0->height & 1)) return VX_ERROR_INVALID_DIMENSION;
        const int idx = channel_index(sc_enum(p[1]));
        if (!is_valid(p[1], VX_TYPE_SCALAR) || idx < 0 || idx > (f == VX_DF_IMAGE_RGBX ? 3 : 2)) return VX_ERROR_INVALID_VALUE;
        uint32_t w = i0->width, h = i0->height;
        if (idx > 0 && (f == VX_DF_IMAGE_NV12 || f == VX_DF_IMAGE_NV21 || f == VX_DF_IMAGE_IYUV)) { w >>= 1; h >>= 1; }
        if (idx > 0 && (f == VX_DF_IMAGE_YUYV || f == VX_DF_IMAGE_UYVY)) w >>= 1;
        return set_meta(o, w, h, VX_DF_IMAGE_U8);
    }
    case VX_KERNEL_HISTOGRAM:                           // agoKernel_Histogram_DATA_U8: ValidateArguments_Img_1IN(U8)
        if (!fmt_is(p[0], VX_DF_IMAGE_U8)) return VX_ERROR_INVALID_FORMAT;
        return is_valid(p[1], VX_TYPE_DISTRIBUTION) ? VX_SUCCESS : VX_ERROR_INVALID_PARAMETERS;
    case VX_KERNEL_INTEGRAL_IMAGE:                      // ValidateArguments_Img_1OUT_1IN(U32, U8)
        if (!fmt_is(p[0], VX_DF_IMAGE_U8)) return VX_ERROR_INVALID_FORMAT;
        return set_meta(img(1), img(0)->width, img(0)->height, VX_DF_IMAGE_U32);
    case VX_KERNEL_CUSTOM_CONVOLUTION: {                // agoKernel_Convolve_{U8,S16}_U8 validate (:15615)
        if (!fmt_is(p[0], VX_DF_IMAGE_U8)) return VX_ERROR_INVALID_FORMAT;
        const Convolution *cv = static_cast<Convolution *>(p[1]);
        if (!(cv->rows & 1) || !(cv->columns & 1)) return VX_ERROR_INVALID_DIMENSION;
        Image *o = img(2);
        // the divide picks the U8 kernel for a U8 output and the S16 one otherwise
        // (ago_drama_divide.cpp:892), whose meta sets S16
        const vx_df_image f = o && o->format == VX_DF_IMAGE_U8 ? VX_DF_IMAGE_U8 : VX_DF_IMAGE_S16;
        return set_meta(o, img(0)->width, img(0)->height, f);
    }
    case VX_KERNEL_TABLE_LOOKUP: {                      // ovxKernel_TableLookup (ago_kernel_api.cpp)
        Image *i0 = img(0);
        if (!is_valid(p[1], VX_TYPE_LUT) || !i0 || !i0->num_planes) return VX_ERROR_INVALID_PARAMETERS;
        const Lut *l = static_cast<Lut *>(p[1]);
        const bool u8 = i0->format == VX_DF_IMAGE_U8 && l->data_type == VX_TYPE_UINT8;
        if (!u8 && !(i0->format == VX_DF_IMAGE_S16 && l->data_type == VX_TYPE_INT16)) return VX_ERROR_INVALID_FORMAT;
        // a U8 table shorter than 256 entries would be read past its end (undefined): refused
        if (u8 && l->count != 256) return VX_ERROR_NOT_SUPPORTED;
        return set_meta(img(2), i0->width, i0->height, i0->format);
    }
    case VX_KERNEL_CHANNEL_COMBINE: {                   // ovxKernel_ChannelCombine (ago_kernel_api.cpp)
        Image *o = img(4);
        if (!o || o->format == VX_DF_IMAGE_VIRT) return VX_ERROR_INVALID_FORMAT;
        const vx_df_image f = o->format;
        int sx = 0, sy = 0;
        if (f == VX_DF_IMAGE_IYUV || f == VX_DF_IMAGE_NV12 || f == VX_DF_IMAGE_NV21) sx = sy = 1;
        else if (f == VX_DF_IMAGE_YUYV || f == VX_DF_IMAGE_UYVY) sx = 1;
        else if (f != VX_DF_IMAGE_RGB && f != VX_DF_IMAGE_RGBX && f != VX_DF_IMAGE_YUV4) return VX_ERROR_INVALID_FORMAT;
        const int planes = 2 + (img(2) ? 1 : 0) + (img(2) && img(3) ? 1 : 0);
        if ((!img(2) && img(3)) || planes != (f == VX_DF_IMAGE_RGBX ? 4 : 3)) return VX_ERROR_INVALID_PARAMETERS;
        Image *i0 = img(0);
        if (!fmt_is(i0, VX_DF_IMAGE_U8)) return VX_ERROR_INVALID_FORMAT;
        for (int k = 1; k < planes; k++) {
            if (!fmt_is(img(k), VX_DF_IMAGE_U8)) return VX_ERROR_INVALID_FORMAT;
            if ((img(k)->width << sx) != i0->width || (img(k)->height << sy) != i0->height) return VX_ERROR_INVALID_DIMENSION;
        }
        return set_meta(o, i0->width, i0->height, f);
    }
    case VX_KERNEL_SCALE_IMAGE: {
        Image *i0 = img(0), *o = img(1);
        if (!fmt_is(i0, VX_DF_IMAGE_U8) || !o || !o->width || !o->height) return VX_ERROR_INVALID_PARAMETERS;
        return set_meta(o, o->width, o->height, VX_DF_IMAGE_U8);
    }
    case VX_KERNEL_HALFSCALE_GAUSSIAN: {
        Image *i0 = img(0);
        if (!fmt_is(i0, VX_DF_IMAGE_U8)) return VX_ERROR_INVALID_FORMAT;
        if (sc_i32(p[2]) != 5) return VX_ERROR_NOT_SUPPORTED;
        return set_meta(img(1), (i0->width + 1) / 2, (i0->height + 1) / 2, VX_DF_IMAGE_U8);
    }
    case VX_KERNEL_WARP_AFFINE: case VX_KERNEL_WARP_PERSPECTIVE: {
        Image *i0 = img(0), *o = img(3);
        if (!fmt_is(i0, VX_DF_IMAGE_U8) || !o || !o->width || !o->height) return VX_ERROR_INVALID_PARAMETERS;
        Matrix *m = is_valid(p[1], VX_TYPE_MATRIX) ? static_cast<Matrix *>(p[1]) : nullptr;
        const vx_size rows = n->kernel == VX_KERNEL_WARP_AFFINE ? 3 : 3, cols = n->kernel == VX_KERNEL_WARP_AFFINE ? 2 : 3;
        if (!m || m->data_type != VX_TYPE_FLOAT32 || m->rows != rows || m->columns != cols) return VX_ERROR_INVALID_PARAMETERS;
        return set_meta(o, o->width, o->height, VX_DF_IMAGE_U8);
    }
    case VX_KERNEL_REMAP: {
        Image *i0 = img(0), *o = img(3);
        Remap *r = is_valid(p[1], VX_TYPE_REMAP) ? static_cast<Remap *>(p[1]) : nullptr;
        if (!fmt_is(i0, VX_DF_IMAGE_U8) || !r || !o) return VX_ERROR_INVALID_PARAMETERS;
        if (r->src_width != i0->width || r->src_height != i0->height) return VX_ERROR_INVALID_DIMENSION;
        return set_meta(o, r->dst_width, r->dst_height, VX_DF_IMAGE_U8);
    }
    case VX_KERNEL_GAUSSIAN_PYRAMID: {
        Image *i0 = img(0);
        Pyramid *py = is_valid(p[1], VX_TYPE_PYRAMID) ? static_cast<Pyramid *>(p[1]) : nullptr;
        if (!fmt_is(i0, VX_DF_IMAGE_U8) || !py) return VX_ERROR_INVALID_PARAMETERS;
        if (py->width != i0->width || py->height != i0->height || py->format != VX_DF_IMAGE_U8) return VX_ERROR_INVALID_DIMENSION;
        return VX_SUCCESS;
    }
    case VX_KERNEL_OPTICAL_FLOW_PYR_LK: {
        for (int i = 0; i < 2; i++) if (!is_valid(p[i], VX_TYPE_PYRAMID)) return VX_ERROR_INVALID_PARAMETERS;
        Pyramid *a = static_cast<Pyramid *>(p[0]), *b = static_cast<Pyramid *>(p[1]);
        if (a->levels != b->levels || a->width != b->width || a->height != b->height) return VX_ERROR_INVALID_DIMENSION;
        for (int i = 2; i <= 4; i++) if (!is_valid(p[i], VX_TYPE_ARRAY)) return VX_ERROR_INVALID_PARAMETERS;
        Array *o = static_cast<Array *>(p[4]);
        if (o->item_type == VX_TYPE_INVALID && o->is_virtual) { o->item_type = VX_TYPE_KEYPOINT; o->item_size = sizeof(vx_keypoint_t); }
        if (static_cast<Array *>(p[2])->item_type != VX_TYPE_KEYPOINT || o->item_type != VX_TYPE_KEYPOINT) return VX_ERROR_INVALID_TYPE;
        const vx_size win = static_cast<Scalar *>(p[9])->v.sz;
        if (win < 3 || win > AGOCUDA_LK_MAX_WINDOW) return VX_ERROR_INVALID_VALUE;   // ago_kernel_api.cpp:20624
        if (a->levels > AGOCUDA_LK_MAX_LEVELS) return VX_ERROR_NOT_SUPPORTED;
        // the reference's Scharr pass loops on `x <= width - 8` in unsigned arithmetic
        // (ago_haf_cpu_opticalflow.cpp:95), so it cannot process a level narrower than 8
        for (Image *lv : a->level) if (lv->width < 8 || lv->height < 3) return VX_ERROR_INVALID_DIMENSION;
        return VX_SUCCESS;
    }
    default:
        return VX_ERROR_NOT_SUPPORTED;
    }
}

// ------------------------------------------------------------------------------------
// divide (ago/ago_drama_divide.cpp)
// ------------------------------------------------------------------------------------
static Scalar *virt_scalar(Graph *g, vx_enum type, uint64_t value)
{
    Scalar *s = make_scalar(g->ctx, g, type, &value);
    s->is_virtual = true;
    s->ext_count = 0;
    graph_own(g, s);
    return s;
}

static Image *virt_image(Graph *g, uint32_t w, uint32_t h, vx_df_image f)
{
    Image *img = make_image(g->ctx, g, w, h, f, true);
    img->ext_count = 0;
    graph_own(g, img);
    return img;
}

static Array *virt_array(Graph *g, vx_enum item, vx_size cap)
{
    Array *a = make_array(g->ctx, g, item, cap, true);
    a->ext_count = 0;
    graph_own(g, a);
    return a;
}

// Item type of AGO's internal Canny stack / Harris XYS lists (sizes of ago_coord2d_ushort_t
// and ago_keypoint_xys_t, ago/ago_haf_cpu.h).
constexpr vx_enum kItemCoord2dU16 = 0x7F01;
constexpr vx_enum kItemKeypointXYS = 0x7F02;

static vx_status divide_node(Graph *g, Node *n, std::vector<LNode> &out)
{
    auto &p = n->params;
    auto add = [&](LK k, std::vector<Ref *> args) {
        LNode ln; ln.k = k; ln.p = std::move(args); ln.origin = n; ln.border = n->border;
        out.push_back(std::move(ln));
    };
    if (n->ukernel) {
        // one host step; outputs first (the lowered-node convention), the callback gets the
        // node's own parameter order.  Bidirectional parameters count as inputs here.
        LNode ln;
        ln.k = LK::USER_KERNEL;
        ln.origin = n;
        ln.border = n->border;
        for (size_t i = 0; i < p.size(); i++) if (n->ukernel->uparams[i].dir == VX_OUTPUT) ln.p.push_back(p[i]);
        ln.nout = (int)ln.p.size();
        for (size_t i = 0; i < p.size(); i++) if (n->ukernel->uparams[i].dir != VX_OUTPUT) ln.p.push_back(p[i]);
        out.push_back(std::move(ln));
        return VX_SUCCESS;
    }
    switch (n->kernel) {
    case VX_KERNEL_GAUSSIAN_3x3: add(LK::GAUSSIAN_U8_U8_3x3, {p[1], p[0]}); return VX_SUCCESS;   // :863
    case VX_KERNEL_SOBEL_3x3:                                                                      // :509
        if (p[1]) add(LK::SOBEL_S16_U8_3x3_GX, {p[1], p[0]});
        if (p[2]) add(LK::SOBEL_S16_U8_3x3_GY, {p[2], p[0]});
        return VX_SUCCESS;
    case VX_KERNEL_MAGNITUDE: add(LK::MAGNITUDE_S16_S16S16, {p[2], p[0], p[1]}); return VX_SUCCESS;
    case VX_KERNEL_CONVERTDEPTH: {                                                                 // :1166
        Image *i0 = IMG(p[0]);
        if (i0->format == VX_DF_IMAGE_U8) { add(LK::COLOR_DEPTH_S16_U8, {p[1], p[0], p[3]}); return VX_SUCCESS; }
        add(sc_enum(p[2]) == VX_CONVERT_POLICY_WRAP ? LK::COLOR_DEPTH_U8_S16_WRAP : LK::COLOR_DEPTH_U8_S16_SAT, {p[1], p[0], p[3]});
        return VX_SUCCESS;
    }
    case VX_KERNEL_THRESHOLD:                                                                          // :741
        add(static_cast<Threshold *>(p[1])->thresh_type == VX_THRESHOLD_TYPE_RANGE ? LK::THRESHOLD_U8_U8_RANGE
                                                                                 : LK::THRESHOLD_U8_U8_BINARY,
            {p[2], p[0], p[1]});
        return VX_SUCCESS;
    case VX_KERNEL_BOX_3x3: add(LK::BOX_U8_U8_3x3, {p[1], p[0]}); return VX_SUCCESS;                  // :849
    case VX_KERNEL_MEDIAN_3x3: add(LK::MEDIAN_U8_U8_3x3, {p[1], p[0]}); return VX_SUCCESS;            // :835
    case VX_KERNEL_DILATE_3x3: add(LK::DILATE_U8_U8_3x3, {p[1], p[0]}); return VX_SUCCESS;            // :786
    case VX_KERNEL_ERODE_3x3: add(LK::ERODE_U8_U8_3x3, {p[1], p[0]}); return VX_SUCCESS;              // :810
    case VX_KERNEL_NOT: add(LK::NOT_U8_U8, {p[1], p[0]}); return VX_SUCCESS;                          // :1293
    case VX_KERNEL_AND: add(LK::AND_U8_U8U8, {p[2], p[0], p[1]}); return VX_SUCCESS;                  // :1191
    case VX_KERNEL_OR: add(LK::OR_U8_U8U8, {p[2], p[0], p[1]}); return VX_SUCCESS;                    // :1225
    case VX_KERNEL_XOR: add(LK::XOR_U8_U8U8, {p[2], p[0], p[1]}); return VX_SUCCESS;                  // :1259
    case VX_KERNEL_ABSDIFF:                                                                            // :689
        add(IMG(p[2])->format == VX_DF_IMAGE_U8 ? LK::ABS_DIFF_U8_U8U8 : LK::ABS_DIFF_S16_S16S16_SAT, {p[2], p[0], p[1]});
        return VX_SUCCESS;
    case VX_KERNEL_ADD: case VX_KERNEL_SUBTRACT: {                                                     // :1386, :1428
        const vx_df_image fa = IMG(p[0])->format, fb = IMG(p[1])->format, fo = IMG(p[3])->format;
        const bool sat = sc_enum(p[2]) == VX_CONVERT_POLICY_SATURATE;
        const bool u8a = fa == VX_DF_IMAGE_U8, u8b = fb == VX_DF_IMAGE_U8;
        Ref *A = p[0], *B = p[1];
        LK k = LK::INVALID;
        if (n->kernel == VX_KERNEL_ADD) {
            if (fo == VX_DF_IMAGE_U8) k = sat ? LK::ADD_U8_U8U8_SAT : LK::ADD_U8_U8U8_WRAP;
            else if (u8a && u8b) k = LK::ADD_S16_U8U8;
            else if (u8a || u8b) {
                k = sat ? LK::ADD_S16_S16U8_SAT : LK::ADD_S16_S16U8_WRAP;
                if (u8a) std::swap(A, B);   // the S16 operand goes first
            } else k = sat ? LK::ADD_S16_S16S16_SAT : LK::ADD_S16_S16S16_WRAP;
        } else {
            if (fo == VX_DF_IMAGE_U8) k = sat ? LK::SUB_U8_U8U8_SAT : LK::SUB_U8_U8U8_WRAP;
            else if (u8a && u8b) k = LK::SUB_S16_U8U8;
            else if (u8b) k = sat ? LK::SUB_S16_S16U8_SAT : LK::SUB_S16_S16U8_WRAP;
            else if (u8a) k = sat ? LK::SUB_S16_U8S16_SAT : LK::SUB_S16_U8S16_WRAP;
            else k = sat ? LK::SUB_S16_S16S16_SAT : LK::SUB_S16_S16S16_WRAP;
        }
        add(k, {p[3], A, B});
        return VX_SUCCESS;
    }
    case VX_KERNEL_CANNY_EDGE_DETECTOR: {                                                              // :1618
        Image *i0 = IMG(p[0]);
        Array *stack = virt_array(g, kItemCoord2dU16, (vx_size)i0->width * i0->height);
        stack->item_size = 4;
        Image *sob = virt_image(g, i0->width, i0->height, VX_DF_IMAGE_U16);
        const int gs = sc_i32(p[2]);
        const bool l1 = sc_enum(p[3]) == VX_NORM_L1;
        const LK sobel = gs == 3 ? (l1 ? LK::CANNY_SOBEL_U16_U8_3x3_L1NORM : LK::CANNY_SOBEL_U16_U8_3x3_L2NORM)
                       : gs == 5 ? (l1 ? LK::CANNY_SOBEL_U16_U8_5x5_L1NORM : LK::CANNY_SOBEL_U16_U8_5x5_L2NORM)
                                 : (l1 ? LK::CANNY_SOBEL_U16_U8_7x7_L1NORM : LK::CANNY_SOBEL_U16_U8_7x7_L2NORM);
        add(sobel, {sob, p[0]});
        // 7x7 gradients use the suppression variant that quarters the thresholds (:1690)
        add(gs == 7 ? LK::CANNY_SUPP_THRESHOLD_U8XY_U16_7x7 : LK::CANNY_SUPP_THRESHOLD_U8XY_U16_3x3, {p[4], stack, sob, p[1], p[2]});
        add(LK::CANNY_EDGE_TRACE_U8_U8XY, {p[4], stack});
        return VX_SUCCESS;
    }
    case VX_KERNEL_HARRIS_CORNERS: {                                                                   // :1703
        Image *i0 = IMG(p[0]);
        Image *hg3 = virt_image(g, i0->width, i0->height, VX_DF_IMAGE('F', '3', '3', '2'));
        Image *hvc = virt_image(g, i0->width, i0->height, VX_DF_IMAGE_F32_AMD);
        Array *xys = virt_array(g, kItemKeypointXYS, (vx_size)i0->width * i0->height);
        xys->item_size = 8;
        Scalar *sw = virt_scalar(g, VX_TYPE_UINT32, i0->width), *sh = virt_scalar(g, VX_TYPE_UINT32, i0->height);
        const int32_t gs = sc_i32(p[4]), bs = sc_i32(p[5]);
        add(gs == 3 ? LK::HARRIS_SOBEL_HG3_U8_3x3 : gs == 5 ? LK::HARRIS_SOBEL_HG3_U8_5x5 : LK::HARRIS_SOBEL_HG3_U8_7x7,
            {hg3, p[0]});
        add(bs == 3 ? LK::HARRIS_SCORE_HVC_HG3_3x3 : bs == 5 ? LK::HARRIS_SCORE_HVC_HG3_5x5 : LK::HARRIS_SCORE_HVC_HG3_7x7,
            {hvc, hg3, p[3], p[1], p[4]});
        add(LK::NON_MAX_SUPP_XY_ANY_3x3, {xys, hvc});
        add(LK::HARRIS_MERGE_SORT_AND_PICK_XY_XYS, {p[6], p.size() > 7 ? p[7] : nullptr, xys, p[2], sw, sh});
        return VX_SUCCESS;
    }
    case VX_KERNEL_FAST_CORNERS: {                                                                     // :1789
        // {corners, num_corners, input, strength}; the suppression flag picks the kernel
        const bool sup = static_cast<Scalar *>(p[2])->v.i32 != 0;
        add(sup ? LK::FAST_CORNERS_XY_U8_SUPRESSION : LK::FAST_CORNERS_XY_U8_NOSUPRESSION,
            {p[3], p.size() > 4 ? p[4] : nullptr, p[0], p[1]});
        return VX_SUCCESS;
    }
    case VX_KERNEL_COLOR_CONVERT: {                                                                    // :200-256
        Image *o = IMG(p[1]);
        if (o->format == VX_DF_IMAGE_NV12) {
            add(LK::COLOR_CONVERT_Y_RGB, {o->children[0], p[0]});
            add(LK::COLOR_CONVERT_UV12_RGB, {o->children[1], p[0]});
        } else {
            add(LK::COLOR_CONVERT_Y_RGB, {o->children[0], p[0]});
            add(LK::COLOR_CONVERT_IU_RGB, {o->children[1], p[0]});
            add(LK::COLOR_CONVERT_IV_RGB, {o->children[2], p[0]});
        }
        return VX_SUCCESS;
    }
    case VX_KERNEL_CHANNEL_EXTRACT: {                                                                  // :342
        Image *i0 = IMG(p[0]);
        const int idx = channel_index(sc_enum(p[1]));
        const vx_df_image f = i0->format;
        static const LK u24[3] = {LK::CHANNEL_EXTRACT_U8_U24_POS0, LK::CHANNEL_EXTRACT_U8_U24_POS1, LK::CHANNEL_EXTRACT_U8_U24_POS2};
        static const LK u32[4] = {LK::CHANNEL_EXTRACT_U8_U32_POS0, LK::CHANNEL_EXTRACT_U8_U32_POS1, LK::CHANNEL_EXTRACT_U8_U32_POS2,
                                  LK::CHANNEL_EXTRACT_U8_U32_POS3};
        if (f == VX_DF_IMAGE_RGB) add(u24[idx], {p[2], p[0]});
        else if (f == VX_DF_IMAGE_RGBX) add(u32[idx], {p[2], p[0]});
        else if (f == VX_DF_IMAGE_NV12 || f == VX_DF_IMAGE_NV21) {
            if (idx == 0) add(LK::CHANNEL_COPY_U8_U8, {p[2], i0->children[0]});
            else add((idx == 1) == (f == VX_DF_IMAGE_NV12) ? LK::CHANNEL_EXTRACT_U8_U16_POS0 : LK::CHANNEL_EXTRACT_U8_U16_POS1,
                     {p[2], i0->children[1]});
        } else if (f == VX_DF_IMAGE_UYVY) {
            add(idx == 0 ? LK::CHANNEL_EXTRACT_U8_U16_POS1 : idx == 1 ? LK::CHANNEL_EXTRACT_U8_U32_POS0 : LK::CHANNEL_EXTRACT_U8_U32_POS2,
                {p[2], p[0]});
        } else if (f == VX_DF_IMAGE_YUYV) {
            add(idx == 0 ? LK::CHANNEL_EXTRACT_U8_U16_POS0 : idx == 1 ? LK::CHANNEL_EXTRACT_U8_U32_POS1 : LK::CHANNEL_EXTRACT_U8_U32_POS3,
                {p[2], p[0]});
        } else {
            add(LK::CHANNEL_COPY_U8_U8, {p[2], i0->children[idx]});
        }
        return VX_SUCCESS;
    }
    case VX_KERNEL_INTEGRAL_IMAGE: add(LK::INTEGRAL_IMAGE_U32_U8, {p[1], p[0]}); return VX_SUCCESS;     // :772
    case VX_KERNEL_HISTOGRAM: add(LK::HISTOGRAM_DATA_U8, {p[1], p[0]}); return VX_SUCCESS;             // :639
    case VX_KERNEL_CUSTOM_CONVOLUTION:                                                                 // :877
        add(IMG(p[2])->format == VX_DF_IMAGE_U8 ? LK::CONVOLVE_U8_U8 : LK::CONVOLVE_S16_U8, {p[2], p[0], p[1]});
        return VX_SUCCESS;
    case VX_KERNEL_TABLE_LOOKUP:                                                                       // :618
        add(IMG(p[0])->format == VX_DF_IMAGE_U8 ? LK::LUT_U8_U8 : LK::LUT_S16_S16, {p[2], p[0], p[1]});
        return VX_SUCCESS;
    case VX_KERNEL_CHANNEL_COMBINE: {                                                                  // :416
        Image *o = IMG(p[4]);
        const vx_df_image f = o->format;
        auto plane0 = [](Ref *r) -> Ref * { return IMG(r)->children.empty() ? r : (Ref *)IMG(r)->children[0]; };
        if (f == VX_DF_IMAGE_RGB) add(LK::CHANNEL_COMBINE_U24_U8U8U8_RGB, {p[4], p[0], p[1], p[2]});
        else if (f == VX_DF_IMAGE_RGBX) add(LK::CHANNEL_COMBINE_U32_U8U8U8U8_RGBX, {p[4], p[0], p[1], p[2], p[3]});
        else if (f == VX_DF_IMAGE_UYVY) add(LK::CHANNEL_COMBINE_U32_U8U8U8_UYVY, {p[4], p[0], p[1], p[2]});
        else if (f == VX_DF_IMAGE_YUYV) add(LK::CHANNEL_COMBINE_U32_U8U8U8_YUYV, {p[4], p[0], p[1], p[2]});
        else if (f == VX_DF_IMAGE_NV12 || f == VX_DF_IMAGE_NV21) {
            add(LK::CHANNEL_COPY_U8_U8, {o->children[0], plane0(p[0])});
            add(LK::CHANNEL_COMBINE_U16_U8U8, f == VX_DF_IMAGE_NV12 ? std::vector<Ref *>{o->children[1], p[1], p[2]}
                                                                     : std::vector<Ref *>{o->children[1], p[2], p[1]});
        } else {                                                    // IYUV, YUV4: plane copies
            for (int k = 0; k < 3; k++) add(LK::CHANNEL_COPY_U8_U8, {o->children[k], plane0(p[k])});
        }
        return VX_SUCCESS;
    }
    case VX_KERNEL_SCALE_IMAGE: {                                                                      // :563
        Image *i0 = IMG(p[0]), *o = IMG(p[1]);
        if (i0->width == o->width && i0->height == o->height) { add(LK::CHANNEL_COPY_U8_U8, {p[1], p[0]}); return VX_SUCCESS; }
        vx_enum t = sc_enum(p[2]);
        if (n->border.mode != VX_BORDER_UNDEFINED && t == VX_INTERPOLATION_BILINEAR) return VX_ERROR_NOT_SUPPORTED;
        LK k = t == VX_INTERPOLATION_NEAREST_NEIGHBOR ? LK::SCALE_IMAGE_U8_U8_NEAREST
             : t == VX_INTERPOLATION_BILINEAR ? LK::SCALE_IMAGE_U8_U8_BILINEAR : LK::SCALE_IMAGE_U8_U8_AREA;
        add(k, {p[1], p[0]});
        return VX_SUCCESS;
    }
    case VX_KERNEL_HALFSCALE_GAUSSIAN:
        add(LK::SCALE_GAUSSIAN_HALF_U8_U8_5x5, {p[1], p[0]});
        return VX_SUCCESS;
    case VX_KERNEL_WARP_AFFINE: case VX_KERNEL_WARP_PERSPECTIVE: {                                    // :1542
        const bool aff = n->kernel == VX_KERNEL_WARP_AFFINE;
        vx_enum t = sc_enum(p[2]);
        if (n->border.mode == VX_BORDER_CONSTANT) {
            Scalar *b = virt_scalar(g, VX_TYPE_UINT8, n->border.constant_value.U8);
            LK k = aff ? (t == VX_INTERPOLATION_BILINEAR ? LK::WARP_AFFINE_U8_U8_BILINEAR_CONSTANT : LK::WARP_AFFINE_U8_U8_NEAREST_CONSTANT)
                       : (t == VX_INTERPOLATION_BILINEAR ? LK::WARP_PERSPECTIVE_U8_U8_BILINEAR_CONSTANT : LK::WARP_PERSPECTIVE_U8_U8_NEAREST_CONSTANT);
            add(k, {p[3], p[0], p[1], b});
        } else if (n->border.mode == VX_BORDER_UNDEFINED) {
            LK k = aff ? (t == VX_INTERPOLATION_BILINEAR ? LK::WARP_AFFINE_U8_U8_BILINEAR : LK::WARP_AFFINE_U8_U8_NEAREST)
                       : (t == VX_INTERPOLATION_BILINEAR ? LK::WARP_PERSPECTIVE_U8_U8_BILINEAR : LK::WARP_PERSPECTIVE_U8_U8_NEAREST);
            add(k, {p[3], p[0], p[1]});
        } else {
            return VX_ERROR_NOT_SUPPORTED;
        }
        return VX_SUCCESS;
    }
    case VX_KERNEL_REMAP: {                                                                            // :1490
        const bool bl = sc_enum(p[2]) == VX_INTERPOLATION_BILINEAR;
        if (n->border.mode == VX_BORDER_CONSTANT) {
            Scalar *b = virt_scalar(g, VX_TYPE_UINT8, n->border.constant_value.U8);
            add(bl ? LK::REMAP_U8_U8_BILINEAR_CONSTANT : LK::REMAP_U8_U8_NEAREST_CONSTANT, {p[3], p[0], p[1], b});
        } else if (n->border.mode == VX_BORDER_UNDEFINED) {
            add(bl ? LK::REMAP_U8_U8_BILINEAR : LK::REMAP_U8_U8_NEAREST, {p[3], p[0], p[1]});
        } else {
            return VX_ERROR_NOT_SUPPORTED;
        }
        return VX_SUCCESS;
    }
    case VX_KERNEL_GAUSSIAN_PYRAMID: {                                                                 // :900
        Pyramid *py = static_cast<Pyramid *>(p[1]);
        Ref *next = p[0];
        for (vx_size l = 0; l < py->levels; l++) {
            add(l == 0 ? LK::CHANNEL_COPY_U8_U8 : LK::SCALE_GAUSSIAN_HALF_U8_U8_5x5, {py->level[l], next});
            next = py->level[l];
        }
        return VX_SUCCESS;
    }
    case VX_KERNEL_OPTICAL_FLOW_PYR_LK: {                                                              // :1810
        // AGO order: new points, old pyramid, new pyramid, old points, new estimates,
        //            termination, epsilon, num_iterations, use_initial_estimate, window
        add(LK::OPTICAL_FLOW_PYR_LK_XY_XY, {p[4], p[0], p[1], p[2], p[3], p[5], p[6], p[7], p[8], p[9]});
        return VX_SUCCESS;
    }
    default:
        return VX_ERROR_NOT_SUPPORTED;
    }
}

// ------------------------------------------------------------------------------------
// data usage bookkeeping
// ------------------------------------------------------------------------------------
static bool is_canny_supp(LK k)
{
    return k == LK::CANNY_SUPP_THRESHOLD_U8XY_U16_3x3 || k == LK::CANNY_SUPP_THRESHOLD_U8XY_U16_7x7;
}

static int num_outputs_k(LK k)
{
    switch (k) {
    case LK::SOBEL_S16S16_U8_3x3_GXY: case LK::COLOR_CONVERT_NV12_RGB: return 2;
    case LK::COLOR_CONVERT_IYUV_RGB: return 3;
    case LK::CANNY_SUPP_THRESHOLD_U8XY_U16_3x3: case LK::CANNY_SUPP_THRESHOLD_U8XY_U16_7x7: return 2;
    case LK::HARRIS_MERGE_SORT_AND_PICK_XY_XYS: return 2;
    case LK::FAST_CORNERS_XY_U8_SUPRESSION: case LK::FAST_CORNERS_XY_U8_NOSUPRESSION: return 2;
    default: return 1;
    }
}

static int num_outputs(const LNode &ln) { return ln.nout >= 0 ? ln.nout : num_outputs_k(ln.k); }

bool lnode_is_output(const LNode &ln, size_t i) { return (int)i < num_outputs(ln); }

// the root data object a reference aliases (planes alias their image, levels their pyramid)
static Ref *root_of(Ref *r)
{
    if (r && r->type == VX_TYPE_IMAGE && IMG(r)->parent) return IMG(r)->parent;
    return r;
}

static int input_uses(Graph *g, Ref *d, const LNode *except_a = nullptr, const LNode *except_b = nullptr)
{
    int n = 0;
    for (const LNode &ln : g->lnodes) {
        if (ln.removed || &ln == except_a || &ln == except_b) continue;
        for (size_t i = num_outputs(ln); i < ln.p.size(); i++) if (ln.p[i] == d) n++;
        // Canny edge trace reads-modifies-writes its image; the stack is its input
        if (ln.k == LK::CANNY_EDGE_TRACE_U8_U8XY && ln.p[0] == d) n++;
    }
    // pyramids used whole (optical flow) keep their levels alive
    for (const LNode &ln : g->lnodes) {
        if (ln.removed || ln.k != LK::OPTICAL_FLOW_PYR_LK_XY_XY) continue;
        for (int i : {1, 2}) {
            Pyramid *py = static_cast<Pyramid *>(ln.p[i]);
            for (Image *lv : py->level) if (lv == d) n++;
        }
    }
    return n;
}

// ------------------------------------------------------------------------------------
// merge rules (ago/ago_drama_remove.cpp:38-) and copy / unused-output removal
// ------------------------------------------------------------------------------------
static bool merge_pass(Graph *g)
{
    auto &L = g->lnodes;
    for (size_t i = 0; i < L.size(); i++) {
        if (L[i].removed) continue;
        for (size_t j = 0; j < L.size(); j++) {
            if (j == i || L[j].removed) continue;
            LNode &a = L[i], &b = L[j];
            // SOBEL GX + GY = GXY (:147)
            if (a.k == LK::SOBEL_S16_U8_3x3_GX && b.k == LK::SOBEL_S16_U8_3x3_GY && a.p[1] == b.p[1]) {
                a.k = LK::SOBEL_S16S16_U8_3x3_GXY;
                a.p = {a.p[0], b.p[0], a.p[1]};
                b.removed = true;
                return true;
            }
            // SOBEL + MAGNITUDE = SOBEL_MAGNITUDE (:165) when gx/gy are virtual and solitary
            if (a.k == LK::SOBEL_S16S16_U8_3x3_GXY && b.k == LK::MAGNITUDE_S16_S16S16 && b.p[1] == a.p[0] && b.p[2] == a.p[1] &&
                a.p[0]->is_virtual && a.p[1]->is_virtual && input_uses(g, a.p[0], &b) == 0 && input_uses(g, a.p[1], &b) == 0) {
                a.k = LK::SOBEL_MAGNITUDE_S16_U8_3x3;
                a.p = {b.p[0], a.p[2]};
                a.border = b.border;
                b.removed = true;
                return true;
            }
            // RGB to NV12 (:49)
            if (a.k == LK::COLOR_CONVERT_Y_RGB && b.k == LK::COLOR_CONVERT_UV12_RGB && a.p[1] == b.p[1]) {
                a.k = LK::COLOR_CONVERT_NV12_RGB;
                a.p = {a.p[0], b.p[0], a.p[1]};
                b.removed = true;
                return true;
            }
            // RGB to IYUV (:58)
            if (a.k == LK::COLOR_CONVERT_Y_RGB && b.k == LK::COLOR_CONVERT_IU_RGB && a.p[1] == b.p[1]) {
                for (size_t k = 0; k < L.size(); k++) {
                    LNode &c = L[k];
                    if (k == i || k == j || c.removed || c.k != LK::COLOR_CONVERT_IV_RGB || c.p[1] != a.p[1]) continue;
                    a.k = LK::COLOR_CONVERT_IYUV_RGB;
                    a.p = {a.p[0], b.p[0], c.p[0], a.p[1]};
                    b.removed = c.removed = true;
                    return true;
                }
            }
        }
    }
    return false;
}

static void replace_data(Graph *g, Ref *from, Ref *to)
{
    g->replaced[from] = to;
    for (auto &kv : g->replaced) if (kv.second == from) kv.second = to;
    for (LNode &ln : g->lnodes)
        for (Ref *&r : ln.p) if (r == from) r = to;
}

static bool remove_copy_pass(Graph *g)
{
    // a copy into a virtual image is replaced by its source (ago_drama_remove.cpp:926)
    for (LNode &ln : g->lnodes) {
        if (ln.removed || ln.k != LK::CHANNEL_COPY_U8_U8) continue;
        Ref *dst = ln.p[0], *src = ln.p[1];
        if (dst->is_virtual && !IMG(dst)->parent) {
            ln.removed = true;
            replace_data(g, dst, src);
            return true;
        }
    }
    return false;
}

static bool remove_unused_pass(Graph *g)
{
    for (LNode &ln : g->lnodes) {
        if (ln.removed) continue;
        bool all_unused = true;
        for (int i = 0; i < num_outputs(ln); i++) {
            Ref *o = ln.p[i];
            if (!o) continue;
            Ref *root = root_of(o);
            if (!o->is_virtual || input_uses(g, o) > 0) { all_unused = false; break; }
            if (root != o) {   // a plane of a multi-plane virtual image: any plane used keeps it
                for (Image *c : IMG(root)->children) if (input_uses(g, c) > 0) all_unused = false;
                if (input_uses(g, root) > 0) all_unused = false;
            }
        }
        if (ln.k == LK::CANNY_EDGE_TRACE_U8_U8XY || ln.k == LK::OPTICAL_FLOW_PYR_LK_XY_XY) {
            if (!ln.p[0]->is_virtual || input_uses(g, ln.p[0]) > 0) all_unused = false;
        }
        if (all_unused) { ln.removed = true; return true; }
    }
    return false;
}

// topological order with hierarchical levels (ago/ago_drama.cpp:287)
static vx_status sort_lnodes(Graph *g)
{
    auto &L = g->lnodes;
    std::vector<LNode> live;
    for (LNode &ln : L) if (!ln.removed) live.push_back(ln);
    const size_t n = live.size();
    std::vector<int> level(n, -1);
    // writer of each data object
    std::map<Ref *, int> writer;
    for (size_t i = 0; i < n; i++)
        for (int k = 0; k < num_outputs(live[i]); k++) {
            Ref *o = live[i].p[k];
            if (!o) continue;
            if (writer.count(o) && live[i].k != LK::CANNY_EDGE_TRACE_U8_U8XY && !is_canny_supp(live[writer[o]].k))
                return VX_ERROR_MULTIPLE_WRITERS;
            // edge trace updates the image written by suppression: it runs after it
            if (!writer.count(o) || live[i].k == LK::CANNY_EDGE_TRACE_U8_U8XY) writer[o] = (int)i;
        }
    std::function<int(size_t, int)> lev = [&](size_t i, int depth) -> int {
        if (depth > (int)n + 1) return -2;
        if (level[i] >= 0) return level[i];
        int lv = 0;
        for (size_t k = num_outputs(live[i]); k < live[i].p.size(); k++) {
            Ref *d = live[i].p[k];
            if (!d) continue;
            std::vector<Ref *> deps{d};
            if (d->type == VX_TYPE_PYRAMID) for (Image *lvimg : static_cast<Pyramid *>(d)->level) deps.push_back(lvimg);
            for (Ref *x : deps) {
                auto it = writer.find(x);
                if (it == writer.end() || it->second == (int)i) continue;
                int l = lev(it->second, depth + 1);
                if (l < 0) return -2;
                lv = std::max(lv, l + 1);
            }
        }
        if (live[i].k == LK::CANNY_EDGE_TRACE_U8_U8XY) {
            for (size_t j = 0; j < n; j++)
                if (is_canny_supp(live[j].k) && live[j].p[0] == live[i].p[0]) {
                    int l = lev(j, depth + 1);
                    if (l < 0) return -2;
                    lv = std::max(lv, l + 1);
                }
        }
        return level[i] = lv;
    };
    for (size_t i = 0; i < n; i++) if (lev(i, 0) < 0) return VX_ERROR_INVALID_GRAPH;   // cycle
    std::vector<size_t> order(n);
    for (size_t i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return level[a] < level[b]; });
    std::vector<LNode> sorted;
    for (size_t i : order) { live[i].level = level[i]; sorted.push_back(live[i]); }
    L.swap(sorted);
    return VX_SUCCESS;
}

vx_status lower_graph(Graph *g)
{
    g->lnodes.clear();
    g->replaced.clear();
    graph_release_owned(g);       // the previous lowering's virtual data (no plan names it any more)
    for (Node *n : g->nodes) {
        if (n->removed) continue;
        vx_status s = validate_node(g, n);
        if (s) { log_error(n, s, "ERROR: vxVerifyGraph: node validation failed (%d)\n", s); return s; }
        s = divide_node(g, n, g->lnodes);
        if (s) { log_error(n, s, "ERROR: vxVerifyGraph: node is not supported by the B200 target (%d)\n", s); return s; }
    }
    for (bool changed = true; changed;) {
        changed = false;
        if (!(g->optimizer_flags & kOptNoRemoveCopy) && remove_copy_pass(g)) { changed = true; continue; }
        if (!(g->optimizer_flags & kOptNoRemoveUnused) && remove_unused_pass(g)) { changed = true; continue; }
        if (!(g->optimizer_flags & kOptNoMerge) && merge_pass(g)) { changed = true; continue; }
    }
    return sort_lnodes(g);
}

// ------------------------------------------------------------------------------------
// valid rectangles (ago/ago_interface.cpp:1734 + each kernel's valid_rect_callback)
// ------------------------------------------------------------------------------------
static void shrink_from(Image *out, const Image *in, uint32_t n)
{
    const uint32_t w = out->width, h = out->height;
    out->valid.start_x = std::min(in->valid.start_x + n, w);
    out->valid.start_y = std::min(in->valid.start_y + n, h);
    out->valid.end_x = (uint32_t)std::max((int)in->valid.end_x - (int)n, 0);
    out->valid.end_y = (uint32_t)std::max((int)in->valid.end_y - (int)n, 0);
}

static void copy_rect(Image *out, const Image *in) { out->valid = in->valid; }

static void scale_rect(Image *a, Image *b)
{
    // ago_kernel_api.cpp:19956 (Bilinear), :20558 (Area), :19847 (Nearest): the callback
    // reads paramList[0] (the destination) as its "input" and writes paramList[1] (the
    // source) -- kept as the reference does it.
    const float wo = (float)b->width, ho = (float)b->height, wi = (float)a->width, hi = (float)a->height;
    vx_rectangle_t r;
    r.start_x = (uint32_t)(((a->valid.start_x + 0.5f) * wo / wi) - 0.5f);
    r.start_y = (uint32_t)(((a->valid.start_y + 0.5f) * ho / hi) - 0.5f);
    r.end_x = (uint32_t)(((a->valid.end_x + 0.5f) * wo / wi) - 0.5f);
    r.end_y = (uint32_t)(((a->valid.end_y + 0.5f) * ho / hi) - 0.5f);
    b->valid = r;
}

vx_status propagate_valid_rects(Graph *g)
{
    for (LNode &ln : g->lnodes) {
        auto I = [&](int i) { return IMG(ln.p[i]); };
        switch (ln.k) {
        case LK::GAUSSIAN_U8_U8_3x3: case LK::SOBEL_S16_U8_3x3_GX: case LK::SOBEL_S16_U8_3x3_GY:
        case LK::SOBEL_MAGNITUDE_S16_U8_3x3: case LK::CANNY_SOBEL_U16_U8_3x3_L1NORM: case LK::CANNY_SOBEL_U16_U8_3x3_L2NORM:
        case LK::HARRIS_SOBEL_HG3_U8_3x3: case LK::HARRIS_SCORE_HVC_HG3_3x3:
            shrink_from(I(0), I(1), 1); break;
        case LK::SOBEL_S16S16_U8_3x3_GXY:
            // ago_kernel_api.cpp:16154 clamps with the input's size
            shrink_from(I(0), I(2), 1); shrink_from(I(1), I(2), 1); break;
        case LK::CANNY_SOBEL_U16_U8_5x5_L1NORM: case LK::CANNY_SOBEL_U16_U8_5x5_L2NORM:   // :17701
        case LK::HARRIS_SOBEL_HG3_U8_5x5: case LK::HARRIS_SCORE_HVC_HG3_5x5:            // :16850, :17046
            shrink_from(I(0), I(1), 2); break;
        case LK::HARRIS_SOBEL_HG3_U8_7x7: case LK::HARRIS_SCORE_HVC_HG3_7x7:
            shrink_from(I(0), I(1), 3); break;
        case LK::CANNY_SOBEL_U16_U8_7x7_L1NORM: case LK::CANNY_SOBEL_U16_U8_7x7_L2NORM:
            shrink_from(I(0), I(1), 3); break;
        case LK::CANNY_SUPP_THRESHOLD_U8XY_U16_3x3: case LK::CANNY_SUPP_THRESHOLD_U8XY_U16_7x7: shrink_from(I(0), I(2), 1); break;
        case LK::MAGNITUDE_S16_S16S16: {
            Image *o = I(0), *a = I(1), *b = I(2);
            o->valid = vx_rectangle_t{std::max(a->valid.start_x, b->valid.start_x), std::max(a->valid.start_y, b->valid.start_y),
                                      std::min(a->valid.end_x, b->valid.end_x), std::min(a->valid.end_y, b->valid.end_y)};
            break;
        }
        case LK::COLOR_DEPTH_U8_S16_SAT: case LK::COLOR_DEPTH_U8_S16_WRAP: case LK::COLOR_DEPTH_S16_U8:
        case LK::THRESHOLD_U8_U8_BINARY: case LK::CHANNEL_COPY_U8_U8:
        case LK::THRESHOLD_U8_U8_RANGE: case LK::NOT_U8_U8: case LK::LUT_U8_U8: case LK::LUT_S16_S16:
        case LK::INTEGRAL_IMAGE_U32_U8:
        case LK::CHANNEL_EXTRACT_U8_U16_POS0: case LK::CHANNEL_EXTRACT_U8_U16_POS1: case LK::CHANNEL_EXTRACT_U8_U24_POS0:
        case LK::CHANNEL_EXTRACT_U8_U24_POS1: case LK::CHANNEL_EXTRACT_U8_U24_POS2: case LK::CHANNEL_EXTRACT_U8_U32_POS0:
        case LK::CHANNEL_EXTRACT_U8_U32_POS1: case LK::CHANNEL_EXTRACT_U8_U32_POS2: case LK::CHANNEL_EXTRACT_U8_U32_POS3:
        case LK::CHANNEL_COMBINE_U32_U8U8U8_UYVY: case LK::CHANNEL_COMBINE_U32_U8U8U8_YUYV:   // :11847 (first input)
            copy_rect(I(0), I(1)); break;
        case LK::CHANNEL_COMBINE_U16_U8U8: case LK::CHANNEL_COMBINE_U24_U8U8U8_RGB: case LK::CHANNEL_COMBINE_U32_U8U8U8U8_RGBX: {
            Image *o = I(0);                                     // :11693, :11767: intersection of the inputs
            o->valid = I(1)->valid;
            for (size_t k = 2; k < ln.p.size(); k++) {
                const vx_rectangle_t &r = I((int)k)->valid;
                o->valid = vx_rectangle_t{std::max(o->valid.start_x, r.start_x), std::max(o->valid.start_y, r.start_y),
                                          std::min(o->valid.end_x, r.end_x), std::min(o->valid.end_y, r.end_y)};
            }
            break;
        }
        case LK::BOX_U8_U8_3x3: case LK::DILATE_U8_U8_3x3: case LK::ERODE_U8_U8_3x3: case LK::MEDIAN_U8_U8_3x3:
            shrink_from(I(0), I(1), 1); break;                  // e.g. :15033 (Box)
        case LK::CONVOLVE_U8_U8: case LK::CONVOLVE_S16_U8: {   // :15654: columns / 2 and rows / 2
            Image *o = I(0);
            const Image *in = I(1);
            const Convolution *cv = static_cast<const Convolution *>(ln.p[2]);
            const uint32_t M = (uint32_t)cv->columns >> 1, N = (uint32_t)cv->rows >> 1;
            o->valid.start_x = std::min(in->valid.start_x + M, o->width);
            o->valid.start_y = std::min(in->valid.start_y + N, o->height);
            o->valid.end_x = (uint32_t)std::max((int)in->valid.end_x - (int)M, 0);
            o->valid.end_y = (uint32_t)std::max((int)in->valid.end_y - (int)N, 0);
            break;
        }
        case LK::ABS_DIFF_U8_U8U8: case LK::ABS_DIFF_S16_S16S16_SAT:
        case LK::ADD_U8_U8U8_WRAP: case LK::ADD_U8_U8U8_SAT: case LK::ADD_S16_U8U8: case LK::ADD_S16_S16U8_WRAP:
        case LK::ADD_S16_S16U8_SAT: case LK::ADD_S16_S16S16_WRAP: case LK::ADD_S16_S16S16_SAT:
        case LK::SUB_U8_U8U8_WRAP: case LK::SUB_U8_U8U8_SAT: case LK::SUB_S16_U8U8: case LK::SUB_S16_S16U8_WRAP:
        case LK::SUB_S16_S16U8_SAT: case LK::SUB_S16_U8S16_WRAP: case LK::SUB_S16_U8S16_SAT:
        case LK::SUB_S16_S16S16_WRAP: case LK::SUB_S16_S16S16_SAT:
        case LK::AND_U8_U8U8: case LK::OR_U8_U8U8: case LK::XOR_U8_U8U8: {   // e.g. :4514 (Add_U8_U8U8_Wrap)
            Image *o = I(0), *a = I(1), *b = I(2);
            o->valid = vx_rectangle_t{std::max(a->valid.start_x, b->valid.start_x), std::max(a->valid.start_y, b->valid.start_y),
                                      std::min(a->valid.end_x, b->valid.end_x), std::min(a->valid.end_y, b->valid.end_y)};
            break;
        }
        case LK::COLOR_CONVERT_NV12_RGB: {                      // :13953
            Image *in = I(2);
            copy_rect(I(0), in);
            I(1)->valid = vx_rectangle_t{(in->valid.start_x + 1) >> 1, (in->valid.start_y + 1) >> 1,
                                         (in->valid.end_x + 1) >> 1, (in->valid.end_y + 1) >> 1};
            break;
        }
        case LK::COLOR_CONVERT_IYUV_RGB: {                      // :13506
            Image *in = I(3);
            copy_rect(I(0), in);
            for (int c = 1; c <= 2; c++)
                I(c)->valid = vx_rectangle_t{(in->valid.start_x + 1) >> 1, (in->valid.start_y + 1) >> 1,
                                             in->valid.end_x >> 1, in->valid.end_y >> 1};
            break;
        }
        case LK::SCALE_IMAGE_U8_U8_NEAREST: case LK::SCALE_IMAGE_U8_U8_BILINEAR: case LK::SCALE_IMAGE_U8_U8_AREA:
            scale_rect(I(0), I(1)); break;
        case LK::SCALE_GAUSSIAN_HALF_U8_U8_5x5: {               // :15477
            Image *o = I(0), *in = I(1);
            o->valid = vx_rectangle_t{std::min((in->valid.start_x + 1) >> 1, o->width), std::min((in->valid.start_y + 1) >> 1, o->height),
                                      (in->valid.end_x + 1) >> 1, (in->valid.end_y + 1) >> 1};
            break;
        }
        case LK::USER_KERNEL:                                  // AGO_KERNEL_FLAG_VALID_RECT_RESET (vx_api.cpp:2601)
            for (int i = 0; i < ln.nout; i++)
                if (ln.p[i] && ln.p[i]->type == VX_TYPE_IMAGE) I(i)->valid = vx_rectangle_t{0, 0, I(i)->width, I(i)->height};
            break;
        default: break;   // no callback in the reference: the output keeps its rectangle
        }
    }
    // multi-plane images report the rectangle of plane 0
    for (LNode &ln : g->lnodes)
        for (int i = 0; i < num_outputs(ln); i++)
            if (ln.p[i] && ln.p[i]->type == VX_TYPE_IMAGE && IMG(ln.p[i])->parent && IMG(ln.p[i])->parent->children[0] == ln.p[i])
                IMG(ln.p[i])->parent->valid = IMG(ln.p[i])->valid;
    return VX_SUCCESS;
}

}  // namespace agovx
