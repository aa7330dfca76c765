// gdf.cpp -- graph import from AGO's text graph description (GDF), the format runvx and
// vxSetGraphAttribute(VX_GRAPH_ATTRIBUTE_AMD_IMPORT_FROM_TEXT) read
// (ago/ago_interface.cpp:456 agoReadGraphFromStringInternal; data descriptions
// ago/ago_util.cpp:1026-1760 agoCreateDataFromDescription).
//
// Supported statements: `data <name> = <description>` and `node <kernel> <args...>`, with
// `#` comments.  Descriptions: image / image-virtual (FORMAT,W,H as the library reads them,
// or runvx's W,H,FORMAT), pyramid / pyramid-virtual (FORMAT,W,H,levels,scale or
// levels,scale,W,H,FORMAT), array / array-virtual (TYPE,capacity), scalar (TYPE,value),
// threshold (BINARY|RANGE,in,out[:INIT,v[,v2]]; formats as codes or numbers), matrix
// (TYPE,columns,rows[:INIT,{a;b;...}]), lut (TYPE,count), distribution (bins,offset,range).
// INIT values are applied here (the reference library leaves them to the application's
// data-registry callback, which still receives them).  A description's trailing
// `:<params>` (runvx's READ/WRITE/INIT requests) goes to the data-registry callback, as in
// the reference.  Node arguments: data names, `null`, `!ENUM_NAME` (an enum scalar, e.g.
// !CHANNEL_Y, !NORM_L1), `$N` (the N-th reference passed in AgoGraphImportInfo), and
// `attr:BORDER_MODE:UNDEFINED|REPLICATE|CONSTANT,<value>`.  Macros, loops, conditionals,
// sub-graph files and the AMD low-level kernel names are not read (an error is logged).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>

#include "vx_internal.h"

namespace agovx {

Node *graph_add_node(Graph *g, vx_enum kernel, const std::vector<Ref *> &params);
Image *make_image(Context *ctx, Graph *scope, uint32_t w, uint32_t h, vx_df_image fmt, bool virt);
Array *make_array(Context *ctx, Graph *scope, vx_enum item_type, vx_size capacity, bool virt);
Scalar *make_scalar(Context *ctx, Graph *scope, vx_enum type, const void *ptr);
vx_size type_size(vx_enum t);

namespace {

struct NamedEnum { const char *name; vx_enum value; };

// Enum names a GDF writes (with or without the VX_ prefix; ago_util.cpp agoName2Enum)
const NamedEnum kEnums[] = {
    {"TYPE_INT8", VX_TYPE_INT8}, {"TYPE_UINT8", VX_TYPE_UINT8}, {"TYPE_INT16", VX_TYPE_INT16},
    {"TYPE_UINT16", VX_TYPE_UINT16}, {"TYPE_INT32", VX_TYPE_INT32}, {"TYPE_UINT32", VX_TYPE_UINT32},
    {"TYPE_INT64", VX_TYPE_INT64}, {"TYPE_UINT64", VX_TYPE_UINT64}, {"TYPE_FLOAT32", VX_TYPE_FLOAT32},
    {"TYPE_FLOAT64", VX_TYPE_FLOAT64}, {"TYPE_ENUM", VX_TYPE_ENUM}, {"TYPE_SIZE", VX_TYPE_SIZE},
    {"TYPE_DF_IMAGE", VX_TYPE_DF_IMAGE}, {"TYPE_BOOL", VX_TYPE_BOOL}, {"TYPE_KEYPOINT", VX_TYPE_KEYPOINT},
    {"TYPE_COORDINATES2D", VX_TYPE_COORDINATES2D}, {"TYPE_COORDINATES2DF", VX_TYPE_COORDINATES2DF},
    {"TYPE_RECTANGLE", VX_TYPE_RECTANGLE},
    {"CHANNEL_0", VX_CHANNEL_0}, {"CHANNEL_1", VX_CHANNEL_1}, {"CHANNEL_2", VX_CHANNEL_2}, {"CHANNEL_3", VX_CHANNEL_3},
    {"CHANNEL_R", VX_CHANNEL_R}, {"CHANNEL_G", VX_CHANNEL_G}, {"CHANNEL_B", VX_CHANNEL_B}, {"CHANNEL_A", VX_CHANNEL_A},
    {"CHANNEL_Y", VX_CHANNEL_Y}, {"CHANNEL_U", VX_CHANNEL_U}, {"CHANNEL_V", VX_CHANNEL_V},
    {"NORM_L1", VX_NORM_L1}, {"NORM_L2", VX_NORM_L2},
    {"CONVERT_POLICY_WRAP", VX_CONVERT_POLICY_WRAP}, {"CONVERT_POLICY_SATURATE", VX_CONVERT_POLICY_SATURATE},
    {"INTERPOLATION_NEAREST_NEIGHBOR", VX_INTERPOLATION_NEAREST_NEIGHBOR},
    {"INTERPOLATION_BILINEAR", VX_INTERPOLATION_BILINEAR}, {"INTERPOLATION_AREA", VX_INTERPOLATION_AREA},
    {"TERM_CRITERIA_ITERATIONS", VX_TERM_CRITERIA_ITERATIONS}, {"TERM_CRITERIA_EPSILON", VX_TERM_CRITERIA_EPSILON},
    {"TERM_CRITERIA_BOTH", VX_TERM_CRITERIA_BOTH},
    {"THRESHOLD_TYPE_BINARY", VX_THRESHOLD_TYPE_BINARY}, {"THRESHOLD_TYPE_RANGE", VX_THRESHOLD_TYPE_RANGE},
    {"BINARY", VX_THRESHOLD_TYPE_BINARY}, {"RANGE", VX_THRESHOLD_TYPE_RANGE},
    {"BORDER_UNDEFINED", VX_BORDER_UNDEFINED}, {"BORDER_CONSTANT", VX_BORDER_CONSTANT},
    {"BORDER_REPLICATE", VX_BORDER_REPLICATE},
    // the reference's own short names (ago_util.cpp name table)
    {"WRAP", VX_CONVERT_POLICY_WRAP}, {"SATURATE", VX_CONVERT_POLICY_SATURATE},
    {"NEAREST_NEIGHBOR", VX_INTERPOLATION_NEAREST_NEIGHBOR}, {"BILINEAR", VX_INTERPOLATION_BILINEAR},
    {"AREA", VX_INTERPOLATION_AREA}, {"CRITERIA_ITERATIONS", VX_TERM_CRITERIA_ITERATIONS},
    {"CRITERIA_EPSILON", VX_TERM_CRITERIA_EPSILON}, {"CRITERIA_BOTH", VX_TERM_CRITERIA_BOTH},
    {"BORDER_MODE_UNDEFINED", VX_BORDER_UNDEFINED}, {"BORDER_MODE_REPLICATE", VX_BORDER_REPLICATE},
    {"BORDER_MODE_CONSTANT", VX_BORDER_CONSTANT},
    // short type names of descriptions (array:KEYPOINT, scalar:FLOAT32, ...)
    {"INT8", VX_TYPE_INT8}, {"UINT8", VX_TYPE_UINT8}, {"INT16", VX_TYPE_INT16}, {"UINT16", VX_TYPE_UINT16},
    {"INT32", VX_TYPE_INT32}, {"UINT32", VX_TYPE_UINT32}, {"INT64", VX_TYPE_INT64}, {"UINT64", VX_TYPE_UINT64},
    {"FLOAT32", VX_TYPE_FLOAT32}, {"FLOAT64", VX_TYPE_FLOAT64}, {"ENUM", VX_TYPE_ENUM}, {"SIZE", VX_TYPE_SIZE},
    {"DF_IMAGE", VX_TYPE_DF_IMAGE}, {"BOOL", VX_TYPE_BOOL}, {"KEYPOINT", VX_TYPE_KEYPOINT},
    {"COORDINATES2D", VX_TYPE_COORDINATES2D}, {"COORDINATES2DF", VX_TYPE_COORDINATES2DF},
    {"RECTANGLE", VX_TYPE_RECTANGLE},
};

const NamedEnum kKernels[] = {
    {"color_convert", VX_KERNEL_COLOR_CONVERT}, {"channel_extract", VX_KERNEL_CHANNEL_EXTRACT},
    {"channel_combine", VX_KERNEL_CHANNEL_COMBINE}, {"sobel_3x3", VX_KERNEL_SOBEL_3x3},
    {"magnitude", VX_KERNEL_MAGNITUDE}, {"scale_image", VX_KERNEL_SCALE_IMAGE},
    {"table_lookup", VX_KERNEL_TABLE_LOOKUP}, {"histogram", VX_KERNEL_HISTOGRAM}, {"absdiff", VX_KERNEL_ABSDIFF},
    {"threshold", VX_KERNEL_THRESHOLD}, {"integral_image", VX_KERNEL_INTEGRAL_IMAGE},
    {"dilate_3x3", VX_KERNEL_DILATE_3x3}, {"erode_3x3", VX_KERNEL_ERODE_3x3}, {"median_3x3", VX_KERNEL_MEDIAN_3x3},
    {"box_3x3", VX_KERNEL_BOX_3x3}, {"gaussian_3x3", VX_KERNEL_GAUSSIAN_3x3},
    {"gaussian_pyramid", VX_KERNEL_GAUSSIAN_PYRAMID}, {"convertdepth", VX_KERNEL_CONVERTDEPTH},
    {"canny_edge_detector", VX_KERNEL_CANNY_EDGE_DETECTOR}, {"and", VX_KERNEL_AND}, {"or", VX_KERNEL_OR},
    {"xor", VX_KERNEL_XOR}, {"not", VX_KERNEL_NOT}, {"add", VX_KERNEL_ADD}, {"subtract", VX_KERNEL_SUBTRACT},
    {"warp_affine", VX_KERNEL_WARP_AFFINE}, {"warp_perspective", VX_KERNEL_WARP_PERSPECTIVE},
    {"harris_corners", VX_KERNEL_HARRIS_CORNERS}, {"optical_flow_pyr_lk", VX_KERNEL_OPTICAL_FLOW_PYR_LK},
    {"fast_corners", VX_KERNEL_FAST_CORNERS},
    {"remap", VX_KERNEL_REMAP}, {"halfscale_gaussian", VX_KERNEL_HALFSCALE_GAUSSIAN},
};

bool enum_by_name(std::string n, vx_enum &v)
{
    if (n.compare(0, 3, "VX_") == 0) n = n.substr(3);
    for (const NamedEnum &e : kEnums)
        if (n == e.name) { v = e.value; return true; }
    return false;
}

std::vector<std::string> split(const std::string &s, char sep)
{
    std::vector<std::string> out;
    std::string cur;
    for (char ch : s) {
        if (ch == sep) { out.push_back(cur); cur.clear(); }
        else cur += ch;
    }
    out.push_back(cur);
    return out;
}

bool to_u32(const std::string &s, uint32_t &v)
{
    char *end = nullptr;
    const unsigned long x = strtoul(s.c_str(), &end, 0);
    if (s.empty() || *end) return false;
    v = (uint32_t)x;
    return true;
}

vx_df_image fourcc(const std::string &s)
{
    return s.size() == 4 ? (vx_df_image)VX_DF_IMAGE(s[0], s[1], s[2], s[3]) : 0;
}

struct Importer {
    Graph *g;
    Context *c;
    const AgoGraphImportInfo *info;
    std::map<std::string, Ref *> names;
    int lineno = 0;
    std::string line;

    vx_status fail(vx_status st, const char *what)
    {
        log_error(g, st, "ERROR: agoReadGraph: line %d: %s\n>>>> %s\n", lineno, what, line.c_str());
        return st;
    }

    // W,H,FORMAT (runvx order) or FORMAT,W,H
    bool image_config(const std::vector<std::string> &f, uint32_t &w, uint32_t &h, vx_df_image &fmt)
    {
        if (f.size() != 3) return false;
        if (f[0].size() == 4 && !isdigit((unsigned char)f[0][0])) return (fmt = fourcc(f[0])) && to_u32(f[1], w) && to_u32(f[2], h);
        return to_u32(f[0], w) && to_u32(f[1], h) && (fmt = fourcc(f[2]));
    }

    Ref *make_data(const std::string &desc, std::string &app_params, vx_status &err)
    {
        err = VX_ERROR_NOT_SUPPORTED;
        const size_t c1 = desc.find(':');
        if (c1 == std::string::npos) return nullptr;
        std::string kind = desc.substr(0, c1), rest = desc.substr(c1 + 1), extra;
        const size_t c2 = rest.find(':');
        if (c2 != std::string::npos) { extra = rest.substr(c2 + 1); rest = rest.substr(0, c2); }
        app_params = extra;
        bool virt = false;
        const std::string vsuf = "-virtual";
        if (kind.size() > vsuf.size() && kind.compare(kind.size() - vsuf.size(), vsuf.size(), vsuf) == 0) {
            virt = true;
            kind = kind.substr(0, kind.size() - vsuf.size());
        }
        const std::vector<std::string> f = split(rest, ',');
        std::vector<std::string> init;
        if (extra.compare(0, 5, "INIT,") == 0) init = split(extra.substr(5), ',');
        err = VX_ERROR_INVALID_PARAMETERS;
        if (kind == "image") {
            uint32_t w, h;
            vx_df_image fmt;
            if (!image_config(f, w, h, fmt)) return nullptr;
            if (virt) return (Ref *)vxCreateVirtualImage((vx_graph)g, w, h, fmt);
            return (Ref *)vxCreateImage((vx_context)c, w, h, fmt);
        }
        if (kind == "pyramid") {   // FORMAT,W,H,levels,scale (library form) or levels,scale,W,H,FORMAT (runvx)
            if (f.size() != 5) return nullptr;
            const bool fmt_first = f[0].size() == 4 && !isdigit((unsigned char)f[0][0]);
            const std::string &sl = fmt_first ? f[3] : f[0], &ss = fmt_first ? f[4] : f[1];
            const std::string &sw = fmt_first ? f[1] : f[2], &sh = fmt_first ? f[2] : f[3], &sf = fmt_first ? f[0] : f[4];
            uint32_t levels, w, h;
            if (!to_u32(sl, levels) || !to_u32(sw, w) || !to_u32(sh, h)) return nullptr;
            float scale = 0.5f;
            if (ss == "half" || ss == "HALF") scale = 0.5f;
            else if (ss == "orb" || ss == "ORB") scale = 0.8408964f;
            else scale = (float)atof(ss.c_str());
            const vx_df_image fmt = fourcc(sf);
            if (virt) return (Ref *)vxCreateVirtualPyramid((vx_graph)g, levels, scale, w, h, fmt);
            return (Ref *)vxCreatePyramid((vx_context)c, levels, scale, w, h, fmt);
        }
        if (kind == "array") {                            // TYPE,capacity
            vx_enum t;
            uint32_t cap;
            if (f.size() != 2 || !enum_by_name(f[0], t) || !to_u32(f[1], cap)) return nullptr;
            if (virt) return (Ref *)vxCreateVirtualArray((vx_graph)g, t, cap);
            return (Ref *)vxCreateArray((vx_context)c, t, cap);
        }
        if (kind == "scalar") {                           // TYPE,value
            vx_enum t;
            if (f.size() < 2 || !enum_by_name(f[0], t)) return nullptr;
            const std::string &v = f[1];
            uint8_t raw[16] = {};
            if (t == VX_TYPE_FLOAT32) { const float x = (float)atof(v.c_str()); memcpy(raw, &x, 4); }
            else if (t == VX_TYPE_FLOAT64) { const double x = atof(v.c_str()); memcpy(raw, &x, 8); }
            else if (t == VX_TYPE_BOOL) {
                const vx_bool b = (v == "TRUE" || v == "true" || v == "1") ? vx_true_e : vx_false_e;
                memcpy(raw, &b, sizeof b);
            } else if (t == VX_TYPE_ENUM) {
                vx_enum e;
                if (!enum_by_name(v, e)) { uint32_t x; if (!to_u32(v, x)) return nullptr; e = (vx_enum)x; }
                memcpy(raw, &e, sizeof e);
            } else if (t == VX_TYPE_DF_IMAGE) {
                const vx_df_image d = fourcc(v);
                memcpy(raw, &d, sizeof d);
            } else {
                const long long x = strtoll(v.c_str(), nullptr, 0);
                memcpy(raw, &x, type_size(t) ? type_size(t) : 4);
            }
            return (Ref *)vxCreateScalar((vx_context)c, t, raw);
        }
        if (kind == "threshold") {                        // BINARY|RANGE,in,out[:INIT,...]
            vx_enum t;
            if (f.empty() || !enum_by_name(f[0], t)) return nullptr;
            // formats as four-character codes or as the numeric vx_df_image (the library form)
            auto fmt_of = [&](size_t i) -> vx_df_image {
                if (f.size() <= i) return VX_DF_IMAGE_U8;
                if (f[i].size() == 4 && !isdigit((unsigned char)f[i][0])) return fourcc(f[i]);
                uint32_t v = 0;
                return to_u32(f[i], v) ? (vx_df_image)v : 0;
            };
            vx_threshold th = vxCreateThresholdForImage((vx_context)c, t, fmt_of(1), fmt_of(2));
            if (!th) return nullptr;
            uint32_t a = 0, b = 0;
            if (t == VX_THRESHOLD_TYPE_BINARY && init.size() >= 1 && to_u32(init[0], a)) {
                vx_int32 v = (vx_int32)a;
                vxSetThresholdAttribute(th, VX_THRESHOLD_THRESHOLD_VALUE, &v, sizeof v);
            } else if (t == VX_THRESHOLD_TYPE_RANGE && init.size() >= 2 && to_u32(init[0], a) && to_u32(init[1], b)) {
                vx_int32 lo = (vx_int32)a, hi = (vx_int32)b;
                vxSetThresholdAttribute(th, VX_THRESHOLD_THRESHOLD_LOWER, &lo, sizeof lo);
                vxSetThresholdAttribute(th, VX_THRESHOLD_THRESHOLD_UPPER, &hi, sizeof hi);
            }
            return (Ref *)th;
        }
        if (kind == "matrix") {                           // TYPE,columns,rows[:INIT,{a;b;...}]
            vx_enum t;
            uint32_t cols, rows;
            if (f.size() != 3 || !enum_by_name(f[0], t) || !to_u32(f[1], cols) || !to_u32(f[2], rows)) return nullptr;
            vx_matrix m = vxCreateMatrix((vx_context)c, t, cols, rows);
            if (!m) return nullptr;
            const size_t lb = extra.find('{'), rb = extra.find('}');
            if (extra.compare(0, 5, "INIT,") == 0 && lb != std::string::npos && rb != std::string::npos && rb > lb) {
                const std::vector<std::string> vals = split(extra.substr(lb + 1, rb - lb - 1), ';');
                if (vals.size() != (size_t)cols * rows) return nullptr;
                std::vector<uint8_t> buf((size_t)cols * rows * type_size(t));
                for (size_t i = 0; i < vals.size(); i++) {
                    if (t == VX_TYPE_FLOAT32) { const float x = (float)atof(vals[i].c_str()); memcpy(&buf[i * 4], &x, 4); }
                    else if (t == VX_TYPE_INT32) { const int32_t x = (int32_t)strtol(vals[i].c_str(), nullptr, 0); memcpy(&buf[i * 4], &x, 4); }
                    else buf[i] = (uint8_t)strtol(vals[i].c_str(), nullptr, 0);
                }
                vxCopyMatrix(m, buf.data(), VX_WRITE_ONLY, VX_MEMORY_TYPE_HOST);
            }
            return (Ref *)m;
        }
        if (kind == "lut") {                              // TYPE,count
            vx_enum t;
            uint32_t n;
            if (f.size() != 2 || !enum_by_name(f[0], t) || !to_u32(f[1], n)) return nullptr;
            return virt ? (Ref *)vxCreateVirtualLUT((vx_graph)g, t, n) : (Ref *)vxCreateLUT((vx_context)c, t, n);
        }
        if (kind == "distribution") {                     // bins,offset,range
            uint32_t bins, range;
            if (f.size() != 3 || !to_u32(f[0], bins) || !to_u32(f[2], range)) return nullptr;
            const vx_int32 off = (vx_int32)strtol(f[1].c_str(), nullptr, 0);
            return virt ? (Ref *)vxCreateVirtualDistribution((vx_graph)g, bins, off, range)
                        : (Ref *)vxCreateDistribution((vx_context)c, bins, off, range);
        }
        err = VX_ERROR_NOT_SUPPORTED;
        return nullptr;
    }

    vx_status statement(const std::vector<std::string> &a)
    {
        if (a.size() == 4 && a[0] == "data" && a[2] == "=") {
            std::string params;
            vx_status err = VX_SUCCESS;
            Ref *r = make_data(a[3], params, err);
            if (!r || vxGetStatus((vx_reference)r) != VX_SUCCESS) return fail(err ? err : VX_FAILURE, "data type not supported");
            r->name = a[1];
            names[a[1]] = r;
            if (info->data_registry_callback_f && !params.empty())
                info->data_registry_callback_f(info->data_registry_callback_obj, (vx_reference)r, a[1].c_str(), params.c_str());
            return VX_SUCCESS;
        }
        if (a.size() >= 2 && a[0] == "node") {
            std::string kn = a[1];
            const std::string pre = "org.khronos.openvx.";
            if (kn.compare(0, pre.size(), pre) == 0) kn = kn.substr(pre.size());
            vx_enum kernel = 0;
            for (const NamedEnum &e : kKernels)
                if (kn == e.name) kernel = e.value;
            if (!kernel) return fail(VX_ERROR_NOT_SUPPORTED, "kernel not supported");
            std::vector<Ref *> params;
            vx_border_t border{VX_BORDER_UNDEFINED, {}};
            bool has_border = false;
            for (size_t i = 2; i < a.size(); i++) {
                const std::string &arg = a[i];
                if (arg.compare(0, 5, "attr:") == 0) {
                    if (arg.compare(5, 12, "BORDER_MODE:") != 0) return fail(VX_ERROR_NOT_SUPPORTED, "unsupported node attribute");
                    const std::string m = arg.substr(17);
                    has_border = true;
                    if (m == "UNDEFINED") border.mode = VX_BORDER_UNDEFINED;
                    else if (m == "REPLICATE") border.mode = VX_BORDER_REPLICATE;
                    else if (m.compare(0, 9, "CONSTANT,") == 0) {
                        border.mode = VX_BORDER_CONSTANT;
                        border.constant_value.U32 = (vx_uint32)strtoul(m.c_str() + 9, nullptr, 0);
                    } else {
                        return fail(VX_ERROR_INVALID_VALUE, "invalid/unsupported border mode attribute");
                    }
                    continue;
                }
                if (arg == "null") { params.push_back(nullptr); continue; }
                if (arg[0] == '!') {
                    vx_enum e;
                    if (!enum_by_name(arg.substr(1), e)) return fail(VX_ERROR_INVALID_VALUE, "unknown enum name");
                    Scalar *s = make_scalar(c, g, VX_TYPE_ENUM, &e);
                    s->ext_count = 0;             // held by the node it is passed to
                    params.push_back(s);
                    continue;
                }
                if (arg[0] == '$') {
                    const int k = atoi(arg.c_str() + 1);
                    if (k < 1 || (uint32_t)k > info->num_ref || !info->ref) return fail(VX_ERROR_INVALID_PARAMETERS, "invalid $ reference");
                    params.push_back((Ref *)info->ref[k - 1]);
                    continue;
                }
                auto it = names.find(arg);
                if (it == names.end()) return fail(VX_ERROR_INVALID_PARAMETERS, "unknown data name");
                params.push_back(it->second);
            }
            Node *n = graph_add_node(g, kernel, params);
            if (!n) return fail(VX_FAILURE, "node creation failed");
            if (has_border) n->border = border;
            return VX_SUCCESS;
        }
        return fail(VX_ERROR_NOT_SUPPORTED, "statement not supported");
    }
};

}  // namespace

vx_status graph_import_text(Graph *g, const AgoGraphImportInfo *info)
{
    if (!info || !info->text) return VX_ERROR_INVALID_PARAMETERS;
    Importer im{g, g->ctx, info, {}};
    std::istringstream in(info->text);
    std::string raw;
    while (std::getline(in, raw)) {
        im.lineno++;
        im.line = raw;
        const size_t hash = raw.find('#');
        if (hash != std::string::npos) raw = raw.substr(0, hash);
        std::istringstream ws(raw);
        std::vector<std::string> a;
        for (std::string t; ws >> t;) a.push_back(t);
        if (a.empty()) continue;
        vx_status s = im.statement(a);
        if (s) return s;
    }
    return VX_SUCCESS;
}

}  // namespace agovx
