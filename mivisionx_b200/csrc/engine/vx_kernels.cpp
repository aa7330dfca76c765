// vx_kernels.cpp -- the kernel registry: vxGetKernelByName / vxGetKernelByEnum, kernel
// queries, generic nodes (vxCreateGenericNode + vxSetParameterByIndex) and parameter
// objects, the path runvx takes for every GDF node (utilities/runvx/vxEngine.cpp:923-928).
//
// The table lists the OpenVX 1.x vision kernels under the names of the Khronos registry
// ("org.khronos.openvx.<name>", as ago/ago_kernel_list.cpp registers them), each with its
// parameter signature.  A kernel this target does not execute is still found, so graphs
// build as with the reference; vxVerifyGraph then reports it as not supported.
#include <dlfcn.h>

#include <cstdio>
#include <cstring>
#include <string>

#include "vx_internal.h"

using namespace agovx;

namespace agovx {
Node *graph_add_node(Graph *g, vx_enum kernel, const std::vector<Ref *> &params);

namespace {

// One entry per kernel.  `sig` has two characters per parameter: the direction ('i' input,
// 'o' output, 'b' bidirectional; upper case = optional) and the object type ('I' image,
// 'S' scalar, 'T' threshold, 'M' matrix, 'A' array, 'P' pyramid, 'L' lut, 'D' distribution,
// 'C' convolution, 'R' remap, '*' any reference).
struct KernelSpec { vx_enum id; const char *name; const char *sig; };

const KernelSpec kSpecs[] = {
    {VX_KERNEL_COLOR_CONVERT, "color_convert", "iIoI"},
    {VX_KERNEL_CHANNEL_EXTRACT, "channel_extract", "iIiSoI"},
    {VX_KERNEL_CHANNEL_COMBINE, "channel_combine", "iIiIIIIIoI"},
    {VX_KERNEL_SOBEL_3x3, "sobel_3x3", "iIOIOI"},
    {VX_KERNEL_MAGNITUDE, "magnitude", "iIiIoI"},
    {VX_KERNEL_PHASE, "phase", "iIiIoI"},
    {VX_KERNEL_SCALE_IMAGE, "scale_image", "iIoIiS"},
    {VX_KERNEL_TABLE_LOOKUP, "table_lookup", "iIiLoI"},
    {VX_KERNEL_HISTOGRAM, "histogram", "iIoD"},
    {VX_KERNEL_EQUALIZE_HISTOGRAM, "equalize_histogram", "iIoI"},
    {VX_KERNEL_ABSDIFF, "absdiff", "iIiIoI"},
    {VX_KERNEL_MEAN_STDDEV, "mean_stddev", "iIoSOS"},
    {VX_KERNEL_THRESHOLD, "threshold", "iIiToI"},
    {VX_KERNEL_INTEGRAL_IMAGE, "integral_image", "iIoI"},
    {VX_KERNEL_DILATE_3x3, "dilate_3x3", "iIoI"},
    {VX_KERNEL_ERODE_3x3, "erode_3x3", "iIoI"},
    {VX_KERNEL_MEDIAN_3x3, "median_3x3", "iIoI"},
    {VX_KERNEL_BOX_3x3, "box_3x3", "iIoI"},
    {VX_KERNEL_GAUSSIAN_3x3, "gaussian_3x3", "iIoI"},
    {VX_KERNEL_CUSTOM_CONVOLUTION, "custom_convolution", "iIiCoI"},
    {VX_KERNEL_GAUSSIAN_PYRAMID, "gaussian_pyramid", "iIoP"},
    {VX_KERNEL_ACCUMULATE, "accumulate", "iIbI"},
    {VX_KERNEL_ACCUMULATE_WEIGHTED, "accumulate_weighted", "iIiSbI"},
    {VX_KERNEL_ACCUMULATE_SQUARE, "accumulate_square", "iIiSbI"},
    {VX_KERNEL_MINMAXLOC, "minmaxloc", "iIoSoSOAOAOSOS"},
    {VX_KERNEL_CONVERTDEPTH, "convertdepth", "iIoIiSiS"},
    {VX_KERNEL_CANNY_EDGE_DETECTOR, "canny_edge_detector", "iIiTiSiSoI"},
    {VX_KERNEL_AND, "and", "iIiIoI"},
    {VX_KERNEL_OR, "or", "iIiIoI"},
    {VX_KERNEL_XOR, "xor", "iIiIoI"},
    {VX_KERNEL_NOT, "not", "iIoI"},
    {VX_KERNEL_MULTIPLY, "multiply", "iIiIiSiSiSoI"},
    {VX_KERNEL_ADD, "add", "iIiIiSoI"},
    {VX_KERNEL_SUBTRACT, "subtract", "iIiIiSoI"},
    {VX_KERNEL_WARP_AFFINE, "warp_affine", "iIiMiSoI"},
    {VX_KERNEL_WARP_PERSPECTIVE, "warp_perspective", "iIiMiSoI"},
    {VX_KERNEL_HARRIS_CORNERS, "harris_corners", "iIiSiSiSiSiSoAOS"},
    {VX_KERNEL_FAST_CORNERS, "fast_corners", "iIiSiSoAOS"},
    {VX_KERNEL_OPTICAL_FLOW_PYR_LK, "optical_flow_pyr_lk", "iPiPiAiAoAiSiSiSiSiS"},
    {VX_KERNEL_REMAP, "remap", "iIiRiSoI"},
    {VX_KERNEL_HALFSCALE_GAUSSIAN, "halfscale_gaussian", "iIoIiS"},
    {VX_KERNEL_WEIGHTED_AVERAGE, "weighted_average", "iIiSiIoI"},
};
constexpr size_t kNumSpecs = sizeof(kSpecs) / sizeof(kSpecs[0]);
constexpr const char *kKhronosPrefix = "org.khronos.openvx.";

const KernelSpec *spec_by_name(const char *name)
{
    if (!name) return nullptr;
    std::string n(name);
    if (n.compare(0, strlen(kKhronosPrefix), kKhronosPrefix) == 0) n = n.substr(strlen(kKhronosPrefix));
    else if (n.find('.') != std::string::npos) return nullptr;     // another vendor's name space
    for (const KernelSpec &k : kSpecs)
        if (n == k.name) return &k;
    return nullptr;
}

const KernelSpec *spec_by_enum(vx_enum id)
{
    for (const KernelSpec &k : kSpecs)
        if (k.id == id) return &k;
    return nullptr;
}

vx_enum type_of(char t)
{
    switch (t) {
    case 'I': return VX_TYPE_IMAGE;
    case 'S': return VX_TYPE_SCALAR;
    case 'T': return VX_TYPE_THRESHOLD;
    case 'M': return VX_TYPE_MATRIX;
    case 'A': return VX_TYPE_ARRAY;
    case 'P': return VX_TYPE_PYRAMID;
    case 'L': return VX_TYPE_LUT;
    case 'D': return VX_TYPE_DISTRIBUTION;
    case 'C': return VX_TYPE_CONVOLUTION;
    case 'R': return VX_TYPE_REMAP;
    default: return VX_TYPE_REFERENCE;
    }
}

vx_enum direction_of(char d)
{
    switch (d | 0x20) {
    case 'o': return VX_OUTPUT;
    case 'b': return VX_BIDIRECTIONAL;
    default: return VX_INPUT;
    }
}

// The context's kernel objects, one per table entry, made on first use and held by the
// context (an internal reference) so that handles stay valid after vxReleaseKernel.
Kernel *context_kernel(Context *c, const KernelSpec *s)
{
    for (Kernel *k : c->kernels)
        if (k->id == s->id) return k;
    Kernel *k = new Kernel();
    k->type = VX_TYPE_KERNEL;
    k->id = s->id;
    k->kname = std::string(kKhronosPrefix) + s->name;
    k->sig = s->sig;
    k->num_params = (int)(strlen(s->sig) / 2);
    k->ext_count = 0;
    k->int_count = 1;
    add_ref(c, k);
    c->kernels.push_back(k);
    return k;
}

template <class T> T *as(void *h) { return static_cast<T *>(static_cast<Ref *>(h)); }

}  // namespace

// Every required parameter of the node is set and every parameter has its declared type.
vx_status check_node_params(Node *n)
{
    const KernelSpec *s = spec_by_enum(n->kernel);
    if (!s) return VX_SUCCESS;       // not in the table: the kernel's own validation decides
    const size_t np = strlen(s->sig) / 2;
    if (n->params.size() != np) return VX_ERROR_INVALID_PARAMETERS;
    for (size_t i = 0; i < np; i++) {
        const char dir = s->sig[2 * i], t = s->sig[2 * i + 1];
        Ref *r = n->params[i];
        if (!r) {
            if (dir >= 'a' && dir <= 'z') {
                log_error(n, VX_ERROR_NOT_SUFFICIENT, "ERROR: vxVerifyGraph: %s: required parameter %zu is not set\n", s->name, i);
                return VX_ERROR_NOT_SUFFICIENT;
            }
            continue;
        }
        if (!is_ref(r)) return VX_ERROR_INVALID_REFERENCE;
        const vx_enum want = type_of(t);
        if (want != VX_TYPE_REFERENCE && r->type != want) {
            log_error(n, VX_ERROR_INVALID_TYPE, "ERROR: vxVerifyGraph: %s: parameter %zu has type 0x%x, expected 0x%x\n",
                      s->name, i, r->type, want);
            return VX_ERROR_INVALID_TYPE;
        }
    }
    return VX_SUCCESS;
}

// Parameter objects (vxGetParameterByIndex / vxGetKernelParameterByIndex): a node or a
// kernel and an index.
struct Parameter : Ref {
    Node *node = nullptr;
    Kernel *kernel = nullptr;
    uint32_t index = 0;
};

}  // namespace agovx

#define CHECK_REF(h, T) if (!is_valid(h, T)) return VX_ERROR_INVALID_REFERENCE

extern "C" {

vx_kernel vxGetKernelByName(vx_context context, const vx_char *name)
{
    if (!is_valid(context, VX_TYPE_CONTEXT)) return nullptr;
    const KernelSpec *s = spec_by_name(name);
    if (!s) {
        log_error(as<Ref>(context), VX_ERROR_INVALID_PARAMETERS, "ERROR: vxGetKernelByName: kernel %s is not known\n",
                  name ? name : "(null)");
        return nullptr;
    }
    Kernel *k = context_kernel(as<Context>(context), s);
    k->ext_count++;
    k->released = false;
    return (vx_kernel)k;
}

vx_kernel vxGetKernelByEnum(vx_context context, vx_enum kernel)
{
    if (!is_valid(context, VX_TYPE_CONTEXT)) return nullptr;
    const KernelSpec *s = spec_by_enum(kernel);
    if (!s) return nullptr;
    Kernel *k = context_kernel(as<Context>(context), s);
    k->ext_count++;
    k->released = false;
    return (vx_kernel)k;
}

vx_status vxReleaseKernel(vx_kernel *kernel)
{
    if (!kernel || !is_valid(*kernel, VX_TYPE_KERNEL)) return VX_ERROR_INVALID_REFERENCE;
    Kernel *k = as<Kernel>(*kernel);
    if (k->ext_count <= 0) return VX_ERROR_INVALID_REFERENCE;
    k->ext_count--;                  // the context keeps the object
    *kernel = nullptr;
    return VX_SUCCESS;
}

vx_status vxQueryKernel(vx_kernel kernel, vx_enum attribute, void *ptr, vx_size size)
{
    CHECK_REF(kernel, VX_TYPE_KERNEL);
    Kernel *k = as<Kernel>(kernel);
    if (!ptr) return VX_ERROR_INVALID_PARAMETERS;
    switch (attribute) {
    case VX_KERNEL_PARAMETERS: if (size != sizeof(vx_uint32)) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint32 *)ptr = (vx_uint32)k->num_params; return VX_SUCCESS;
    case VX_KERNEL_NAME:
        if (size < VX_MAX_KERNEL_NAME) return VX_ERROR_INVALID_PARAMETERS;
        snprintf((char *)ptr, size, "%s", k->kname.c_str());
        return VX_SUCCESS;
    case VX_KERNEL_ENUM: if (size != sizeof(vx_enum)) return VX_ERROR_INVALID_PARAMETERS; *(vx_enum *)ptr = k->id; return VX_SUCCESS;
    case VX_KERNEL_LOCAL_DATA_SIZE: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = 0; return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_node vxCreateGenericNode(vx_graph graph, vx_kernel kernel)
{
    if (!is_valid(graph, VX_TYPE_GRAPH) || !is_valid(kernel, VX_TYPE_KERNEL)) return nullptr;
    Kernel *k = as<Kernel>(kernel);
    std::vector<Ref *> params((size_t)k->num_params, nullptr);
    return (vx_node)graph_add_node(as<Graph>(graph), k->id, params);
}

vx_status vxSetParameterByIndex(vx_node node, vx_uint32 index, vx_reference value)
{
    CHECK_REF(node, VX_TYPE_NODE);
    Node *n = as<Node>(node);
    if (index >= n->params.size()) return VX_ERROR_INVALID_PARAMETERS;
    if (value && !is_ref(value)) return VX_ERROR_INVALID_REFERENCE;
    const KernelSpec *s = spec_by_enum(n->kernel);
    if (value && s) {
        const vx_enum want = type_of(s->sig[2 * index + 1]);
        const vx_enum got = as<Ref>(value)->type;
        if (want != VX_TYPE_REFERENCE && got != want) {
            log_error(n, VX_ERROR_INVALID_TYPE, "ERROR: vxSetParameterByIndex: parameter %u of %s takes type 0x%x, got 0x%x\n",
                      index, s->name, want, got);
            return VX_ERROR_INVALID_TYPE;
        }
    }
    Ref *old = n->params[index];
    if (value) retain_internal(as<Ref>(value));
    n->params[index] = value ? as<Ref>(value) : nullptr;
    release_internal(old);
    if (n->scope) graph_invalidate(n->scope);
    return VX_SUCCESS;
}

vx_parameter vxGetParameterByIndex(vx_node node, vx_uint32 index)
{
    if (!is_valid(node, VX_TYPE_NODE)) return nullptr;
    Node *n = as<Node>(node);
    if (index >= n->params.size()) return nullptr;
    Parameter *p = new Parameter();
    p->type = VX_TYPE_PARAMETER;
    p->node = n;
    p->index = index;
    add_ref(n->ctx, p);
    return (vx_parameter)p;
}

vx_parameter vxGetKernelParameterByIndex(vx_kernel kernel, vx_uint32 index)
{
    if (!is_valid(kernel, VX_TYPE_KERNEL)) return nullptr;
    Kernel *k = as<Kernel>(kernel);
    if ((int)index >= k->num_params) return nullptr;
    Parameter *p = new Parameter();
    p->type = VX_TYPE_PARAMETER;
    p->kernel = k;
    p->index = index;
    add_ref(k->ctx, p);
    return (vx_parameter)p;
}

vx_status vxSetParameterByReference(vx_parameter parameter, vx_reference value)
{
    CHECK_REF(parameter, VX_TYPE_PARAMETER);
    Parameter *p = as<Parameter>(parameter);
    if (!p->node || !is_valid(p->node, VX_TYPE_NODE)) return VX_ERROR_INVALID_PARAMETERS;
    return vxSetParameterByIndex((vx_node)p->node, p->index, value);
}

vx_status vxQueryParameter(vx_parameter parameter, vx_enum attribute, void *ptr, vx_size size)
{
    CHECK_REF(parameter, VX_TYPE_PARAMETER);
    Parameter *p = as<Parameter>(parameter);
    if (!ptr) return VX_ERROR_INVALID_PARAMETERS;
    const KernelSpec *s = spec_by_enum(p->node ? p->node->kernel : p->kernel->id);
    const char *sig = s ? s->sig + 2 * p->index : "i*";
    switch (attribute) {
    case VX_PARAMETER_INDEX: if (size != sizeof(vx_uint32)) return VX_ERROR_INVALID_PARAMETERS; *(vx_uint32 *)ptr = p->index; return VX_SUCCESS;
    case VX_PARAMETER_DIRECTION: if (size != sizeof(vx_enum)) return VX_ERROR_INVALID_PARAMETERS; *(vx_enum *)ptr = direction_of(sig[0]); return VX_SUCCESS;
    case VX_PARAMETER_TYPE: if (size != sizeof(vx_enum)) return VX_ERROR_INVALID_PARAMETERS; *(vx_enum *)ptr = type_of(sig[1]); return VX_SUCCESS;
    case VX_PARAMETER_STATE:
        if (size != sizeof(vx_enum)) return VX_ERROR_INVALID_PARAMETERS;
        *(vx_enum *)ptr = (sig[0] >= 'A' && sig[0] <= 'Z') ? VX_PARAMETER_STATE_OPTIONAL : VX_PARAMETER_STATE_REQUIRED;
        return VX_SUCCESS;
    case VX_PARAMETER_REF:
        if (size != sizeof(vx_reference) || !p->node) return VX_ERROR_INVALID_PARAMETERS;
        *(vx_reference *)ptr = (vx_reference)p->node->params[p->index];
        if (p->node->params[p->index]) p->node->params[p->index]->ext_count++;
        return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxReleaseParameter(vx_parameter *param)
{
    if (!param || !is_valid(*param, VX_TYPE_PARAMETER)) return VX_ERROR_INVALID_REFERENCE;
    vx_status s = vxReleaseReference((vx_reference *)param);
    return s;
}

// vxLoadKernels (vx_api.cpp:2325 -> agoLoadModule, ago_interface.cpp:1128): open the module
// library and call its vxPublishKernels.  User kernels (vxAddUserKernel) are not part of
// this target, so a module that publishes any fails to load.
vx_status vxLoadKernels(vx_context context, const vx_char *module)
{
    CHECK_REF(context, VX_TYPE_CONTEXT);
    if (!module || !*module) return VX_ERROR_INVALID_PARAMETERS;
    std::string file = std::string("lib") + module + ".so";
    void *h = dlopen(file.c_str(), RTLD_NOW | RTLD_LOCAL);
    if (!h) h = dlopen(module, RTLD_NOW | RTLD_LOCAL);
    if (!h) {
        log_error(as<Ref>(context), VX_ERROR_INVALID_PARAMETERS, "ERROR: vxLoadKernels: cannot load %s: %s\n", module, dlerror());
        return VX_ERROR_INVALID_PARAMETERS;
    }
    using Publish = vx_status (*)(vx_context);
    Publish pub = (Publish)dlsym(h, "vxPublishKernels");
    if (!pub) {
        dlclose(h);
        log_error(as<Ref>(context), VX_ERROR_INVALID_MODULE, "ERROR: vxLoadKernels: %s has no vxPublishKernels\n", module);
        return VX_ERROR_INVALID_MODULE;
    }
    return pub(context);
}

}  // extern "C"
