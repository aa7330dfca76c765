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

constexpr vx_uint32 kMaxUserParams = 32;   // AGO_MAX_PARAMS

// a user kernel of the context by name (exact) or by enumeration
Kernel *user_kernel(Context *c, const char *name, vx_enum id, bool byName)
{
    for (Kernel *k : c->kernels)
        if (k->user && (byName ? (name && k->kname == name) : k->id == id)) return k;
    return nullptr;
}

}  // namespace

// Parameters a node of a user kernel must have: every required one set, types as declared
// (VX_TYPE_REFERENCE accepts any object).
static vx_status check_user_params(Node *n)
{
    Kernel *k = n->ukernel;
    if (n->params.size() != k->uparams.size()) return VX_ERROR_INVALID_PARAMETERS;
    for (size_t i = 0; i < n->params.size(); i++) {
        const UserParam &up = k->uparams[i];
        Ref *r = n->params[i];
        if (!r) {
            if (up.state == VX_PARAMETER_STATE_REQUIRED) {
                log_error(n, VX_ERROR_NOT_SUFFICIENT, "ERROR: vxVerifyGraph: %s: required parameter %zu is not set\n",
                          k->kname.c_str(), i);
                return VX_ERROR_NOT_SUFFICIENT;
            }
            continue;
        }
        if (!is_ref(r)) return VX_ERROR_INVALID_REFERENCE;
        if (up.type != VX_TYPE_REFERENCE && r->type != up.type) {
            log_error(n, VX_ERROR_INVALID_TYPE, "ERROR: vxVerifyGraph: %s: parameter %zu has type 0x%x, expected 0x%x\n",
                      k->kname.c_str(), i, r->type, up.type);
            return VX_ERROR_INVALID_TYPE;
        }
    }
    return VX_SUCCESS;
}

// Every required parameter of the node is set and every parameter has its declared type.
vx_status check_node_params(Node *n)
{
    if (n->ukernel) return check_user_params(n);
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
    if (Kernel *u = user_kernel(as<Context>(context), name, 0, true)) {
        u->ext_count++;
        u->released = false;
        return (vx_kernel)u;
    }
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
    if (Kernel *u = user_kernel(as<Context>(context), nullptr, kernel, false)) {
        u->ext_count++;
        u->released = false;
        return (vx_kernel)u;
    }
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
    case VX_KERNEL_LOCAL_DATA_SIZE: if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS; *(vx_size *)ptr = k->local_size; return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_node vxCreateGenericNode(vx_graph graph, vx_kernel kernel)
{
    if (!is_valid(graph, VX_TYPE_GRAPH) || !is_valid(kernel, VX_TYPE_KERNEL)) return nullptr;
    Kernel *k = as<Kernel>(kernel);
    if (k->user && !k->finalized) return nullptr;
    std::vector<Ref *> params((size_t)k->num_params, nullptr);
    Node *n = graph_add_node(as<Graph>(graph), k->id, params);
    if (n && k->user) n->ukernel = k;
    return (vx_node)n;
}

vx_status vxSetParameterByIndex(vx_node node, vx_uint32 index, vx_reference value)
{
    CHECK_REF(node, VX_TYPE_NODE);
    Node *n = as<Node>(node);
    if (index >= n->params.size()) return VX_ERROR_INVALID_PARAMETERS;
    if (value && !is_ref(value)) return VX_ERROR_INVALID_REFERENCE;
    const KernelSpec *s = n->ukernel ? nullptr : spec_by_enum(n->kernel);
    if (value && n->ukernel) {
        const vx_enum want = n->ukernel->uparams[index].type, got = as<Ref>(value)->type;
        if (want != VX_TYPE_REFERENCE && got != want) return VX_ERROR_INVALID_TYPE;
    }
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
    Kernel *uk = p->node ? p->node->ukernel : (p->kernel->user ? p->kernel : nullptr);
    const KernelSpec *s = uk ? nullptr : spec_by_enum(p->node ? p->node->kernel : p->kernel->id);
    const char *sig = s ? s->sig + 2 * p->index : "i*";
    if (uk) {
        const UserParam &up = uk->uparams[p->index];
        switch (attribute) {
        case VX_PARAMETER_DIRECTION: if (size != sizeof(vx_enum)) return VX_ERROR_INVALID_PARAMETERS; *(vx_enum *)ptr = up.dir; return VX_SUCCESS;
        case VX_PARAMETER_TYPE: if (size != sizeof(vx_enum)) return VX_ERROR_INVALID_PARAMETERS; *(vx_enum *)ptr = up.type; return VX_SUCCESS;
        case VX_PARAMETER_STATE: if (size != sizeof(vx_enum)) return VX_ERROR_INVALID_PARAMETERS; *(vx_enum *)ptr = up.state; return VX_SUCCESS;
        default: break;
        }
    }
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
// library and call its vxPublishKernels, which adds its kernels with vxAddUserKernel.
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

// ---------------------------------------------------------------- user kernels
// vxAddUserKernel / vxAddParameterToKernel / vxFinalizeKernel / vxRemoveKernel /
// vxSetKernelAttribute (vx_api.cpp:2584-2800).  A user kernel's node runs its kernel_f on the
// host when the graph executes; with VX_KERNEL_ATTRIBUTE_AMD_GPU_BUFFER_ACCESS_ENABLE it gets
// device buffers (VX_IMAGE_ATTRIBUTE_AMD_HIP_BUFFER) and the graph's CUDA stream
// (VX_NODE_ATTRIBUTE_AMD_HIP_STREAM) instead of host access.
vx_kernel vxAddUserKernel(vx_context context, const vx_char name[VX_MAX_KERNEL_NAME], vx_enum enumeration,
                          vx_kernel_f func_ptr, vx_uint32 numParams, vx_kernel_validate_f validate,
                          vx_kernel_initialize_f init, vx_kernel_deinitialize_f deinit)
{
    if (!is_valid(context, VX_TYPE_CONTEXT) || !name || !func_ptr || !validate || numParams == 0 ||
        numParams > kMaxUserParams)
        return nullptr;
    Context *c = as<Context>(context);
    if (user_kernel(c, name, 0, true) || user_kernel(c, nullptr, enumeration, false) || spec_by_enum(enumeration) ||
        spec_by_name(name)) {
        log_error(as<Ref>(context), VX_ERROR_INVALID_PARAMETERS, "ERROR: vxAddUserKernel: %s / 0x%x is already a kernel\n",
                  name, enumeration);
        return nullptr;
    }
    Kernel *k = new Kernel();
    k->type = VX_TYPE_KERNEL;
    k->id = enumeration;
    k->kname = name;
    k->user = true;
    k->func = func_ptr;
    k->validate = validate;
    k->init = init;
    k->deinit = deinit;
    k->num_params = (int)numParams;
    k->uparams.resize(numParams);
    k->ext_count = 1;
    k->int_count = 1;                // the context's kernel list
    add_ref(c, k);
    c->kernels.push_back(k);
    return (vx_kernel)k;
}

vx_status vxAddParameterToKernel(vx_kernel kernel, vx_uint32 index, vx_enum dir, vx_enum data_type, vx_enum state)
{
    CHECK_REF(kernel, VX_TYPE_KERNEL);
    Kernel *k = as<Kernel>(kernel);
    if (!k->user || k->finalized || index >= kMaxUserParams) return VX_ERROR_INVALID_PARAMETERS;
    if (dir != VX_INPUT && dir != VX_OUTPUT && dir != VX_BIDIRECTIONAL) return VX_ERROR_INVALID_PARAMETERS;
    if (state != VX_PARAMETER_STATE_REQUIRED && state != VX_PARAMETER_STATE_OPTIONAL) return VX_ERROR_INVALID_PARAMETERS;
    if (data_type == VX_TYPE_DELAY && dir != VX_INPUT) return VX_ERROR_INVALID_PARAMETERS;
    if (index >= k->uparams.size()) k->uparams.resize(index + 1);
    k->uparams[index] = UserParam{dir, data_type, state, true};
    k->num_params = (int)k->uparams.size();
    return VX_SUCCESS;
}

vx_status vxFinalizeKernel(vx_kernel kernel)
{
    CHECK_REF(kernel, VX_TYPE_KERNEL);
    Kernel *k = as<Kernel>(kernel);
    if (!k->user || k->finalized || k->uparams.empty()) return VX_ERROR_INVALID_REFERENCE;
    for (const UserParam &up : k->uparams)
        if (!up.set) return VX_ERROR_INVALID_REFERENCE;
    k->finalized = true;
    return VX_SUCCESS;
}

vx_status vxRemoveKernel(vx_kernel kernel)
{
    CHECK_REF(kernel, VX_TYPE_KERNEL);
    Kernel *k = as<Kernel>(kernel);
    if (!k->user) return VX_ERROR_INVALID_PARAMETERS;      // built-in kernels stay
    Context *c = k->ctx;
    for (size_t i = 0; i < c->kernels.size(); i++)
        if (c->kernels[i] == k) { c->kernels.erase(c->kernels.begin() + (long)i); break; }
    k->finalized = false;            // no new nodes; existing nodes keep their callbacks
    k->ext_count = 0;
    return VX_SUCCESS;
}

vx_status vxSetKernelAttribute(vx_kernel kernel, vx_enum attribute, const void *ptr, vx_size size)
{
    CHECK_REF(kernel, VX_TYPE_KERNEL);
    Kernel *k = as<Kernel>(kernel);
    if (!ptr) return VX_ERROR_INVALID_PARAMETERS;
    switch (attribute) {
    case VX_KERNEL_LOCAL_DATA_SIZE:
        if (size != sizeof(vx_size)) return VX_ERROR_INVALID_PARAMETERS;
        k->local_size = *(const vx_size *)ptr;
        return VX_SUCCESS;
    case VX_KERNEL_ATTRIBUTE_AMD_GPU_BUFFER_ACCESS_ENABLE:
        if (size != sizeof(vx_bool)) return VX_ERROR_INVALID_PARAMETERS;
        if (!k->user || k->finalized) return VX_ERROR_NOT_SUPPORTED;
        k->gpu_access = *(const vx_bool *)ptr == vx_true_e;
        return VX_SUCCESS;
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

// ---------------------------------------------------------------- meta formats
static MetaFormat *meta_of(vx_meta_format m)
{
    MetaFormat *f = reinterpret_cast<MetaFormat *>(m);
    return f && f->magic == MetaFormat{}.magic ? f : nullptr;
}

vx_status vxSetMetaFormatAttribute(vx_meta_format meta, vx_enum attribute, const void *ptr, vx_size size)
{
    MetaFormat *m = meta_of(meta);
    if (!m) return VX_ERROR_INVALID_REFERENCE;
    if (!ptr) return VX_ERROR_INVALID_PARAMETERS;
    auto take = [&](auto &dst, vx_enum type) {
        if (size != sizeof(dst)) return VX_ERROR_INVALID_PARAMETERS;
        memcpy(&dst, ptr, sizeof(dst));
        if (type) m->type = type;
        return VX_SUCCESS;
    };
    switch (attribute) {
    case VX_IMAGE_FORMAT: return take(m->format, VX_TYPE_IMAGE);
    case VX_IMAGE_WIDTH: return take(m->width, VX_TYPE_IMAGE);
    case VX_IMAGE_HEIGHT: return take(m->height, VX_TYPE_IMAGE);
    case VX_ARRAY_ITEMTYPE: return take(m->item_type, VX_TYPE_ARRAY);
    case VX_ARRAY_CAPACITY: return take(m->capacity, VX_TYPE_ARRAY);
    case VX_SCALAR_TYPE: return take(m->scalar_type, VX_TYPE_SCALAR);
    case VX_PYRAMID_LEVELS: return take(m->levels, VX_TYPE_PYRAMID);
    case VX_PYRAMID_SCALE: return take(m->scale, VX_TYPE_PYRAMID);
    case VX_PYRAMID_FORMAT: return take(m->format, VX_TYPE_PYRAMID);
    case VX_PYRAMID_WIDTH: return take(m->width, VX_TYPE_PYRAMID);
    case VX_PYRAMID_HEIGHT: return take(m->height, VX_TYPE_PYRAMID);
    case VX_VALID_RECT_CALLBACK: return take(m->valid_rect, 0);
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxQueryMetaFormatAttribute(vx_meta_format meta, vx_enum attribute, void *ptr, vx_size size)
{
    MetaFormat *m = meta_of(meta);
    if (!m) return VX_ERROR_INVALID_REFERENCE;
    if (!ptr) return VX_ERROR_INVALID_PARAMETERS;
    auto give = [&](const auto &src) {
        if (size != sizeof(src)) return VX_ERROR_INVALID_PARAMETERS;
        memcpy(ptr, &src, sizeof(src));
        return VX_SUCCESS;
    };
    switch (attribute) {
    case VX_IMAGE_FORMAT: case VX_PYRAMID_FORMAT: return give(m->format);
    case VX_IMAGE_WIDTH: case VX_PYRAMID_WIDTH: return give(m->width);
    case VX_IMAGE_HEIGHT: case VX_PYRAMID_HEIGHT: return give(m->height);
    case VX_ARRAY_ITEMTYPE: return give(m->item_type);
    case VX_ARRAY_CAPACITY: return give(m->capacity);
    case VX_SCALAR_TYPE: return give(m->scalar_type);
    case VX_PYRAMID_LEVELS: return give(m->levels);
    case VX_PYRAMID_SCALE: return give(m->scale);
    case VX_VALID_RECT_CALLBACK: return give(m->valid_rect);
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

vx_status vxSetMetaFormatFromReference(vx_meta_format meta, vx_reference exemplar)
{
    MetaFormat *m = meta_of(meta);
    if (!m) return VX_ERROR_INVALID_REFERENCE;
    if (!is_ref(exemplar)) return VX_ERROR_INVALID_REFERENCE;
    Ref *r = as<Ref>(exemplar);
    switch (r->type) {
    case VX_TYPE_IMAGE: {
        Image *img = static_cast<Image *>(r);
        m->type = VX_TYPE_IMAGE; m->format = img->format; m->width = img->width; m->height = img->height;
        return VX_SUCCESS;
    }
    case VX_TYPE_ARRAY: {
        Array *a = static_cast<Array *>(r);
        m->type = VX_TYPE_ARRAY; m->item_type = a->item_type; m->capacity = a->capacity;
        return VX_SUCCESS;
    }
    case VX_TYPE_SCALAR:
        m->type = VX_TYPE_SCALAR; m->scalar_type = static_cast<Scalar *>(r)->data_type;
        return VX_SUCCESS;
    case VX_TYPE_PYRAMID: {
        Pyramid *py = static_cast<Pyramid *>(r);
        m->type = VX_TYPE_PYRAMID; m->levels = py->levels; m->scale = py->scale; m->format = py->format;
        m->width = py->width; m->height = py->height;
        return VX_SUCCESS;
    }
    default: return VX_ERROR_NOT_SUPPORTED;
    }
}

}  // extern "C"
