// vx_internal.h -- object model of the B200 OpenVX/AGO engine.
//
// Objects are C++ structs behind the opaque OpenVX handles.  Data lives in device memory
// (HBM) first: every non-virtual image/array owns a device buffer and a lazily allocated
// pinned host mirror; `host_valid` / `dev_valid` track which copy is current, and copies
// happen only at the API boundary (copy/map/unmap) or just before a graph launch -- the
// same role AGO's agoDataSyncFromGpuToCpu / COPY_TO_HIPMEM play (ago/ago_interface.cpp:2005).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "agocuda.h"
#include "agovx.h"

namespace agovx {

constexpr uint32_t kMagic = 0xB200A60u;

struct Graph;
struct Context;

struct Ref {
    uint32_t magic = kMagic;
    vx_enum type = VX_TYPE_REFERENCE;
    Context *ctx = nullptr;
    Graph *scope = nullptr;          // owning graph for virtual objects
    int ext_count = 1;               // application references
    int int_count = 0;               // references held by graphs / nodes / parents
    bool is_virtual = false;
    bool released = false;           // application released its last reference
    std::string name;
    virtual ~Ref() = default;
};

bool is_valid(const void *r, vx_enum type);
inline bool is_ref(const void *r) { return r && static_cast<const Ref *>(r)->magic == kMagic; }

void log_error(Ref *ref, vx_status st, const char *fmt, ...);

// ------------------------------------------------------------------------------------
// Data objects
// ------------------------------------------------------------------------------------
struct Plane {
    uint32_t width = 0, height = 0;   // plane size in pixels
    uint32_t bpp = 1;                 // bytes per pixel (all channels)
    uint32_t dev_stride = 0;          // bytes
    uint32_t host_stride = 0;         // bytes
    uint8_t *dev = nullptr;           // device pointer to pixel (0,0)
    uint8_t *host = nullptr;          // host pointer to pixel (0,0)
    bool dev_owned = false, host_owned = false;
    size_t dev_bytes() const { return (size_t)dev_stride * height; }
    size_t host_bytes() const { return (size_t)host_stride * height; }
};

struct MapInfo { uint32_t plane; vx_rectangle_t rect; vx_enum usage; uint8_t *ptr; };

struct Image : Ref {
    uint32_t width = 0, height = 0;
    vx_df_image format = VX_DF_IMAGE_VIRT;
    vx_enum color_space = VX_COLOR_SPACE_BT709, color_range = VX_CHANNEL_RANGE_FULL;
    int num_planes = 0;
    Plane planes[3];
    vx_rectangle_t valid{0, 0, 0, 0};
    bool host_valid = false, dev_valid = false;
    bool uniform = false;
    vx_pixel_value_t uniform_value{};
    vx_enum import_type = VX_MEMORY_TYPE_NONE;  // HOST / HIP(device) for images from handle
    Image *parent = nullptr;          // pyramid/channel parent (shares memory)
    Image *view_of = nullptr;         // image this ROI / channel view holds an internal reference on
    std::vector<Image *> views;       // ROI views of this image (vxCreateImageFromROI): share its storage
    uint32_t view_x = 0, view_y = 0;  // a ROI view's offset in its parent's plane 0, in pixels
    bool roi_view = false;
    std::vector<Image *> children;    // planes of multi-plane images as U8 images (AGO children)
    std::map<vx_map_id, MapInfo> maps;
    vx_map_id next_map = 1;
    bool allocated() const { return num_planes > 0 && planes[0].dev != nullptr; }
    ~Image() override;
};

struct Scalar : Ref {
    vx_enum data_type = VX_TYPE_INVALID;
    union { vx_int8 i8; vx_uint8 u8; vx_int16 i16; vx_uint16 u16; vx_int32 i32; vx_uint32 u32; vx_int64 i64;
            vx_uint64 u64; vx_float32 f32; vx_float64 f64; vx_enum e; vx_size sz; vx_df_image df; vx_bool b;
            uint8_t raw[16]; } v{};
    uint32_t *dev = nullptr;          // device word for values written by kernels (sizes/counts)
    bool dev_newer = false;
    uint64_t version = 0;
    ~Scalar() override;
};

struct Threshold : Ref {
    vx_enum thresh_type = VX_THRESHOLD_TYPE_BINARY;
    vx_enum data_type = VX_TYPE_UINT8;
    vx_df_image input_format = VX_DF_IMAGE_U8, output_format = VX_DF_IMAGE_U8;
    vx_pixel_value_t value{}, lower{}, upper{}, true_value{}, false_value{};
    uint64_t version = 0;
};

struct Matrix : Ref {
    vx_enum data_type = VX_TYPE_FLOAT32;
    vx_size columns = 0, rows = 0;
    std::vector<uint8_t> data;
    uint64_t version = 0;
};

struct Array : Ref {
    vx_enum item_type = VX_TYPE_INVALID;
    vx_size item_size = 0, capacity = 0;
    // Device layout: items at `dev`; the item count lives in a separate device word so
    // kernels can append with atomics.  num_items is the host view of that count.
    uint8_t *dev = nullptr;
    uint32_t *dev_count = nullptr;
    std::vector<uint8_t> host;
    vx_size num_items = 0;
    bool host_valid = true, dev_valid = false;
    uint8_t *host_mapped = nullptr;   // device alias of `host` once it is page-locked (graph staging)
    std::map<vx_map_id, std::pair<vx_size, vx_enum>> maps;
    vx_map_id next_map = 1;
    ~Array() override;
};

struct Pyramid : Ref {
    vx_size levels = 0;
    vx_float32 scale = 0.5f;
    uint32_t width = 0, height = 0;
    vx_df_image format = VX_DF_IMAGE_U8;
    std::vector<Image *> level;
};

// Counts live on the device (written by the histogram kernel) and are read back on demand.
struct Distribution : Ref {
    vx_size bins = 0;
    vx_int32 offset = 0;
    vx_uint32 range = 0, window = 0;  // window = ceil(range / bins) (ago_util.cpp:2396)
    std::vector<uint32_t> host;
    uint32_t *dev = nullptr;
    bool dev_newer = false;
    std::map<vx_map_id, vx_enum> maps;
    vx_map_id next_map = 1;
    ~Distribution() override;
};

// vxCreateDelay: slot objects shaped like the exemplar.  vxGetReferenceFromDelay(-k) is the
// slot object k; ageing rotates the data storage among the slot objects (AGO's agoAgeDelay
// likewise moves buffers among the delay's children), so references handed out stay valid
// and graphs re-plan for the new device pointers.
struct Delay : Ref {
    vx_enum item_type = VX_TYPE_INVALID;
    std::vector<Ref *> slots;
};
vx_status delay_age(Delay *d);
struct Graph;
vx_status graph_import_text(Graph *g, const AgoGraphImportInfo *info);

struct Lut : Ref {
    vx_enum data_type = VX_TYPE_UINT8;  // UINT8 (count <= 256) or INT16 (count <= 65536)
    vx_size count = 0;
    uint32_t offset = 0;              // index of element 0: 0 for UINT8, count / 2 for INT16
    std::vector<uint8_t> data;
    uint64_t version = 0;
    std::map<vx_map_id, vx_enum> maps;
    vx_map_id next_map = 1;
};

struct Remap : Ref {
    uint32_t src_width = 0, src_height = 0, dst_width = 0, dst_height = 0;
    std::vector<vx_coordinates2df_t> table;     // dst_width * dst_height
    uint64_t version = 0;
};

// ------------------------------------------------------------------------------------
// Kernels, nodes and graphs
// ------------------------------------------------------------------------------------
// A parameter a user kernel declares (vxAddParameterToKernel).
struct UserParam {
    vx_enum dir = 0, type = 0, state = 0;
    bool set = false;
};

struct Kernel : Ref {
    vx_enum id = 0;
    std::string kname;
    int num_params = 0;
    const char *sig = "";             // parameter directions and types (vx_kernels.cpp)
    // user kernels (vxAddUserKernel, vx_api.cpp:2584): host callbacks and declared parameters
    bool user = false, finalized = false;
    bool gpu_access = false;          // VX_KERNEL_ATTRIBUTE_AMD_GPU_BUFFER_ACCESS_ENABLE: works on device buffers
    vx_kernel_f func = nullptr;
    vx_kernel_validate_f validate = nullptr;
    vx_kernel_initialize_f init = nullptr;
    vx_kernel_deinitialize_f deinit = nullptr;
    std::vector<UserParam> uparams;
    vx_size local_size = 0;           // VX_KERNEL_LOCAL_DATA_SIZE
};

// vx_meta_format: what a user kernel's validator says about one output parameter.
struct MetaFormat {
    uint32_t magic = 0x4d455441u;
    vx_enum type = 0;                 // VX_TYPE_IMAGE / ARRAY / SCALAR / PYRAMID (0: not set)
    vx_df_image format = 0;
    vx_uint32 width = 0, height = 0;
    vx_enum item_type = 0;
    vx_size capacity = 0;
    vx_enum scalar_type = 0;
    vx_size levels = 0;
    vx_float32 scale = 0.f;
    vx_kernel_image_valid_rectangle_f valid_rect = nullptr;
};

struct Convolution : Ref {
    vx_size columns = 0, rows = 0;
    vx_uint32 scale = 1;
    std::vector<vx_int16> coeffs;     // rows x columns, row-major as the application writes them
    uint64_t version = 0;
};

struct Node : Ref {
    vx_enum kernel = 0;               // OpenVX kernel enum (VX_KERNEL_*)
    std::vector<Ref *> params;
    vx_border_t border{VX_BORDER_UNDEFINED, {}};
    uint32_t affinity = 0;            // AGO_TARGET_AFFINITY_* (0 = graph default)
    vx_status status = VX_SUCCESS;
    vx_perf_t perf{};
    vx_size extra = 0;                // OpticalFlowPyrLK window_dimension
    int32_t iparam[2] = {0, 0};       // Canny: gradient_size / norm; Harris: gradient/block size
    vx_enum eparam = 0;               // interpolation / channel / policy / termination
    bool removed = false;
    // Device state that outlives a plan, as AGO's node scratch (localDataPtr) outlives
    // executions: LK's Scharr row buffer and level-0 derivative carry.  Zeroed once.
    void *state[2] = {nullptr, nullptr};
    size_t state_bytes[2] = {0, 0};
    void *node_state(int slot, size_t bytes);
    // user-kernel nodes: the kernel object, VX_NODE_LOCAL_DATA_SIZE / _PTR and whether the
    // kernel's initialize callback has run for the current verification
    Kernel *ukernel = nullptr;
    vx_size local_size = 0;
    void *local_ptr = nullptr;
    bool local_owned = false, initialized = false;
    ~Node() override;
};

// Low-level AGO kernels (names follow ago/ago_kernels.h) the OpenVX nodes lower to.
enum class LK : int {
    INVALID = 0,
    GAUSSIAN_U8_U8_3x3, SOBEL_S16_U8_3x3_GX, SOBEL_S16_U8_3x3_GY, SOBEL_S16S16_U8_3x3_GXY,
    MAGNITUDE_S16_S16S16, SOBEL_MAGNITUDE_S16_U8_3x3, COLOR_DEPTH_U8_S16_SAT, COLOR_DEPTH_U8_S16_WRAP,
    COLOR_DEPTH_S16_U8, THRESHOLD_U8_U8_BINARY, CHANNEL_COPY_U8_U8,
    CANNY_SOBEL_U16_U8_3x3_L1NORM, CANNY_SOBEL_U16_U8_3x3_L2NORM, CANNY_SUPP_THRESHOLD_U8XY_U16_3x3,
    CANNY_EDGE_TRACE_U8_U8XY,
    HARRIS_SOBEL_HG3_U8_3x3, HARRIS_SCORE_HVC_HG3_3x3, NON_MAX_SUPP_XY_ANY_3x3, HARRIS_MERGE_SORT_AND_PICK_XY_XYS,
    COLOR_CONVERT_Y_RGB, COLOR_CONVERT_UV12_RGB, COLOR_CONVERT_IU_RGB, COLOR_CONVERT_IV_RGB,
    COLOR_CONVERT_NV12_RGB, COLOR_CONVERT_IYUV_RGB,
    SCALE_IMAGE_U8_U8_NEAREST, SCALE_IMAGE_U8_U8_BILINEAR, SCALE_IMAGE_U8_U8_AREA,
    WARP_AFFINE_U8_U8_NEAREST, WARP_AFFINE_U8_U8_NEAREST_CONSTANT, WARP_AFFINE_U8_U8_BILINEAR,
    WARP_AFFINE_U8_U8_BILINEAR_CONSTANT, WARP_PERSPECTIVE_U8_U8_NEAREST_CONSTANT,
    WARP_PERSPECTIVE_U8_U8_BILINEAR_CONSTANT, REMAP_U8_U8_NEAREST_CONSTANT, REMAP_U8_U8_BILINEAR_CONSTANT,
    SCALE_GAUSSIAN_HALF_U8_U8_5x5, OPTICAL_FLOW_PYR_LK_XY_XY,
    WARP_PERSPECTIVE_U8_U8_NEAREST, WARP_PERSPECTIVE_U8_U8_BILINEAR, REMAP_U8_U8_NEAREST, REMAP_U8_U8_BILINEAR,
    BOX_U8_U8_3x3, DILATE_U8_U8_3x3, ERODE_U8_U8_3x3, MEDIAN_U8_U8_3x3,
    ABS_DIFF_U8_U8U8, ABS_DIFF_S16_S16S16_SAT,
    ADD_U8_U8U8_WRAP, ADD_U8_U8U8_SAT, ADD_S16_U8U8, ADD_S16_S16U8_WRAP, ADD_S16_S16U8_SAT,
    ADD_S16_S16S16_WRAP, ADD_S16_S16S16_SAT,
    SUB_U8_U8U8_WRAP, SUB_U8_U8U8_SAT, SUB_S16_U8U8, SUB_S16_S16U8_WRAP, SUB_S16_S16U8_SAT,
    SUB_S16_U8S16_WRAP, SUB_S16_U8S16_SAT, SUB_S16_S16S16_WRAP, SUB_S16_S16S16_SAT,
    AND_U8_U8U8, OR_U8_U8U8, XOR_U8_U8U8, NOT_U8_U8, THRESHOLD_U8_U8_RANGE,
    CHANNEL_EXTRACT_U8_U16_POS0, CHANNEL_EXTRACT_U8_U16_POS1, CHANNEL_EXTRACT_U8_U24_POS0, CHANNEL_EXTRACT_U8_U24_POS1,
    CHANNEL_EXTRACT_U8_U24_POS2, CHANNEL_EXTRACT_U8_U32_POS0, CHANNEL_EXTRACT_U8_U32_POS1, CHANNEL_EXTRACT_U8_U32_POS2,
    CHANNEL_EXTRACT_U8_U32_POS3, CHANNEL_COMBINE_U16_U8U8, CHANNEL_COMBINE_U24_U8U8U8_RGB,
    CHANNEL_COMBINE_U32_U8U8U8_UYVY, CHANNEL_COMBINE_U32_U8U8U8_YUYV, CHANNEL_COMBINE_U32_U8U8U8U8_RGBX,
    LUT_U8_U8, LUT_S16_S16, INTEGRAL_IMAGE_U32_U8, HISTOGRAM_DATA_U8,
    CANNY_SOBEL_U16_U8_5x5_L1NORM, CANNY_SOBEL_U16_U8_5x5_L2NORM, CANNY_SOBEL_U16_U8_7x7_L1NORM,
    CANNY_SOBEL_U16_U8_7x7_L2NORM, CANNY_SUPP_THRESHOLD_U8XY_U16_7x7,
    CONVOLVE_U8_U8, CONVOLVE_S16_U8,
    HARRIS_SOBEL_HG3_U8_5x5, HARRIS_SOBEL_HG3_U8_7x7, HARRIS_SCORE_HVC_HG3_5x5, HARRIS_SCORE_HVC_HG3_7x7,
    FAST_CORNERS_XY_U8_SUPRESSION, FAST_CORNERS_XY_U8_NOSUPRESSION,
    USER_KERNEL,                      // a vxAddUserKernel node, run on the host
    COUNT
};
const char *lk_name(LK k);

// A lowered node: AGO argument order (outputs first, ago/ago_drama_divide.cpp).
struct LNode {
    LK k = LK::INVALID;
    std::vector<Ref *> p;
    Node *origin = nullptr;
    vx_border_t border{VX_BORDER_UNDEFINED, {}};
    bool removed = false;
    int level = 0;                    // hierarchical level (longest path from graph inputs)
    int nout = -1;                    // outputs first; -1: the count the kernel kind implies
};

// One unit of device work in the execution plan: recorded into the CUDA graph.
// A piece of a step that can be ordered on its own: a batched step over independent
// frames splits into one part per frame.
struct Part {
    std::function<int(cudaStream_t)> launch;
    std::vector<LNode *> nodes;                 // lowered nodes the part covers
};

struct Step {
    std::string name;
    std::function<int(cudaStream_t)> launch;   // returns 0 or an agocuda/cuda error
    int num_kernels = 1;
    std::vector<LNode *> nodes;                 // lowered nodes this step covers
    std::vector<Part> parts;                    // optional split of `launch`, in launch order
};

// A verified plan and its captured CUDA graph, kept while another plan runs: ageing a delay
// alternates the graph between a few storage layouts, each with its own plan.
struct PlanState {
    std::vector<Step> steps;
    std::vector<void *> dev_scratch;
    cudaGraph_t cgraph = nullptr;
    cudaGraphExec_t cexec = nullptr;
    std::vector<Ref *> inputs, outputs;
    std::vector<Image *> streamed_in, streamed_out;
    std::vector<Array *> staged_in, staged_out;
    std::string plan_text;
    uint64_t use = 0;                            // last use, for eviction
};

struct Graph : Ref {
    std::vector<Node *> nodes;
    std::vector<LNode> lnodes;
    std::map<Ref *, Ref *> replaced;  // virtual data the copy-removal pass replaced by the copy's source
    std::vector<Step> steps;
    std::vector<Ref *> inputs, outputs;          // non-virtual data read / written by the graph
    std::vector<Ref *> owned_virtual;            // virtual data created for lowering
    std::vector<void *> dev_scratch;             // device allocations owned by the plan
    bool verified = false;
    bool host_steps = false;          // the plan calls user kernels on the host: launches are not captured
    vx_enum state = VX_GRAPH_STATE_UNVERIFIED;
    uint32_t optimizer_flags = 0;
    uint32_t affinity = 0;
    cudaStream_t stream = nullptr;
    cudaGraph_t cgraph = nullptr;
    cudaGraphExec_t cexec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaStream_t> lanes;             // streams forked from `stream` during capture
    std::vector<cudaEvent_t> cap_events;         // fork/join/dependency events of the capture
    std::vector<Image *> streamed_in, streamed_out;  // host images copied inside the CUDA graph
    // arrays copied inside the CUDA graph through their page-locked host buffers, with one
    // mapped count slot each (io_slots_host[i] <-> staged_in / staged_out in that order)
    std::vector<Array *> staged_in, staged_out;
    uint32_t *io_slots_host = nullptr, *io_slots_dev = nullptr;
    bool scheduled = false;
    vx_status last_status = VX_SUCCESS;
    vx_perf_t perf{};
    float gpu_ms_last = 0.f;
    double gpu_ns_total = 0.0;                   // device time of all launches (the AVG attribute)
    uint64_t gpu_runs = 0;
    uint64_t param_signature = 0;                // hash of by-value kernel parameters at capture
    // Device-side status word (mapped pinned memory): kernels set bits on bounded-wait
    // expiry or capacity overflow; checked after every launch.
    uint32_t *status_host = nullptr, *status_dev = nullptr;
    std::string plan_text;                       // human-readable plan (for tests / debugging)
    std::vector<Delay *> auto_age;               // delays aged after every execution (vxRegisterAutoAging)
    std::map<uint64_t, PlanState> plan_cache;    // other plans by parameter signature
    uint64_t plan_uses = 0;
    std::recursive_mutex lock;
    ~Graph() override;
};

struct Context : Ref {
    int device = 0;
    std::vector<vx_size> user_structs;   // vxRegisterUserStruct sizes, by enum - VX_TYPE_USER_STRUCT_START
    std::vector<Ref *> refs;          // every object created in this context
    vx_log_callback_f log_cb = nullptr;
    bool log_reentrant = false;
    std::mutex log_mutex;
    vx_border_t immediate_border{VX_BORDER_UNDEFINED, {}};
    uint32_t affinity = AGO_TARGET_AFFINITY_GPU;
    std::vector<Kernel *> kernels;
    bool tearing_down = false;        // vxReleaseContext deletes every object itself
    int in_user_kernel = 0;           // > 0 while a user kernel's callback runs: virtual data may be accessed
};

// Optimizer flag bits of VX_GRAPH_ATTRIBUTE_AMD_OPTIMIZER_FLAGS (ago/ago_internal.h:123-129),
// plus the bits this target adds.
constexpr uint32_t kOptNoDivide = 0x1, kOptNoRemoveCopy = 0x2, kOptNoRemoveUnused = 0x4, kOptNoMerge = 0x8;
constexpr uint32_t kOptNoFusion = 0x00010000;       // one launch per lowered node ("plain" form)
constexpr uint32_t kOptNoGraphCapture = 0x00020000; // launch steps directly instead of a CUDA graph
constexpr uint32_t kOptSerial = 0x00040000;         // capture on one stream (no concurrent branches)
constexpr uint32_t kOptNoTma = 0x00080000;          // pixel chains and pyramid levels load tiles without TMA

// helpers implemented in vx_objects.cpp
void add_ref(Context *ctx, Ref *r);
void retain_internal(Ref *r);
void release_internal(Ref *r);
void destroy_ref(Ref *r);
void graph_own(Graph *g, Ref *r);             // the graph's lowering holds r until re-lowered or released
void graph_release_owned(Graph *g);
vx_status image_alloc_device(Image *img);
void image_refresh_views(Image *root);
vx_status image_sync_to_device(Image *img, cudaStream_t s);
vx_status image_sync_to_host(Image *img);
void user_nodes_deinit(Graph *g);                 // vx_graph.cpp
int run_user_node(Graph *g, Node *n, cudaStream_t q);
vx_status array_alloc_device(Array *a);
vx_status array_sync_to_device(Array *a, cudaStream_t s);
vx_status array_sync_to_host(Array *a);
vx_status scalar_sync_to_host(Scalar *s);
vx_status scalar_alloc_device(Scalar *s);
Image *make_image(Context *ctx, Graph *scope, uint32_t w, uint32_t h, vx_df_image fmt, bool virt);
Array *make_array(Context *ctx, Graph *scope, vx_enum item_type, vx_size capacity, bool virt);
Scalar *make_scalar(Context *ctx, Graph *scope, vx_enum type, const void *ptr);
int format_planes(vx_df_image f, uint32_t w, uint32_t h, Plane *pl);
vx_size type_size(vx_enum t);
uint32_t align_up(uint32_t v, uint32_t a);

// implemented in vx_graph.cpp / plan.cpp
vx_status graph_verify(Graph *g);
vx_status graph_process(Graph *g, bool wait);
vx_status graph_wait(Graph *g);
void graph_invalidate(Graph *g);
vx_status lower_graph(Graph *g);
vx_status plan_graph(Graph *g);
vx_status propagate_valid_rects(Graph *g);
bool lnode_is_output(const LNode &ln, size_t i);

// scalar value accessors
inline int32_t sc_i32(Ref *r) { return static_cast<Scalar *>(r)->v.i32; }
inline float sc_f32(Ref *r) { return static_cast<Scalar *>(r)->v.f32; }
inline vx_enum sc_enum(Ref *r) { return static_cast<Scalar *>(r)->v.e; }
inline Image *IMG(Ref *r) { return static_cast<Image *>(r); }

}  // namespace agovx

// opaque-handle structs of the public ABI are the internal ones
struct _vx_reference : agovx::Ref {};
