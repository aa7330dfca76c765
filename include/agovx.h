/*
 * agovx.h -- the OpenVX 1.3 C API subset (plus the AMD extensions this path uses) exported
 * by mivisionx_b200's libopenvx.so.
 *
 * This is an ABI declaration written for this project: names, enum values, struct layouts
 * and function signatures are those of the Khronos OpenVX 1.3 headers and AMD's
 * vx_ext_amd.h as shipped by the reference (amd_openvx/openvx/include/VX/vx_types.h,
 * vx_api.h, vx_nodes.h, vx_kernels.h, include/vx_ext_amd.h), so a program compiled against
 * the Khronos headers links against this library unchanged.  tests/test_abi_header.py
 * compares every enum value here with the reference headers.
 */
#ifndef AGOVX_H
#define AGOVX_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- base types (vx_types.h) ---------------- */
typedef char vx_char;
typedef uint8_t vx_uint8;
typedef uint16_t vx_uint16;
typedef uint32_t vx_uint32;
typedef uint64_t vx_uint64;
typedef int8_t vx_int8;
typedef int16_t vx_int16;
typedef int32_t vx_int32;
typedef int64_t vx_int64;
typedef float vx_float32;
typedef double vx_float64;
typedef int32_t vx_enum;
typedef size_t vx_size;
typedef uint32_t vx_df_image;
typedef uintptr_t vx_map_id;
typedef vx_enum vx_bool;
typedef vx_enum vx_status;
typedef vx_enum vx_action;

enum { vx_false_e = 0, vx_true_e = 1 };

typedef struct _vx_reference *vx_reference;
typedef struct _vx_context *vx_context;
typedef struct _vx_graph *vx_graph;
typedef struct _vx_node *vx_node;
typedef struct _vx_kernel *vx_kernel;
typedef struct _vx_parameter *vx_parameter;
typedef struct _vx_image *vx_image;
typedef struct _vx_scalar *vx_scalar;
typedef struct _vx_threshold *vx_threshold;
typedef struct _vx_matrix *vx_matrix;
typedef struct _vx_array *vx_array;
typedef struct _vx_pyramid *vx_pyramid;
typedef struct _vx_remap *vx_remap;
typedef struct _vx_convolution *vx_convolution;
typedef struct _vx_delay *vx_delay;
typedef struct _vx_lut *vx_lut;
typedef struct _vx_distribution *vx_distribution;

#define VX_ID_KHRONOS 0x000
#define VX_ID_AMD 0x00D
#define VX_ATTRIBUTE_BASE(vendor, object) ((vx_int32)(((vx_uint32)(vendor) << 20) | ((vx_uint32)(object) << 8)))
#define VX_KERNEL_BASE(vendor, lib) ((vx_int32)(((vx_uint32)(vendor) << 20) | ((vx_uint32)(lib) << 12)))
#define VX_ENUM_BASE(vendor, id) ((vx_int32)(((vx_uint32)(vendor) << 20) | ((vx_uint32)(id) << 12)))
#define VX_DF_IMAGE(a, b, c, d) ((vx_uint32)(vx_uint8)(a) | ((vx_uint32)(vx_uint8)(b) << 8U) | \
                                 ((vx_uint32)(vx_uint8)(c) << 16U) | ((vx_uint32)(vx_uint8)(d) << 24U))
#define VX_SCALE_UNITY (1024u)
#define VX_SCALE_PYRAMID_HALF (0.5f)
#define VX_MAX_LOG_MESSAGE_LEN (1024)

enum vx_type_e {
    VX_TYPE_INVALID = 0x000, VX_TYPE_CHAR = 0x001, VX_TYPE_INT8 = 0x002, VX_TYPE_UINT8 = 0x003,
    VX_TYPE_INT16 = 0x004, VX_TYPE_UINT16 = 0x005, VX_TYPE_INT32 = 0x006, VX_TYPE_UINT32 = 0x007,
    VX_TYPE_INT64 = 0x008, VX_TYPE_UINT64 = 0x009, VX_TYPE_FLOAT32 = 0x00A, VX_TYPE_FLOAT64 = 0x00B,
    VX_TYPE_ENUM = 0x00C, VX_TYPE_SIZE = 0x00D, VX_TYPE_DF_IMAGE = 0x00E, VX_TYPE_FLOAT16 = 0x00F,
    VX_TYPE_BOOL = 0x010, VX_TYPE_RECTANGLE = 0x020, VX_TYPE_KEYPOINT = 0x021,
    VX_TYPE_COORDINATES2D = 0x022, VX_TYPE_COORDINATES3D = 0x023, VX_TYPE_COORDINATES2DF = 0x024,
    VX_TYPE_REFERENCE = 0x800, VX_TYPE_CONTEXT = 0x801, VX_TYPE_GRAPH = 0x802, VX_TYPE_NODE = 0x803,
    VX_TYPE_KERNEL = 0x804, VX_TYPE_PARAMETER = 0x805, VX_TYPE_DELAY = 0x806, VX_TYPE_LUT = 0x807,
    VX_TYPE_DISTRIBUTION = 0x808, VX_TYPE_PYRAMID = 0x809, VX_TYPE_THRESHOLD = 0x80A,
    VX_TYPE_MATRIX = 0x80B, VX_TYPE_CONVOLUTION = 0x80C, VX_TYPE_SCALAR = 0x80D, VX_TYPE_ARRAY = 0x80E,
    VX_TYPE_IMAGE = 0x80F, VX_TYPE_REMAP = 0x810, VX_TYPE_ERROR = 0x811, VX_TYPE_META_FORMAT = 0x812,
    VX_TYPE_OBJECT_ARRAY = 0x813,
};

enum vx_status_e {
    VX_STATUS_MIN = -25, VX_ERROR_REFERENCE_NONZERO = -24, VX_ERROR_MULTIPLE_WRITERS = -23,
    VX_ERROR_GRAPH_ABANDONED = -22, VX_ERROR_GRAPH_SCHEDULED = -21, VX_ERROR_INVALID_SCOPE = -20,
    VX_ERROR_INVALID_NODE = -19, VX_ERROR_INVALID_GRAPH = -18, VX_ERROR_INVALID_TYPE = -17,
    VX_ERROR_INVALID_VALUE = -16, VX_ERROR_INVALID_DIMENSION = -15, VX_ERROR_INVALID_FORMAT = -14,
    VX_ERROR_INVALID_LINK = -13, VX_ERROR_INVALID_REFERENCE = -12, VX_ERROR_INVALID_MODULE = -11,
    VX_ERROR_INVALID_PARAMETERS = -10, VX_ERROR_OPTIMIZED_AWAY = -9, VX_ERROR_NO_MEMORY = -8,
    VX_ERROR_NO_RESOURCES = -7, VX_ERROR_NOT_COMPATIBLE = -6, VX_ERROR_NOT_ALLOCATED = -5,
    VX_ERROR_NOT_SUFFICIENT = -4, VX_ERROR_NOT_SUPPORTED = -3, VX_ERROR_NOT_IMPLEMENTED = -2,
    VX_FAILURE = -1, VX_SUCCESS = 0,
};

enum vx_enum_e {
    VX_ENUM_DIRECTION = 0x00, VX_ENUM_ACTION = 0x01, VX_ENUM_HINT = 0x02, VX_ENUM_DIRECTIVE = 0x03,
    VX_ENUM_INTERPOLATION = 0x04, VX_ENUM_OVERFLOW = 0x05, VX_ENUM_COLOR_SPACE = 0x06,
    VX_ENUM_COLOR_RANGE = 0x07, VX_ENUM_PARAMETER_STATE = 0x08, VX_ENUM_CHANNEL = 0x09,
    VX_ENUM_CONVERT_POLICY = 0x0A, VX_ENUM_THRESHOLD_TYPE = 0x0B, VX_ENUM_BORDER = 0x0C,
    VX_ENUM_COMPARISON = 0x0D, VX_ENUM_MEMORY_TYPE = 0x0E, VX_ENUM_TERM_CRITERIA = 0x0F,
    VX_ENUM_NORM_TYPE = 0x10, VX_ENUM_ACCESSOR = 0x11, VX_ENUM_ROUND_POLICY = 0x12,
    VX_ENUM_TARGET = 0x13, VX_ENUM_BORDER_POLICY = 0x14, VX_ENUM_GRAPH_STATE = 0x15,
};

#define VX__E(id, n) (VX_ENUM_BASE(VX_ID_KHRONOS, id) + (n))
#define VX__A(obj, n) (VX_ATTRIBUTE_BASE(VX_ID_KHRONOS, obj) + (n))

enum { VX_INPUT = VX__E(VX_ENUM_DIRECTION, 0), VX_OUTPUT = VX__E(VX_ENUM_DIRECTION, 1),
       VX_BIDIRECTIONAL = VX__E(VX_ENUM_DIRECTION, 2) };
enum { VX_ACTION_CONTINUE = VX__E(VX_ENUM_ACTION, 0), VX_ACTION_ABANDON = VX__E(VX_ENUM_ACTION, 1) };
enum { VX_DIRECTIVE_DISABLE_LOGGING = VX__E(VX_ENUM_DIRECTIVE, 0), VX_DIRECTIVE_ENABLE_LOGGING = VX__E(VX_ENUM_DIRECTIVE, 1),
       VX_DIRECTIVE_DISABLE_PERFORMANCE = VX__E(VX_ENUM_DIRECTIVE, 2), VX_DIRECTIVE_ENABLE_PERFORMANCE = VX__E(VX_ENUM_DIRECTIVE, 3) };
enum { VX_INTERPOLATION_NEAREST_NEIGHBOR = VX__E(VX_ENUM_INTERPOLATION, 0),
       VX_INTERPOLATION_BILINEAR = VX__E(VX_ENUM_INTERPOLATION, 1),
       VX_INTERPOLATION_AREA = VX__E(VX_ENUM_INTERPOLATION, 2) };
enum { VX_COLOR_SPACE_NONE = VX__E(VX_ENUM_COLOR_SPACE, 0), VX_COLOR_SPACE_BT601_525 = VX__E(VX_ENUM_COLOR_SPACE, 1),
       VX_COLOR_SPACE_BT601_625 = VX__E(VX_ENUM_COLOR_SPACE, 2), VX_COLOR_SPACE_BT709 = VX__E(VX_ENUM_COLOR_SPACE, 3),
       VX_COLOR_SPACE_DEFAULT = VX__E(VX_ENUM_COLOR_SPACE, 3) };
enum { VX_CHANNEL_RANGE_FULL = VX__E(VX_ENUM_COLOR_RANGE, 0), VX_CHANNEL_RANGE_RESTRICTED = VX__E(VX_ENUM_COLOR_RANGE, 1) };
enum { VX_PARAMETER_STATE_REQUIRED = VX__E(VX_ENUM_PARAMETER_STATE, 0), VX_PARAMETER_STATE_OPTIONAL = VX__E(VX_ENUM_PARAMETER_STATE, 1) };
enum { VX_CHANNEL_0 = VX__E(VX_ENUM_CHANNEL, 0), VX_CHANNEL_1 = VX__E(VX_ENUM_CHANNEL, 1),
       VX_CHANNEL_2 = VX__E(VX_ENUM_CHANNEL, 2), VX_CHANNEL_3 = VX__E(VX_ENUM_CHANNEL, 3),
       VX_CHANNEL_R = VX__E(VX_ENUM_CHANNEL, 0x10), VX_CHANNEL_G = VX__E(VX_ENUM_CHANNEL, 0x11),
       VX_CHANNEL_B = VX__E(VX_ENUM_CHANNEL, 0x12), VX_CHANNEL_A = VX__E(VX_ENUM_CHANNEL, 0x13),
       VX_CHANNEL_Y = VX__E(VX_ENUM_CHANNEL, 0x14), VX_CHANNEL_U = VX__E(VX_ENUM_CHANNEL, 0x15),
       VX_CHANNEL_V = VX__E(VX_ENUM_CHANNEL, 0x16) };
enum { VX_CONVERT_POLICY_WRAP = VX__E(VX_ENUM_CONVERT_POLICY, 0), VX_CONVERT_POLICY_SATURATE = VX__E(VX_ENUM_CONVERT_POLICY, 1) };
enum { VX_THRESHOLD_TYPE_BINARY = VX__E(VX_ENUM_THRESHOLD_TYPE, 0), VX_THRESHOLD_TYPE_RANGE = VX__E(VX_ENUM_THRESHOLD_TYPE, 1) };
enum { VX_BORDER_UNDEFINED = VX__E(VX_ENUM_BORDER, 0), VX_BORDER_CONSTANT = VX__E(VX_ENUM_BORDER, 1),
       VX_BORDER_REPLICATE = VX__E(VX_ENUM_BORDER, 2) };
enum { VX_MEMORY_TYPE_NONE = VX__E(VX_ENUM_MEMORY_TYPE, 0), VX_MEMORY_TYPE_HOST = VX__E(VX_ENUM_MEMORY_TYPE, 1),
       VX_MEMORY_TYPE_OPENCL = VX__E(VX_ENUM_MEMORY_TYPE, 2),
       /* AMD: device memory import (vx_ext_amd.h vx_memory_type_amd_e); on this target it
        * means CUDA device memory of the context's device. */
       VX_MEMORY_TYPE_HIP = VX__E(VX_ENUM_MEMORY_TYPE, 3) };
enum { VX_TERM_CRITERIA_ITERATIONS = VX__E(VX_ENUM_TERM_CRITERIA, 0), VX_TERM_CRITERIA_EPSILON = VX__E(VX_ENUM_TERM_CRITERIA, 1),
       VX_TERM_CRITERIA_BOTH = VX__E(VX_ENUM_TERM_CRITERIA, 2) };
enum { VX_NORM_L1 = VX__E(VX_ENUM_NORM_TYPE, 0), VX_NORM_L2 = VX__E(VX_ENUM_NORM_TYPE, 1) };
enum { VX_READ_ONLY = VX__E(VX_ENUM_ACCESSOR, 1), VX_WRITE_ONLY = VX__E(VX_ENUM_ACCESSOR, 2),
       VX_READ_AND_WRITE = VX__E(VX_ENUM_ACCESSOR, 3) };
enum { VX_TARGET_ANY = VX__E(VX_ENUM_TARGET, 0), VX_TARGET_STRING = VX__E(VX_ENUM_TARGET, 1) };
enum { VX_GRAPH_STATE_UNVERIFIED = VX__E(VX_ENUM_GRAPH_STATE, 0), VX_GRAPH_STATE_VERIFIED = VX__E(VX_ENUM_GRAPH_STATE, 1),
       VX_GRAPH_STATE_RUNNING = VX__E(VX_ENUM_GRAPH_STATE, 2), VX_GRAPH_STATE_ABANDONED = VX__E(VX_ENUM_GRAPH_STATE, 3),
       VX_GRAPH_STATE_COMPLETED = VX__E(VX_ENUM_GRAPH_STATE, 4) };
enum { VX_NOGAP_X = 1 };

enum vx_df_image_e {
    VX_DF_IMAGE_VIRT = VX_DF_IMAGE('V', 'I', 'R', 'T'), VX_DF_IMAGE_RGB = VX_DF_IMAGE('R', 'G', 'B', '2'),
    VX_DF_IMAGE_RGBX = VX_DF_IMAGE('R', 'G', 'B', 'A'), VX_DF_IMAGE_NV12 = VX_DF_IMAGE('N', 'V', '1', '2'),
    VX_DF_IMAGE_NV21 = VX_DF_IMAGE('N', 'V', '2', '1'), VX_DF_IMAGE_UYVY = VX_DF_IMAGE('U', 'Y', 'V', 'Y'),
    VX_DF_IMAGE_YUYV = VX_DF_IMAGE('Y', 'U', 'Y', 'V'), VX_DF_IMAGE_IYUV = VX_DF_IMAGE('I', 'Y', 'U', 'V'),
    VX_DF_IMAGE_YUV4 = VX_DF_IMAGE('Y', 'U', 'V', '4'), VX_DF_IMAGE_U1 = VX_DF_IMAGE('U', '0', '0', '1'),
    VX_DF_IMAGE_U8 = VX_DF_IMAGE('U', '0', '0', '8'), VX_DF_IMAGE_U16 = VX_DF_IMAGE('U', '0', '1', '6'),
    VX_DF_IMAGE_S16 = VX_DF_IMAGE('S', '0', '1', '6'), VX_DF_IMAGE_U32 = VX_DF_IMAGE('U', '0', '3', '2'),
    VX_DF_IMAGE_S32 = VX_DF_IMAGE('S', '0', '3', '2'),
    /* AMD formats (vx_ext_amd.h): F32 planes used by the float warp/remap path */
    VX_DF_IMAGE_F32_AMD = VX_DF_IMAGE('F', '0', '3', '2'),
};

/* attributes */
enum { VX_REFERENCE_COUNT = VX__A(VX_TYPE_REFERENCE, 0), VX_REFERENCE_TYPE = VX__A(VX_TYPE_REFERENCE, 1),
       VX_REFERENCE_NAME = VX__A(VX_TYPE_REFERENCE, 2) };
enum { VX_CONTEXT_VENDOR_ID = VX__A(VX_TYPE_CONTEXT, 0), VX_CONTEXT_VERSION = VX__A(VX_TYPE_CONTEXT, 1),
       VX_CONTEXT_UNIQUE_KERNELS = VX__A(VX_TYPE_CONTEXT, 2), VX_CONTEXT_MODULES = VX__A(VX_TYPE_CONTEXT, 3),
       VX_CONTEXT_REFERENCES = VX__A(VX_TYPE_CONTEXT, 4), VX_CONTEXT_IMPLEMENTATION = VX__A(VX_TYPE_CONTEXT, 5),
       VX_CONTEXT_IMMEDIATE_BORDER = VX__A(VX_TYPE_CONTEXT, 0xA) };
enum { VX_GRAPH_NUMNODES = VX__A(VX_TYPE_GRAPH, 0), VX_GRAPH_PERFORMANCE = VX__A(VX_TYPE_GRAPH, 2),
       VX_GRAPH_NUMPARAMETERS = VX__A(VX_TYPE_GRAPH, 3), VX_GRAPH_STATE = VX__A(VX_TYPE_GRAPH, 4) };
enum { VX_NODE_STATUS = VX__A(VX_TYPE_NODE, 0), VX_NODE_PERFORMANCE = VX__A(VX_TYPE_NODE, 1),
       VX_NODE_BORDER = VX__A(VX_TYPE_NODE, 2), VX_NODE_LOCAL_DATA_SIZE = VX__A(VX_TYPE_NODE, 3),
       VX_NODE_LOCAL_DATA_PTR = VX__A(VX_TYPE_NODE, 4), VX_NODE_PARAMETERS = VX__A(VX_TYPE_NODE, 5) };
enum { VX_IMAGE_WIDTH = VX__A(VX_TYPE_IMAGE, 0), VX_IMAGE_HEIGHT = VX__A(VX_TYPE_IMAGE, 1),
       VX_IMAGE_FORMAT = VX__A(VX_TYPE_IMAGE, 2), VX_IMAGE_PLANES = VX__A(VX_TYPE_IMAGE, 3),
       VX_IMAGE_SPACE = VX__A(VX_TYPE_IMAGE, 4), VX_IMAGE_RANGE = VX__A(VX_TYPE_IMAGE, 5),
       VX_IMAGE_SIZE = VX__A(VX_TYPE_IMAGE, 6), VX_IMAGE_MEMORY_TYPE = VX__A(VX_TYPE_IMAGE, 7),
       VX_IMAGE_IS_UNIFORM = VX__A(VX_TYPE_IMAGE, 8), VX_IMAGE_UNIFORM_VALUE = VX__A(VX_TYPE_IMAGE, 9) };
enum { VX_SCALAR_TYPE = VX__A(VX_TYPE_SCALAR, 0) };
enum { VX_THRESHOLD_TYPE = VX__A(VX_TYPE_THRESHOLD, 0), VX_THRESHOLD_THRESHOLD_VALUE = VX__A(VX_TYPE_THRESHOLD, 1),
       VX_THRESHOLD_THRESHOLD_LOWER = VX__A(VX_TYPE_THRESHOLD, 2), VX_THRESHOLD_THRESHOLD_UPPER = VX__A(VX_TYPE_THRESHOLD, 3),
       VX_THRESHOLD_TRUE_VALUE = VX__A(VX_TYPE_THRESHOLD, 4), VX_THRESHOLD_FALSE_VALUE = VX__A(VX_TYPE_THRESHOLD, 5),
       VX_THRESHOLD_DATA_TYPE = VX__A(VX_TYPE_THRESHOLD, 6), VX_THRESHOLD_INPUT_FORMAT = VX__A(VX_TYPE_THRESHOLD, 7),
       VX_THRESHOLD_OUTPUT_FORMAT = VX__A(VX_TYPE_THRESHOLD, 8) };
enum { VX_DISTRIBUTION_DIMENSIONS = VX__A(VX_TYPE_DISTRIBUTION, 0), VX_DISTRIBUTION_OFFSET = VX__A(VX_TYPE_DISTRIBUTION, 1),
       VX_DISTRIBUTION_RANGE = VX__A(VX_TYPE_DISTRIBUTION, 2), VX_DISTRIBUTION_BINS = VX__A(VX_TYPE_DISTRIBUTION, 3),
       VX_DISTRIBUTION_WINDOW = VX__A(VX_TYPE_DISTRIBUTION, 4), VX_DISTRIBUTION_SIZE = VX__A(VX_TYPE_DISTRIBUTION, 5) };
enum { VX_LUT_TYPE = VX__A(VX_TYPE_LUT, 0), VX_LUT_COUNT = VX__A(VX_TYPE_LUT, 1), VX_LUT_SIZE = VX__A(VX_TYPE_LUT, 2),
       VX_LUT_OFFSET = VX__A(VX_TYPE_LUT, 3) };
enum { VX_MATRIX_TYPE = VX__A(VX_TYPE_MATRIX, 0), VX_MATRIX_ROWS = VX__A(VX_TYPE_MATRIX, 1),
       VX_MATRIX_COLUMNS = VX__A(VX_TYPE_MATRIX, 2), VX_MATRIX_SIZE = VX__A(VX_TYPE_MATRIX, 3) };
enum { VX_PYRAMID_LEVELS = VX__A(VX_TYPE_PYRAMID, 0), VX_PYRAMID_SCALE = VX__A(VX_TYPE_PYRAMID, 1),
       VX_PYRAMID_WIDTH = VX__A(VX_TYPE_PYRAMID, 2), VX_PYRAMID_HEIGHT = VX__A(VX_TYPE_PYRAMID, 3),
       VX_PYRAMID_FORMAT = VX__A(VX_TYPE_PYRAMID, 4) };
enum { VX_REMAP_SOURCE_WIDTH = VX__A(VX_TYPE_REMAP, 0), VX_REMAP_SOURCE_HEIGHT = VX__A(VX_TYPE_REMAP, 1),
       VX_REMAP_DESTINATION_WIDTH = VX__A(VX_TYPE_REMAP, 2), VX_REMAP_DESTINATION_HEIGHT = VX__A(VX_TYPE_REMAP, 3) };
enum { VX_ARRAY_ITEMTYPE = VX__A(VX_TYPE_ARRAY, 0), VX_ARRAY_NUMITEMS = VX__A(VX_TYPE_ARRAY, 1),
       VX_ARRAY_CAPACITY = VX__A(VX_TYPE_ARRAY, 2), VX_ARRAY_ITEMSIZE = VX__A(VX_TYPE_ARRAY, 3) };

/* AMD vendor attributes and directives (include/vx_ext_amd.h) */
#define AGO_TARGET_AFFINITY_CPU 0x0010
#define AGO_TARGET_AFFINITY_GPU 0x0020
enum { VX_CONTEXT_ATTRIBUTE_AMD_AFFINITY = VX_ATTRIBUTE_BASE(VX_ID_AMD, VX_TYPE_CONTEXT) + 0x02,
       VX_CONTEXT_ATTRIBUTE_AMD_HIP_DEVICE = VX_ATTRIBUTE_BASE(VX_ID_AMD, VX_TYPE_CONTEXT) + 0x07 };
enum { VX_GRAPH_ATTRIBUTE_AMD_AFFINITY = VX_ATTRIBUTE_BASE(VX_ID_AMD, VX_TYPE_GRAPH) + 0x01,
       VX_GRAPH_ATTRIBUTE_AMD_IMPORT_FROM_TEXT = VX_ATTRIBUTE_BASE(VX_ID_AMD, VX_TYPE_GRAPH) + 0x02,
       VX_GRAPH_ATTRIBUTE_AMD_EXPORT_TO_TEXT = VX_ATTRIBUTE_BASE(VX_ID_AMD, VX_TYPE_GRAPH) + 0x03,
       VX_GRAPH_ATTRIBUTE_AMD_OPTIMIZER_FLAGS = VX_ATTRIBUTE_BASE(VX_ID_AMD, VX_TYPE_GRAPH) + 0x04,
       VX_GRAPH_ATTRIBUTE_AMD_PERFORMANCE_INTERNAL_LAST = VX_ATTRIBUTE_BASE(VX_ID_AMD, VX_TYPE_GRAPH) + 0x05,
       VX_GRAPH_ATTRIBUTE_AMD_PERFORMANCE_INTERNAL_AVG = VX_ATTRIBUTE_BASE(VX_ID_AMD, VX_TYPE_GRAPH) + 0x06,
       VX_GRAPH_ATTRIBUTE_AMD_PERFORMANCE_INTERNAL_PROFILE = VX_ATTRIBUTE_BASE(VX_ID_AMD, VX_TYPE_GRAPH) + 0x07 };
enum { VX_NODE_ATTRIBUTE_AMD_AFFINITY = VX_ATTRIBUTE_BASE(VX_ID_AMD, VX_TYPE_NODE) + 0x01,
       VX_NODE_ATTRIBUTE_AMD_HIP_STREAM = VX_ATTRIBUTE_BASE(VX_ID_AMD, VX_TYPE_NODE) + 0x03 };
enum { VX_IMAGE_ATTRIBUTE_AMD_GPU_BUFFER_OFFSET = VX_ATTRIBUTE_BASE(VX_ID_AMD, VX_TYPE_IMAGE) + 0x02,
       VX_IMAGE_ATTRIBUTE_AMD_GPU_BUFFER_STRIDE = VX_ATTRIBUTE_BASE(VX_ID_AMD, VX_TYPE_IMAGE) + 0x04,
       VX_IMAGE_ATTRIBUTE_AMD_HIP_BUFFER = VX_ATTRIBUTE_BASE(VX_ID_AMD, VX_TYPE_IMAGE) + 0x06 };
enum { VX_DIRECTIVE_AMD_READ_ONLY = VX_ENUM_BASE(VX_ID_AMD, VX_ENUM_DIRECTIVE) + 0x01,
       VX_DIRECTIVE_AMD_COPY_TO_HIPMEM = VX_ENUM_BASE(VX_ID_AMD, VX_ENUM_DIRECTIVE) + 0x02,
       VX_DIRECTIVE_AMD_ENABLE_PROFILE_CAPTURE = VX_ENUM_BASE(VX_ID_AMD, VX_ENUM_DIRECTIVE) + 0x03,
       VX_DIRECTIVE_AMD_DISABLE_PROFILE_CAPTURE = VX_ENUM_BASE(VX_ID_AMD, VX_ENUM_DIRECTIVE) + 0x04,
       VX_DIRECTIVE_AMD_DISABLE_GPU_FLUSH = VX_ENUM_BASE(VX_ID_AMD, VX_ENUM_DIRECTIVE) + 0x05 };

typedef struct {
    vx_uint32 device_type;  /* AGO_TARGET_AFFINITY_CPU or AGO_TARGET_AFFINITY_GPU */
    vx_uint32 device_info, group, reserved;
} AgoTargetAffinityInfo;

/* VX_GRAPH_ATTRIBUTE_AMD_IMPORT_FROM_TEXT argument (vx_ext_amd.h AgoGraphImportInfo) */
typedef struct {
    vx_char *text;
    vx_uint32 num_ref;
    vx_reference *ref;
    vx_int32 dumpToConsole;
    void (*data_registry_callback_f)(void *obj, vx_reference ref, const char *name, const char *app_params);
    void *data_registry_callback_obj;
} AgoGraphImportInfo;

/* kernels (vx_kernels.h) */
#define VX__K(n) (VX_KERNEL_BASE(VX_ID_KHRONOS, 0) + (n))
enum vx_kernel_e {
    VX_KERNEL_COLOR_CONVERT = VX__K(0x1), VX_KERNEL_CHANNEL_EXTRACT = VX__K(0x2), VX_KERNEL_CHANNEL_COMBINE = VX__K(0x3),
    VX_KERNEL_SOBEL_3x3 = VX__K(0x4), VX_KERNEL_MAGNITUDE = VX__K(0x5), VX_KERNEL_PHASE = VX__K(0x6),
    VX_KERNEL_SCALE_IMAGE = VX__K(0x7), VX_KERNEL_TABLE_LOOKUP = VX__K(0x8), VX_KERNEL_ABSDIFF = VX__K(0xB), VX_KERNEL_THRESHOLD = VX__K(0xD),
    VX_KERNEL_INTEGRAL_IMAGE = VX__K(0xE), VX_KERNEL_HISTOGRAM = VX__K(0x9),
    VX_KERNEL_DILATE_3x3 = VX__K(0xF), VX_KERNEL_ERODE_3x3 = VX__K(0x10), VX_KERNEL_MEDIAN_3x3 = VX__K(0x11),
    VX_KERNEL_BOX_3x3 = VX__K(0x12), VX_KERNEL_AND = VX__K(0x1C), VX_KERNEL_OR = VX__K(0x1D), VX_KERNEL_XOR = VX__K(0x1E),
    VX_KERNEL_NOT = VX__K(0x1F), VX_KERNEL_ADD = VX__K(0x21), VX_KERNEL_SUBTRACT = VX__K(0x22),
    VX_KERNEL_GAUSSIAN_3x3 = VX__K(0x13), VX_KERNEL_GAUSSIAN_PYRAMID = VX__K(0x15),
    VX_KERNEL_CONVERTDEPTH = VX__K(0x1A), VX_KERNEL_CANNY_EDGE_DETECTOR = VX__K(0x1B),
    VX_KERNEL_WARP_AFFINE = VX__K(0x23), VX_KERNEL_WARP_PERSPECTIVE = VX__K(0x24),
    VX_KERNEL_HARRIS_CORNERS = VX__K(0x25), VX_KERNEL_OPTICAL_FLOW_PYR_LK = VX__K(0x27),
    VX_KERNEL_REMAP = VX__K(0x28), VX_KERNEL_HALFSCALE_GAUSSIAN = VX__K(0x29),
    VX_KERNEL_EQUALIZE_HISTOGRAM = VX__K(0xA), VX_KERNEL_MEAN_STDDEV = VX__K(0xC), VX_KERNEL_CUSTOM_CONVOLUTION = VX__K(0x14),
    VX_KERNEL_ACCUMULATE = VX__K(0x16), VX_KERNEL_ACCUMULATE_WEIGHTED = VX__K(0x17), VX_KERNEL_ACCUMULATE_SQUARE = VX__K(0x18),
    VX_KERNEL_MINMAXLOC = VX__K(0x19), VX_KERNEL_MULTIPLY = VX__K(0x20), VX_KERNEL_FAST_CORNERS = VX__K(0x26),
    VX_KERNEL_WEIGHTED_AVERAGE = VX__K(0x40),
};

/* structures */
typedef struct _vx_imagepatch_addressing_t {
    vx_uint32 dim_x, dim_y;
    vx_int32 stride_x, stride_y;
    vx_uint32 scale_x, scale_y;
    vx_uint32 step_x;
    vx_uint16 step_y;
    vx_uint16 stride_x_bits;
} vx_imagepatch_addressing_t;
typedef struct _vx_perf_t { vx_uint64 tmp, beg, end, sum, avg, min, num, max; } vx_perf_t;
typedef struct _vx_keypoint_t {
    vx_int32 x, y;
    vx_float32 strength, scale, orientation;
    vx_int32 tracking_status;
    vx_float32 error;
} vx_keypoint_t;
typedef struct _vx_rectangle_t { vx_uint32 start_x, start_y, end_x, end_y; } vx_rectangle_t;
typedef struct _vx_coordinates2d_t { vx_uint32 x, y; } vx_coordinates2d_t;
typedef struct _vx_coordinates2df_t { vx_float32 x, y; } vx_coordinates2df_t;
typedef union _vx_pixel_value_t {
    vx_uint8 RGB[3]; vx_uint8 RGBX[4]; vx_uint8 YUV[3]; vx_bool U1; vx_uint8 U8; vx_uint16 U16;
    vx_int16 S16; vx_uint32 U32; vx_int32 S32; vx_uint8 reserved[16];
} vx_pixel_value_t;
typedef struct _vx_border_t { vx_enum mode; vx_pixel_value_t constant_value; } vx_border_t;
typedef void (*vx_log_callback_f)(vx_context context, vx_reference ref, vx_status status, const vx_char string[]);

/* ---------------- API (vx_api.h) ---------------- */
vx_context vxCreateContext(void);
vx_status vxReleaseContext(vx_context *context);
vx_context vxGetContext(vx_reference reference);
vx_status vxGetStatus(vx_reference reference);
vx_status vxQueryContext(vx_context context, vx_enum attribute, void *ptr, vx_size size);
vx_status vxSetContextAttribute(vx_context context, vx_enum attribute, const void *ptr, vx_size size);
vx_status vxDirective(vx_reference reference, vx_enum directive);
vx_status vxQueryReference(vx_reference ref, vx_enum attribute, void *ptr, vx_size size);
vx_status vxReleaseReference(vx_reference *ref_ptr);
vx_status vxRetainReference(vx_reference ref);
vx_status vxSetReferenceName(vx_reference ref, const vx_char *name);
void vxRegisterLogCallback(vx_context context, vx_log_callback_f callback, vx_bool reentrant);
void vxAddLogEntry(vx_reference ref, vx_status status, const char *message, ...);

vx_image vxCreateImage(vx_context context, vx_uint32 width, vx_uint32 height, vx_df_image color);
vx_image vxCreateVirtualImage(vx_graph graph, vx_uint32 width, vx_uint32 height, vx_df_image color);
vx_image vxCreateUniformImage(vx_context context, vx_uint32 width, vx_uint32 height, vx_df_image color, const vx_pixel_value_t *value);
vx_image vxCreateImageFromHandle(vx_context context, vx_df_image color, const vx_imagepatch_addressing_t addrs[],
                                 void *const ptrs[], vx_enum memory_type);
vx_status vxSwapImageHandle(vx_image image, void *const new_ptrs[], void *prev_ptrs[], vx_size num_planes);
vx_status vxQueryImage(vx_image image, vx_enum attribute, void *ptr, vx_size size);
vx_status vxReleaseImage(vx_image *image);
vx_status vxCopyImagePatch(vx_image image, const vx_rectangle_t *image_rect, vx_uint32 image_plane_index,
                           const vx_imagepatch_addressing_t *user_addr, void *user_ptr, vx_enum usage, vx_enum user_mem_type);
vx_status vxMapImagePatch(vx_image image, const vx_rectangle_t *rect, vx_uint32 plane_index, vx_map_id *map_id,
                          vx_imagepatch_addressing_t *addr, void **ptr, vx_enum usage, vx_enum mem_type, vx_uint32 flags);
vx_status vxUnmapImagePatch(vx_image image, vx_map_id map_id);
vx_status vxGetValidRegionImage(vx_image image, vx_rectangle_t *rect);
vx_status vxSetImageValidRectangle(vx_image image, const vx_rectangle_t *rect);

vx_graph vxCreateGraph(vx_context context);
vx_status vxReleaseGraph(vx_graph *graph);
vx_status vxVerifyGraph(vx_graph graph);
vx_status vxProcessGraph(vx_graph graph);
vx_status vxScheduleGraph(vx_graph graph);
vx_status vxWaitGraph(vx_graph graph);
vx_status vxQueryGraph(vx_graph graph, vx_enum attribute, void *ptr, vx_size size);
vx_status vxSetGraphAttribute(vx_graph graph, vx_enum attribute, const void *ptr, vx_size size);
vx_bool vxIsGraphVerified(vx_graph graph);

vx_status vxQueryNode(vx_node node, vx_enum attribute, void *ptr, vx_size size);
vx_status vxSetNodeAttribute(vx_node node, vx_enum attribute, const void *ptr, vx_size size);
vx_status vxReleaseNode(vx_node *node);
vx_status vxRemoveNode(vx_node *node);
vx_status vxSetNodeTarget(vx_node node, vx_enum target_enum, const char *target_string);

vx_scalar vxCreateScalar(vx_context context, vx_enum data_type, const void *ptr);
vx_status vxReleaseScalar(vx_scalar *scalar);
vx_status vxQueryScalar(vx_scalar scalar, vx_enum attribute, void *ptr, vx_size size);
vx_status vxCopyScalar(vx_scalar scalar, void *user_ptr, vx_enum usage, vx_enum user_mem_type);

vx_threshold vxCreateThreshold(vx_context c, vx_enum thresh_type, vx_enum data_type);
vx_threshold vxCreateThresholdForImage(vx_context context, vx_enum thresh_type, vx_df_image input_format, vx_df_image output_format);
vx_status vxReleaseThreshold(vx_threshold *thresh);
vx_status vxSetThresholdAttribute(vx_threshold thresh, vx_enum attribute, const void *ptr, vx_size size);
vx_status vxQueryThreshold(vx_threshold thresh, vx_enum attribute, void *ptr, vx_size size);
vx_status vxCopyThresholdValue(vx_threshold thresh, vx_pixel_value_t *value_ptr, vx_enum usage, vx_enum user_mem_type);
vx_status vxCopyThresholdRange(vx_threshold thresh, vx_pixel_value_t *lower_value_ptr, vx_pixel_value_t *upper_value_ptr,
                               vx_enum usage, vx_enum user_mem_type);

enum { VX_DELAY_TYPE = VX__A(VX_TYPE_DELAY, 0), VX_DELAY_SLOTS = VX__A(VX_TYPE_DELAY, 1) };
vx_delay vxCreateDelay(vx_context context, vx_reference exemplar, vx_size num_slots);
vx_status vxReleaseDelay(vx_delay *delay);
vx_status vxQueryDelay(vx_delay delay, vx_enum attribute, void *ptr, vx_size size);
vx_reference vxGetReferenceFromDelay(vx_delay delay, vx_int32 index);
vx_status vxAgeDelay(vx_delay delay);
vx_status vxRegisterAutoAging(vx_graph graph, vx_delay delay);

vx_distribution vxCreateDistribution(vx_context context, vx_size numBins, vx_int32 offset, vx_uint32 range);
vx_distribution vxCreateVirtualDistribution(vx_graph graph, vx_size numBins, vx_int32 offset, vx_uint32 range);
vx_status vxReleaseDistribution(vx_distribution *distribution);
vx_status vxQueryDistribution(vx_distribution distribution, vx_enum attribute, void *ptr, vx_size size);
vx_status vxCopyDistribution(vx_distribution distribution, void *user_ptr, vx_enum usage, vx_enum user_mem_type);
vx_status vxMapDistribution(vx_distribution distribution, vx_map_id *map_id, void **ptr, vx_enum usage, vx_enum mem_type,
                            vx_uint32 flags);
vx_status vxUnmapDistribution(vx_distribution distribution, vx_map_id map_id);

vx_lut vxCreateLUT(vx_context context, vx_enum data_type, vx_size count);
vx_lut vxCreateVirtualLUT(vx_graph graph, vx_enum data_type, vx_size count);
vx_status vxReleaseLUT(vx_lut *lut);
vx_status vxQueryLUT(vx_lut lut, vx_enum attribute, void *ptr, vx_size size);
vx_status vxCopyLUT(vx_lut lut, void *user_ptr, vx_enum usage, vx_enum user_mem_type);
vx_status vxMapLUT(vx_lut lut, vx_map_id *map_id, void **ptr, vx_enum usage, vx_enum mem_type, vx_uint32 flags);
vx_status vxUnmapLUT(vx_lut lut, vx_map_id map_id);

vx_matrix vxCreateMatrix(vx_context c, vx_enum data_type, vx_size columns, vx_size rows);
vx_status vxReleaseMatrix(vx_matrix *mat);
vx_status vxQueryMatrix(vx_matrix mat, vx_enum attribute, void *ptr, vx_size size);
vx_status vxCopyMatrix(vx_matrix matrix, void *user_ptr, vx_enum usage, vx_enum user_mem_type);

vx_array vxCreateArray(vx_context context, vx_enum item_type, vx_size capacity);
vx_array vxCreateVirtualArray(vx_graph graph, vx_enum item_type, vx_size capacity);
vx_status vxReleaseArray(vx_array *arr);
vx_status vxQueryArray(vx_array arr, vx_enum attribute, void *ptr, vx_size size);
vx_status vxAddArrayItems(vx_array arr, vx_size count, const void *ptr, vx_size stride);
vx_status vxTruncateArray(vx_array arr, vx_size new_num_items);
vx_status vxCopyArrayRange(vx_array array, vx_size range_start, vx_size range_end, vx_size user_stride, void *user_ptr,
                           vx_enum usage, vx_enum user_mem_type);
vx_status vxMapArrayRange(vx_array array, vx_size range_start, vx_size range_end, vx_map_id *map_id, vx_size *stride,
                          void **ptr, vx_enum usage, vx_enum mem_type, vx_uint32 flags);
vx_status vxUnmapArrayRange(vx_array array, vx_map_id map_id);

vx_pyramid vxCreatePyramid(vx_context context, vx_size levels, vx_float32 scale, vx_uint32 width, vx_uint32 height, vx_df_image format);
vx_pyramid vxCreateVirtualPyramid(vx_graph graph, vx_size levels, vx_float32 scale, vx_uint32 width, vx_uint32 height, vx_df_image format);
vx_image vxGetPyramidLevel(vx_pyramid pyr, vx_uint32 index);
vx_status vxQueryPyramid(vx_pyramid pyr, vx_enum attribute, void *ptr, vx_size size);
vx_status vxReleasePyramid(vx_pyramid *pyr);

vx_remap vxCreateRemap(vx_context context, vx_uint32 src_width, vx_uint32 src_height, vx_uint32 dst_width, vx_uint32 dst_height);
vx_status vxReleaseRemap(vx_remap *table);
vx_status vxSetRemapPoint(vx_remap table, vx_uint32 dst_x, vx_uint32 dst_y, vx_float32 src_x, vx_float32 src_y);
vx_status vxCopyRemapPatch(vx_remap remap, const vx_rectangle_t *rect, vx_size user_stride_y, void *user_ptr,
                           vx_enum user_coordinate_type, vx_enum usage, vx_enum user_mem_type);
vx_status vxQueryRemap(vx_remap table, vx_enum attribute, void *ptr, vx_size size);

/* Graph time as VX_GRAPH_ATTRIBUTE_AMD_PERFORMANCE_INTERNAL_{LAST,AVG} report it, in ns (vx_ext_amd.h) */
typedef struct {
    vx_uint64 kernel_enqueue;
    vx_uint64 kernel_wait;
    vx_uint64 buffer_read;
    vx_uint64 buffer_write;
} AgoGraphPerfInternalInfo;

/* ---------------- kernels, generic nodes, parameters (vx_api.h group_kernel / group_parameter) ---------------- */
#define VX_MAX_KERNEL_NAME (256)
enum { VX_KERNEL_PARAMETERS = VX__A(VX_TYPE_KERNEL, 0), VX_KERNEL_NAME = VX__A(VX_TYPE_KERNEL, 1),
       VX_KERNEL_ENUM = VX__A(VX_TYPE_KERNEL, 2), VX_KERNEL_LOCAL_DATA_SIZE = VX__A(VX_TYPE_KERNEL, 3) };
enum { VX_PARAMETER_INDEX = VX__A(VX_TYPE_PARAMETER, 0), VX_PARAMETER_DIRECTION = VX__A(VX_TYPE_PARAMETER, 1),
       VX_PARAMETER_TYPE = VX__A(VX_TYPE_PARAMETER, 2), VX_PARAMETER_STATE = VX__A(VX_TYPE_PARAMETER, 3),
       VX_PARAMETER_REF = VX__A(VX_TYPE_PARAMETER, 4) };
vx_kernel vxGetKernelByName(vx_context context, const vx_char *name);
vx_kernel vxGetKernelByEnum(vx_context context, vx_enum kernel);
vx_status vxQueryKernel(vx_kernel kernel, vx_enum attribute, void *ptr, vx_size size);
vx_status vxReleaseKernel(vx_kernel *kernel);
vx_status vxLoadKernels(vx_context context, const vx_char *module);
vx_node vxCreateGenericNode(vx_graph graph, vx_kernel kernel);
vx_status vxSetParameterByIndex(vx_node node, vx_uint32 index, vx_reference value);
vx_parameter vxGetParameterByIndex(vx_node node, vx_uint32 index);
vx_parameter vxGetKernelParameterByIndex(vx_kernel kernel, vx_uint32 index);
vx_status vxSetParameterByReference(vx_parameter parameter, vx_reference value);
vx_status vxQueryParameter(vx_parameter parameter, vx_enum attribute, void *ptr, vx_size size);
vx_status vxReleaseParameter(vx_parameter *param);

/* ---------------- user kernels (vx_api.h group_user_kernels; vx_ext_amd.h) ---------------- */
typedef struct _vx_meta_format *vx_meta_format;
typedef vx_status (*vx_kernel_f)(vx_node node, const vx_reference *parameters, vx_uint32 num);
typedef vx_status (*vx_kernel_initialize_f)(vx_node node, const vx_reference *parameters, vx_uint32 num);
typedef vx_status (*vx_kernel_deinitialize_f)(vx_node node, const vx_reference *parameters, vx_uint32 num);
typedef vx_status (*vx_kernel_validate_f)(vx_node node, const vx_reference parameters[], vx_uint32 num, vx_meta_format metas[]);
typedef vx_status (*vx_kernel_image_valid_rectangle_f)(vx_node node, vx_uint32 index, const vx_rectangle_t *const input_valid[],
                                                       vx_rectangle_t *const output_valid[]);
typedef vx_status (*vx_publish_kernels_f)(vx_context context);
enum { VX_VALID_RECT_CALLBACK = VX__A(VX_TYPE_META_FORMAT, 1) };
enum { VX_KERNEL_ATTRIBUTE_AMD_GPU_BUFFER_ACCESS_ENABLE = VX_ATTRIBUTE_BASE(VX_ID_AMD, VX_TYPE_KERNEL) + 0x05 };
vx_kernel vxAddUserKernel(vx_context context, const vx_char name[VX_MAX_KERNEL_NAME], vx_enum enumeration,
                          vx_kernel_f func_ptr, vx_uint32 numParams, vx_kernel_validate_f validate,
                          vx_kernel_initialize_f init, vx_kernel_deinitialize_f deinit);
vx_status vxAddParameterToKernel(vx_kernel kernel, vx_uint32 index, vx_enum dir, vx_enum data_type, vx_enum state);
vx_status vxFinalizeKernel(vx_kernel kernel);
vx_status vxRemoveKernel(vx_kernel kernel);
vx_status vxSetKernelAttribute(vx_kernel kernel, vx_enum attribute, const void *ptr, vx_size size);
vx_status vxSetMetaFormatAttribute(vx_meta_format meta, vx_enum attribute, const void *ptr, vx_size size);
vx_status vxQueryMetaFormatAttribute(vx_meta_format meta, vx_enum attribute, void *ptr, vx_size size);
vx_status vxSetMetaFormatFromReference(vx_meta_format meta, vx_reference exemplar);

/* ---------------- image views, convolutions, legacy access (vx_api.h, vx_compatibility.h, vx_ext_amd.h) ---------------- */
enum { VX_CONVOLUTION_ROWS = VX__A(VX_TYPE_CONVOLUTION, 0), VX_CONVOLUTION_COLUMNS = VX__A(VX_TYPE_CONVOLUTION, 1),
       VX_CONVOLUTION_SCALE = VX__A(VX_TYPE_CONVOLUTION, 2), VX_CONVOLUTION_SIZE = VX__A(VX_TYPE_CONVOLUTION, 3) };
typedef struct {
    vx_size components;
    vx_size planes;
    vx_size pixelSizeInBitsNum;
    vx_enum colorSpace;
    vx_enum channelRange;
    vx_size pixelSizeInBitsDenom;
} AgoImageFormatDescription;
typedef struct _vx_tensor_t *vx_tensor;
vx_image vxCreateImageFromROI(vx_image img, const vx_rectangle_t *rect);
vx_image vxCreateImageFromChannel(vx_image img, vx_enum channel);
vx_status vxSetImageAttribute(vx_image image, vx_enum attribute, const void *ptr, vx_size size);
void *vxFormatImagePatchAddress2d(void *ptr, vx_uint32 x, vx_uint32 y, const vx_imagepatch_addressing_t *addr);
vx_status vxGetContextImageFormatDescription(vx_context context, vx_df_image format, AgoImageFormatDescription *desc);
vx_status vxAccessImagePatch(vx_image image, const vx_rectangle_t *rect, vx_uint32 plane_index,
                             vx_imagepatch_addressing_t *addr, void **ptr, vx_enum usage);
vx_status vxCommitImagePatch(vx_image image, const vx_rectangle_t *rect, vx_uint32 plane_index,
                             const vx_imagepatch_addressing_t *addr, const void *ptr);
vx_status vxAccessArrayRange(vx_array arr, vx_size start, vx_size end, vx_size *stride, void **ptr, vx_enum usage);
vx_status vxCommitArrayRange(vx_array arr, vx_size start, vx_size end, const void *ptr);
vx_status vxAccessDistribution(vx_distribution distribution, void **ptr, vx_enum usage);
vx_status vxCommitDistribution(vx_distribution distribution, const void *ptr);
vx_status vxAccessLUT(vx_lut lut, void **ptr, vx_enum usage);
vx_status vxCommitLUT(vx_lut lut, const void *ptr);
vx_status vxReadMatrix(vx_matrix mat, void *array);
vx_status vxWriteMatrix(vx_matrix mat, const void *array);
vx_status vxReadScalarValue(vx_scalar ref, void *ptr);
vx_status vxWriteScalarValue(vx_scalar ref, const void *ptr);
vx_status vxGetRemapPoint(vx_remap table, vx_uint32 dst_x, vx_uint32 dst_y, vx_float32 *src_x, vx_float32 *src_y);
vx_status vxGetReferenceName(vx_reference ref, vx_char name[], vx_size size);
vx_enum vxRegisterUserStruct(vx_context context, vx_size size);
vx_convolution vxCreateConvolution(vx_context context, vx_size columns, vx_size rows);
vx_status vxReleaseConvolution(vx_convolution *conv);
vx_status vxQueryConvolution(vx_convolution conv, vx_enum attribute, void *ptr, vx_size size);
vx_status vxSetConvolutionAttribute(vx_convolution conv, vx_enum attribute, const void *ptr, vx_size size);
vx_status vxCopyConvolutionCoefficients(vx_convolution conv, void *user_ptr, vx_enum usage, vx_enum user_mem_type);
vx_status vxReadConvolutionCoefficients(vx_convolution conv, vx_int16 *array);
vx_status vxWriteConvolutionCoefficients(vx_convolution conv, const vx_int16 *array);
/* Tensors are outside this target's vision path: creation returns NULL, the other calls
 * VX_ERROR_NOT_SUPPORTED (the symbols exist so that applications such as runvx link). */
vx_tensor vxCreateTensor(vx_context context, vx_size number_of_dims, const vx_size *dims, vx_enum data_type,
                         vx_int8 fixed_point_position);
vx_tensor vxCreateVirtualTensor(vx_graph graph, vx_size number_of_dims, const vx_size *dims, vx_enum data_type,
                                vx_int8 fixed_point_position);
vx_tensor vxCreateTensorFromView(vx_tensor tensor, vx_size number_of_dims, const vx_size *view_start, const vx_size *view_end);
vx_tensor vxCreateTensorFromHandle(vx_context context, vx_size number_of_dims, const vx_size *dims, vx_enum data_type,
                                   vx_int8 fixed_point_position, const vx_size *stride, void *ptr, vx_enum memory_type);
vx_status vxQueryTensor(vx_tensor tensor, vx_enum attribute, void *ptr, vx_size size);
vx_status vxReleaseTensor(vx_tensor *tensor);
vx_status vxSwapTensorHandle(vx_tensor tensor, void *new_ptr, void **prev_ptr);
vx_status vxCopyTensorPatch(vx_tensor tensor, vx_size number_of_dims, const vx_size *view_start, const vx_size *view_end,
                            const vx_size *user_stride, void *user_ptr, vx_enum usage, vx_enum user_memory_type);
vx_status vxMapTensorPatch(vx_tensor tensor, vx_size number_of_dims, const vx_size *view_start, const vx_size *view_end,
                           vx_map_id *map_id, vx_size *stride, void **ptr, vx_enum usage, vx_enum mem_type);
vx_status vxUnmapTensorPatch(vx_tensor tensor, const vx_map_id map_id);

/* ---------------- node factories (vx_nodes.h) ---------------- */
vx_node vxColorConvertNode(vx_graph graph, vx_image input, vx_image output);
vx_node vxChannelExtractNode(vx_graph graph, vx_image input, vx_enum channel, vx_image output);
vx_node vxSobel3x3Node(vx_graph graph, vx_image input, vx_image output_x, vx_image output_y);
vx_node vxMagnitudeNode(vx_graph graph, vx_image grad_x, vx_image grad_y, vx_image mag);
vx_node vxScaleImageNode(vx_graph graph, vx_image src, vx_image dst, vx_enum type);
vx_node vxThresholdNode(vx_graph graph, vx_image input, vx_threshold thresh, vx_image output);
vx_node vxGaussian3x3Node(vx_graph graph, vx_image input, vx_image output);
vx_node vxGaussianPyramidNode(vx_graph graph, vx_image input, vx_pyramid gaussian);
vx_node vxConvertDepthNode(vx_graph graph, vx_image input, vx_image output, vx_enum policy, vx_scalar shift);
vx_node vxCannyEdgeDetectorNode(vx_graph graph, vx_image input, vx_threshold hyst, vx_int32 gradient_size,
                                vx_enum norm_type, vx_image output);
vx_node vxWarpAffineNode(vx_graph graph, vx_image input, vx_matrix matrix, vx_enum type, vx_image output);
vx_node vxWarpPerspectiveNode(vx_graph graph, vx_image input, vx_matrix matrix, vx_enum type, vx_image output);
vx_node vxHarrisCornersNode(vx_graph graph, vx_image input, vx_scalar strength_thresh, vx_scalar min_distance,
                            vx_scalar sensitivity, vx_int32 gradient_size, vx_int32 block_size, vx_array corners,
                            vx_scalar num_corners);
vx_node vxFastCornersNode(vx_graph graph, vx_image input, vx_scalar strength_thresh, vx_bool nonmax_suppression,
                          vx_array corners, vx_scalar num_corners);
vx_node vxOpticalFlowPyrLKNode(vx_graph graph, vx_pyramid old_images, vx_pyramid new_images, vx_array old_points,
                               vx_array new_points_estimates, vx_array new_points, vx_enum termination, vx_scalar epsilon,
                               vx_scalar num_iterations, vx_scalar use_initial_estimate, vx_size window_dimension);
vx_node vxRemapNode(vx_graph graph, vx_image input, vx_remap table, vx_enum policy, vx_image output);
vx_node vxHalfScaleGaussianNode(vx_graph graph, vx_image input, vx_image output, vx_int32 kernel_size);
vx_node vxBox3x3Node(vx_graph graph, vx_image input, vx_image output);
vx_node vxMedian3x3Node(vx_graph graph, vx_image input, vx_image output);
vx_node vxDilate3x3Node(vx_graph graph, vx_image input, vx_image output);
vx_node vxErode3x3Node(vx_graph graph, vx_image input, vx_image output);
vx_node vxAbsDiffNode(vx_graph graph, vx_image in1, vx_image in2, vx_image out);
vx_node vxAddNode(vx_graph graph, vx_image in1, vx_image in2, vx_enum policy, vx_image out);
vx_node vxSubtractNode(vx_graph graph, vx_image in1, vx_image in2, vx_enum policy, vx_image out);
vx_node vxAndNode(vx_graph graph, vx_image in1, vx_image in2, vx_image out);
vx_node vxOrNode(vx_graph graph, vx_image in1, vx_image in2, vx_image out);
vx_node vxXorNode(vx_graph graph, vx_image in1, vx_image in2, vx_image out);
vx_node vxNotNode(vx_graph graph, vx_image input, vx_image output);
vx_node vxTableLookupNode(vx_graph graph, vx_image input, vx_lut lut, vx_image output);
vx_node vxIntegralImageNode(vx_graph graph, vx_image input, vx_image output);
vx_node vxHistogramNode(vx_graph graph, vx_image input, vx_distribution distribution);
vx_node vxChannelCombineNode(vx_graph graph, vx_image plane0, vx_image plane1, vx_image plane2, vx_image plane3,
                             vx_image output);
vx_node vxConvolveNode(vx_graph graph, vx_image input, vx_convolution conv, vx_image output);

#ifdef __cplusplus
}
#endif
#endif /* AGOVX_H */
