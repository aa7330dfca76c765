"""ctypes binding of the OpenVX 1.3 C API subset in include/agovx.h.

The binding takes the library as an argument, so the same graph-building code drives this
package's libopenvx.so (the B200 target) and any other OpenVX library with the same ABI --
the parity tests use it on the reference AMD OpenVX build as well.

    from mivisionx_b200 import vx
    api = vx.OpenVX()                     # this package's libopenvx.so
    ctx = api.vxCreateContext()
"""
from __future__ import annotations

import ctypes as C

import numpy as np

# ---------------------------------------------------------------- constants (include/agovx.h)
def _enum_base(vendor, eid):
    return (vendor << 20) | (eid << 12)


def _attr_base(vendor, obj):
    return (vendor << 20) | (obj << 8)


def _df(a, b, c, d):
    return ord(a) | (ord(b) << 8) | (ord(c) << 16) | (ord(d) << 24)


VX_ID_KHRONOS, VX_ID_AMD = 0x000, 0x00D
VX_SUCCESS, VX_FAILURE = 0, -1
VX_ERROR_INVALID_PARAMETERS, VX_ERROR_NOT_SUPPORTED, VX_ERROR_NOT_IMPLEMENTED = -10, -3, -2
VX_ERROR_INVALID_FORMAT, VX_ERROR_INVALID_REFERENCE, VX_ERROR_INVALID_GRAPH = -14, -12, -18

VX_TYPE_INT8, VX_TYPE_UINT8, VX_TYPE_INT16, VX_TYPE_UINT16 = 0x002, 0x003, 0x004, 0x005
VX_TYPE_INT32, VX_TYPE_UINT32, VX_TYPE_FLOAT32, VX_TYPE_ENUM, VX_TYPE_SIZE = 0x006, 0x007, 0x00A, 0x00C, 0x00D
VX_TYPE_BOOL, VX_TYPE_KEYPOINT, VX_TYPE_COORDINATES2DF = 0x010, 0x021, 0x024
VX_TYPE_GRAPH, VX_TYPE_IMAGE, VX_TYPE_ARRAY = 0x802, 0x80F, 0x80E

VX_DF_IMAGE_U8 = _df('U', '0', '0', '8')
VX_DF_IMAGE_U16 = _df('U', '0', '1', '6')
VX_DF_IMAGE_S16 = _df('S', '0', '1', '6')
VX_DF_IMAGE_RGB = _df('R', 'G', 'B', '2')
VX_DF_IMAGE_RGBX = _df('R', 'G', 'B', 'A')
VX_DF_IMAGE_NV12 = _df('N', 'V', '1', '2')
VX_DF_IMAGE_IYUV = _df('I', 'Y', 'U', 'V')
VX_DF_IMAGE_VIRT = _df('V', 'I', 'R', 'T')
VX_DF_IMAGE_F32_AMD = _df('F', '0', '3', '2')
VX_DF_IMAGE_U32 = _df('U', '0', '3', '2')

VX_CONVERT_POLICY_WRAP = _enum_base(0, 0x0A) + 0
VX_CONVERT_POLICY_SATURATE = _enum_base(0, 0x0A) + 1
VX_THRESHOLD_TYPE_BINARY = _enum_base(0, 0x0B) + 0
VX_THRESHOLD_TYPE_RANGE = _enum_base(0, 0x0B) + 1
VX_BORDER_UNDEFINED = _enum_base(0, 0x0C) + 0
VX_BORDER_CONSTANT = _enum_base(0, 0x0C) + 1
VX_BORDER_REPLICATE = _enum_base(0, 0x0C) + 2
VX_MEMORY_TYPE_HOST = _enum_base(0, 0x0E) + 1
VX_MEMORY_TYPE_HIP = _enum_base(0, 0x0E) + 3
VX_TERM_CRITERIA_ITERATIONS = _enum_base(0, 0x0F) + 0
VX_TERM_CRITERIA_EPSILON = _enum_base(0, 0x0F) + 1
VX_TERM_CRITERIA_BOTH = _enum_base(0, 0x0F) + 2
VX_SCALE_PYRAMID_HALF = 0.5
VX_NORM_L1 = _enum_base(0, 0x10) + 0
VX_NORM_L2 = _enum_base(0, 0x10) + 1
VX_READ_ONLY = _enum_base(0, 0x11) + 1
VX_WRITE_ONLY = _enum_base(0, 0x11) + 2
VX_READ_AND_WRITE = _enum_base(0, 0x11) + 3
VX_INTERPOLATION_NEAREST_NEIGHBOR = _enum_base(0, 0x04) + 0
VX_INTERPOLATION_BILINEAR = _enum_base(0, 0x04) + 1
VX_INTERPOLATION_AREA = _enum_base(0, 0x04) + 2
VX_CHANNEL_Y = _enum_base(0, 0x09) + 0x14
VX_CHANNEL_U = _enum_base(0, 0x09) + 0x15
VX_CHANNEL_V = _enum_base(0, 0x09) + 0x16

VX_IMAGE_WIDTH = _attr_base(0, VX_TYPE_IMAGE) + 0
VX_IMAGE_HEIGHT = _attr_base(0, VX_TYPE_IMAGE) + 1
VX_IMAGE_FORMAT = _attr_base(0, VX_TYPE_IMAGE) + 2
VX_ARRAY_NUMITEMS = _attr_base(0, VX_TYPE_ARRAY) + 1
VX_ARRAY_CAPACITY = _attr_base(0, VX_TYPE_ARRAY) + 2
VX_NODE_BORDER = _attr_base(0, 0x803) + 2
VX_GRAPH_PERFORMANCE = _attr_base(0, VX_TYPE_GRAPH) + 2
VX_THRESHOLD_THRESHOLD_VALUE = _attr_base(0, 0x80A) + 1
VX_THRESHOLD_THRESHOLD_LOWER = _attr_base(0, 0x80A) + 2
VX_THRESHOLD_THRESHOLD_UPPER = _attr_base(0, 0x80A) + 3
VX_GRAPH_ATTRIBUTE_AMD_AFFINITY = _attr_base(VX_ID_AMD, VX_TYPE_GRAPH) + 0x01
VX_GRAPH_ATTRIBUTE_AMD_EXPORT_TO_TEXT = _attr_base(VX_ID_AMD, VX_TYPE_GRAPH) + 0x03
VX_GRAPH_ATTRIBUTE_AMD_OPTIMIZER_FLAGS = _attr_base(VX_ID_AMD, VX_TYPE_GRAPH) + 0x04
VX_GRAPH_ATTRIBUTE_AMD_IMPORT_FROM_TEXT = _attr_base(VX_ID_AMD, VX_TYPE_GRAPH) + 0x02
VX_GRAPH_ATTRIBUTE_AMD_PERFORMANCE_INTERNAL_LAST = _attr_base(VX_ID_AMD, VX_TYPE_GRAPH) + 0x05
AGO_TARGET_AFFINITY_CPU, AGO_TARGET_AFFINITY_GPU = 0x10, 0x20

VX_INPUT, VX_OUTPUT, VX_BIDIRECTIONAL = _enum_base(0, 0x00) + 0, _enum_base(0, 0x00) + 1, _enum_base(0, 0x00) + 2
VX_PARAMETER_STATE_REQUIRED, VX_PARAMETER_STATE_OPTIONAL = _enum_base(0, 0x08) + 0, _enum_base(0, 0x08) + 1
VX_KERNEL_LOCAL_DATA_SIZE = _attr_base(0, 0x804) + 3
VX_NODE_STATUS = _attr_base(0, 0x803) + 0
VX_NODE_LOCAL_DATA_SIZE = _attr_base(0, 0x803) + 3
VX_NODE_LOCAL_DATA_PTR = _attr_base(0, 0x803) + 4
VX_NODE_ATTRIBUTE_AMD_HIP_STREAM = _attr_base(VX_ID_AMD, 0x803) + 0x03
VX_KERNEL_ATTRIBUTE_AMD_GPU_BUFFER_ACCESS_ENABLE = _attr_base(VX_ID_AMD, 0x804) + 0x05
VX_IMAGE_ATTRIBUTE_AMD_GPU_BUFFER_STRIDE = _attr_base(VX_ID_AMD, VX_TYPE_IMAGE) + 0x04
VX_IMAGE_ATTRIBUTE_AMD_HIP_BUFFER = _attr_base(VX_ID_AMD, VX_TYPE_IMAGE) + 0x06
VX_ID_USER = 0xFFE
VX_KERNEL_BASE_USER = _enum_base(VX_ID_USER, 0)   # VX_KERNEL_BASE(VX_ID_USER, 0): enumerations for user kernels

# optimizer flag bits this target adds to VX_GRAPH_ATTRIBUTE_AMD_OPTIMIZER_FLAGS
OPT_NO_FUSION = 0x00010000        # one launch per lowered node ("plain" form)
OPT_NO_GRAPH_CAPTURE = 0x00020000  # launch the steps directly instead of one CUDA graph
OPT_NO_TMA = 0x00080000            # pixel chains and pyramid levels load their tiles without TMA


# ---------------------------------------------------------------- structures
class AgoGraphPerfInternalInfo(C.Structure):
    _fields_ = [("kernel_enqueue", C.c_uint64), ("kernel_wait", C.c_uint64), ("buffer_read", C.c_uint64),
                ("buffer_write", C.c_uint64)]


class vx_imagepatch_addressing_t(C.Structure):
    _fields_ = [("dim_x", C.c_uint32), ("dim_y", C.c_uint32), ("stride_x", C.c_int32), ("stride_y", C.c_int32),
                ("scale_x", C.c_uint32), ("scale_y", C.c_uint32), ("step_x", C.c_uint32), ("step_y", C.c_uint16),
                ("stride_x_bits", C.c_uint16)]


class vx_rectangle_t(C.Structure):
    _fields_ = [("start_x", C.c_uint32), ("start_y", C.c_uint32), ("end_x", C.c_uint32), ("end_y", C.c_uint32)]


class vx_keypoint_t(C.Structure):
    _fields_ = [("x", C.c_int32), ("y", C.c_int32), ("strength", C.c_float), ("scale", C.c_float),
                ("orientation", C.c_float), ("tracking_status", C.c_int32), ("error", C.c_float)]


KEYPOINT_DTYPE = np.dtype([("x", "<i4"), ("y", "<i4"), ("strength", "<f4"), ("scale", "<f4"),
                           ("orientation", "<f4"), ("tracking_status", "<i4"), ("error", "<f4")])


class vx_pixel_value_t(C.Union):
    _fields_ = [("U8", C.c_uint8), ("U16", C.c_uint16), ("S16", C.c_int16), ("U32", C.c_uint32), ("S32", C.c_int32),
                ("reserved", C.c_uint8 * 16)]


class vx_border_t(C.Structure):
    _fields_ = [("mode", C.c_int32), ("constant_value", vx_pixel_value_t)]


class vx_perf_t(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("tmp", "beg", "end", "sum", "avg", "min", "num", "max")]


GDF_CALLBACK = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_char_p, C.c_char_p)


class AgoGraphImportInfo(C.Structure):
    _fields_ = [("text", C.c_char_p), ("num_ref", C.c_uint32), ("ref", C.POINTER(C.c_void_p)),
                ("dumpToConsole", C.c_int32), ("data_registry_callback_f", GDF_CALLBACK),
                ("data_registry_callback_obj", C.c_void_p)]


class AgoTargetAffinityInfo(C.Structure):
    _fields_ = [("device_type", C.c_uint32), ("device_info", C.c_uint32), ("group", C.c_uint32), ("reserved", C.c_uint32)]


vp, i32, u32, sz, f32 = C.c_void_p, C.c_int32, C.c_uint32, C.c_size_t, C.c_float
_SIGS = {
    "vxCreateContext": (vp, []), "vxReleaseContext": (i32, [C.POINTER(vp)]),
    "vxGetStatus": (i32, [vp]),
    "vxCreateImage": (vp, [vp, u32, u32, u32]), "vxCreateVirtualImage": (vp, [vp, u32, u32, u32]),
    "vxCreateImageFromHandle": (vp, [vp, u32, vp, vp, i32]),
    "vxSwapImageHandle": (i32, [vp, vp, vp, sz]),
    "vxReleaseImage": (i32, [C.POINTER(vp)]), "vxQueryImage": (i32, [vp, i32, vp, sz]),
    "vxCopyImagePatch": (i32, [vp, vp, u32, vp, vp, i32, i32]),
    "vxMapImagePatch": (i32, [vp, vp, u32, C.POINTER(C.c_size_t), vp, C.POINTER(vp), i32, i32, u32]),
    "vxUnmapImagePatch": (i32, [vp, C.c_size_t]),
    "vxGetValidRegionImage": (i32, [vp, vp]), "vxSetImageValidRectangle": (i32, [vp, vp]),
    "vxCreateGraph": (vp, [vp]), "vxReleaseGraph": (i32, [C.POINTER(vp)]),
    "vxVerifyGraph": (i32, [vp]), "vxProcessGraph": (i32, [vp]), "vxScheduleGraph": (i32, [vp]),
    "vxWaitGraph": (i32, [vp]), "vxQueryGraph": (i32, [vp, i32, vp, sz]), "vxSetGraphAttribute": (i32, [vp, i32, vp, sz]),
    "vxSetNodeAttribute": (i32, [vp, i32, vp, sz]), "vxReleaseNode": (i32, [C.POINTER(vp)]),
    "vxCreateScalar": (vp, [vp, i32, vp]), "vxCopyScalar": (i32, [vp, vp, i32, i32]),
    "vxCreateThresholdForImage": (vp, [vp, i32, u32, u32]), "vxCreateThreshold": (vp, [vp, i32, i32]),
    "vxSetThresholdAttribute": (i32, [vp, i32, vp, sz]),
    "vxCopyThresholdValue": (i32, [vp, vp, i32, i32]), "vxCopyThresholdRange": (i32, [vp, vp, vp, i32, i32]),
    "vxCreateMatrix": (vp, [vp, i32, sz, sz]), "vxCopyMatrix": (i32, [vp, vp, i32, i32]),
    "vxCreateArray": (vp, [vp, i32, sz]), "vxCreateVirtualArray": (vp, [vp, i32, sz]),
    "vxQueryArray": (i32, [vp, i32, vp, sz]), "vxAddArrayItems": (i32, [vp, sz, vp, sz]),
    "vxCopyArrayRange": (i32, [vp, sz, sz, sz, vp, i32, i32]), "vxTruncateArray": (i32, [vp, sz]),
    "vxCreatePyramid": (vp, [vp, sz, f32, u32, u32, u32]), "vxCreateVirtualPyramid": (vp, [vp, sz, f32, u32, u32, u32]),
    "vxGetPyramidLevel": (vp, [vp, u32]),
    "vxCreateRemap": (vp, [vp, u32, u32, u32, u32]), "vxCopyRemapPatch": (i32, [vp, vp, sz, vp, i32, i32, i32]),
    "vxGaussian3x3Node": (vp, [vp, vp, vp]), "vxSobel3x3Node": (vp, [vp, vp, vp, vp]),
    "vxMagnitudeNode": (vp, [vp, vp, vp, vp]), "vxConvertDepthNode": (vp, [vp, vp, vp, i32, vp]),
    "vxThresholdNode": (vp, [vp, vp, vp, vp]),
    "vxCannyEdgeDetectorNode": (vp, [vp, vp, vp, i32, i32, vp]),
    "vxHarrisCornersNode": (vp, [vp, vp, vp, vp, vp, i32, i32, vp, vp]),
    "vxFastCornersNode": (vp, [vp, vp, vp, i32, vp, vp]),
    "vxColorConvertNode": (vp, [vp, vp, vp]), "vxChannelExtractNode": (vp, [vp, vp, i32, vp]),
    "vxScaleImageNode": (vp, [vp, vp, vp, i32]), "vxWarpAffineNode": (vp, [vp, vp, vp, i32, vp]),
    "vxWarpPerspectiveNode": (vp, [vp, vp, vp, i32, vp]), "vxRemapNode": (vp, [vp, vp, vp, i32, vp]),
    "vxGaussianPyramidNode": (vp, [vp, vp, vp]), "vxHalfScaleGaussianNode": (vp, [vp, vp, vp, i32]),
    "vxOpticalFlowPyrLKNode": (vp, [vp, vp, vp, vp, vp, vp, i32, vp, vp, vp, sz]),
    "vxBox3x3Node": (vp, [vp, vp, vp]), "vxMedian3x3Node": (vp, [vp, vp, vp]),
    "vxDilate3x3Node": (vp, [vp, vp, vp]), "vxErode3x3Node": (vp, [vp, vp, vp]),
    "vxAbsDiffNode": (vp, [vp, vp, vp, vp]), "vxAndNode": (vp, [vp, vp, vp, vp]), "vxOrNode": (vp, [vp, vp, vp, vp]),
    "vxXorNode": (vp, [vp, vp, vp, vp]), "vxNotNode": (vp, [vp, vp, vp]),
    "vxAddNode": (vp, [vp, vp, vp, i32, vp]), "vxSubtractNode": (vp, [vp, vp, vp, i32, vp]),
    "vxChannelCombineNode": (vp, [vp, vp, vp, vp, vp, vp]),
    "vxConvolveNode": (vp, [vp, vp, vp, vp]),
    "vxCreateConvolution": (vp, [vp, sz, sz]), "vxCopyConvolutionCoefficients": (i32, [vp, vp, i32, i32]),
    "vxSetConvolutionAttribute": (i32, [vp, i32, vp, sz]), "vxReleaseConvolution": (i32, [C.POINTER(vp)]),
    "vxCreateLUT": (vp, [vp, i32, sz]), "vxCopyLUT": (i32, [vp, vp, i32, i32]), "vxQueryLUT": (i32, [vp, i32, vp, sz]),
    "vxTableLookupNode": (vp, [vp, vp, vp, vp]), "vxIntegralImageNode": (vp, [vp, vp, vp]),
    "vxCreateDistribution": (vp, [vp, sz, i32, u32]), "vxCopyDistribution": (i32, [vp, vp, i32, i32]),
    "vxHistogramNode": (vp, [vp, vp, vp]),
    "vxCreateDelay": (vp, [vp, vp, sz]), "vxGetReferenceFromDelay": (vp, [vp, i32]), "vxAgeDelay": (i32, [vp]),
    "vxRegisterAutoAging": (i32, [vp, vp]), "vxQueryDelay": (i32, [vp, i32, vp, sz]),
    # kernels, generic nodes and user kernels
    "vxGetKernelByName": (vp, [vp, C.c_char_p]), "vxGetKernelByEnum": (vp, [vp, i32]),
    "vxReleaseKernel": (i32, [C.POINTER(vp)]), "vxQueryKernel": (i32, [vp, i32, vp, sz]),
    "vxCreateGenericNode": (vp, [vp, vp]), "vxSetParameterByIndex": (i32, [vp, u32, vp]),
    "vxQueryNode": (i32, [vp, i32, vp, sz]),
    "vxAddUserKernel": (vp, [vp, C.c_char_p, i32, vp, u32, vp, vp, vp]),
    "vxAddParameterToKernel": (i32, [vp, u32, i32, i32, i32]), "vxFinalizeKernel": (i32, [vp]),
    "vxRemoveKernel": (i32, [vp]), "vxSetKernelAttribute": (i32, [vp, i32, vp, sz]),
    "vxSetMetaFormatAttribute": (i32, [vp, i32, vp, sz]), "vxSetMetaFormatFromReference": (i32, [vp, vp]),
    "vxQueryMetaFormatAttribute": (i32, [vp, i32, vp, sz]),
}

# user-kernel callbacks (vx_types.h vx_kernel_f / vx_kernel_validate_f / vx_kernel_initialize_f)
KernelF = C.CFUNCTYPE(i32, vp, C.POINTER(vp), u32)
KernelValidateF = C.CFUNCTYPE(i32, vp, C.POINTER(vp), u32, C.POINTER(vp))

_PIX = {VX_DF_IMAGE_U8: (np.uint8, 1), VX_DF_IMAGE_U16: (np.uint16, 1), VX_DF_IMAGE_S16: (np.int16, 1),
        VX_DF_IMAGE_RGB: (np.uint8, 3), VX_DF_IMAGE_RGBX: (np.uint8, 4), VX_DF_IMAGE_F32_AMD: (np.float32, 1),
        VX_DF_IMAGE_U32: (np.uint32, 1)}


def image_plane_layout(fmt, width: int, height: int):
    """[(rows, pixels per row, bytes per pixel)] of each plane of a U8, RGB, NV12 or IYUV image."""
    if fmt == VX_DF_IMAGE_U8:
        return [(height, width, 1)]
    if fmt == VX_DF_IMAGE_RGB:
        return [(height, width, 3)]
    if fmt == VX_DF_IMAGE_NV12:
        return [(height, width, 1), (height // 2, width // 2, 2)]
    if fmt == VX_DF_IMAGE_IYUV:
        return [(height, width, 1), (height // 2, width // 2, 1), (height // 2, width // 2, 1)]
    raise ValueError(f"no plane layout for format {fmt:#x}")


class OpenVX:
    """Typed access to an OpenVX library plus numpy helpers for data exchange."""

    def __init__(self, lib: C.CDLL | None = None):
        if lib is None:
            from . import native
            lib = native.openvx()
        self.lib = lib
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
            setattr(self, name, fn)

    # ---- checks
    @staticmethod
    def ok(status: int, what: str = "") -> None:
        if status != VX_SUCCESS:
            raise RuntimeError(f"{what} failed with vx_status {status}")

    def obj(self, h, what: str = "object"):
        if not h or self.vxGetStatus(h) != VX_SUCCESS:
            raise RuntimeError(f"creating {what} failed")
        return h

    # ---- scalars / thresholds
    def scalar(self, ctx, vtype, value):
        ct = {VX_TYPE_INT32: C.c_int32, VX_TYPE_UINT32: C.c_uint32, VX_TYPE_FLOAT32: C.c_float, VX_TYPE_ENUM: C.c_int32,
              VX_TYPE_SIZE: C.c_size_t, VX_TYPE_BOOL: C.c_int32, VX_TYPE_UINT8: C.c_uint8}[vtype]
        v = ct(value)
        return self.obj(self.vxCreateScalar(ctx, vtype, C.byref(v)), "scalar")

    def read_scalar(self, s, ctype=C.c_size_t):
        v = ctype(0)
        self.ok(self.vxCopyScalar(s, C.byref(v), VX_READ_ONLY, VX_MEMORY_TYPE_HOST), "vxCopyScalar")
        return v.value

    def threshold_binary(self, ctx, value):
        t = self.obj(self.vxCreateThresholdForImage(ctx, VX_THRESHOLD_TYPE_BINARY, VX_DF_IMAGE_U8, VX_DF_IMAGE_U8), "threshold")
        v = C.c_int32(value)
        self.ok(self.vxSetThresholdAttribute(t, VX_THRESHOLD_THRESHOLD_VALUE, C.byref(v), 4), "threshold value")
        return t

    def threshold_range(self, ctx, lower, upper):
        t = self.obj(self.vxCreateThresholdForImage(ctx, VX_THRESHOLD_TYPE_RANGE, VX_DF_IMAGE_U8, VX_DF_IMAGE_U8), "threshold")
        for attr, val in ((VX_THRESHOLD_THRESHOLD_LOWER, lower), (VX_THRESHOLD_THRESHOLD_UPPER, upper)):
            v = C.c_int32(val)
            self.ok(self.vxSetThresholdAttribute(t, attr, C.byref(v), 4), "threshold range")
        return t

    def matrix_f32(self, ctx, m: np.ndarray):
        m = np.ascontiguousarray(m, dtype=np.float32)
        rows, cols = m.shape
        h = self.obj(self.vxCreateMatrix(ctx, VX_TYPE_FLOAT32, cols, rows), "matrix")
        self.ok(self.vxCopyMatrix(h, m.ctypes.data, VX_WRITE_ONLY, VX_MEMORY_TYPE_HOST), "vxCopyMatrix")
        return h

    def convolution(self, ctx, coeffs: np.ndarray, scale: int = 1):
        """vx_convolution of `coeffs` (rows x columns int16) with `scale` (a power of two)."""
        k = np.ascontiguousarray(coeffs, dtype=np.int16)
        rows, cols = k.shape
        c = self.obj(self.vxCreateConvolution(ctx, cols, rows), "convolution")
        self.ok(self.vxCopyConvolutionCoefficients(c, k.ctypes.data, VX_WRITE_ONLY, VX_MEMORY_TYPE_HOST), "coefficients")
        v = C.c_uint32(scale)
        self.ok(self.vxSetConvolutionAttribute(c, _attr_base(0, 0x80C) + 2, C.byref(v), 4), "scale")
        return c

    def set_border(self, node, mode, value=0):
        b = vx_border_t()
        b.mode = mode
        b.constant_value.U32 = value
        self.ok(self.vxSetNodeAttribute(node, VX_NODE_BORDER, C.byref(b), C.sizeof(b)), "border")

    def set_optimizer_flags(self, graph, flags):
        v = C.c_uint32(flags)
        self.ok(self.vxSetGraphAttribute(graph, VX_GRAPH_ATTRIBUTE_AMD_OPTIMIZER_FLAGS, C.byref(v), 4), "optimizer flags")

    def set_graph_affinity(self, graph, device_type):
        a = AgoTargetAffinityInfo(device_type, 0, 0, 0)
        return self.vxSetGraphAttribute(graph, VX_GRAPH_ATTRIBUTE_AMD_AFFINITY, C.byref(a), C.sizeof(a))

    def import_gdf(self, graph, text: str, on_data=None, refs=()):
        """Read a text graph description into `graph` (VX_GRAPH_ATTRIBUTE_AMD_IMPORT_FROM_TEXT).
        Returns (status, {name: (reference, params)}) for the data that carry `:<params>` (the
        data registry callback of the reference's importer); `on_data(ref, name, params)` runs
        inside that callback, while the text is read (where runvx applies INIT requests);
        `refs` are the references `$1`, `$2`, ... of the text."""
        found = {}

        def cb(obj, ref, name, params):
            found[name.decode()] = (ref, params.decode())
            if on_data is not None:
                on_data(ref, name.decode(), params.decode())

        fn = GDF_CALLBACK(cb)
        arr = (C.c_void_p * max(1, len(refs)))(*refs)
        info = AgoGraphImportInfo(text.encode(), len(refs), C.cast(arr, C.POINTER(C.c_void_p)) if refs else None, 0, fn,
                                  None)
        st = self.vxSetGraphAttribute(graph, VX_GRAPH_ATTRIBUTE_AMD_IMPORT_FROM_TEXT, C.byref(info), C.sizeof(info))
        return st, found

    def plan(self, graph):
        """The verified execution plan of a graph on this target: [(step name, kernels per run)]."""
        buf = C.create_string_buffer(1 << 20)
        if self.vxQueryGraph(graph, VX_GRAPH_ATTRIBUTE_AMD_EXPORT_TO_TEXT, buf, len(buf)) != VX_SUCCESS:
            return []
        steps = []
        for line in buf.value.decode().splitlines():
            name, _, k = line.partition("\t")
            steps.append((name, int(k or 0)))
        return steps

    def plan_text(self, graph) -> str:
        return "\n".join(name for name, _ in self.plan(graph))

    def set_device(self, ctx, device: int):
        """Select the CUDA device of a context (VX_CONTEXT_ATTRIBUTE_AMD_HIP_DEVICE)."""
        v = C.c_int32(device)
        attr = _attr_base(VX_ID_AMD, 0x801) + 0x07
        self.lib.vxSetContextAttribute.argtypes = [vp, i32, vp, sz]
        self.ok(self.lib.vxSetContextAttribute(ctx, attr, C.byref(v), 4), "set device")

    def gpu_ms_last(self, graph) -> float:
        """Device time of the graph's last launch (CUDA events on its stream), in ms."""
        p = AgoGraphPerfInternalInfo()
        self.ok(self.vxQueryGraph(graph, VX_GRAPH_ATTRIBUTE_AMD_PERFORMANCE_INTERNAL_LAST, C.byref(p), C.sizeof(p)), "perf")
        return p.kernel_wait / 1e6

    # ---- images
    def query_image(self, img):
        w, h, f = C.c_uint32(), C.c_uint32(), C.c_uint32()
        self.ok(self.vxQueryImage(img, VX_IMAGE_WIDTH, C.byref(w), 4), "query")
        self.ok(self.vxQueryImage(img, VX_IMAGE_HEIGHT, C.byref(h), 4), "query")
        self.ok(self.vxQueryImage(img, VX_IMAGE_FORMAT, C.byref(f), 4), "query")
        return w.value, h.value, f.value

    def image_from_host(self, ctx, arr, fmt=None, width=None, height=None):
        """vxCreateImageFromHandle(VX_MEMORY_TYPE_HOST) over application-owned buffers: one
        (H, W) uint8 array for a U8 image, else a list of per-plane arrays shaped (plane rows,
        plane row bytes) with `width` x `height` the image size (U8: the array's).  The
        buffers must outlive the image; when page-locked, graphs copy them in (and, for
        outputs, back) inside their CUDA graph."""
        fmt = VX_DF_IMAGE_U8 if fmt is None else fmt
        planes = [arr] if isinstance(arr, np.ndarray) else list(arr)
        if width is None:
            height, width = planes[0].shape[:2]
        layout = image_plane_layout(fmt, width, height)
        addrs = (vx_imagepatch_addressing_t * len(planes))()
        for a, pl, (ph, pw, bpp) in zip(addrs, planes, layout):
            a.dim_x, a.dim_y, a.stride_x, a.stride_y = pw, ph, bpp, pl.strides[0]
            a.scale_x = a.scale_y = 1024
            a.step_x = a.step_y = 1
        ptrs = (C.c_void_p * len(planes))(*[pl.ctypes.data for pl in planes])
        return self.obj(self.vxCreateImageFromHandle(ctx, fmt, addrs, ptrs, VX_MEMORY_TYPE_HOST), "image from handle")

    def write_plane(self, img, arr: np.ndarray, plane: int = 0, full_w=None, full_h=None):
        """Copy host pixels into plane `plane` (vxCopyImagePatch WRITE_ONLY)."""
        arr = np.ascontiguousarray(arr)
        w, h, _ = self.query_image(img)
        ph, pw = arr.shape[:2]
        addr = vx_imagepatch_addressing_t()
        addr.dim_x, addr.dim_y = pw, ph
        addr.stride_x = arr.strides[1] if arr.ndim > 1 else arr.itemsize
        addr.stride_y = arr.strides[0]
        addr.scale_x = addr.scale_y = 1024
        addr.step_x = addr.step_y = 1
        rect = vx_rectangle_t(0, 0, w, h)
        self.ok(self.vxCopyImagePatch(img, C.byref(rect), plane, C.byref(addr), arr.ctypes.data, VX_WRITE_ONLY,
                                      VX_MEMORY_TYPE_HOST), "vxCopyImagePatch(write)")

    def read_plane(self, img, plane: int = 0, dtype=None, channels=None, shape=None) -> np.ndarray:
        w, h, f = self.query_image(img)
        if dtype is None:
            dtype, channels = _PIX.get(f, (np.uint8, 1))
        if shape is None:
            shape = (h, w) if plane == 0 or f not in (VX_DF_IMAGE_NV12, VX_DF_IMAGE_IYUV) else ((h + 1) // 2, (w + 1) // 2)
            if f == VX_DF_IMAGE_NV12 and plane == 1:
                channels = 2
        ph, pw = shape
        out = np.zeros((ph, pw, channels) if channels and channels > 1 else (ph, pw), dtype=dtype)
        addr = vx_imagepatch_addressing_t()
        addr.dim_x, addr.dim_y = pw, ph
        addr.stride_x = out.itemsize * (channels or 1)
        addr.stride_y = out.strides[0]
        addr.scale_x = addr.scale_y = 1024
        addr.step_x = addr.step_y = 1
        rect = vx_rectangle_t(0, 0, w, h)
        self.ok(self.vxCopyImagePatch(img, C.byref(rect), plane, C.byref(addr), out.ctypes.data, VX_READ_ONLY,
                                      VX_MEMORY_TYPE_HOST), "vxCopyImagePatch(read)")
        return out

    def valid_region(self, img):
        r = vx_rectangle_t()
        self.ok(self.vxGetValidRegionImage(img, C.byref(r)), "vxGetValidRegionImage")
        return (r.start_x, r.start_y, r.end_x, r.end_y)

    # ---- arrays
    def array_items(self, arr, dtype=KEYPOINT_DTYPE) -> np.ndarray:
        n = C.c_size_t(0)
        self.ok(self.vxQueryArray(arr, VX_ARRAY_NUMITEMS, C.byref(n), C.sizeof(n)), "vxQueryArray")
        out = np.zeros(n.value, dtype=dtype)
        if n.value:
            self.ok(self.vxCopyArrayRange(arr, 0, n.value, dtype.itemsize, out.ctypes.data, VX_READ_ONLY,
                                          VX_MEMORY_TYPE_HOST), "vxCopyArrayRange")
        return out

    def array_set(self, arr, items: np.ndarray):
        items = np.ascontiguousarray(items)
        self.ok(self.vxTruncateArray(arr, 0), "vxTruncateArray")
        if len(items):
            self.ok(self.vxAddArrayItems(arr, len(items), items.ctypes.data, items.dtype.itemsize), "vxAddArrayItems")

    def perf(self, graph) -> vx_perf_t:
        p = vx_perf_t()
        self.ok(self.vxQueryGraph(graph, VX_GRAPH_PERFORMANCE, C.byref(p), C.sizeof(p)), "perf")
        return p
