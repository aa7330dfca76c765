"""Loading of the in-tree native libraries (no fallback: a missing library is an error)."""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(PKG, "lib")
AGOCUDA_SO = os.path.join(LIBDIR, "libagocuda.so")
OPENVX_SO = os.path.join(LIBDIR, "libopenvx.so")

_agocuda = None
_openvx = None

u32, i32, u64, vp, f32 = C.c_uint32, C.c_int32, C.c_uint64, C.c_void_p, C.c_float

# name -> argtypes (all return int unless listed in _RESTYPES)
AGOCUDA_SIGNATURES = {
    "agocuda_abi_version": [],
    "agocuda_launch_count": [],
    "agocuda_Gaussian_U8_U8_3x3": [vp, u32, u32, vp, u32, vp, u32],
    "agocuda_Sobel_S16S16_U8_3x3_GXY": [vp, u32, u32, vp, u32, vp, u32, vp, u32],
    "agocuda_SobelMagnitude_S16_U8_3x3": [vp, u32, u32, vp, u32, vp, u32],
    "agocuda_Magnitude_S16_S16S16": [vp, u32, u32, vp, u32, vp, u32, vp, u32],
    "agocuda_ColorDepth_U8_S16_Sat": [vp, u32, u32, vp, u32, vp, u32, i32],
    "agocuda_Threshold_U8_U8_Binary": [vp, u32, u32, vp, u32, vp, u32, i32],
    "agocuda_fused_GaussSobelMagDepthThresh": [vp, vp, u32, u32, u32, i32, i32],
    "agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_size": [u32],
    "agocuda_fused_GaussSobelMagDepthThresh_tensor_maps": [vp, u32, vp, C.c_size_t],
    "agocuda_fused_GaussSobelMagDepthThresh_tma": [vp, vp, vp, u32, u32, u32, i32, i32, vp],
}
_RESTYPES = {"agocuda_launch_count": u64, "agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_size": C.c_size_t}


class AgoFrame(C.Structure):
    """Mirror of `agocuda_frame` (include/agocuda.h)."""
    _fields_ = [("src", vp), ("dst", vp), ("width", u32), ("height", u32),
                ("srcStride", u32), ("dstStride", u32), ("simdBegin", i32), ("simdEnd", i32)]


LK_MAX_LEVELS = 12


class PyramidLevel(C.Structure):
    """Mirror of `agocuda_pyramid_level`."""
    _fields_ = [("image", vp), ("width", u32), ("height", u32), ("stride", u32), ("reserved", u32)]


class HalfJob(C.Structure):
    """Mirror of `agocuda_half_job`."""
    _fields_ = [("src", vp), ("dst", vp), ("srcW", u32), ("srcH", u32), ("srcStride", u32), ("dstW", u32),
                ("dstH", u32), ("dstStride", u32), ("tileBegin", u32), ("reserved", u32)]


class LkFrame(C.Structure):
    """Mirror of `agocuda_lk_frame`."""
    _fields_ = [("oldPyr", PyramidLevel * LK_MAX_LEVELS), ("newPyr", PyramidLevel * LK_MAX_LEVELS),
                ("oldPoints", vp), ("estPoints", vp), ("newPoints", vp), ("pOldCount", vp), ("pEstCount", vp),
                ("pNewCount", vp), ("scharrRows", vp), ("newCapacity", u32), ("levels", u32), ("termination", i32),
                ("epsilon", f32), ("numIterations", u32), ("useInitialEstimate", i32), ("windowDimension", i32),
                ("count", u32), ("scharrWords", (u32 * 2) * LK_MAX_LEVELS), ("carry", vp), ("carryRows", u32)]


def agocuda() -> C.CDLL:
    """The CUDA kernel library (include/agocuda.h).  Raises if it has not been built."""
    global _agocuda
    if _agocuda is None:
        if not os.path.exists(AGOCUDA_SO):
            raise RuntimeError(f"{AGOCUDA_SO} is missing: run `python -m mivisionx_b200.build` first")
        lib = C.CDLL(AGOCUDA_SO, mode=C.RTLD_GLOBAL)
        for name, args in AGOCUDA_SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, C.c_int)
        _agocuda = lib
    return _agocuda


def openvx() -> C.CDLL:
    """The OpenVX host engine (libopenvx.so of this package).  Raises if not built."""
    global _openvx
    if _openvx is None:
        if not os.path.exists(OPENVX_SO):
            raise RuntimeError(f"{OPENVX_SO} is missing: run `python -m mivisionx_b200.build` first")
        agocuda()
        _openvx = C.CDLL(OPENVX_SO, mode=C.RTLD_LOCAL)
    return _openvx
