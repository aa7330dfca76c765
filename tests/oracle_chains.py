"""Graph-level compositions of the oracle kernels, called the way the AGO kernel wrappers
call the HAF CPU kernels (ago/ago_kernel_api.cpp) on AGO-style buffers (16-byte aligned
rows, so the HAF scalar prefix is empty).  Each returns the output image(s) and the OpenVX
valid rectangle (start_x, start_y, end_x, end_y)."""
from __future__ import annotations

import ctypes as C

import numpy as np

import oracle as O
from imgbuf import Img

u32, i32, vp, u8 = C.c_uint32, C.c_int32, C.c_void_p, C.c_uint8

_SIGS = {
    "Gaussian_U8_U8_3x3": [u32, u32, vp, u32, vp, u32],
    "SobelMagnitude_S16_U8_3x3": [u32, u32, vp, u32, vp, u32],
    "Sobel_S16S16_U8_3x3_GXY": [u32, u32, vp, u32, vp, u32, vp, u32],
    "Magnitude_S16_S16S16": [u32, u32, vp, u32, vp, u32, vp, u32],
    "ColorDepth_U8_S16_Sat": [u32, u32, vp, u32, vp, u32, i32],
    "Threshold_U8_U8_Binary": [u32, u32, vp, u32, vp, u32, u8],
}


def fn(name):
    lib = O.oracle_lib()
    f = getattr(lib, "oracle_" + name)
    if name in _SIGS:
        f.argtypes = _SIGS[name]
    f.restype = C.c_int
    return f


def ago_img(h, w, dtype=np.uint8, channels=1):
    return Img(h, w, dtype, channels=channels, align_off=0)


def shrink(rect, n):
    sx, sy, ex, ey = rect
    return (sx + n, sy + n, ex - n, ey - n)


def gaussian3x3(src: Img) -> Img:
    out = ago_img(src.h, src.w)
    fn("Gaussian_U8_U8_3x3")(src.w, src.h - 2, out.row_ptr(1), out.stride, src.row_ptr(1), src.stride)
    return out


def sobel_magnitude(src: Img) -> Img:
    out = ago_img(src.h, src.w, np.int16)
    fn("SobelMagnitude_S16_U8_3x3")(src.w, src.h - 2, out.row_ptr(1), out.stride, src.row_ptr(1), src.stride)
    return out


def sobel_gxy(src: Img):
    gx, gy = ago_img(src.h, src.w, np.int16), ago_img(src.h, src.w, np.int16)
    fn("Sobel_S16S16_U8_3x3_GXY")(src.w, src.h - 2, gx.row_ptr(1), gx.stride, gy.row_ptr(1), gy.stride,
                                  src.row_ptr(1), src.stride)
    return gx, gy


def magnitude(gx: Img, gy: Img) -> Img:
    out = ago_img(gx.h, gx.w, np.int16)
    fn("Magnitude_S16_S16S16")(gx.w, gx.h, out.ptr, out.stride, gx.ptr, gx.stride, gy.ptr, gy.stride)
    return out


def colordepth_sat(src: Img, shift: int) -> Img:
    out = ago_img(src.h, src.w)
    fn("ColorDepth_U8_S16_Sat")(src.w, src.h, out.ptr, out.stride, src.ptr, src.stride, shift)
    return out


def threshold_binary(src: Img, thr: int) -> Img:
    out = ago_img(src.h, src.w)
    fn("Threshold_U8_U8_Binary")(src.w, src.h, out.ptr, out.stride, src.ptr, src.stride, thr & 0xFF)
    return out


def cfg1_chain(img: np.ndarray, shift: int = 0, thr: int = 128):
    """Gaussian3x3 -> Sobel3x3 -> Magnitude -> ConvertDepth(SATURATE) -> Threshold(BINARY)
    with virtual intermediates: AGO lowers Sobel+Magnitude to SobelMagnitude
    (ago/ago_drama_remove.cpp:165)."""
    h, w = img.shape
    src = ago_img(h, w)
    src.set(img)
    g = gaussian3x3(src)
    m = sobel_magnitude(g)
    d = colordepth_sat(m, shift)
    t = threshold_binary(d, thr)
    return t.get(), shrink((0, 0, w, h), 2)
