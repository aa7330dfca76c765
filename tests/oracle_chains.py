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
    """Buffer laid out as AGO allocates images: 16-byte row pitch, zero padding around."""
    bpp = np.dtype(dtype).itemsize * channels
    return Img(h, w, dtype, channels=channels, stride=((w * bpp + 15) // 16) * 16, pad=4, align_off=0)


_SIGS.update({
    "CannySobel_U16_U8_3x3_L1NORM": [u32, u32, vp, u32, vp, u32],
    "CannySuppThreshold_U8XY_U16_3x3": [u32, vp, C.POINTER(C.c_uint32), u32, u32, vp, u32, vp, u32, C.c_uint16, C.c_uint16],
    "CannyEdgeTrace_U8_U8XY": [u32, u32, vp, u32, u32, vp, u32],
    "HarrisSobel_HG3_U8_3x3": [u32, u32, vp, u32, vp, u32],
    "HarrisScore_HVC_HG3_3x3": [u32, u32, vp, u32, vp, u32, C.c_float, C.c_float, C.c_float],
    "HarrisSobel_HG3_U8_NxN": [u32, u32, vp, u32, vp, u32, u32],
    "HarrisScore_HVC_HG3_NxN": [u32, u32, vp, u32, vp, u32, C.c_float, C.c_float, C.c_float, u32],
    "NonMaxSupp_XY_ANY_3x3": [u32, vp, C.POINTER(C.c_uint32), u32, u32, vp, u32],
    "HarrisMergeSortAndPick_XY_XYS": [u32, vp, C.POINTER(C.c_uint32), vp, u32, C.c_float, u32, u32],
})

XYS = np.dtype([("x", "<i2"), ("y", "<i2"), ("s", "<f4")])
KP = np.dtype([("x", "<i4"), ("y", "<i4"), ("strength", "<f4"), ("scale", "<f4"), ("orientation", "<f4"),
               ("tracking_status", "<i4"), ("error", "<f4")])


def harris_norm(gs=3):
    f = fn("harris_norm_factor")
    f.argtypes = [i32]
    f.restype = C.c_float
    return f(gs)


def canny_parts(img: np.ndarray, lower=80, upper=100):
    """CannySobel, CannySuppThreshold, CannyEdgeTrace as AGO calls them; returns the packed
    gradient plane, the 0/127/255 map, the strong stack and the final edge map."""
    h, w = img.shape
    src = ago_img(h, w); src.set(img)
    sob = ago_img(h, w, np.uint16)
    out = ago_img(h, w)
    stack = np.zeros(w * h, np.uint32)
    top = C.c_uint32(0)
    fn("CannySobel_U16_U8_3x3_L1NORM")(w, h, sob.ptr, sob.stride, src.ptr, src.stride)
    fn("CannySuppThreshold_U8XY_U16_3x3")(w * h, stack.ctypes.data, C.byref(top), w, h, out.ptr, out.stride,
                                          sob.ptr, sob.stride, lower, upper)
    supp = out.get()
    strong = stack[:top.value].copy()
    fn("CannyEdgeTrace_U8_U8XY")(w, h, out.ptr, out.stride, w * h, stack.ctypes.data, top.value)
    return sob.get(), supp, strong, out.get()


def canny(img: np.ndarray, lower=80, upper=100):
    """vxCannyEdgeDetectorNode (3x3, L1): edge map and valid rectangle."""
    h, w = img.shape
    return canny_parts(img, lower, upper)[3], (2, 2, w - 2, h - 2)


def harris_norm_block(gs, bs):
    f = O.oracle_lib().oracle_harris_norm_factor_block
    f.argtypes, f.restype = [i32, i32], C.c_float
    return f(gs, bs)


def harris_parts(img: np.ndarray, k=0.04, tc=1e-3, gs=3, bs=3):
    """HarrisSobel_HG3_U8_{gs}x{gs}, HarrisScore_HVC_HG3_{bs}x{bs} (normalised by
    (255 * 2^(gs-1) * bs)^4) and NonMaxSupp_XY_ANY_3x3 on AGO-laid-out zeroed buffers."""
    h, w = img.shape
    src = ago_img(h, w); src.set(img)
    hg3 = ago_img(h, w, np.float32, 3)
    hvc = ago_img(h, w, np.float32)
    lst = np.zeros(w * h, XYS)
    cnt = C.c_uint32(0)
    if gs == 3:
        fn("HarrisSobel_HG3_U8_3x3")(w, h, hg3.ptr, hg3.stride, src.ptr, src.stride)
    else:
        fn("HarrisSobel_HG3_U8_NxN")(w, h, hg3.ptr, hg3.stride, src.ptr, src.stride, gs)
    if bs == 3:
        fn("HarrisScore_HVC_HG3_3x3")(w, h, hvc.ptr, hvc.stride, hg3.ptr, hg3.stride, k, tc, harris_norm_block(gs, 3))
    else:
        fn("HarrisScore_HVC_HG3_NxN")(w, h, hvc.ptr, hvc.stride, hg3.ptr, hg3.stride, k, tc, harris_norm_block(gs, bs), bs)
    fn("NonMaxSupp_XY_ANY_3x3")(w * h, lst.ctypes.data, C.byref(cnt), w, h, hvc.ptr, hvc.stride)
    return hg3.get(), hvc.get(), lst[:cnt.value].copy()


def harris_pick(lst: np.ndarray, w, h, min_distance=5.0, capacity=1 << 20):
    lst = lst.copy()
    out = np.zeros(max(1, capacity), KP)
    cnt = C.c_uint32(0)
    fn("HarrisMergeSortAndPick_XY_XYS")(capacity, out.ctypes.data, C.byref(cnt), lst.ctypes.data, len(lst),
                                        min_distance, w, h)
    return out[:min(cnt.value, capacity)], cnt.value


def _sfn(name, args):
    f = getattr(O.oracle_lib(), "oracle_" + name)
    f.argtypes = args
    f.restype = C.c_int
    return f


def scale_matrix(kind, sw, sh, dw, dh):
    m = (C.c_float * 4)()
    f = O.oracle_lib().oracle_scale_matrix
    f.argtypes = [C.c_int, u32, u32, u32, u32, vp]
    f.restype = None
    f(kind, sw, sh, dw, dh, C.cast(m, vp))
    return m


def color_scale_warp(rgb: np.ndarray, matrix: np.ndarray):
    """The configuration-3 graph as AGO runs it: NV12 and IYUV from RGB, ScaleImage of the NV12
    Y plane (the ChannelExtract copy is removed), both warps of the bilinear result."""
    h, w = rgb.shape[:2]
    src = ago_img(h, w, np.uint8, 3); src.set(rgb)
    y, uv = ago_img(h, w), ago_img(h // 2, w // 2, np.uint8, 2)
    y2, u, v = ago_img(h, w), ago_img(h // 2, w // 2), ago_img(h // 2, w // 2)
    a8 = [u32, u32, vp, u32, vp, u32, vp, u32]
    _sfn("ColorConvert_NV12_RGB", a8)(w, h, y.ptr, y.stride, uv.ptr, uv.stride, src.ptr, src.stride)
    _sfn("ColorConvert_IYUV_RGB", a8 + [vp, u32])(w, h, y2.ptr, y2.stride, u.ptr, u.stride, v.ptr, v.stride, src.ptr, src.stride)
    out = {"nv12_y": y.get(), "nv12_uv": uv.get(), "iyuv_y": y2.get(), "iyuv_u": u.get(), "iyuv_v": v.get()}
    dw, dh = w // 2, h // 2
    sargs = [u32, u32, vp, u32, u32, u32, vp, u32, vp]
    sb, sa = ago_img(dh, dw), ago_img(dh, dw)
    _sfn("ScaleImage_U8_U8_Bilinear", sargs)(dw, dh, sb.ptr, sb.stride, w, h, y.ptr, y.stride, C.cast(scale_matrix(1, w, h, dw, dh), vp))
    _sfn("ScaleImage_U8_U8_Area", sargs)(dw, dh, sa.ptr, sa.stride, w, h, y.ptr, y.stride, C.cast(scale_matrix(2, w, h, dw, dh), vp))
    out["scale_bilinear"], out["scale_area"] = sb.get(), sa.get()
    m = np.ascontiguousarray(matrix, np.float32)
    wn, wb = ago_img(dh, dw), ago_img(dh, dw)
    _sfn("WarpAffine_U8_U8_Nearest_Constant", [u32, u32, vp, u32, u32, u32, vp, u32, vp, u8, u32, u32, u32, u32])(
        dw, dh, wn.ptr, wn.stride, dw, dh, sb.ptr, sb.stride, m.ctypes.data, 0, 0, 0, dw, dh)
    _sfn("WarpAffine_U8_U8_Bilinear_Constant", [u32, u32, vp, u32, u32, u32, vp, u32, vp, u8])(
        dw, dh, wb.ptr, wb.stride, dw, dh, sb.ptr, sb.stride, m.ctypes.data, 0)
    out["warp_nearest"], out["warp_bilinear"] = wn.get(), wb.get()
    # Pixels whose bilinear footprint reaches below the last source row: the reference reads
    # past its buffer there (geometric.cpp:1190, psrc + stride), so its value is undefined.
    f = np.float32
    xs_ = np.arange(((dw + 3) // 4) * 4, dtype=f)[None, :dw]
    ys_ = np.arange(dh, dtype=f)[:, None]
    with np.errstate(invalid="ignore"):
        yd = ys_ * m[1, 1] + m[2, 1]
        ysrc = (m[0, 1] * xs_).astype(f) + yd.astype(f)
        xd = ys_ * m[1, 0] + m[2, 0]
        xsrc = (m[0, 0] * xs_).astype(f) + xd.astype(f)
    inside = (xsrc >= 0) & (xsrc < dw) & (ysrc >= 0) & (ysrc < dh)
    out["warp_bilinear_undefined_in_reference"] = inside & (np.trunc(ysrc) >= dh - 1)
    full = (0, 0, dw, dh)
    for k in ("scale_bilinear", "scale_area", "warp_nearest", "warp_bilinear"):
        out[k + "_rect"] = full
    return out


def harris(img: np.ndarray, k=0.04, tc=1e-3, min_distance=5.0, capacity=1 << 20, gs=3, bs=3):
    """vxHarrisCornersNode (gradient gs, block bs): (corners, num_corners)."""
    h, w = img.shape
    return harris_pick(harris_parts(img, k, tc, gs, bs)[2], w, h, min_distance, capacity)


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
