"""Pin the colour-conversion, scaling and warp restatements (oracle/agooracle_geometry.c)
to the reference HAF CPU kernels on AGO-layout buffers."""
import ctypes as C
import math

import numpy as np
import pytest

import oracle as O
from imgbuf import Img
from mivisionx_b200 import workloads as WL

u32, vp, u8, f32 = C.c_uint32, C.c_void_p, C.c_uint8, C.c_float


class Rect(C.Structure):
    _fields_ = [("sx", u32), ("sy", u32), ("ex", u32), ("ey", u32)]


def ago_img(h, w, dtype=np.uint8, ch=1):
    bpp = np.dtype(dtype).itemsize * ch
    return Img(h, w, dtype, channels=ch, stride=((w * bpp + 15) // 16) * 16, pad=4, align_off=0)


def ofn(name, args):
    f = getattr(O.oracle_lib(), name)
    f.argtypes = args
    f.restype = C.c_int
    return f


def rfn(name, args):
    f = O.ref_haf(name)
    f.argtypes = args
    f.restype = C.c_int
    return f


@pytest.mark.parametrize("W,H", [(64, 32), (38, 10), (132, 66), (3840, 16)])
def test_pin_color_convert(ref, W, H):
    rgb = WL.cfg3_frame(seed=W + H, width=W, height=H)
    src = ago_img(H, W, np.uint8, 3); src.set(rgb)
    outs = {}
    for who in ("ref", "oracle"):
        y, uv = ago_img(H, W), ago_img(H // 2, W // 2, np.uint8, 2)
        y2, u, v = ago_img(H, W), ago_img(H // 2, W // 2), ago_img(H // 2, W // 2)
        args8 = [u32, u32, vp, u32, vp, u32, vp, u32]
        args10 = [u32, u32, vp, u32, vp, u32, vp, u32, vp, u32]
        f1 = rfn("HafCpu_ColorConvert_NV12_RGB", args8) if who == "ref" else ofn("oracle_ColorConvert_NV12_RGB", args8)
        f2 = rfn("HafCpu_ColorConvert_IYUV_RGB", args10) if who == "ref" else ofn("oracle_ColorConvert_IYUV_RGB", args10)
        f1(W, H, y.ptr, y.stride, uv.ptr, uv.stride, src.ptr, src.stride)
        f2(W, H, y2.ptr, y2.stride, u.ptr, u.stride, v.ptr, v.stride, src.ptr, src.stride)
        outs[who] = [a.get() for a in (y, uv, y2, u, v)]
    for a, b in zip(outs["ref"], outs["oracle"]):
        np.testing.assert_array_equal(a, b)


def _matrix(kind, sw, sh, dw, dh):
    m = (C.c_float * 4)()
    f = O.oracle_lib().oracle_scale_matrix
    f.argtypes = [C.c_int, u32, u32, u32, u32, vp]
    f.restype = None
    f(kind, sw, sh, dw, dh, C.cast(m, vp))
    return m


@pytest.mark.parametrize("kind,name", [(0, "Nearest"), (1, "Bilinear"), (2, "Area")])
@pytest.mark.parametrize("sw,sh,dw,dh", [(128, 64, 64, 32), (3840, 32, 1920, 16), (100, 60, 50, 30), (64, 48, 96, 72),
                                         (90, 50, 40, 30)])
def test_pin_scale(ref, kind, name, sw, sh, dw, dh):
    if name == "Area" and not ((sw == 2 * dw and sh == 2 * dh) or (sw == dw and sh == dh)):
        pytest.skip("area restatement covers the exact 1x and 2x paths")
    img = WL.cfg1_image(seed=sw * 3 + dh, width=sw, height=sh)
    src = ago_img(sh, sw); src.set(img)
    m = _matrix(kind, sw, sh, dw, dh)
    a, b = ago_img(dh, dw), ago_img(dh, dw)
    buf = np.zeros(16 + ((dw + 15) & ~15) * 8 + 4 * dh + 64, np.uint8)
    buf[:16] = np.frombuffer(bytes(m), np.uint8)
    args = [u32, u32, vp, u32, u32, u32, vp, u32, vp]
    assert rfn("HafCpu_ScaleImage_U8_U8_" + name, args)(dw, dh, a.ptr, a.stride, sw, sh, src.ptr, src.stride, buf.ctypes.data) == 0
    assert ofn("oracle_ScaleImage_U8_U8_" + name, args)(dw, dh, b.ptr, b.stride, sw, sh, src.ptr, src.stride, C.cast(m, vp)) == 0
    np.testing.assert_array_equal(b.get(), a.get())


def _affine(seed, sw, sh, dw, dh):
    u = WL.uniform01(seed, 4, stream=23)
    th = math.radians((u[0] * 2 - 1) * 15)
    s = 0.8 + 0.4 * u[1]
    a, b = s * math.cos(th), s * math.sin(th)
    cx, cy = dw / 2, dh / 2
    c0 = sw / 2 - a * cx + b * cy + (u[2] * 2 - 1) * 0.05 * sw
    c1 = sh / 2 - b * cx - a * cy + (u[3] * 2 - 1) * 0.05 * sh
    return np.array([[a, b], [-b, a], [c0, c1]], np.float32)


@pytest.mark.parametrize("sw,sh,dw,dh,seed", [(64, 48, 64, 48, 1), (200, 120, 160, 100, 2), (96, 64, 96, 64, 3),
                                              (96, 64, 48, 32, 4)])
@pytest.mark.parametrize("valid", [None, (3, 2, 90, 60)])
def test_pin_warp_affine(ref, sw, sh, dw, dh, seed, valid):
    img = WL.cfg1_image(seed=seed, width=sw, height=sh)
    src = ago_img(sh, sw); src.set(img)
    m = _affine(seed, sw, sh, dw, dh)
    local = np.zeros(2 * 4 * dw + 256, np.uint8)
    rect = Rect(*(valid or (0, 0, sw, sh)))
    for name in ("Nearest_Constant", "Bilinear_Constant"):
        a, b = ago_img(dh, dw), ago_img(dh, dw)
        if name == "Nearest_Constant":
            rfn("HafCpu_WarpAffine_U8_U8_" + name, [u32, u32, vp, u32, u32, u32, vp, u32, vp, u8, Rect, vp])(
                dw, dh, a.ptr, a.stride, sw, sh, src.ptr, src.stride, m.ctypes.data, 7, rect, local.ctypes.data)
            ofn("oracle_WarpAffine_U8_U8_" + name, [u32, u32, vp, u32, u32, u32, vp, u32, vp, u8, u32, u32, u32, u32])(
                dw, dh, b.ptr, b.stride, sw, sh, src.ptr, src.stride, m.ctypes.data, 7, rect.sx, rect.sy, rect.ex, rect.ey)
        else:
            rfn("HafCpu_WarpAffine_U8_U8_" + name, [u32, u32, vp, u32, u32, u32, vp, u32, vp, u8, vp])(
                dw, dh, a.ptr, a.stride, sw, sh, src.ptr, src.stride, m.ctypes.data, 7, local.ctypes.data)
            ofn("oracle_WarpAffine_U8_U8_" + name, [u32, u32, vp, u32, u32, u32, vp, u32, vp, u8])(
                dw, dh, b.ptr, b.stride, sw, sh, src.ptr, src.stride, m.ctypes.data, 7)
        np.testing.assert_array_equal(b.get(), a.get(), err_msg=name)
