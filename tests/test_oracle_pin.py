"""Pin the C restatement (oracle/agooracle.c) to the reference AGO CPU kernels compiled from
the reference's own sources (oracle/_ref/libopenvx_ref.so): identical inputs, identical
output-address alignment (the HAF kernels choose their SIMD/scalar split from it), and
every processed pixel must match bit for bit -- including the border columns the reference
computes from the padding bytes around the image."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from imgbuf import Img

u32, i32, vp, u8 = C.c_uint32, C.c_int32, C.c_void_p, C.c_uint8

SHAPES = [(16, 5), (17, 7), (31, 6), (64, 9), (100, 8), (19, 3)]
ALIGNS = [0, 2, 5, 8, 14]


def _fn(lib, name, argtypes):
    f = getattr(lib, name) if not name.startswith("HafCpu") else O.ref_haf(name)
    f.argtypes = argtypes
    f.restype = C.c_int
    return f


def _pair(oracle, name, argtypes, ref_argtypes=None):
    a = _fn(oracle, "oracle_" + name, argtypes)
    b = _fn(None, "HafCpu_" + name, ref_argtypes or argtypes)
    return a, b


@pytest.mark.parametrize("W,H", SHAPES)
@pytest.mark.parametrize("al", ALIGNS)
def test_pin_gaussian3x3(oracle, ref, rng, W, H, al):
    f_o, f_r = _pair(oracle, "Gaussian_U8_U8_3x3", [u32, u32, vp, u32, vp, u32], [u32, u32, vp, u32, vp, u32, vp])
    src = Img(H, W, rng=rng)
    d0, d1 = Img(H, W, align_off=al), Img(H, W, align_off=al)
    scratch = np.zeros(3 * 2 * (W + 16) + 64, np.uint8)
    f_o(W, H - 2, d0.row_ptr(1), d0.stride, src.row_ptr(1), src.stride)
    f_r(W, H - 2, d1.row_ptr(1), d1.stride, src.row_ptr(1), src.stride, scratch.ctypes.data)
    np.testing.assert_array_equal(d0.get(), d1.get())


@pytest.mark.parametrize("W,H", SHAPES)
@pytest.mark.parametrize("al", [0])   # the reference's aligned SSE loads/stores need al == 0
def test_pin_sobel_magnitude(oracle, ref, rng, W, H, al):
    f_o, f_r = _pair(oracle, "SobelMagnitude_S16_U8_3x3", [u32, u32, vp, u32, vp, u32])
    src = Img(H, W, rng=rng)
    d0, d1 = Img(H, W, np.int16, align_off=al), Img(H, W, np.int16, align_off=al)
    f_o(W, H - 2, d0.row_ptr(1), d0.stride, src.row_ptr(1), src.stride)
    f_r(W, H - 2, d1.row_ptr(1), d1.stride, src.row_ptr(1), src.stride)
    np.testing.assert_array_equal(d0.get(), d1.get())


@pytest.mark.parametrize("W,H", SHAPES)
@pytest.mark.parametrize("al", [0])   # aligned SSE stores in the reference need al == 0
def test_pin_sobel_gxy(oracle, ref, rng, W, H, al):
    f_o, f_r = _pair(oracle, "Sobel_S16S16_U8_3x3_GXY", [u32, u32, vp, u32, vp, u32, vp, u32],
                     [u32, u32, vp, u32, vp, u32, vp, u32, vp])
    src = Img(H, W, rng=rng)
    gx0, gy0 = Img(H, W, np.int16, align_off=al), Img(H, W, np.int16, align_off=al)
    gx1, gy1 = Img(H, W, np.int16, align_off=al), Img(H, W, np.int16, align_off=al)
    scratch = np.zeros(6 * 2 * (W + 16) + 64, np.uint8)
    f_o(W, H - 2, gx0.row_ptr(1), gx0.stride, gy0.row_ptr(1), gy0.stride, src.row_ptr(1), src.stride)
    f_r(W, H - 2, gx1.row_ptr(1), gx1.stride, gy1.row_ptr(1), gy1.stride, src.row_ptr(1), src.stride,
        scratch.ctypes.data)
    np.testing.assert_array_equal(gx0.get(), gx1.get())
    np.testing.assert_array_equal(gy0.get(), gy1.get())


@pytest.mark.parametrize("W,H", SHAPES)
@pytest.mark.parametrize("al", [0, 2, 6, 10])
@pytest.mark.parametrize("amp", [1020, 32767])
def test_pin_magnitude(oracle, ref, rng, W, H, al, amp):
    f_o, f_r = _pair(oracle, "Magnitude_S16_S16S16", [u32, u32, vp, u32, vp, u32, vp, u32])
    gx = Img(H, W, np.int16, fill=rng.integers(-amp, amp + 1, (H, W)))
    gy = Img(H, W, np.int16, fill=rng.integers(-amp, amp + 1, (H, W)))
    d0, d1 = Img(H, W, np.int16, align_off=al), Img(H, W, np.int16, align_off=al)
    f_o(W, H, d0.ptr, d0.stride, gx.ptr, gx.stride, gy.ptr, gy.stride)
    f_r(W, H, d1.ptr, d1.stride, gx.ptr, gx.stride, gy.ptr, gy.stride)
    np.testing.assert_array_equal(d0.get(), d1.get())


@pytest.mark.parametrize("W,H", SHAPES)
@pytest.mark.parametrize("al", [0, 3, 9])
@pytest.mark.parametrize("shift", [0, 1, 3, 7])
def test_pin_colordepth_sat(oracle, ref, rng, W, H, al, shift):
    f_o, f_r = _pair(oracle, "ColorDepth_U8_S16_Sat", [u32, u32, vp, u32, vp, u32, i32])
    src = Img(H, W, np.int16, fill=rng.integers(-32768, 32768, (H, W)))
    d0, d1 = Img(H, W, align_off=al), Img(H, W, align_off=al)
    f_o(W, H, d0.ptr, d0.stride, src.ptr, src.stride, shift)
    f_r(W, H, d1.ptr, d1.stride, src.ptr, src.stride, shift)
    np.testing.assert_array_equal(d0.get(), d1.get())


@pytest.mark.parametrize("W,H", SHAPES)
@pytest.mark.parametrize("al", [0, 3])
@pytest.mark.parametrize("thr", [0, 1, 127, 128, 200, 255])
def test_pin_threshold_binary(oracle, ref, rng, W, H, al, thr):
    f_o, f_r = _pair(oracle, "Threshold_U8_U8_Binary", [u32, u32, vp, u32, vp, u32, u8])
    src = Img(H, W, rng=rng, align_off=al)
    d0, d1 = Img(H, W, align_off=al), Img(H, W, align_off=al)
    f_o(W, H, d0.ptr, d0.stride, src.ptr, src.stride, thr)
    f_r(W, H, d1.ptr, d1.stride, src.ptr, src.stride, thr)
    np.testing.assert_array_equal(d0.get(), d1.get())
