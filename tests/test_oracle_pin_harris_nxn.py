"""Pin the Harris 5x5 / 7x7 restatements (oracle_HarrisSobel_HG3_U8_NxN,
oracle_HarrisScore_HVC_HG3_NxN) to the reference's HafCpu_HarrisSobel_HG3_U8_{5x5,7x7}
(ago_haf_cpu_harris.cpp:333, :455) and HafCpu_HarrisScore_HVC_HG3_{5x5,7x7} (:661, :731),
built from its own sources: the gradient products of every written row and column
(including the columns whose taps leave the row) and the scores of every pixel.  Buffers use
AGO's row pitch (ALIGN16 of the row), which for W % 4 == 0 is exactly 12 W bytes for the
gradient products: the reference's gradient loops step from one row's end straight into the
next row's start."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from imgbuf import Img

u32, vp, f32 = C.c_uint32, C.c_void_p, C.c_float


def _ref(name, args):
    f = O.ref_haf(name)
    f.argtypes, f.restype = args, C.c_int
    return f


def _orc(name, args):
    f = getattr(O.oracle_lib(), name)
    f.argtypes, f.restype = args, C.c_int
    return f


@pytest.mark.parametrize("gs", [5, 7])
@pytest.mark.parametrize("W,H", [(64, 20), (48, 33), (96, 12)])
def test_pin_harris_sobel(ref, rng, gs, W, H):
    src = Img(H, W, rng=rng)
    st = ((12 * W + 15) // 16) * 16
    d0, d1 = Img(H, W, np.float32, channels=3, stride=st), Img(H, W, np.float32, channels=3, stride=st)
    scratch = np.zeros(16 * ((W + 15) & ~15) * 8 + 256, np.uint8)
    _orc("oracle_HarrisSobel_HG3_U8_NxN", [u32, u32, vp, u32, vp, u32, u32])(W, H, d0.ptr, d0.stride, src.ptr, src.stride, gs)
    _ref(f"HafCpu_HarrisSobel_HG3_U8_{gs}x{gs}", [u32, u32, vp, u32, vp, u32, vp])(W, H, d1.ptr, d1.stride, src.ptr,
                                                                                    src.stride, scratch.ctypes.data)
    r = gs // 2
    np.testing.assert_array_equal(d0.get()[r:H - r], d1.get()[r:H - r])


@pytest.mark.parametrize("bs", [5, 7])
@pytest.mark.parametrize("W,H", [(64, 20), (48, 33)])
def test_pin_harris_score(ref, rng, bs, W, H):
    g = Img(H, W, np.float32, channels=3, stride=((12 * W + 15) // 16) * 16)
    g.set(rng.integers(0, 1 << 20, (H, W, 3)).astype(np.float32) * np.float32(37.0))
    d0, d1 = Img(H, W, np.float32), Img(H, W, np.float32)
    f = O.oracle_lib().oracle_harris_norm_factor_block
    f.argtypes, f.restype = [C.c_int32, C.c_int32], C.c_float
    norm = f(5, bs)
    args = [u32, u32, vp, u32, vp, u32, f32, f32, f32]
    _orc("oracle_HarrisScore_HVC_HG3_NxN", args + [u32])(W, H, d0.ptr, d0.stride, g.ptr, g.stride, 0.04, 1e-9, norm, bs)
    _ref(f"HafCpu_HarrisScore_HVC_HG3_{bs}x{bs}", args)(W, H, d1.ptr, d1.stride, g.ptr, g.stride, 0.04, 1e-9, norm)
    out = d0.get()
    np.testing.assert_array_equal(out, d1.get())
    assert (out > 0).mean() > 0.01
