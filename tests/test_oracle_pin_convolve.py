"""Pin the convolution restatement (oracle_Convolve_{U8,S16}_U8, oracle/agooracle.c) to the
reference's HafCpu_Convolve_{U8,S16}_U8_{3,5,7,9}xN (ago_haf_cpu_filter.cpp:2676-3830) built
from its own sources: every width, several heights, both output types, shifts 0 and 3,
negative coefficients, widths with a scalar tail -- all processed pixels bit for bit,
including the SIMD-body logical shift and the unshifted scalar columns."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from imgbuf import Img

u32, i32, vp = C.c_uint32, C.c_int32, C.c_void_p
SZ = C.c_size_t


def _ref(out, cols):
    f = O.ref_haf(f"HafCpu_Convolve_{out}_U8_{cols}xN")
    f.argtypes, f.restype = [u32, u32, vp, u32, vp, u32, vp, SZ, i32], C.c_int
    return f


def _orc(out):
    f = getattr(O.oracle_lib(), f"oracle_Convolve_{out}_U8")
    f.argtypes, f.restype = [u32, u32, vp, u32, vp, u32, vp, u32, u32, i32], C.c_int
    return f


def coefficients(cols, rows, seed, big=False):
    rng = np.random.default_rng(seed)
    hi = 2000 if big else 9
    return rng.integers(-hi, hi + 1, cols * rows).astype(np.int16)


@pytest.mark.parametrize("out", ["U8", "S16"])
@pytest.mark.parametrize("cols", [3, 5, 7, 9])
@pytest.mark.parametrize("rows", [3, 5, 9])
@pytest.mark.parametrize("shift,big", [(0, False), (3, False), (0, True), (5, True)])
@pytest.mark.parametrize("W,H", [(64, 20), (45, 17)])
def test_pin_convolve(ref, rng, out, cols, rows, shift, big, W, H):
    if O.ref_lib() is None:
        pytest.skip("reference library not built")
    dt = np.uint8 if out == "U8" else np.int16
    src = Img(H, W, rng=rng)
    conv = coefficients(cols, rows, cols * 100 + rows * 10 + shift, big)
    d0, d1 = Img(H, W, dt), Img(H, W, dt)
    hy = rows // 2
    _orc(out)(W, H - rows + 1, d0.row_ptr(hy), d0.stride, src.row_ptr(hy), src.stride, conv.ctypes.data, cols, rows, shift)
    _ref(out, cols)(W, H - rows + 1, d1.row_ptr(hy), d1.stride, src.row_ptr(hy), src.stride, conv.ctypes.data, rows, shift)
    np.testing.assert_array_equal(d0.get(), d1.get())
