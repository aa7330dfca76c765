"""Pin the Canny and Harris restatements (oracle/agooracle.c) to the reference HAF CPU
kernels built from the reference sources, on buffers laid out as AGO lays them out
(16-byte row strides, zero padding around the image) -- the reference reads one pixel
outside each row at the image borders, and those values reach the interior through
hysteresis and non-maximum suppression, so the layout is part of the semantics."""
import ctypes as C
import math

import numpy as np
import pytest

import oracle as O
from imgbuf import Img
from mivisionx_b200 import workloads as WL

u32, i32, u16, vp, f32 = C.c_uint32, C.c_int32, C.c_uint16, C.c_void_p, C.c_float
P = C.POINTER(C.c_uint32)

XYS = np.dtype([("x", "<i2"), ("y", "<i2"), ("s", "<f4")])
KP = np.dtype([("x", "<i4"), ("y", "<i4"), ("strength", "<f4"), ("scale", "<f4"), ("orientation", "<f4"),
               ("tracking_status", "<i4"), ("error", "<f4")])

SHAPES = [(16, 8), (48, 20), (37, 19), (64, 64), (100, 41)]


def ago_img(h, w, dtype=np.uint8, ch=1):
    bpp = np.dtype(dtype).itemsize * ch
    return Img(h, w, dtype, channels=ch, stride=((w * bpp + 15) // 16) * 16, pad=4, align_off=0)


def fn(lib, name, args):
    f = getattr(lib, name) if lib is not None else O.ref_haf(name)
    f.argtypes = args
    f.restype = C.c_int
    return f


def scene(W, H, seed):
    img = WL.cfg2_scene(seed=seed, width=W, height=H, rects=max(2, W * H // 400))
    return img


def canny_front(lib_or_ref, img):
    """CannySobel + CannySuppThreshold as the AGO wrappers call them; returns (sobel, map, stack)."""
    H, W = img.shape
    src = ago_img(H, W); src.set(img)
    sob = ago_img(H, W, np.uint16)
    out = ago_img(H, W)
    stack = np.zeros(W * H, dtype=np.uint32)
    top = C.c_uint32(0)
    if lib_or_ref == "ref":
        local = np.zeros(((W + 15) & ~15) * 4 + 128, np.uint8)
        fn(None, "HafCpu_CannySobel_U16_U8_3x3_L1NORM", [u32, u32, vp, u32, vp, u32, vp])(
            W, H, sob.ptr, sob.stride, src.ptr, src.stride, local.ctypes.data)
        fn(None, "HafCpu_CannySuppThreshold_U8XY_U16_3x3", [u32, vp, P, u32, u32, vp, u32, vp, u32, u16, u16])(
            W * H, stack.ctypes.data, C.byref(top), W, H, out.ptr, out.stride, sob.ptr, sob.stride, 80, 100)
    else:
        o = O.oracle_lib()
        fn(o, "oracle_CannySobel_U16_U8_3x3_L1NORM", [u32, u32, vp, u32, vp, u32])(W, H, sob.ptr, sob.stride, src.ptr, src.stride)
        fn(o, "oracle_CannySuppThreshold_U8XY_U16_3x3", [u32, vp, P, u32, u32, vp, u32, vp, u32, u16, u16])(
            W * H, stack.ctypes.data, C.byref(top), W, H, out.ptr, out.stride, sob.ptr, sob.stride, 80, 100)
    return sob, out, stack, top.value


@pytest.mark.parametrize("W,H", SHAPES)
def test_pin_canny(ref, W, H):
    img = scene(W, H, seed=W + H)
    rs, ro, rst, rtop = canny_front("ref", img)
    os_, oo, ost, otop = canny_front("oracle", img)
    np.testing.assert_array_equal(os_.get()[1:H - 1], rs.get()[1:H - 1])
    np.testing.assert_array_equal(oo.get(), ro.get())
    assert otop == rtop
    np.testing.assert_array_equal(ost[:otop], rst[:rtop])
    # edge trace
    fn(None, "HafCpu_CannyEdgeTrace_U8_U8XY", [u32, u32, vp, u32, u32, vp, u32])(W, H, ro.ptr, ro.stride, W * H, rst.ctypes.data, rtop)
    fn(O.oracle_lib(), "oracle_CannyEdgeTrace_U8_U8XY", [u32, u32, vp, u32, u32, vp, u32])(W, H, oo.ptr, oo.stride, W * H, ost.ctypes.data, otop)
    np.testing.assert_array_equal(oo.get(), ro.get())


def harris_front(which, img, k=0.04, tc=1e-3):
    H, W = img.shape
    src = ago_img(H, W); src.set(img)
    hg3 = ago_img(H, W, np.float32, 3)
    hvc = ago_img(H, W, np.float32)
    lst = np.zeros(W * H, XYS)
    cnt = C.c_uint32(0)
    norm = fn(O.oracle_lib(), "oracle_harris_norm_factor", [i32])
    norm.restype = C.c_float
    nf = norm(3)
    if which == "ref":
        scratch = np.zeros(3 * 2 * 2 * ((W + 15) & ~15) + 64, np.int16)
        fn(None, "HafCpu_HarrisSobel_HG3_U8_3x3", [u32, u32, vp, u32, vp, u32, vp])(W, H, hg3.ptr, hg3.stride, src.ptr, src.stride, scratch.ctypes.data)
        fn(None, "HafCpu_HarrisScore_HVC_HG3_3x3", [u32, u32, vp, u32, vp, u32, f32, f32, f32])(W, H, hvc.ptr, hvc.stride, hg3.ptr, hg3.stride, k, tc, nf)
        fn(None, "HafCpu_NonMaxSupp_XY_ANY_3x3", [u32, vp, P, u32, u32, vp, u32])(W * H, lst.ctypes.data, C.byref(cnt), W, H, hvc.ptr, hvc.stride)
    else:
        o = O.oracle_lib()
        fn(o, "oracle_HarrisSobel_HG3_U8_3x3", [u32, u32, vp, u32, vp, u32])(W, H, hg3.ptr, hg3.stride, src.ptr, src.stride)
        fn(o, "oracle_HarrisScore_HVC_HG3_3x3", [u32, u32, vp, u32, vp, u32, f32, f32, f32])(W, H, hvc.ptr, hvc.stride, hg3.ptr, hg3.stride, k, tc, nf)
        fn(o, "oracle_NonMaxSupp_XY_ANY_3x3", [u32, vp, P, u32, u32, vp, u32])(W * H, lst.ctypes.data, C.byref(cnt), W, H, hvc.ptr, hvc.stride)
    return hg3, hvc, lst[:cnt.value].copy()


def ref_pick(lst, W, H, mind, cap):
    lst = lst.copy()
    out = np.zeros(max(cap, 1), KP)
    cnt = C.c_uint32(0)
    if mind > 2.0:
        cell = int(math.floor(mind / math.sqrt(2)))
        gw, gh = (W + cell - 1) // cell, (H + cell - 1) // cell
        hdr = np.array([gw, gh, cell, gw * gh * 4], np.uint32)
        grid = np.zeros(gw * gh * 2 + 8, np.int16)
        gi, gb = hdr.ctypes.data, grid.ctypes.data
    else:
        hdr = grid = None
        gi = gb = None
    fn(None, "HafCpu_HarrisMergeSortAndPick_XY_XYS", [u32, vp, P, vp, u32, f32, vp, vp])(
        cap, out.ctypes.data, C.byref(cnt), lst.ctypes.data, len(lst), mind, gi, gb)
    return out[:min(cnt.value, cap)], cnt.value


def oracle_pick(lst, W, H, mind, cap):
    lst = lst.copy()
    out = np.zeros(max(cap, 1), KP)
    cnt = C.c_uint32(0)
    fn(O.oracle_lib(), "oracle_HarrisMergeSortAndPick_XY_XYS", [u32, vp, P, vp, u32, f32, u32, u32])(
        cap, out.ctypes.data, C.byref(cnt), lst.ctypes.data, len(lst), mind, W, H)
    return out[:min(cnt.value, cap)], cnt.value


# Widths that are not a multiple of 4 are excluded: the reference then steps rows of its
# F32x3 buffer by floor(stride / 12) elements (ago_haf_cpu_harris.cpp:167 and :611) while the
# row-1 pointer uses the byte stride, so HarrisScore reads a misaligned layout.  The oracle and
# the GPU path implement the row layout the code intends.
@pytest.mark.parametrize("W,H", [(16, 8), (48, 20), (36, 19), (64, 64), (100, 41)])
def test_pin_harris(ref, W, H):
    img = scene(W, H, seed=3 * W + H)
    rg, rv, rl = harris_front("ref", img)
    og, ov, ol = harris_front("oracle", img)
    np.testing.assert_array_equal(og.get()[1:H - 1], rg.get()[1:H - 1])
    np.testing.assert_array_equal(ov.get(), rv.get())
    np.testing.assert_array_equal(ol, rl)
    for mind, cap in ((5.0, 10000), (5.0, 3), (1.5, 10000), (9.5, 7)):
        a, na = ref_pick(rl, W, H, mind, cap)
        b, nb = oracle_pick(ol, W, H, mind, cap)
        assert na == nb
        np.testing.assert_array_equal(a, b)


def test_pin_harris_pick_synthetic(ref):
    """Dense random candidates (many conflicts, ties on strength) on a 300x200 image."""
    rng = np.random.default_rng(5)
    n = 5000
    lst = np.zeros(n, XYS)
    lst["x"] = rng.integers(1, 299, n)
    lst["y"] = rng.integers(1, 199, n)
    lst["s"] = rng.integers(1, 50, n).astype(np.float32) / 7
    for mind, cap in ((5.0, 100000), (3.0, 50), (12.0, 100000)):
        a, na = ref_pick(lst, 300, 200, mind, cap)
        b, nb = oracle_pick(lst, 300, 200, mind, cap)
        assert na == nb
        np.testing.assert_array_equal(a, b)


CANNY_VARIANTS = [(3, 1), (5, 0), (5, 1), (7, 0), (7, 1)]


def canny_sobel_nxn(which, img, gsize, l2):
    """The packed Canny gradient of one window size / norm on an AGO-laid-out buffer."""
    H, W = img.shape
    src = ago_img(H, W); src.set(img)
    sob = ago_img(H, W, np.uint16)
    if which == "ref":
        local = np.zeros(((W + 15) & ~15) * 4 + 128, np.uint8)
        name = f"HafCpu_CannySobel_U16_U8_{gsize}x{gsize}_{'L2' if l2 else 'L1'}NORM"
        fn(None, name, [u32, u32, vp, u32, vp, u32, vp])(W, H, sob.ptr, sob.stride, src.ptr, src.stride, local.ctypes.data)
    else:
        fn(O.oracle_lib(), "oracle_CannySobel_U16_U8_NxN", [u32, u32, vp, u32, vp, u32, u32, u32])(
            W, H, sob.ptr, sob.stride, src.ptr, src.stride, gsize, l2)
    return sob.get()


@pytest.mark.parametrize("W,H", SHAPES + [(333, 47), (1920, 24)])
@pytest.mark.parametrize("gsize,l2", CANNY_VARIANTS)
def test_pin_canny_sobel_variants(ref, gsize, l2, W, H):
    """3x3 L2, 5x5 and 7x7 gradients: every written row [R, H-R) equals the reference,
    on textured scenes and on noise (which saturates the 7x7 sums)."""
    R = gsize // 2
    for img in (scene(W, H, seed=W * gsize + l2),
                np.random.default_rng(W + H + gsize).integers(0, 256, (H, W), dtype=np.int32).astype(np.uint8)):
        want = canny_sobel_nxn("ref", img, gsize, l2)
        got = canny_sobel_nxn("oracle", img, gsize, l2)
        np.testing.assert_array_equal(got[R:H - R], want[R:H - R])


@pytest.mark.parametrize("W,H", SHAPES)
def test_oracle_canny_nxn_matches_3x3_l1(W, H):
    """The generic restatement at 3x3 L1 reproduces the pinned 3x3 L1 one."""
    img = scene(W, H, seed=W)
    a = canny_sobel_nxn("oracle", img, 3, 0)
    b, _, _, _ = canny_front("oracle", img)
    np.testing.assert_array_equal(a[1:H - 1], b.get()[1:H - 1])
