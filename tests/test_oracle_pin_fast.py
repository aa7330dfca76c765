"""Pin the FAST-9 restatement (oracle_FastCorners_XY_U8_{NoSupression,Supression}) to the
reference's HafCpu_FastCorners_XY_U8_NoSupression / _Supression
(ago_haf_cpu_fast_corners.cpp:414, :599), built from its own sources, on AGO-laid-out
buffers: the keypoint lists (order, coordinates, strengths and the other fields) and the
counts, including the capacity cut-off.  The reference's SIMD body and scalar tail both run
(widths with W % 8 and (W - 6) % 8 non-zero)."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import oracle_chains as OC
from mivisionx_b200 import workloads as WL

u32, f32, vp = C.c_uint32, C.c_float, C.c_void_p
P32 = C.POINTER(C.c_uint32)


def _ref(name, extra=()):
    f = O.ref_haf(name)
    f.argtypes, f.restype = [u32, vp, P32, u32, u32, vp, u32, f32] + list(extra), C.c_int
    return f


def _orc(name):
    f = getattr(O.oracle_lib(), name)
    f.argtypes, f.restype = [u32, vp, P32, u32, u32, vp, u32, f32], C.c_int
    return f


def _images(W, H, seed):
    rng = np.random.default_rng(seed)
    noise = rng.integers(0, 256, (H, W), dtype=np.int32).astype(np.uint8)
    scene = WL.cfg2_scene(seed=seed, width=W, height=H, rects=max(4, W * H // 200))
    return {"noise": noise, "scene": scene}


def run_both(img, thr, suppress, capacity):
    H, W = img.shape
    src = OC.ago_img(H, W); src.set(img)
    out = []
    for which in ("oracle", "ref"):
        kp = np.zeros(max(capacity, 1), OC.KP)
        n = C.c_uint32(0)
        if which == "oracle":
            _orc(f"oracle_FastCorners_XY_U8_{'Supression' if suppress else 'NoSupression'}")(
                capacity, kp.ctypes.data, C.byref(n), W, H, src.ptr, src.stride, thr)
        elif suppress:
            scratch = np.zeros(W * H + 64, np.uint8)
            _ref("HafCpu_FastCorners_XY_U8_Supression", [vp])(capacity, kp.ctypes.data, C.byref(n), W, H, src.ptr,
                                                              src.stride, thr, scratch.ctypes.data)
        else:
            _ref("HafCpu_FastCorners_XY_U8_NoSupression")(capacity, kp.ctypes.data, C.byref(n), W, H, src.ptr,
                                                           src.stride, thr)
        out.append((kp[:min(n.value, capacity)], n.value))
    return out


@pytest.mark.parametrize("suppress", [False, True])
@pytest.mark.parametrize("thr", [10.0, 25.7, 60.0])
@pytest.mark.parametrize("W,H", [(64, 20), (75, 33), (128, 48), (201, 17)])
def test_pin_fast(ref, suppress, thr, W, H):
    for kind, img in _images(W, H, W * 7 + H).items():
        (a, na), (b, nb) = run_both(img, thr, suppress, capacity=1 << 16)
        assert na == nb, (kind, na, nb)
        np.testing.assert_array_equal(a, b)
        if kind == "noise" and thr < 30:
            assert na > 0


@pytest.mark.parametrize("suppress", [False, True])
def test_pin_fast_capacity(ref, suppress):
    img = _images(96, 40, 3)["noise"]
    (a, na), (b, nb) = run_both(img, 12.0, suppress, capacity=17)
    assert na == nb and na > 17
    np.testing.assert_array_equal(a, b)


def test_pin_fast_full_size_scene(ref):
    """A 1920x1080 scene, suppression on and off."""
    img = WL.cfg2_scene(seed=11, width=1920, height=1080, rects=4000)
    for suppress in (False, True):
        (a, na), (b, nb) = run_both(img, 20.0, suppress, capacity=1 << 18)
        assert na == nb and na > 100
        np.testing.assert_array_equal(a, b)
