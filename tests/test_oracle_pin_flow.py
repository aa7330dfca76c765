"""Pin the pyramid-level and pyramidal-LK restatements (oracle/agooracle_flow.c) to the
reference HAF CPU kernels built from the reference sources.

ScaleGaussianHalf reads two pixels outside each row, so both run on AGO-layout buffers
(16-byte row pitch, zero padding).  LK is called twice in a row on one persistent node
scratch, as a graph node is across executions: the reference's Scharr pass reads scratch
words that earlier levels and earlier calls left behind, and the restatement must agree on
those too."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from imgbuf import Img
from mivisionx_b200 import workloads as WL

u32, i32, vp, f32, cbool = C.c_uint32, C.c_int32, C.c_void_p, C.c_float, C.c_bool
KP = WL.KEYPOINT_DTYPE
TERM_ITER, TERM_EPS, TERM_BOTH = 0xF000, 0xF001, 0xF002   # VX_TERM_CRITERIA_*


class PyrLevel(C.Structure):
    """ago_pyramid_u8_t (ago/ago_haf_cpu.h:75)."""
    _fields_ = [("width", u32), ("height", u32), ("stride", u32), ("image", vp), ("computed", i32)]


def ago_img(h, w):
    return Img(h, w, np.uint8, stride=((w + 15) // 16) * 16, pad=4, align_off=0)


def half_level(impl, src: Img, dst: Img):
    """One ScaleGaussianHalf level as agoKernel_ScaleGaussianHalf_U8_U8_5x5 calls it
    (ago_kernel_api.cpp:15420): destination rows 1..H-2, source from row 2."""
    first_row, first_col = bool(src.h & 1), bool(src.w & 1)
    args = (dst.w, dst.h - 2, dst.row_ptr(1), dst.stride, src.row_ptr(2), src.stride, first_row, first_col)
    if impl == "ref":
        f = O.ref_haf("HafCpu_ScaleGaussianHalf_U8_U8_5x5")
        f.argtypes = [u32, u32, vp, u32, vp, u32, cbool, cbool, vp]
        f.restype = C.c_int
        scratch = np.zeros(20 * ((dst.stride + 15) & ~15) + 64, np.uint8)
        assert f(*args, scratch.ctypes.data) == 0
    else:
        f = O.oracle_lib().oracle_ScaleGaussianHalf_U8_U8_5x5
        f.argtypes = [u32, u32, vp, u32, vp, u32, C.c_int, C.c_int]
        f.restype = C.c_int
        assert f(*args) == 0


@pytest.mark.parametrize("W,H", [(37, 19), (64, 48), (100, 41), (129, 67), (241, 135), (640, 480)])
def test_scale_gaussian_half_matches_reference(ref, W, H):
    rng = np.random.default_rng(W * 7 + H)
    src = ago_img(H, W)
    src.set(rng.integers(0, 256, (H, W), dtype=np.uint8))
    oW, oH = (W + 1) >> 1, (H + 1) >> 1
    outs = {}
    for impl in ("ref", "oracle"):
        dst = ago_img(oH, oW)
        half_level(impl, src, dst)
        outs[impl] = dst.get()
    np.testing.assert_array_equal(outs["oracle"], outs["ref"])
    assert not outs["ref"][0].any() and not outs["ref"][-1].any()   # rows 0 and H-1 are not written


def build_pyramid(img: np.ndarray, levels: int):
    """Level 0 is a copy of the frame; higher levels come from the restatement (pinned above)."""
    H, W = img.shape
    lv = [ago_img(H, W)]
    lv[0].set(img)
    for (w, h) in WL.pyramid_sizes(W, H, levels)[1:]:
        d = ago_img(h, w)
        half_level("oracle", lv[-1], d)
        lv.append(d)
    desc = (PyrLevel * levels)(*[PyrLevel(l.w, l.h, l.stride, l.ptr, 1) for l in lv])
    return lv, desc


def lk_call(impl, new_kp, old_pyr, new_pyr, levels, old_kp, est_kp, term, eps, iters, use_est, W0, scratch, win):
    args = (new_kp.ctypes.data, 0.5, levels, C.cast(old_pyr, vp), C.cast(new_pyr, vp), len(old_kp), old_kp.ctypes.data,
            est_kp.ctypes.data, term, eps, iters, use_est, W0 * 4, scratch.ctypes.data, win)
    types = [vp, f32, u32, vp, vp, u32, vp, vp, i32, f32, u32, i32, u32, vp, i32]
    if impl == "ref":
        f = O.ref_haf("HafCpu_OpticalFlowPyrLK_XY_XY_Generic")
    else:
        f = O.oracle_lib().oracle_OpticalFlowPyrLK_XY_XY
    f.argtypes = types
    f.restype = C.c_int
    assert f(*args) == 0


def lk_scratch(W0, H0, cap):
    n = O.oracle_lib().oracle_OpticalFlowPyrLK_scratch_size
    n.argtypes, n.restype = [u32, u32, u32], C.c_size_t
    raw = np.zeros(int(n(W0, H0, cap)) + 64, np.uint8)
    off = (-raw.ctypes.data) % 32          # agoAllocMemory returns 32-byte aligned memory
    return raw[off:off + int(n(W0, H0, cap))]


def points(seed, W, H, n, lost_every=0):
    kp = WL.cfg4_points(seed, W, H, n)
    if lost_every:
        kp["tracking_status"][::lost_every] = 0
    kp["strength"] = np.arange(n, dtype=np.float32)
    return kp


CASES = [
    # W, H, levels, window, termination, epsilon, iterations, use_initial_estimate
    (160, 120, 5, 9, TERM_BOTH, 0.01, 20, 0),
    (320, 240, 4, 9, TERM_ITER, 0.01, 10, 1),
    (250, 170, 3, 7, TERM_BOTH, 0.01, 20, 0),      # level widths 250, 125, 63: W % 8 in {2, 5, 7}
    (200, 100, 3, 8, TERM_BOTH, 0.001, 15, 0),     # even window: 8-lane group and no scalar tail
    (128, 96, 3, 15, TERM_BOTH, 0.01, 20, 1),
    (96, 80, 2, 3, TERM_ITER, 0.01, 5, 0),
    (144, 112, 3, 4, TERM_BOTH, 0.5, 20, 0),
    (176, 136, 4, 11, TERM_BOTH, 0.0001, 30, 0),
]


@pytest.mark.parametrize("W,H,levels,win,term,eps,iters,use_est", CASES)
def test_lk_matches_reference_across_two_calls(ref, W, H, levels, win, term, eps, iters, use_est):
    n = 600
    scratch = {impl: lk_scratch(W, H, n) for impl in ("ref", "oracle")}
    for call in range(2):                                   # same node scratch, two frames
        f1, f2, (dx, dy) = WL.cfg4_pair(seed=100 * W + H + call, width=W, height=H, max_shift=3.0)
        old_lv, old_desc = build_pyramid(f1, levels)
        new_lv, new_desc = build_pyramid(f2, levels)
        old_kp = points(W + H + call, W, H, n, lost_every=17)
        est_kp = old_kp.copy()
        est_kp["x"] = np.clip(old_kp["x"] + int(round(dx)), 0, W - 1)
        est_kp["y"] = np.clip(old_kp["y"] + int(round(dy)), 0, H - 1)
        est_kp["tracking_status"][5::23] = 0
        est_kp["strength"] += 1000
        out = {}
        for impl in ("ref", "oracle"):
            kp = np.zeros(n, KP)
            kp.view(np.uint8)[:] = 0xA5                     # fields the kernel leaves alone stay visible
            lk_call(impl, kp, old_desc, new_desc, levels, old_kp, est_kp, term, eps, iters, use_est, W,
                    scratch[impl], win)
            out[impl] = kp
        assert out["oracle"].tobytes() == out["ref"].tobytes(), (
            f"call {call}: {np.count_nonzero(out['oracle'] != out['ref'])} keypoints differ")
        tracked = out["ref"]["tracking_status"] != 0
        assert tracked.sum() > n // 3                         # the case exercises real tracking
