"""The allocation-free hysteresis (agocuda_CannyEdgeTrace_U8_U8XY_noalloc) must produce
exactly what the regular entry point produces with caller-allocated scratch, on calls in a
row of different sizes and content (its fixed scratch array is shared by every call and keeps
the previous call's contents), and must refuse images above its size limit without launching.

This file is collected last on purpose so a stop-at-first-failure run has already run every
other test; it also passes on its own in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from mivisionx_b200 import workloads as WL

pytestmark = pytest.mark.gpu

u32, vp, u16, sz = C.c_uint32, C.c_void_p, C.c_uint16, C.c_size_t


@pytest.fixture(scope="module")
def lib(cuda):
    from mivisionx_b200 import native
    L = native.agocuda()
    sigs = {
        "agocuda_CannySobel_U16_U8_3x3_L1NORM": [vp, u32, u32, vp, u32, vp, u32],
        "agocuda_CannySuppThreshold_U8XY_U16_3x3": [vp, u32, u32, vp, u32, vp, u32, vp, vp, u32, u16, u16],
        "agocuda_CannyEdgeTrace_U8_U8XY": [vp, u32, u32, vp, u32, vp, vp, u32, vp, sz, vp],
        "agocuda_CannyEdgeTrace_U8_U8XY_noalloc": [vp, u32, u32, vp, u32, vp, vp, u32, vp],
    }
    for n, a in sigs.items():
        getattr(L, n).argtypes = a
        getattr(L, n).restype = C.c_int
    L.agocuda_CannyEdgeTrace_scratch_size.argtypes = [u32, u32]
    L.agocuda_CannyEdgeTrace_scratch_size.restype = C.c_size_t
    L.agocuda_CannyEdgeTrace_noalloc_max_pixels.argtypes = []
    L.agocuda_CannyEdgeTrace_noalloc_max_pixels.restype = C.c_size_t
    return L


def _suppressed_map(lib, img):
    """Gradient + suppression on the device: the 0/127/255 map and the strong-pixel stack."""
    import torch

    from devbuf import DevImg, stream_ptr
    H, W = img.shape
    src, sob, out = DevImg(H, W).upload(img), DevImg(H, W, np.uint16), DevImg(H, W)
    stack = torch.zeros(4 * W * H, dtype=torch.uint8, device="cuda")
    cnt = torch.zeros(16, dtype=torch.uint8, device="cuda")
    assert lib.agocuda_CannySobel_U16_U8_3x3_L1NORM(stream_ptr(), W, H, sob.ptr, sob.stride, src.ptr, src.stride) == 0
    assert lib.agocuda_CannySuppThreshold_U8XY_U16_3x3(stream_ptr(), W, H, out.ptr, out.stride, sob.ptr, sob.stride,
                                                       stack.data_ptr(), cnt.data_ptr(), W * H, 80, 100) == 0
    torch.cuda.synchronize()
    return out, stack, cnt


def _copy(img_dev):
    from devbuf import DevImg
    d = DevImg(img_dev.h, img_dev.w)
    d.t.copy_(img_dev.t)
    d.off = img_dev.off
    return d


def _allocating_trace(lib, supp, stack, cnt, W, H):
    """The regular entry point, scratch allocated by the caller: the expected result."""
    import torch

    from devbuf import stream_ptr
    ref = _copy(supp)
    sb = lib.agocuda_CannyEdgeTrace_scratch_size(W, H)
    scratch = torch.zeros(sb + 256, dtype=torch.uint8, device="cuda")
    base = scratch.data_ptr() + (-scratch.data_ptr() % 256)
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    assert lib.agocuda_CannyEdgeTrace_U8_U8XY(stream_ptr(), W, H, ref.ptr, ref.stride, stack.data_ptr(), cnt.data_ptr(),
                                              W * H, base, sb, status.data_ptr()) == 0
    assert int(status[0].item()) == 0
    return ref.download()


def test_noalloc_edge_trace_matches_allocating_entry_point(lib):
    """Calls in a row with different sizes and content: a large image fills most of the
    shared array, the smaller one after it must not see any of those labels or root bits,
    and the third call repeats the first on the array the second left behind."""
    import torch

    from devbuf import stream_ptr
    calls = [(1920, 1080, 11), (640, 480, 29), (1920, 1080, 11)]
    for i, (W, H, seed) in enumerate(calls):
        img = WL.cfg2_scene(seed=seed, width=W, height=H, rects=min(200, W * H // 3000))
        supp, stack, cnt = _suppressed_map(lib, img)
        expected = _allocating_trace(lib, supp, stack, cnt, W, H)
        got = _copy(supp)
        st = torch.zeros(4, dtype=torch.int32, device="cuda")
        assert lib.agocuda_CannyEdgeTrace_U8_U8XY_noalloc(stream_ptr(), W, H, got.ptr, got.stride, stack.data_ptr(),
                                                          cnt.data_ptr(), W * H, st.data_ptr()) == 0
        np.testing.assert_array_equal(got.download(), expected, err_msg=f"call {i} ({W}x{H})")
        assert int(st[0].item()) == 0


def test_noalloc_rejects_images_above_its_limit(lib):
    import torch

    from devbuf import stream_ptr
    limit = lib.agocuda_CannyEdgeTrace_noalloc_max_pixels()
    assert limit == 1 << 21
    W, H = 2048, 1025                         # W*H just above the limit
    buf = torch.zeros(16, dtype=torch.uint8, device="cuda")
    p = buf.data_ptr()
    assert lib.agocuda_CannyEdgeTrace_U8_U8XY_noalloc(stream_ptr(), W, H, p, W, p, p, 1, p) == -15
