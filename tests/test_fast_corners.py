"""vxFastCornersNode (FAST-9, with and without non-maximum suppression).

The node lowers as in the reference (agoDramaDivideFastCornersNode,
ago_drama_divide.cpp:1789) to FastCorners_XY_U8_Supression or _NoSupression; the oracle is
the C restatement pinned to the reference's HafCpu_FastCorners_* in test_oracle_pin_fast.py.

CPU: the reference library's node equals the oracle (list order, fields and count).
GPU: agocuda_FastCorners_XY_U8 equals the oracle on AGO-laid-out images, the capacity cut-off
included, and the engine's graph equals it."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import oracle_chains as OC
from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL

u32, f32, vp, i32, sz = C.c_uint32, C.c_float, C.c_void_p, C.c_int32, C.c_size_t
P32 = C.POINTER(C.c_uint32)


def oracle_fast(img, thr, suppress, capacity):
    H, W = img.shape
    src = OC.ago_img(H, W); src.set(img)
    kp = np.zeros(max(capacity, 1), OC.KP)
    n = C.c_uint32(0)
    f = getattr(O.oracle_lib(), f"oracle_FastCorners_XY_U8_{'Supression' if suppress else 'NoSupression'}")
    f.argtypes, f.restype = [u32, vp, P32, u32, u32, vp, u32, f32], C.c_int
    f(capacity, kp.ctypes.data, C.byref(n), W, H, src.ptr, src.stride, thr)
    return kp[:min(n.value, capacity)], n.value


def run_graph(api, img, thr, suppress, capacity):
    H, W = img.shape
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        src = api.obj(api.vxCreateImage(ctx, W, H, V.VX_DF_IMAGE_U8), "image")
        api.write_plane(src, img)
        arr = api.obj(api.vxCreateArray(ctx, V.VX_TYPE_KEYPOINT, capacity), "array")
        num = api.scalar(ctx, V.VX_TYPE_SIZE, 0)
        g = api.obj(api.vxCreateGraph(ctx), "graph")
        api.obj(api.vxFastCornersNode(g, src, api.scalar(ctx, V.VX_TYPE_FLOAT32, thr), int(suppress), arr, num), "fast")
        api.ok(api.vxVerifyGraph(g), "verify")
        res = []
        for _ in range(2):           # a second execution must not see the first one's corners
            api.ok(api.vxProcessGraph(g), "process")
            res.append((api.array_items(arr).view(OC.KP), api.read_scalar(num)))
        return res
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def _image(kind, W, H, seed):
    if kind == "noise":
        return np.random.default_rng(seed).integers(0, 256, (H, W), dtype=np.int32).astype(np.uint8)
    return WL.cfg2_scene(seed=seed, width=W, height=H, rects=max(4, W * H // 300))


def _check(api, kind, W, H, thr, suppress, capacity=1 << 16):
    img = _image(kind, W, H, W * 3 + H)
    want, want_n = oracle_fast(img, thr, suppress, capacity)
    assert want_n > 0
    for got, n in run_graph(api, img, thr, suppress, capacity):
        assert n == want_n
        np.testing.assert_array_equal(got, want)


# W % 16 in [1, 13]: the circle reads across the row ends land on the row padding, which both
# libraries hold at zero
REF_SIZES = [(100, 60), (333, 97), (644, 360)]


@pytest.mark.parametrize("W,H", REF_SIZES)
@pytest.mark.parametrize("suppress", [False, True])
@pytest.mark.parametrize("kind,thr", [("scene", 20.0), ("noise", 40.5)])
def test_reference_fast_graph(kind, thr, suppress, W, H):
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    _check(V.OpenVX(lib), kind, W, H, thr, suppress)


@pytest.fixture(scope="module")
def agocuda():
    from mivisionx_b200 import native
    L = native.agocuda()
    L.agocuda_FastCorners_scratch_size.argtypes, L.agocuda_FastCorners_scratch_size.restype = [u32, u32], sz
    L.agocuda_FastCorners_XY_U8.argtypes = [vp, u32, u32, vp, u32, f32, i32, vp, u32, vp, vp, vp, sz]
    L.agocuda_FastCorners_XY_U8.restype = C.c_int
    return L


def _kernel(L, img, thr, suppress, capacity, stride_pad=48):
    import torch
    from devbuf import DevImg, stream_ptr
    H, W = img.shape
    src = DevImg(H, W, stride=((W + stride_pad + 3) // 4) * 4).upload(img)
    nb = L.agocuda_FastCorners_scratch_size(W, H)
    scratch = torch.full((nb + 256,), 0xA5, dtype=torch.uint8, device="cuda")   # no zeroing needed
    sp = scratch.data_ptr() + (-scratch.data_ptr() % 256)
    out = torch.zeros(max(capacity, 1) * 28 + 28, dtype=torch.uint8, device="cuda")
    cnt = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = L.agocuda_FastCorners_XY_U8(stream_ptr(), W, H, src.ptr, src.stride, thr, int(suppress), out.data_ptr(),
                                     capacity, cnt.data_ptr(), cnt.data_ptr() + 4, sp, nb)
    assert rc == 0
    torch.cuda.synchronize()
    c = cnt.cpu().numpy().view(np.uint32)
    kp = out.cpu().numpy()[:28 * max(capacity, 1)].view(OC.KP)
    return kp[:c[0]], c[0], c[1]


@pytest.mark.gpu
@pytest.mark.parametrize("W,H", [(64, 48), (100, 60), (333, 97), (37, 21), (7, 7), (1920, 1080), (3840, 2160)])
@pytest.mark.parametrize("suppress", [False, True])
@pytest.mark.parametrize("kind,thr", [("scene", 20.0), ("noise", 40.5), ("noise", 10.0)])
def test_fast_kernel(cuda, agocuda, kind, thr, suppress, W, H):
    """Every image edge case: widths with W % 16 == 0 (reads across the row end reach the next
    row's pixels), narrow and tiny images, and full-size frames."""
    img = _image(kind, W, H, W + H)
    cap = 1 << 21
    want, want_n = oracle_fast(img, thr, suppress, cap)
    got, n_items, n = _kernel(agocuda, img, thr, suppress, cap)
    assert n == want_n and n_items == min(want_n, cap)
    np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("suppress", [False, True])
@pytest.mark.parametrize("cap", [0, 1, 1000, 12345])
def test_fast_kernel_capacity(cuda, agocuda, suppress, cap):
    img = _image("noise", 640, 480, 9)
    want, want_n = oracle_fast(img, 12.0, suppress, max(cap, 1))
    got, n_items, n = _kernel(agocuda, img, 12.0, suppress, cap)
    assert want_n > 12345
    assert n == want_n and n_items == min(want_n, cap)
    np.testing.assert_array_equal(got, want[:cap])


@pytest.mark.gpu
def test_fast_kernel_rejects_bad_arguments(cuda, agocuda):
    from devbuf import stream_ptr
    L = agocuda
    assert L.agocuda_FastCorners_XY_U8(stream_ptr(), 6, 10, 1 << 12, 64, 20.0, 1, 1 << 12, 10, None, None, 1 << 12,
                                       1 << 20) != 0
    assert L.agocuda_FastCorners_XY_U8(stream_ptr(), 64, 10, 1 << 12, 64, 20.0, 1, 1 << 12, 10, None, None, None, 0) != 0
    assert L.agocuda_FastCorners_XY_U8(stream_ptr(), 64, 10, 1 << 12, 64, 20.0, 1, 1 << 12, 10, None, None, 1 << 12,
                                       16) != 0          # scratch too small


@pytest.mark.gpu
@pytest.mark.parametrize("W,H", [(100, 60), (333, 97), (1920, 1080)])
@pytest.mark.parametrize("suppress", [False, True])
@pytest.mark.parametrize("kind,thr", [("scene", 20.0), ("noise", 40.5)])
def test_engine_fast_graph(cuda, kind, thr, suppress, W, H):
    _check(V.OpenVX(), kind, W, H, thr, suppress, capacity=1 << 18)
