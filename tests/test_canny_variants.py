"""vxCannyEdgeDetectorNode with 3x3 L2, 5x5 and 7x7 gradients (L1 and L2).

The node lowers as in the reference (agoDramaDivideCannyEdgeDetectorNode,
ago_drama_divide.cpp:1618): CannySobel_U16_U8_{N}x{N}_{L1,L2}NORM, then
CannySuppThreshold_U8XY_U16_3x3 -- the _7x7 variant for 7x7 gradients, which quarters both
thresholds (ago_kernel_api.cpp:18035) -- then CannyEdgeTrace.  The oracle chain is the C
restatement (oracle_CannySobel_U16_U8_NxN, pinned to the reference HAF kernels in
test_oracle_pin_vision.py) followed by the pinned suppression and trace.

CPU: the reference library's node equals the oracle chain inside the valid rectangle.
GPU: the gradient kernels equal the oracle plane, and the engine's graphs equal the oracle
chain."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from imgbuf import Img
from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL

u32, u16, vp = C.c_uint32, C.c_uint16, C.c_void_p
P32 = C.POINTER(C.c_uint32)
VARIANTS = [(3, "L2"), (5, "L1"), (5, "L2"), (7, "L1"), (7, "L2")]
# thresholds on each variant's magnitude scale (7x7: before the quartering)
THRESH = {3: (20, 40), 5: (600, 1200), 7: (3000, 6000)}


def ago_img(h, w, dtype=np.uint8):
    bpp = np.dtype(dtype).itemsize
    return Img(h, w, dtype, stride=((w * bpp + 15) // 16) * 16, pad=4, align_off=0)


def _f(name, args):
    f = getattr(O.oracle_lib(), name)
    f.argtypes, f.restype = args, C.c_int
    return f


def oracle_gradient(img, gs, l2):
    H, W = img.shape
    src = ago_img(H, W); src.set(img)
    sob = ago_img(H, W, np.uint16)
    _f("oracle_CannySobel_U16_U8_NxN", [u32, u32, vp, u32, vp, u32, u32, u32])(
        W, H, sob.ptr, sob.stride, src.ptr, src.stride, gs, int(l2))
    g = sob.get()
    R = gs // 2
    g[:R] = 0
    g[H - R:] = 0
    return g


def oracle_canny(img, gs, l2, lower, upper):
    """Edge map of the oracle chain."""
    H, W = img.shape
    g = oracle_gradient(img, gs, l2)
    if gs == 7:
        lower, upper = lower // 4, upper // 4
    sob = ago_img(H, W, np.uint16); sob.set(g)
    out = ago_img(H, W)
    stack = np.zeros(W * H, np.uint32)
    top = C.c_uint32(0)
    _f("oracle_CannySuppThreshold_U8XY_U16_3x3", [u32, vp, P32, u32, u32, vp, u32, vp, u32, u16, u16])(
        W * H, stack.ctypes.data, C.byref(top), W, H, out.ptr, out.stride, sob.ptr, sob.stride, lower, upper)
    _f("oracle_CannyEdgeTrace_U8_U8XY", [u32, u32, vp, u32, u32, vp, u32])(
        W, H, out.ptr, out.stride, W * H, stack.ctypes.data, top.value)
    return out.get()


def run_canny(api, img, gs, norm, lower, upper):
    H, W = img.shape
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        src = api.obj(api.vxCreateImage(ctx, W, H, V.VX_DF_IMAGE_U8), "image")
        api.write_plane(src, img)
        dst = api.obj(api.vxCreateImage(ctx, W, H, V.VX_DF_IMAGE_U8), "image")
        g = api.obj(api.vxCreateGraph(ctx), "graph")
        n = V.VX_NORM_L1 if norm == "L1" else V.VX_NORM_L2
        api.obj(api.vxCannyEdgeDetectorNode(g, src, api.threshold_range(ctx, lower, upper), gs, n, dst), "canny")
        api.ok(api.vxVerifyGraph(g), "verify")
        api.ok(api.vxProcessGraph(g), "process")
        return api.read_plane(dst), api.valid_region(dst)
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def _scene(W, H, seed):
    return WL.cfg2_scene(seed=seed, width=W, height=H, rects=max(2, W * H // 2000))


def _check(api, gs, norm, W, H):
    img = _scene(W, H, seed=W * gs + H)
    lo, hi = THRESH[gs]
    got, rect = run_canny(api, img, gs, norm, lo, hi)
    b = gs // 2 + 1
    assert rect == (b, b, W - b, H - b)
    want = oracle_canny(img, gs, norm == "L2", lo, hi)
    np.testing.assert_array_equal(got[b:H - b, b:W - b], want[b:H - b, b:W - b])
    assert (want[b:H - b, b:W - b] == 255).mean() > 0.002   # the case has edges


# W % 16 in [1, 13]: every read the reference makes outside a row lands on its zero padding
REF_SIZES = [(100, 60), (333, 97), (644, 360)]


@pytest.mark.parametrize("W,H", REF_SIZES)
@pytest.mark.parametrize("gs,norm", VARIANTS)
def test_reference_canny_variants(gs, norm, W, H):
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    _check(V.OpenVX(lib), gs, norm, W, H)


@pytest.fixture(scope="module")
def agocuda():
    from mivisionx_b200 import native
    return native.agocuda()


@pytest.mark.gpu
@pytest.mark.parametrize("W,H", [(100, 60), (333, 97), (3840, 2160), (64, 48), (37, 21)])
@pytest.mark.parametrize("gs,norm", VARIANTS)
def test_engine_gradient_kernels(cuda, agocuda, gs, norm, W, H):
    """The agocuda_CannySobel_* kernels on a device plane with a pitch of its own equal the
    oracle's gradient of the AGO-laid-out image, every row (rows outside [R, H-R) are 0)."""
    from devbuf import DevImg, stream_ptr
    img = np.random.default_rng(W + gs).integers(0, 256, (H, W), dtype=np.int32).astype(np.uint8)
    if W > 1000:
        img = _scene(W, H, seed=gs)
    src = DevImg(H, W, stride=W + 48).upload(img)
    dst = DevImg(H, W, np.uint16)
    f = getattr(agocuda, f"agocuda_CannySobel_U16_U8_{gs}x{gs}_{norm}NORM")
    f.argtypes, f.restype = [vp, u32, u32, vp, u32, vp, u32], C.c_int
    assert f(stream_ptr(), W, H, dst.ptr, dst.stride, src.ptr, src.stride) == 0
    np.testing.assert_array_equal(dst.download(), oracle_gradient(img, gs, norm == "L2"))


@pytest.mark.gpu
@pytest.mark.parametrize("W,H", [(100, 60), (333, 97), (644, 360), (3840, 2160)])
@pytest.mark.parametrize("gs,norm", VARIANTS)
def test_engine_canny_variants(cuda, gs, norm, W, H):
    """The engine's graph (gradient, suppression -- quartered thresholds for 7x7 -- and the
    device hysteresis) equals the oracle chain inside the reference's valid rectangle."""
    _check(V.OpenVX(), gs, norm, W, H)


@pytest.mark.gpu
def test_engine_canny_variants_share_a_context(cuda):
    """All variants as graphs of one context, run twice, released one by one and then with
    the context: every graph's teardown leaves the others and the context intact."""
    api = V.OpenVX()
    W, H = 333, 97
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        img = _scene(W, H, seed=5)
        src = api.obj(api.vxCreateImage(ctx, W, H, V.VX_DF_IMAGE_U8), "image")
        api.write_plane(src, img)
        graphs = []
        for gs, norm in VARIANTS:
            dst = api.obj(api.vxCreateImage(ctx, W, H, V.VX_DF_IMAGE_U8), "image")
            g = api.obj(api.vxCreateGraph(ctx), "graph")
            lo, hi = THRESH[gs]
            n = V.VX_NORM_L1 if norm == "L1" else V.VX_NORM_L2
            api.obj(api.vxCannyEdgeDetectorNode(g, src, api.threshold_range(ctx, lo, hi), gs, n, dst), "canny")
            api.ok(api.vxVerifyGraph(g), "verify")
            graphs.append((g, dst, gs, norm, lo, hi))
        for _ in range(2):
            for g, dst, gs, norm, lo, hi in graphs:
                api.ok(api.vxProcessGraph(g), "process")
                b = gs // 2 + 1
                want = oracle_canny(img, gs, norm == "L2", lo, hi)
                np.testing.assert_array_equal(api.read_plane(dst)[b:H - b, b:W - b], want[b:H - b, b:W - b])
        for g, *_ in graphs[::2]:
            api.ok(api.vxReleaseGraph(C.byref(C.c_void_p(g))), "release graph")
        for g, dst, gs, norm, lo, hi in graphs[1::2]:
            api.ok(api.vxProcessGraph(g), "process after other graphs were released")
    finally:
        assert api.vxReleaseContext(C.byref(C.c_void_p(ctx))) == 0
