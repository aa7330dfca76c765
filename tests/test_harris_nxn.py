"""vxHarrisCornersNode with 5x5 / 7x7 gradients and 5x5 / 7x7 blocks.

The node lowers as in the reference (agoDramaDivideHarrisCornersNode,
ago_drama_divide.cpp:1670): HarrisSobel_HG3_U8_{gs}x{gs}, HarrisScore_HVC_HG3_{bs}x{bs}
normalised by (255 * 2^(gs-1) * bs)^4 (ago_kernel_api.cpp:16941, :17012, :17083),
NonMaxSupp_XY_ANY_3x3 and HarrisMergeSortAndPick_XY_XYS.  The oracle chain is the C
restatement pinned to the reference HAF kernels in test_oracle_pin_harris_nxn.py.

CPU: the reference library's node equals the oracle chain (corners and count).
GPU: the gradient and score kernels equal the oracle planes, and the engine's graphs equal
the oracle chain."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import oracle_chains as OC
from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL

u32, f32, vp = C.c_uint32, C.c_float, C.c_void_p
PAIRS = [(5, 3), (7, 3), (3, 5), (5, 5), (3, 7), (5, 7), (7, 5), (7, 7)]
# strength thresholds on each gradient size's normalised score scale
TC = {3: 1e-7, 5: 1e-6, 7: 1e-6}


def run_harris(api, img, gs, bs, tc, k=0.04, min_distance=5.0, capacity=32768):
    H, W = img.shape
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        src = api.obj(api.vxCreateImage(ctx, W, H, V.VX_DF_IMAGE_U8), "image")
        api.write_plane(src, img)
        arr = api.obj(api.vxCreateArray(ctx, V.VX_TYPE_KEYPOINT, capacity), "array")
        num = api.scalar(ctx, V.VX_TYPE_SIZE, 0)
        g = api.obj(api.vxCreateGraph(ctx), "graph")
        api.obj(api.vxHarrisCornersNode(g, src, api.scalar(ctx, V.VX_TYPE_FLOAT32, tc),
                                        api.scalar(ctx, V.VX_TYPE_FLOAT32, min_distance),
                                        api.scalar(ctx, V.VX_TYPE_FLOAT32, k), gs, bs, arr, num), "harris")
        api.ok(api.vxVerifyGraph(g), "verify")
        api.ok(api.vxProcessGraph(g), "process")
        return api.array_items(arr).view(OC.KP), api.read_scalar(num)
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def _scene(W, H, seed):
    return WL.cfg2_scene(seed=seed, width=W, height=H, rects=max(4, W * H // 300))


def _check(api, gs, bs, W, H, capacity=32768):
    img = _scene(W, H, seed=W * gs + H * bs)
    got, num = run_harris(api, img, gs, bs, TC[gs], capacity=capacity)
    want, want_num = OC.harris(img, tc=TC[gs], capacity=capacity, gs=gs, bs=bs)
    assert want_num > 20          # the case has corners
    assert num == want_num
    np.testing.assert_array_equal(got, want)


# W % 4 == 0: the reference's gradient rows are then packed at its 12 W-byte pitch
REF_SIZES = [(100, 60), (332, 97), (644, 360)]


@pytest.mark.parametrize("W,H", REF_SIZES)
@pytest.mark.parametrize("gs,bs", PAIRS)
def test_reference_harris_variants(gs, bs, W, H):
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    _check(V.OpenVX(lib), gs, bs, W, H)


def test_oracle_norm_matches_wrapper_order():
    """(255 * 2^(gs-1) * bs)^4 evaluated left to right in float, as the AGO wrappers do."""
    for gs in (3, 5, 7):
        for bs in (3, 5, 7):
            f = np.float32(255.0) * np.float32(1 << (gs - 1)) * np.float32(bs)
            want = ((f * f) * f) * f
            assert np.float32(OC.harris_norm_block(gs, bs)) == want
    assert OC.harris_norm_block(3, 3) == OC.harris_norm(3)


@pytest.fixture(scope="module")
def agocuda():
    from mivisionx_b200 import native
    return native.agocuda()


def _oracle_gradient(img, gs):
    H, W = img.shape
    src = OC.ago_img(H, W); src.set(img)
    g = OC.ago_img(H, W, np.float32, 3)
    OC.fn("HarrisSobel_HG3_U8_NxN")(W, H, g.ptr, g.stride, src.ptr, src.stride, gs)
    return g.get()


@pytest.mark.gpu
@pytest.mark.parametrize("W,H", [(100, 60), (333, 97), (64, 48), (37, 21), (1920, 1080)])
@pytest.mark.parametrize("gs", [5, 7])
def test_engine_gradient_kernels(cuda, agocuda, gs, W, H):
    """agocuda_HarrisSobel_HG3_U8_NxN on a device plane with a pitch of its own equals the
    oracle's gradient products of the AGO-laid-out image on every row (rows outside
    [R, H-R) are 0), including the columns whose taps leave the row."""
    from devbuf import DevImg, stream_ptr
    img = np.random.default_rng(W + gs).integers(0, 256, (H, W), dtype=np.int32).astype(np.uint8)
    src = DevImg(H, W, stride=W + 48).upload(img)
    dst = DevImg(H, W, np.float32, channels=3)
    f = agocuda.agocuda_HarrisSobel_HG3_U8_NxN
    f.argtypes, f.restype = [vp, u32, u32, vp, u32, vp, u32, u32], C.c_int
    assert f(stream_ptr(), W, H, dst.ptr, dst.stride, src.ptr, src.stride, gs) == 0
    np.testing.assert_array_equal(dst.download(), _oracle_gradient(img, gs))


@pytest.mark.gpu
@pytest.mark.parametrize("W,H", [(100, 60), (333, 97), (1920, 1080)])
@pytest.mark.parametrize("bs", [5, 7])
def test_engine_score_kernels(cuda, agocuda, bs, W, H):
    """agocuda_HarrisScore_HVC_HG3_NxN equals the oracle score on every pixel (the 7x7 block's
    one-column shift included), for large integer-valued products where float rounding of the
    window sums decides the result."""
    from devbuf import DevImg, stream_ptr
    rng = np.random.default_rng(W * bs)
    gv = (rng.integers(0, 1 << 20, (H, W, 3)).astype(np.float32) * np.float32(37.0))
    norm = OC.harris_norm_block(5, bs)
    g = OC.ago_img(H, W, np.float32, 3); g.set(gv)
    want = OC.ago_img(H, W, np.float32)
    OC.fn("HarrisScore_HVC_HG3_NxN")(W, H, want.ptr, want.stride, g.ptr, g.stride, 0.04, 1e-9, norm, bs)
    src = DevImg(H, W, np.float32, channels=3).upload(gv)
    dst = DevImg(H, W, np.float32)
    f = agocuda.agocuda_HarrisScore_HVC_HG3_NxN
    f.argtypes, f.restype = [vp, u32, u32, vp, u32, vp, u32, f32, f32, f32, u32], C.c_int
    assert f(stream_ptr(), W, H, dst.ptr, dst.stride, src.ptr, src.stride, 0.04, 1e-9, norm, bs) == 0
    out = dst.download()
    np.testing.assert_array_equal(out, want.get())
    assert (out > 0).mean() > 0.01


@pytest.mark.gpu
@pytest.mark.parametrize("W,H", [(100, 60), (333, 97), (644, 360), (1920, 1080)])
@pytest.mark.parametrize("gs,bs", PAIRS)
def test_engine_harris_variants(cuda, gs, bs, W, H):
    """The engine's graph (gradient, score, suppression, device pick) equals the oracle chain:
    the same corners in the same order and the same count."""
    _check(V.OpenVX(), gs, bs, W, H)
