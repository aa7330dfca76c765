"""ScaleImage on the GPU: the three agocuda_ScaleImage_U8_U8_* kernels against the oracle
(pinned to the reference HAF kernels in test_oracle_pin_geometry.py), and vxScaleImageNode
with nearest-neighbour interpolation through the engine against the oracle and, for the
valid rectangle, against the reference library."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import oracle_chains as OC
from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL

u32, vp = C.c_uint32, C.c_void_p
NAMES = {0: "Nearest", 1: "Bilinear", 2: "Area"}
KINDS = {V.VX_INTERPOLATION_NEAREST_NEIGHBOR: 0, V.VX_INTERPOLATION_BILINEAR: 1, V.VX_INTERPOLATION_AREA: 2}


def oracle_scale(img, kind, dw, dh):
    sh, sw = img.shape
    src = OC.ago_img(sh, sw); src.set(img)
    dst = OC.ago_img(dh, dw)
    m = OC.scale_matrix(kind, sw, sh, dw, dh)
    f = getattr(O.oracle_lib(), "oracle_ScaleImage_U8_U8_" + NAMES[kind])
    f.argtypes, f.restype = [u32, u32, vp, u32, u32, u32, vp, u32, vp], C.c_int
    assert f(dw, dh, dst.ptr, dst.stride, sw, sh, src.ptr, src.stride, C.cast(m, vp)) == 0
    return dst.get()


SIZES = [(3840, 2160, 1920, 1080), (1920, 1080, 3840, 2160), (640, 480, 333, 97), (100, 60, 50, 30),
         (64, 48, 96, 72), (90, 50, 40, 30), (1280, 720, 1280, 720)]


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [0, 1, 2])
@pytest.mark.parametrize("sw,sh,dw,dh", SIZES)
def test_scale_kernels(cuda, kind, sw, sh, dw, dh):
    if kind == 2 and not ((sw == 2 * dw and sh == 2 * dh) or (sw == dw and sh == dh)):
        pytest.skip("area: the exact 1x and 2x ratios")
    from devbuf import DevImg, stream_ptr
    from mivisionx_b200 import native
    lib = native.agocuda()
    img = WL.cfg1_image(seed=sw + 3 * dh + kind, width=sw, height=sh)
    src, dst = DevImg(sh, sw).upload(img), DevImg(dh, dw)
    f = getattr(lib, "agocuda_ScaleImage_U8_U8_" + NAMES[kind])
    f.argtypes, f.restype = [vp, u32, u32, vp, u32, u32, u32, vp, u32], C.c_int
    assert f(stream_ptr(), dw, dh, dst.ptr, dst.stride, sw, sh, src.ptr, src.stride) == 0
    got, want = dst.download(), oracle_scale(img, kind, dw, dh)
    if kind == 2 and sw == 2 * dw:   # the reference's 2x area path writes the first (W & ~7) columns
        n = dw & ~7
        got, want = got[:, :n], want[:, :n]
    np.testing.assert_array_equal(got, want)


def gauss(img):
    src = OC.ago_img(*img.shape); src.set(img)
    return OC.gaussian3x3(src).get()


def _graph(api, ctx, img, dw, dh, interp, flags=None):
    sh, sw = img.shape
    src = api.obj(api.vxCreateImage(ctx, sw, sh, V.VX_DF_IMAGE_U8), "image")
    dst = api.obj(api.vxCreateImage(ctx, dw, dh, V.VX_DF_IMAGE_U8), "image")
    g = api.obj(api.vxCreateGraph(ctx), "graph")
    if flags is not None:
        api.set_optimizer_flags(g, flags)
    mid = api.obj(api.vxCreateVirtualImage(g, sw, sh, V.VX_DF_IMAGE_U8), "virtual")
    api.obj(api.vxGaussian3x3Node(g, src, mid), "gaussian")     # a valid rectangle smaller than the image
    api.obj(api.vxScaleImageNode(g, mid, dst, interp), "scale")
    api.ok(api.vxVerifyGraph(g), "verify")
    api.write_plane(src, img)
    api.ok(api.vxProcessGraph(g), "process")
    return api.read_plane(dst), api.valid_region(dst)


CASES = [(1920, 1080, 960, 540), (3840, 2160, 1920, 1080), (640, 480, 1000, 700), (200, 120, 77, 33)]


def test_reference_scale_nearest_graph_rect():
    """The reference library's nearest graph equals the oracle chain (Gaussian, then scale)
    on its valid rectangle, and gives the rectangle the engine must give."""
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    api = V.OpenVX(lib)
    ctx = api.obj(api.vxCreateContext(), "context")
    for sw, sh, dw, dh in CASES[:1] + CASES[2:]:
        img = WL.cfg1_image(seed=sw + dh, width=sw, height=sh)
        got, rect = _graph(api, ctx, img, dw, dh, V.VX_INTERPOLATION_NEAREST_NEIGHBOR)
        want = oracle_scale(gauss(img), 0, dw, dh)
        # the callback rewrites the *input's* rectangle (it reads paramList[0], the output, as
        # its input; ago_kernel_api.cpp:19956), so the output keeps its full rectangle
        assert rect == (0, 0, dw, dh), rect
        inner = (slice(2, dh - 2), slice(2, dw - 2))
        np.testing.assert_array_equal(got[inner], want[inner])


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [None, V.OPT_NO_FUSION])
@pytest.mark.parametrize("sw,sh,dw,dh", CASES)
def test_engine_scale_nearest_graph(cuda, flags, sw, sh, dw, dh):
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        img = WL.cfg1_image(seed=sw + dh, width=sw, height=sh)
        got, rect = _graph(api, ctx, img, dw, dh, V.VX_INTERPOLATION_NEAREST_NEIGHBOR, flags)
        assert rect == (0, 0, dw, dh), rect
        want = oracle_scale(gauss(img), 0, dw, dh)
        inner = (slice(2, dh - 2), slice(2, dw - 2))
        np.testing.assert_array_equal(got[inner], want[inner])
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))
