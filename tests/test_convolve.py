"""vxConvolveNode (custom convolution): the reference library's graph equals the oracle chain
(the restatement pinned in test_oracle_pin_convolve.py) inside its valid rectangle; on the
GPU, agocuda_Convolve_{U8,S16}_U8 equal the oracle on every processed pixel, and the engine's
graph equals it inside the valid rectangle, re-planning when the coefficients change."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import oracle_chains as OC
from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL

u32, i32, vp = C.c_uint32, C.c_int32, C.c_void_p


def coefficients(cols, rows, seed, big=False):
    hi = 2000 if big else 9
    return np.random.default_rng(seed).integers(-hi, hi + 1, (rows, cols)).astype(np.int16)


def oracle_convolve(img, conv, shift, out):
    """The AGO node on AGO buffers: rows [rows/2, H - rows/2), all columns."""
    H, W = img.shape
    rows, cols = conv.shape
    dt = np.uint8 if out == "U8" else np.int16
    src = OC.ago_img(H, W); src.set(img)
    dst = OC.ago_img(H, W, dt)
    k = np.ascontiguousarray(conv, np.int16)
    f = getattr(O.oracle_lib(), f"oracle_Convolve_{out}_U8")
    f.argtypes, f.restype = [u32, u32, vp, u32, vp, u32, vp, u32, u32, i32], C.c_int
    hy = rows // 2
    f(W, H - rows + 1, dst.row_ptr(hy), dst.stride, src.row_ptr(hy), src.stride, k.ctypes.data, cols, rows, shift)
    return dst.get()


def run_graph(api, img, conv, scale, out, recolor=None):
    H, W = img.shape
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        src = api.obj(api.vxCreateImage(ctx, W, H, V.VX_DF_IMAGE_U8), "image")
        dst = api.obj(api.vxCreateImage(ctx, W, H, V.VX_DF_IMAGE_U8 if out == "U8" else V.VX_DF_IMAGE_S16), "image")
        api.write_plane(src, img)
        cv = api.convolution(ctx, conv, scale)
        g = api.obj(api.vxCreateGraph(ctx), "graph")
        api.obj(api.vxConvolveNode(g, src, cv, dst), "convolve")
        api.ok(api.vxVerifyGraph(g), "verify")
        api.ok(api.vxProcessGraph(g), "process")
        res = [(api.read_plane(dst), api.valid_region(dst))]
        if recolor is not None:      # new coefficients, same graph: must re-plan
            k = np.ascontiguousarray(recolor, np.int16)
            api.ok(api.vxCopyConvolutionCoefficients(cv, k.ctypes.data, V.VX_WRITE_ONLY, V.VX_MEMORY_TYPE_HOST), "write")
            api.ok(api.vxProcessGraph(g), "process")
            res.append((api.read_plane(dst), api.valid_region(dst)))
        return res
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


CASES = [(3, 3, 1, "U8"), (3, 3, 8, "S16"), (5, 3, 16, "U8"), (7, 5, 1, "S16"), (9, 9, 64, "U8"), (9, 3, 1, "S16")]


def _check(res, img, conv, scale, out):
    (got, rect), = res[:1]
    rows, cols = conv.shape
    H, W = img.shape
    assert rect == (cols // 2, rows // 2, W - cols // 2, H - rows // 2)
    want = oracle_convolve(img, conv, int(np.log2(scale)), out)
    sx, sy, ex, ey = rect
    np.testing.assert_array_equal(got[sy:ey, sx:ex], want[sy:ey, sx:ex])


@pytest.mark.parametrize("cols,rows,scale,out", CASES)
def test_reference_graph_matches_oracle(cols, rows, scale, out):
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    img = WL.cfg1_image(seed=cols * 10 + rows, width=333, height=97)
    conv = coefficients(cols, rows, cols + rows, big=out == "S16")
    _check(run_graph(V.OpenVX(lib), img, conv, scale, out), img, conv, scale, out)


@pytest.mark.gpu
@pytest.mark.parametrize("out", ["U8", "S16"])
@pytest.mark.parametrize("cols", [3, 5, 7, 9])
@pytest.mark.parametrize("rows", [3, 5, 9])
@pytest.mark.parametrize("shift,big", [(0, False), (3, False), (0, True), (5, True)])
@pytest.mark.parametrize("W,H", [(1920, 1080), (45, 17), (333, 97)])
def test_convolve_kernels(cuda, out, cols, rows, shift, big, W, H):
    from devbuf import DevImg, stream_ptr
    from mivisionx_b200 import native
    lib = native.agocuda()
    img = WL.cfg1_image(seed=W + H + cols, width=W, height=H)
    conv = coefficients(cols, rows, cols * 100 + rows * 10 + shift, big)
    dt = np.uint8 if out == "U8" else np.int16
    src, dst = DevImg(H, W).upload(img), DevImg(H, W, dt)
    f = getattr(lib, f"agocuda_Convolve_{out}_U8")
    f.argtypes, f.restype = [vp, u32, u32, vp, u32, vp, u32, vp, u32, u32, i32, i32, i32], C.c_int
    k = np.ascontiguousarray(conv)
    assert f(stream_ptr(), W, H, dst.ptr, dst.stride, src.ptr, src.stride, k.ctypes.data, cols, rows, shift, 0,
             W - W % 16) == 0
    got, want = dst.download(), oracle_convolve(img, conv, shift, out)
    hy, hx = rows // 2, cols // 2
    # every processed row; the columns whose taps stay inside the row (the reference reads the
    # neighbouring rows' bytes for the outer columns, outside the valid region)
    np.testing.assert_array_equal(got[hy:H - hy, hx:W - hx], want[hy:H - hy, hx:W - hx])


@pytest.mark.gpu
@pytest.mark.parametrize("cols,rows,scale,out", CASES)
def test_engine_graph_matches_oracle(cuda, cols, rows, scale, out):
    img = WL.cfg1_image(seed=cols * 10 + rows, width=1920, height=1080)
    conv = coefficients(cols, rows, cols + rows, big=out == "S16")
    conv2 = coefficients(cols, rows, 7 * cols + rows, big=True)
    res = run_graph(V.OpenVX(), img, conv, scale, out, recolor=conv2)
    _check(res[:1], img, conv, scale, out)
    _check(res[1:], img, conv2, scale, out)
