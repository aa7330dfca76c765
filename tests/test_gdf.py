"""Graph import from AGO's text graph description (VX_GRAPH_ATTRIBUTE_AMD_IMPORT_FROM_TEXT,
ago/ago_interface.cpp:456): `data` / `node` statements, inline enum arguments (!NORM_L1),
matrix and threshold initialisers, node border attributes, and the data-registry callback
that hands the application its objects.

CPU: the reference library imports the text and its results equal the same graph built
through the C API in the same library.  GPU: the same for this package's engine."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL

W, H = 320, 240
GDF = f"""
# a small graph touching most statement forms
data src    = image:U008,{W},{H}:IN           # registered with the application (callback)
data gau    = image-virtual:U008,0,0
data bin    = image-virtual:U008,0,0
data inv    = image:U008,{W},{H}:OUT_INV
data gs     = scalar:INT32,3
data edges  = image:U008,{W},{H}:OUT_EDGES
data M      = matrix:FLOAT32,2,3:INIT,{{0.9;0.1;-0.1;0.9;12;-7}}
data med    = image-virtual:U008,0,0
data dil    = image:U008,{W},{H}:OUT_DIL
node org.khronos.openvx.gaussian_3x3 src gau
node org.khronos.openvx.threshold gau $2 bin
node org.khronos.openvx.not bin inv
node org.khronos.openvx.canny_edge_detector src $1 gs !NORM_L1 edges
node org.khronos.openvx.median_3x3 src med attr:BORDER_MODE:UNDEFINED
node org.khronos.openvx.dilate_3x3 med dil
"""


def _lib(ref):
    if ref:
        lib = O.ref_lib()
        if lib is None:
            pytest.skip("reference library not built")
        return V.OpenVX(lib)
    return V.OpenVX()


def imported(api, img):
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        g = api.obj(api.vxCreateGraph(ctx), "graph")
        def on_data(ref, name, params):
            # the application applies INIT requests while the text is read, as runvx does
            # (the reference library reports them through the callback only)
            if name == "M":
                m = np.array([0.9, 0.1, -0.1, 0.9, 12, -7], np.float32)
                api.ok(api.vxCopyMatrix(ref, m.ctypes.data, V.VX_WRITE_ONLY, V.VX_MEMORY_TYPE_HOST), "M")

        # thresholds come from the application ($1, $2): the reference library's text form
        # leaves a threshold's data type unset, which the Canny and Threshold validators refuse
        refs = [api.threshold_range(ctx, 80, 100), api.threshold_binary(ctx, 100)]
        st, found = api.import_gdf(g, GDF, on_data, refs=refs)
        assert st == V.VX_SUCCESS
        assert {k: v[1] for k, v in found.items()} == {
            "src": "IN", "inv": "OUT_INV", "edges": "OUT_EDGES", "dil": "OUT_DIL",
            "M": "INIT,{0.9;0.1;-0.1;0.9;12;-7}"}
        api.write_plane(found["src"][0], img)
        api.ok(api.vxVerifyGraph(g), "verify")
        api.ok(api.vxProcessGraph(g), "process")
        return {k: (api.read_plane(found[k][0]), api.valid_region(found[k][0])) for k in ("inv", "edges", "dil")}
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def built(api, img):
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        g = api.obj(api.vxCreateGraph(ctx), "graph")
        U8 = V.VX_DF_IMAGE_U8
        mk = lambda: api.obj(api.vxCreateImage(ctx, W, H, U8), "image")
        src, inv, edges, dil = mk(), mk(), mk(), mk()
        gau, b, med = (api.vxCreateVirtualImage(g, 0, 0, U8) for _ in range(3))
        api.obj(api.vxGaussian3x3Node(g, src, gau), "n")
        api.obj(api.vxThresholdNode(g, gau, api.threshold_binary(ctx, 100), b), "n")
        api.obj(api.vxNotNode(g, b, inv), "n")
        api.obj(api.vxCannyEdgeDetectorNode(g, src, api.threshold_range(ctx, 80, 100), 3, V.VX_NORM_L1, edges), "n")
        api.obj(api.vxMedian3x3Node(g, src, med), "n")
        api.obj(api.vxDilate3x3Node(g, med, dil), "n")
        api.write_plane(src, img)
        api.ok(api.vxVerifyGraph(g), "verify")
        api.ok(api.vxProcessGraph(g), "process")
        return {k: (api.read_plane(o), api.valid_region(o)) for k, o in
                (("inv", inv), ("edges", edges), ("dil", dil))}
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def _check(api):
    img = WL.cfg2_scene(seed=3, width=W, height=H, rects=40)
    a, b = imported(api, img), built(api, img)
    for k in a:
        (x, rx), (y, ry) = a[k], b[k]
        assert rx == ry, k
        sx, sy, ex, ey = rx
        np.testing.assert_array_equal(x[sy:ey, sx:ex], y[sy:ey, sx:ex], err_msg=k)


def _errors(api):
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        for text in ("data x = image:U008,10,10\nnode org.khronos.openvx.no_such_kernel x x",
                     "data x = image:U008,10,10\nnode org.khronos.openvx.not x missing_name",
                     "data x = bogus:1,2"):
            g = api.obj(api.vxCreateGraph(ctx), "graph")
            assert api.import_gdf(g, text)[0] != V.VX_SUCCESS, text
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def test_reference_import_matches_api():
    _check(_lib(True))


def test_reference_import_errors():
    _errors(_lib(True))


@pytest.mark.gpu
def test_engine_import_matches_api(cuda):
    _check(_lib(False))


@pytest.mark.gpu
def test_engine_import_errors(cuda):
    _errors(_lib(False))
