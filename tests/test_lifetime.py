"""Object lifetime: storage goes back when the last application and internal references are
gone, as agoReleaseData (ago/ago_util.cpp:2771) frees AGO's objects -- a streaming
application that creates and releases images or graphs per frame keeps a flat footprint."""
import ctypes as C

import numpy as np
import pytest

from mivisionx_b200 import vx as V

pytestmark = pytest.mark.gpu


def _free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def test_released_images_return_their_storage(cuda):
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        W, H = 3840, 2160
        row = np.arange(W, dtype=np.uint8)
        frame = np.broadcast_to(row, (H, W))
        base = None
        for i in range(1000):
            img = api.obj(api.vxCreateImage(ctx, W, H, V.VX_DF_IMAGE_U8), "image")
            if i % 50 == 0:
                api.write_plane(img, frame)
                assert np.array_equal(api.read_plane(img)[::997], frame[::997])
            api.ok(api.vxReleaseImage(C.byref(C.c_void_p(img))), "release")
            if i == 10:
                base = _free_bytes()
        # 990 more 8.3 MB images were created and released since `base`
        assert base - _free_bytes() < 64 << 20
        n = C.c_uint32(0)
        q = api.lib.vxQueryContext
        q.argtypes, q.restype = [C.c_void_p, C.c_int32, C.c_void_p, C.c_size_t], C.c_int32
        api.ok(q(ctx, 0x80104, C.byref(n), 4), "references")   # VX_CONTEXT_REFERENCES
        assert n.value < 16, n.value
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def _chain_graph(api, ctx, W, H, src, dst):
    g = api.obj(api.vxCreateGraph(ctx), "graph")
    v1 = api.obj(api.vxCreateVirtualImage(g, W, H, V.VX_DF_IMAGE_U8), "virtual")
    v2 = api.obj(api.vxCreateVirtualImage(g, W, H, V.VX_DF_IMAGE_U8), "virtual")
    api.obj(api.vxGaussian3x3Node(g, src, v1), "gaussian")
    api.obj(api.vxBox3x3Node(g, v1, v2), "box")
    api.obj(api.vxMedian3x3Node(g, v2, dst), "median")
    for v in (v1, v2):
        api.ok(api.vxReleaseImage(C.byref(C.c_void_p(v))), "release virtual")
    return g


def test_released_graphs_return_their_storage(cuda):
    """Per-frame graphs (verify, process, release) with plain-form intermediates that own
    device memory: the graph's plan, its lowered data and its virtual images go with it."""
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        W, H = 1920, 1080
        img = np.random.default_rng(3).integers(0, 256, (H, W), dtype=np.uint8)
        src = api.obj(api.vxCreateImage(ctx, W, H, V.VX_DF_IMAGE_U8), "image")
        dst = api.obj(api.vxCreateImage(ctx, W, H, V.VX_DF_IMAGE_U8), "image")
        api.write_plane(src, img)
        first = None
        base = None
        for i in range(60):
            g = _chain_graph(api, ctx, W, H, src, dst)
            api.set_optimizer_flags(g, 0x10000 | 0x20000)   # plain form: intermediates are materialised
            api.ok(api.vxVerifyGraph(g), "verify")
            api.ok(api.vxProcessGraph(g), "process")
            out = api.read_plane(dst)
            if first is None:
                first = out
            else:
                assert np.array_equal(out, first)
            api.ok(api.vxReleaseGraph(C.byref(C.c_void_p(g))), "release graph")
            if i == 5:
                base = _free_bytes()
        assert base - _free_bytes() < 32 << 20
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))
