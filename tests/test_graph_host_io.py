"""Images created from page-locked application buffers (vxCreateImageFromHandle with
VX_MEMORY_TYPE_HOST, as ago/ago_interface.cpp imports them for the HIP target): the
captured CUDA graph uploads the inputs and downloads the outputs itself, each frame's copies
overlapping other frames' kernels.  Results must equal the oracle -- in the application's
own output buffers, with no read call -- and must follow in-place changes of the input
buffers and vxSwapImageHandle."""
import ctypes as C

import numpy as np
import pytest

import oracle_chains as OC
from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL

pytestmark = pytest.mark.gpu


def pinned(h, w):
    import torch
    return torch.zeros((h, w), dtype=torch.uint8).pin_memory()


def _scene(seed, w, h):
    return WL.cfg2_scene(seed=seed, width=w, height=h, rects=min(200, max(3, w * h // 300)))


def _check_cfg2(edges, corners, num, img):
    h, w = img.shape
    ref_edges, _ = OC.canny(img)
    ref_corners, ref_num = OC.harris(img, capacity=32768)
    np.testing.assert_array_equal(edges[1:h - 1, 1:w - 1], ref_edges[1:h - 1, 1:w - 1])
    assert num == ref_num
    np.testing.assert_array_equal(corners.view(OC.KP), ref_corners)


def test_cfg2_host_buffers(cuda):
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    sizes = [(640, 480), (1280, 720), (648, 360), (200, 120)]
    ins = [pinned(h, w) for w, h in sizes]
    outs = [pinned(h, w) for w, h in sizes]
    g = WL.Cfg2Graph(api, ctx, sizes, host_io={"src": [t.numpy() for t in ins], "edge": [t.numpy() for t in outs]})
    for rnd in range(2):   # the second round rewrites the application's input buffers in place
        frames = [_scene(100 * rnd + i, w, h) for i, (w, h) in enumerate(sizes)]
        for t, f in zip(ins, frames):
            t.numpy()[:] = f
        g.run()
        for i, f in enumerate(frames):
            corners = api.array_items(g.corners[i])
            _check_cfg2(outs[i].numpy(), corners, api.read_scalar(g.num[i]), f)
    # the same results through vxCopyImagePatch reads (host and device copies agree)
    for i, (e, _, _, _) in enumerate(g.results()):
        np.testing.assert_array_equal(e, outs[i].numpy())


def test_swap_handle_recaptures(cuda):
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    w, h = 640, 480
    a_in, b_in, out = pinned(h, w), pinned(h, w), pinned(h, w)
    fa, fb = _scene(7, w, h), _scene(8, w, h)
    a_in.numpy()[:] = fa
    b_in.numpy()[:] = fb
    g = WL.Cfg2Graph(api, ctx, [(w, h)], host_io={"src": [a_in.numpy()], "edge": [out.numpy()]})
    g.run()
    _check_cfg2(out.numpy(), api.array_items(g.corners[0]), api.read_scalar(g.num[0]), fa)
    new = (C.c_void_p * 1)(b_in.data_ptr())
    prev = (C.c_void_p * 1)()
    api.ok(api.vxSwapImageHandle(g.inputs[0], new, prev, 1), "swap")
    assert prev[0] == a_in.data_ptr()
    g.run()
    _check_cfg2(out.numpy(), api.array_items(g.corners[0]), api.read_scalar(g.num[0]), fb)


def test_cfg1_host_buffers_and_pageable_fallback(cuda):
    """Batched chain (one launch for all frames) with page-locked buffers, and the same graph
    over pageable numpy buffers, which take the synchronous copy path."""
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    sizes = [(1920, 1080), (640, 480)]
    frames = [WL.cfg1_image(seed=30 + i, width=w, height=h) for i, (w, h) in enumerate(sizes)]
    want = [OC.cfg1_chain(f) for f in frames]
    for kind in ("pinned", "pageable"):
        if kind == "pinned":
            keep = [pinned(h, w) for w, h in sizes for _ in range(2)]   # owners of the page-locked memory
            ins, outs = [t.numpy() for t in keep[0::2]], [t.numpy() for t in keep[1::2]]
        else:
            ins = [np.zeros((h, w), np.uint8) for w, h in sizes]
            outs = [np.zeros((h, w), np.uint8) for w, h in sizes]
        for b, f in zip(ins, frames):
            b[:] = f
        g = WL.Cfg1Graph(api, ctx, sizes, host_io={"src": ins, "dst": outs})
        g.run()
        for i, ((ref, rect), (got, grect)) in enumerate(zip(want, g.results())):
            assert grect == rect
            sx, sy, ex, ey = rect
            np.testing.assert_array_equal(got[sy:ey, sx:ex], ref[sy:ey, sx:ex], err_msg=f"{kind} frame {i}")
            if kind == "pinned":
                np.testing.assert_array_equal(outs[i][sy:ey, sx:ex], ref[sy:ey, sx:ex])


@pytest.mark.parametrize("host", [False, True])
def test_cfg1_many_frames_in_launch_groups(cuda, host):
    """19 uneven frames: with page-locked application buffers the batched chain runs as
    launches over groups of 8 frames, spread over the capture lanes and interleaved with the
    uploads; device-resident frames share one launch."""
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    sizes = [[(130, 66), (37, 21), (320, 240), (640, 480)][i % 4] for i in range(19)]
    frames = [WL.cfg1_image(seed=60 + i, width=w, height=h) for i, (w, h) in enumerate(sizes)]
    keep = [pinned(h, w) for w, h in sizes for _ in range(2)] if host else []
    host_io = {"src": [t.numpy() for t in keep[0::2]], "dst": [t.numpy() for t in keep[1::2]]} if host else None
    g = WL.Cfg1Graph(api, ctx, sizes, host_io=host_io)
    assert api.plan(g.graph) == [("fused_GaussSobelMagDepthThresh x19", 3 if host else 1)]
    if host:
        for t, f in zip(keep[0::2], frames):
            t.numpy()[:] = f
        g.run()
    else:
        g.run(frames)
    for i, (f, (got, grect)) in enumerate(zip(frames, g.results())):
        ref, rect = OC.cfg1_chain(f)
        assert grect == rect
        sx, sy, ex, ey = rect
        np.testing.assert_array_equal(got[sy:ey, sx:ex], ref[sy:ey, sx:ex], err_msg=f"frame {i}")
        if host:
            np.testing.assert_array_equal(keep[2 * i + 1].numpy()[sy:ey, sx:ex], ref[sy:ey, sx:ex])
