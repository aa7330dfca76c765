"""Images over application-owned device memory (vxCreateImageFromHandle with
VX_MEMORY_TYPE_HIP, vx_api.cpp:1002-1026; here the memory is CUDA device memory): graphs
read and write the application's buffers in place, with no copy; vxSwapImageHandle moves
a graph to other buffers; planes whose layout the kernels cannot take (bases not 256-byte
aligned, row pitches not multiples of 64 bytes) are refused instead of faulting."""
import ctypes as C

import numpy as np
import pytest

import oracle_chains as OC
from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL

pytestmark = pytest.mark.gpu


def dev_plane(h, w, pitch=None):
    """A torch-owned device plane (256-byte aligned base) and its row pitch."""
    import torch
    pitch = pitch or ((w + 63) // 64) * 64
    t = torch.zeros(h * pitch + 256, dtype=torch.uint8, device="cuda")
    off = -t.data_ptr() % 256
    return t, t.data_ptr() + off, pitch, off


def image_from_device(api, ctx, ptr, w, h, pitch):
    addr = V.vx_imagepatch_addressing_t()
    addr.dim_x, addr.dim_y, addr.stride_x, addr.stride_y = w, h, 1, pitch
    addr.scale_x = addr.scale_y = 1024
    addr.step_x = addr.step_y = 1
    ptrs = (C.c_void_p * 1)(ptr)
    return api.vxCreateImageFromHandle(ctx, V.VX_DF_IMAGE_U8, C.byref(addr), ptrs, V.VX_MEMORY_TYPE_HIP)


def _put(t, off, pitch, img):
    import torch
    h, w = img.shape
    rows = t[off: off + h * pitch].view(h, pitch)
    rows[:, :w].copy_(torch.from_numpy(img))


def _get(t, off, pitch, h, w):
    import torch
    torch.cuda.synchronize()
    return t[off: off + h * pitch].view(h, pitch)[:, :w].cpu().numpy()


@pytest.mark.parametrize("flags", [None, V.OPT_NO_FUSION])
def test_cfg1_on_device_buffers(cuda, flags):
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        W, H = 1920, 1080
        bufs = [dev_plane(H, W) for _ in range(4)]           # src A, dst A, src B, dst B
        imgs = [api.obj(image_from_device(api, ctx, p, W, H, pitch), "device image") for _, p, pitch, _ in bufs[:2]]
        graph = api.obj(api.vxCreateGraph(ctx), "graph")
        if flags is not None:
            api.set_optimizer_flags(graph, flags)
        gau = api.vxCreateVirtualImage(graph, W, H, V.VX_DF_IMAGE_U8)
        gx = api.vxCreateVirtualImage(graph, W, H, V.VX_DF_IMAGE_S16)
        gy = api.vxCreateVirtualImage(graph, W, H, V.VX_DF_IMAGE_S16)
        mag = api.vxCreateVirtualImage(graph, W, H, V.VX_DF_IMAGE_S16)
        dep = api.vxCreateVirtualImage(graph, W, H, V.VX_DF_IMAGE_U8)
        api.obj(api.vxGaussian3x3Node(graph, imgs[0], gau), "gaussian")
        api.obj(api.vxSobel3x3Node(graph, gau, gx, gy), "sobel")
        api.obj(api.vxMagnitudeNode(graph, gx, gy, mag), "magnitude")
        api.obj(api.vxConvertDepthNode(graph, mag, dep, V.VX_CONVERT_POLICY_SATURATE, api.scalar(ctx, V.VX_TYPE_INT32, 0)), "depth")
        api.obj(api.vxThresholdNode(graph, dep, api.threshold_binary(ctx, 128), imgs[1]), "threshold")
        api.ok(api.vxVerifyGraph(graph), "verify")
        for rep, seed in enumerate((3, 4)):
            img = WL.cfg1_image(seed=seed, width=W, height=H)
            (ts, _, ps, os_), (td, _, pd, od) = bufs[2 * rep], bufs[2 * rep + 1]
            if rep == 1:   # move the graph to the second pair of buffers
                for im, (_, p, _, _) in zip(imgs, bufs[2:]):
                    new = (C.c_void_p * 1)(p)
                    prev = (C.c_void_p * 1)()
                    api.ok(api.vxSwapImageHandle(im, new, prev, 1), "swap")
            _put(ts, os_, ps, img)
            api.ok(api.vxProcessGraph(graph), "process")
            ref, (sx, sy, ex, ey) = OC.cfg1_chain(img, 0, 128)
            got = _get(td, od, pd, H, W)                     # read straight from the application's buffer
            np.testing.assert_array_equal(got[sy:ey, sx:ex], ref[sy:ey, sx:ex])
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def test_misaligned_device_planes_are_refused(cuda):
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        t, p, pitch, _ = dev_plane(64, 200, pitch=256)
        assert not image_from_device(api, ctx, p + 16, 200, 64, 256)       # base not 256-byte aligned
        assert not image_from_device(api, ctx, p, 200, 64, 224)            # pitch not a multiple of 64
        assert not image_from_device(api, ctx, p, 200, 64, 192)            # pitch below the row
        img = api.obj(image_from_device(api, ctx, p, 200, 64, 256), "device image")
        new = (C.c_void_p * 1)(p + 64)
        assert api.vxSwapImageHandle(img, new, None, 1) == V.VX_ERROR_INVALID_PARAMETERS
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))
