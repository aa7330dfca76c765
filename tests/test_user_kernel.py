"""User kernels (vxAddUserKernel, vx_api.cpp:2584-2800) in this engine's graphs.

A host kernel (the usual plugin form) reads and writes its images through the host access
calls; a device-buffer kernel (VX_KERNEL_ATTRIBUTE_AMD_GPU_BUFFER_ACCESS_ENABLE, the pattern of
amd_custom/source/custom_layer.cpp:138) takes device pointers and the node's CUDA stream
(VX_NODE_ATTRIBUTE_AMD_HIP_STREAM) and enqueues its own work.  Both sit between built-in nodes
(Gaussian3x3 before, Threshold after); the result equals the oracle chain with the user
kernel's arithmetic (255 - v) in the middle.  The callbacks here are Python functions called
from the library through ctypes."""
import ctypes as C

import numpy as np
import pytest

import oracle_chains as OC
from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL

pytestmark = pytest.mark.gpu

u32, vp, sz = C.c_uint32, C.c_void_p, C.c_size_t
INVERT_HOST = V.VX_KERNEL_BASE_USER + 1
INVERT_DEV = V.VX_KERNEL_BASE_USER + 2
FAILS = V.VX_KERNEL_BASE_USER + 3


def _q_u32(api, img, attr):
    v = C.c_uint32(0)
    api.ok(api.vxQueryImage(img, attr, C.byref(v), 4), "query image")
    return v.value


class Plugin:
    """The callbacks of one test's user kernels (kept alive with the object)."""

    def __init__(self, api):
        self.api = api
        self.calls = 0
        self.init_calls = 0
        self.deinit_calls = 0
        self.validate_f = V.KernelValidateF(self.validate)
        self.host_f = V.KernelF(self.invert_on_host)
        self.dev_f = V.KernelF(self.invert_on_device)
        self.fail_f = V.KernelF(lambda node, params, num: -1)     # VX_FAILURE
        self.init_f = V.KernelF(self.init)
        self.deinit_f = V.KernelF(self.deinit)
        from mivisionx_b200 import native
        self.ago = native.agocuda()
        self.ago.agocuda_Not_U8_U8.argtypes = [vp, u32, u32, vp, u32, vp, u32]
        self.ago.agocuda_Not_U8_U8.restype = C.c_int

    # output 1 is a U8 image of the input's size
    def validate(self, node, params, num, metas):
        a = self.api
        src = params[0]
        w, h = _q_u32(a, src, V.VX_IMAGE_WIDTH), _q_u32(a, src, V.VX_IMAGE_HEIGHT)
        fmt = C.c_uint32(V.VX_DF_IMAGE_U8)
        if _q_u32(a, src, V.VX_IMAGE_FORMAT) != V.VX_DF_IMAGE_U8:
            return -14                                            # VX_ERROR_INVALID_FORMAT
        meta = metas[1]
        a.ok(a.vxSetMetaFormatAttribute(meta, V.VX_IMAGE_FORMAT, C.byref(fmt), 4), "meta format")
        a.ok(a.vxSetMetaFormatAttribute(meta, V.VX_IMAGE_WIDTH, C.byref(C.c_uint32(w)), 4), "meta width")
        a.ok(a.vxSetMetaFormatAttribute(meta, V.VX_IMAGE_HEIGHT, C.byref(C.c_uint32(h)), 4), "meta height")
        return 0

    def init(self, node, params, num):
        self.init_calls += 1
        p = C.c_void_p(0)
        self.api.ok(self.api.vxQueryNode(node, V.VX_NODE_LOCAL_DATA_PTR, C.byref(p), C.sizeof(p)), "local ptr")
        if p.value:                                               # kernels that declared local data
            C.cast(p, C.POINTER(C.c_uint32))[0] = 1000
        return 0

    def deinit(self, node, params, num):
        self.deinit_calls += 1
        return 0

    def _map(self, img, usage):
        a = self.api
        w, h = _q_u32(a, img, V.VX_IMAGE_WIDTH), _q_u32(a, img, V.VX_IMAGE_HEIGHT)
        rect = V.vx_rectangle_t(0, 0, w, h)
        mid, addr, ptr = C.c_size_t(0), V.vx_imagepatch_addressing_t(), C.c_void_p(0)
        a.ok(a.vxMapImagePatch(img, C.byref(rect), 0, C.byref(mid), C.byref(addr), C.byref(ptr), usage,
                               V.VX_MEMORY_TYPE_HOST, 0), "map")
        buf = (C.c_uint8 * (addr.stride_y * h)).from_address(ptr.value)
        view = np.frombuffer(buf, np.uint8).reshape(h, addr.stride_y)[:, :w]
        return mid, view

    def invert_on_host(self, node, params, num):
        self.calls += 1
        a = self.api
        m_in, src = self._map(params[0], V.VX_READ_ONLY)
        m_out, dst = self._map(params[1], V.VX_WRITE_ONLY)
        dst[:] = 255 - src
        a.ok(a.vxUnmapImagePatch(params[1], m_out), "unmap out")
        a.ok(a.vxUnmapImagePatch(params[0], m_in), "unmap in")
        p = C.c_void_p(0)
        a.ok(a.vxQueryNode(node, V.VX_NODE_LOCAL_DATA_PTR, C.byref(p), C.sizeof(p)), "local ptr")
        if p.value:
            C.cast(p, C.POINTER(C.c_uint32))[0] += 1
        return 0

    def invert_on_device(self, node, params, num):
        self.calls += 1
        a = self.api
        stream = C.c_void_p(0)
        a.ok(a.vxQueryNode(node, V.VX_NODE_ATTRIBUTE_AMD_HIP_STREAM, C.byref(stream), C.sizeof(stream)), "stream")
        ptrs, pitches = [], []
        for img in (params[0], params[1]):
            d = C.c_void_p(0)
            a.ok(a.vxQueryImage(img, V.VX_IMAGE_ATTRIBUTE_AMD_HIP_BUFFER, C.byref(d), C.sizeof(d)), "device buffer")
            ptrs.append(d.value)
            pitches.append(_q_u32(a, img, V.VX_IMAGE_ATTRIBUTE_AMD_GPU_BUFFER_STRIDE))
        w, h = _q_u32(a, params[0], V.VX_IMAGE_WIDTH), _q_u32(a, params[0], V.VX_IMAGE_HEIGHT)
        return self.ago.agocuda_Not_U8_U8(stream.value, w, h, ptrs[1], pitches[1], ptrs[0], pitches[0])

    def publish(self, ctx, name, enum, func, gpu=False, local_size=0):
        a = self.api
        k = a.vxAddUserKernel(ctx, name.encode(), enum, C.cast(func, vp), 2, C.cast(self.validate_f, vp),
                              C.cast(self.init_f, vp), C.cast(self.deinit_f, vp))
        assert k, name
        if gpu:
            on = C.c_int32(1)
            a.ok(a.vxSetKernelAttribute(k, V.VX_KERNEL_ATTRIBUTE_AMD_GPU_BUFFER_ACCESS_ENABLE, C.byref(on), 4), "gpu access")
        if local_size:
            a.ok(a.vxSetKernelAttribute(k, V.VX_KERNEL_LOCAL_DATA_SIZE, C.byref(C.c_size_t(local_size)), 8), "local size")
        a.ok(a.vxAddParameterToKernel(k, 0, V.VX_INPUT, V.VX_TYPE_IMAGE, V.VX_PARAMETER_STATE_REQUIRED), "param 0")
        a.ok(a.vxAddParameterToKernel(k, 1, V.VX_OUTPUT, V.VX_TYPE_IMAGE, V.VX_PARAMETER_STATE_REQUIRED), "param 1")
        a.ok(a.vxFinalizeKernel(k), "finalize")
        return k


def _oracle(img, thr=128):
    """Gaussian3x3 -> 255 - v -> Threshold(BINARY, thr) on AGO buffers; interior rows/columns."""
    H, W = img.shape
    src = OC.ago_img(H, W); src.set(img)
    g = OC.gaussian3x3(src).get().astype(np.int32)
    return np.where(255 - g > thr, 255, 0).astype(np.uint8)


def _graph(api, ctx, plugin, kernel_name, W, H, flags=None):
    src = api.obj(api.vxCreateImage(ctx, W, H, V.VX_DF_IMAGE_U8), "image")
    dst = api.obj(api.vxCreateImage(ctx, W, H, V.VX_DF_IMAGE_U8), "image")
    g = api.obj(api.vxCreateGraph(ctx), "graph")
    if flags is not None:
        api.set_optimizer_flags(g, flags)
    v1 = api.obj(api.vxCreateVirtualImage(g, W, H, V.VX_DF_IMAGE_U8), "virtual")
    v2 = api.obj(api.vxCreateVirtualImage(g, 0, 0, V.VX_DF_IMAGE_VIRT), "virtual")   # shaped by the validator
    api.obj(api.vxGaussian3x3Node(g, src, v1), "gaussian")
    k = api.obj(api.vxGetKernelByName(ctx, kernel_name.encode()), "kernel")
    node = api.obj(api.vxCreateGenericNode(g, k), "user node")
    api.ok(api.vxSetParameterByIndex(node, 0, v1), "param 0")
    api.ok(api.vxSetParameterByIndex(node, 1, v2), "param 1")
    api.obj(api.vxThresholdNode(g, v2, api.threshold_binary(ctx, 128), dst), "threshold")
    return g, src, dst, node


@pytest.mark.parametrize("gpu", [False, True])
@pytest.mark.parametrize("W,H", [(333, 97), (1920, 1080)])
def test_user_kernel_between_builtin_nodes(cuda, gpu, W, H):
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    plugin = Plugin(api)
    try:
        name = "org.test.invert_dev" if gpu else "org.test.invert_host"
        plugin.publish(ctx, name, INVERT_DEV if gpu else INVERT_HOST, plugin.dev_f if gpu else plugin.host_f,
                       gpu=gpu, local_size=16)
        g, src, dst, node = _graph(api, ctx, plugin, name, W, H)
        api.ok(api.vxVerifyGraph(g), "verify")
        assert plugin.init_calls == 1
        for seed in (1, 2):                                         # two executions, new input each
            img = WL.cfg1_image(seed=seed, width=W, height=H)
            api.write_plane(src, img)
            api.ok(api.vxProcessGraph(g), "process")
            got, want = api.read_plane(dst), _oracle(img)
            np.testing.assert_array_equal(got[1:H - 1, 1:W - 1], want[1:H - 1, 1:W - 1])
        assert plugin.calls == 2
        p = C.c_void_p(0)
        api.ok(api.vxQueryNode(node, V.VX_NODE_LOCAL_DATA_PTR, C.byref(p), C.sizeof(p)), "local ptr")
        n = C.c_size_t(0)
        api.ok(api.vxQueryNode(node, V.VX_NODE_LOCAL_DATA_SIZE, C.byref(n), 8), "local size")
        assert n.value == 16 and p.value
        # init wrote 1000; the host kernel counts its calls there, the device kernel leaves it
        assert C.cast(p, C.POINTER(C.c_uint32))[0] == (1000 if gpu else 1002)
        api.ok(api.vxReleaseGraph(C.byref(C.c_void_p(g))), "release graph")
        assert plugin.deinit_calls == 1
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def test_user_kernel_registration(cuda):
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    plugin = Plugin(api)
    try:
        k = plugin.publish(ctx, "org.test.invert_host", INVERT_HOST, plugin.host_f)
        # names and enumerations are unique, built-in ones included
        assert not api.vxAddUserKernel(ctx, b"org.test.invert_host", INVERT_HOST + 50, C.cast(plugin.host_f, vp), 2,
                                       C.cast(plugin.validate_f, vp), None, None)
        assert not api.vxAddUserKernel(ctx, b"org.khronos.openvx.gaussian_3x3", INVERT_HOST + 51,
                                       C.cast(plugin.host_f, vp), 2, C.cast(plugin.validate_f, vp), None, None)
        assert api.vxGetKernelByEnum(ctx, INVERT_HOST) == k
        for i, (d, t) in enumerate([(V.VX_INPUT, V.VX_TYPE_IMAGE), (V.VX_OUTPUT, V.VX_TYPE_IMAGE)]):
            prm = api.lib.vxGetKernelParameterByIndex
            prm.argtypes, prm.restype = [vp, u32], vp
            q = api.lib.vxQueryParameter
            q.argtypes, q.restype = [vp, C.c_int32, vp, sz], C.c_int32
            h = prm(k, i)
            dv, tv = C.c_int32(0), C.c_int32(0)
            api.ok(q(h, V._attr_base(0, 0x805) + 1, C.byref(dv), 4), "direction")
            api.ok(q(h, V._attr_base(0, 0x805) + 2, C.byref(tv), 4), "type")
            assert (dv.value, tv.value) == (d, t)
        # a kernel with an unset parameter does not finalise and makes no nodes
        k2 = api.vxAddUserKernel(ctx, b"org.test.half", FAILS + 10, C.cast(plugin.host_f, vp), 2,
                                 C.cast(plugin.validate_f, vp), None, None)
        api.ok(api.vxAddParameterToKernel(k2, 0, V.VX_INPUT, V.VX_TYPE_IMAGE, V.VX_PARAMETER_STATE_REQUIRED), "param")
        assert api.vxFinalizeKernel(k2) != 0
        g = api.obj(api.vxCreateGraph(ctx), "graph")
        assert not api.vxCreateGenericNode(g, k2)
        # removed kernels are not found any more
        api.ok(api.vxRemoveKernel(k2), "remove")
        assert not api.vxGetKernelByName(ctx, b"org.test.half")
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def test_user_kernel_failure_abandons_the_graph(cuda):
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    plugin = Plugin(api)
    try:
        plugin.publish(ctx, "org.test.fails", FAILS, plugin.fail_f)
        g, src, dst, node = _graph(api, ctx, plugin, "org.test.fails", 64, 48)
        api.ok(api.vxVerifyGraph(g), "verify")
        api.write_plane(src, WL.cfg1_image(seed=3, width=64, height=48))
        assert api.vxProcessGraph(g) != 0
        st = C.c_int32(0)
        api.ok(api.vxQueryNode(node, V.VX_NODE_STATUS, C.byref(st), 4), "node status")
        assert st.value == -1
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def test_user_kernel_validator_refusal(cuda):
    """The validator sees the input's format: an S16 input fails verification."""
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    plugin = Plugin(api)
    try:
        plugin.publish(ctx, "org.test.invert_host", INVERT_HOST, plugin.host_f)
        g = api.obj(api.vxCreateGraph(ctx), "graph")
        src = api.obj(api.vxCreateImage(ctx, 64, 48, V.VX_DF_IMAGE_S16), "image")
        out = api.obj(api.vxCreateImage(ctx, 64, 48, V.VX_DF_IMAGE_U8), "image")
        node = api.obj(api.vxCreateGenericNode(g, api.vxGetKernelByName(ctx, b"org.test.invert_host")), "node")
        api.ok(api.vxSetParameterByIndex(node, 0, src), "p0")
        api.ok(api.vxSetParameterByIndex(node, 1, out), "p1")
        assert api.vxVerifyGraph(g) != 0
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))
