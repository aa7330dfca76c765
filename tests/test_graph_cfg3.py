"""Colour + geometry graph (configuration 3) through the OpenVX API.

CPU: the reference AGO library runs the graph and must equal the oracle composition on every
output plane, with the same valid rectangles.  GPU: this package's engine, fused and plain,
must equal the oracle bit for bit (bilinear warp included: no +-1 tolerance is needed)."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import oracle_chains as OC
from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL

KEYS = ["nv12_y", "nv12_uv", "iyuv_y", "iyuv_u", "iyuv_v", "scale_bilinear", "scale_area", "warp_nearest", "warp_bilinear"]


def _check(got, ref, w, reference_run=False):
    for k in KEYS:
        a, b = got[k], ref[k]
        if k == "scale_area":   # the reference writes the first (W/2 & ~7) columns only
            n = (w // 2) & ~7
            a, b = a[:, :n], b[:, :n]
        if k == "warp_bilinear" and reference_run:
            # the reference reads past its buffer for footprints below the last row
            keep = ~ref["warp_bilinear_undefined_in_reference"]
            a, b = a[keep], b[keep]
        np.testing.assert_array_equal(a, b, err_msg=k)
    for k in ("scale_bilinear", "scale_area", "warp_nearest", "warp_bilinear"):
        assert got[k + "_rect"] == ref[k + "_rect"], k


@pytest.mark.parametrize("W,H", [(64, 48), (200, 120), (3840, 64)])
def test_reference_graph_matches_oracle(W, H):
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    api = V.OpenVX(lib)
    ctx = api.obj(api.vxCreateContext(), "context")
    rgb = WL.cfg3_frame(seed=W + H, width=W, height=H)
    g = WL.Cfg3Graph(api, ctx, [(W, H)])
    g.run([rgb])
    got, = g.results()
    _check(got, OC.color_scale_warp(rgb, g.matrices[0]), W, reference_run=True)


def test_reference_graph_matches_oracle_full_size():
    """A 3840x2160 configuration-3 frame: the reference library equals the oracle."""
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    api = V.OpenVX(lib)
    ctx = api.obj(api.vxCreateContext(), "context")
    rgb = WL.cfg3_frame(seed=5, width=3840, height=2160)
    g = WL.Cfg3Graph(api, ctx, [(3840, 2160)])
    g.run([rgb])
    got, = g.results()
    _check(got, OC.color_scale_warp(rgb, g.matrices[0]), 3840, reference_run=True)


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [None, V.OPT_NO_FUSION])
def test_engine_cfg3(cuda, flags):
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    sizes = [(3840, 2160), (200, 120), (64, 48)]
    frames = [WL.cfg3_frame(seed=i + 5, width=w, height=h) for i, (w, h) in enumerate(sizes)]
    g = WL.Cfg3Graph(api, ctx, sizes, flags=flags)
    plan = api.plan_text(g.graph)
    if flags is None:
        assert "fused_ColorScale x3" in plan, plan
    else:
        assert "ColorConvert_NV12_RGB" in plan and "ScaleImage_U8_U8_Area" in plan, plan
    for rep in range(2):
        g.run(frames)
        for got, rgb, m, (w, h) in zip(g.results(), frames, g.matrices, sizes):
            _check(got, OC.color_scale_warp(rgb, m), w)


@pytest.mark.gpu
def test_engine_cfg3_ragged_widths(cuda):
    """Widths with W % 8 in {2, 4, 6} (the last 8-column group of the fused kernel holds one to
    three blocks, and W % 4 == 2 puts its last block in the scalar tail)."""
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    sizes = [(202, 40), (196, 22), (198, 34), (36, 20), (1926, 38)]
    frames = [WL.cfg3_frame(seed=i + 11, width=w, height=h) for i, (w, h) in enumerate(sizes)]
    g = WL.Cfg3Graph(api, ctx, sizes)
    assert "fused_ColorScale x5" in api.plan_text(g.graph)
    g.run(frames)
    for got, rgb, m, (w, h) in zip(g.results(), frames, g.matrices, sizes):
        _check(got, OC.color_scale_warp(rgb, m), w)


@pytest.mark.gpu
@pytest.mark.parametrize("W,H", [(3840, 64), (200, 24), (202, 18), (198, 12)])
def test_fused_color_scale_vector_and_byte_forms(cuda, W, H):
    """agocuda_fused_ColorScale_RGB with aligned buffers (8-column vector form) and with
    misaligned ones (one thread per 2x2 block): both equal the oracle's planes."""
    from devbuf import DevImg, stream_ptr
    from mivisionx_b200 import native as N
    lib = N.agocuda()
    rgb = WL.cfg3_frame(seed=W + 3 * H, width=W, height=H)
    ref = OC.color_scale_warp(rgb, np.eye(3, 2, dtype=np.float32))
    for off in (0, 1):
        src = DevImg(H, W, channels=3, align_off=off).upload(rgb)
        ny, y2 = DevImg(H, W, align_off=off), DevImg(H, W, align_off=off)
        nuv = DevImg(H // 2, W // 2, channels=2, align_off=off)
        u, v, sb, sa = (DevImg(H // 2, W // 2, align_off=off) for _ in range(4))
        rc = lib.agocuda_fused_ColorScale_RGB(C.c_void_p(stream_ptr()), W, H, C.c_void_p(src.ptr), src.stride,
                                              C.c_void_p(ny.ptr), ny.stride, C.c_void_p(nuv.ptr), nuv.stride,
                                              C.c_void_p(y2.ptr), y2.stride, C.c_void_p(u.ptr), u.stride,
                                              C.c_void_p(v.ptr), v.stride, C.c_void_p(sb.ptr), sb.stride,
                                              C.c_void_p(sa.ptr), sa.stride)
        assert rc == 0
        n = (W // 2) & ~7
        np.testing.assert_array_equal(ny.download(), ref["nv12_y"], err_msg=f"nv12_y off {off}")
        np.testing.assert_array_equal(nuv.download(), ref["nv12_uv"], err_msg=f"nv12_uv off {off}")
        np.testing.assert_array_equal(y2.download(), ref["iyuv_y"], err_msg=f"iyuv_y off {off}")
        np.testing.assert_array_equal(u.download(), ref["iyuv_u"], err_msg=f"u off {off}")
        np.testing.assert_array_equal(v.download(), ref["iyuv_v"], err_msg=f"v off {off}")
        np.testing.assert_array_equal(sb.download(), ref["scale_bilinear"], err_msg=f"bilinear off {off}")
        np.testing.assert_array_equal(sa.download()[:, :n], ref["scale_area"][:, :n], err_msg=f"area off {off}")
