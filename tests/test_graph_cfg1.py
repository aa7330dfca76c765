"""Graph-level parity of the Gaussian -> Sobel -> Magnitude -> ConvertDepth -> Threshold graph
(configuration 1) through the OpenVX API.

CPU: the reference AGO library (built from source) runs the graph through its own OpenVX
API and must equal the oracle composition, including the valid rectangle -- this pins the
graph-level oracle (lowering + SOBEL+MAGNITUDE merge + valid-rect propagation).
GPU: this package's engine, fused+batched and plain, must equal the oracle bit for bit
inside the valid rectangle."""
import numpy as np
import pytest

import oracle as O
import oracle_chains as OC
from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL


def _ref_api():
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    return V.OpenVX(lib)


@pytest.mark.parametrize("W,H", [(64, 48), (37, 21), (1920, 1080)])
@pytest.mark.parametrize("shift,thr", [(0, 128), (1, 60)])
def test_reference_graph_matches_oracle(W, H, shift, thr):
    api = _ref_api()
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        img = WL.cfg1_image(seed=W * 7 + H, width=W, height=H)
        g = WL.Cfg1Graph(api, ctx, [(W, H)], shift, thr)
        g.run([img])
        (out, rect), = g.results()
        ref, ref_rect = OC.cfg1_chain(img, shift, thr)
        assert rect == ref_rect == (2, 2, W - 2, H - 2)
        sx, sy, ex, ey = rect
        np.testing.assert_array_equal(out[sy:ey, sx:ex], ref[sy:ey, sx:ex])
    finally:
        api.vxReleaseContext(np.ctypeslib.ctypes.byref(np.ctypeslib.ctypes.c_void_p(ctx)))


def test_pcg32_known_answer():
    # pcg32_srandom_r(42, 54) then pcg32_random_r: the first outputs of O'Neill's demo
    out = WL.pcg32(42, 6, stream=54)
    assert [hex(int(v)) for v in out] == ["0xa15c02b7", "0x7b47f409", "0xba1d3330", "0x83d2f293", "0xbfa4784b", "0xcbed606e"]


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [None, V.OPT_NO_FUSION, V.OPT_NO_GRAPH_CAPTURE, V.OPT_NO_TMA])
def test_engine_cfg1_uneven_batch(cuda, flags):
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    sizes = [(1920, 1080), (640, 480), (37, 21), (130, 66)]
    frames = [WL.cfg1_image(seed=i + 3, width=w, height=h) for i, (w, h) in enumerate(sizes)]
    g = WL.Cfg1Graph(api, ctx, sizes, 0, 128, flags=flags)
    plan = api.plan_text(g.graph)
    if flags in (None, V.OPT_NO_GRAPH_CAPTURE, V.OPT_NO_TMA):
        assert plan.strip() == "fused_GaussSobelMagDepthThresh x4", plan
    else:
        assert "SobelMagnitude_S16_U8_3x3" in plan and "fused" not in plan, plan
    for rep in range(2):
        g.run(frames)
        for (out, rect), img in zip(g.results(), frames):
            ref, ref_rect = OC.cfg1_chain(img, 0, 128)
            assert rect == ref_rect
            sx, sy, ex, ey = rect
            np.testing.assert_array_equal(out[sy:ey, sx:ex], ref[sy:ey, sx:ex])


@pytest.mark.gpu
def test_engine_param_change_replans(cuda):
    """Changing the shift scalar after verify must take effect (captured graph re-planned)."""
    import ctypes as C
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    img = WL.cfg1_image(seed=5, width=256, height=64)
    g = WL.Cfg1Graph(api, ctx, [(256, 64)], 0, 40)
    g.run([img])
    v = C.c_int32(2)
    api.ok(api.vxCopyScalar(g.shift, C.byref(v), V.VX_WRITE_ONLY, V.VX_MEMORY_TYPE_HOST), "copy scalar")
    g.run([img])
    (out, rect), = g.results()
    ref, _ = OC.cfg1_chain(img, 2, 40)
    sx, sy, ex, ey = rect
    np.testing.assert_array_equal(out[sy:ey, sx:ex], ref[sy:ey, sx:ex])
