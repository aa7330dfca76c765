"""Canny + Harris graph (configuration 2) through the OpenVX API.

CPU: the reference AGO library runs the graph and must equal the oracle compositions
(edge map inside the valid rectangle, the corner list and count exactly) -- pins the
graph-level oracle, including lowering (Canny -> 3 nodes, Harris -> 4 nodes).
GPU: this package's engine, fused and plain, must equal the oracle: the edge map over the
whole interior [1, W-1) x [1, H-1) (stronger than the valid region) and the corners
exactly, in the same order."""
import numpy as np
import pytest

import oracle as O
import oracle_chains as OC
from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL


def _check(edges, rect, corners, num, img, interior, capacity=32768):
    h, w = img.shape
    ref_edges, ref_rect = OC.canny(img)
    ref_corners, ref_num = OC.harris(img, capacity=capacity)
    assert rect == ref_rect
    if interior:
        np.testing.assert_array_equal(edges[1:h - 1, 1:w - 1], ref_edges[1:h - 1, 1:w - 1])
    else:
        sx, sy, ex, ey = rect
        np.testing.assert_array_equal(edges[sy:ey, sx:ex], ref_edges[sy:ey, sx:ex])
    assert num == ref_num
    got = corners.view(OC.KP)
    np.testing.assert_array_equal(got, ref_corners)


def noise(W, H, seed):
    """Pure noise: the dense-corner case (hundreds of thousands of Harris candidates)."""
    return np.random.default_rng(seed).integers(0, 256, (H, W), dtype=np.int32).astype(np.uint8)


def _reference_run(img, capacity):
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    api = V.OpenVX(lib)
    ctx = api.obj(api.vxCreateContext(), "context")
    h, w = img.shape
    g = WL.Cfg2Graph(api, ctx, [(w, h)], capacity=capacity)
    g.run([img])
    (edges, rect, corners, num), = g.results()
    _check(edges, rect, corners, num, img, interior=False, capacity=capacity)
    return num


@pytest.mark.parametrize("W,H", [(64, 48), (200, 120), (96, 64)])
def test_reference_graph_matches_oracle(W, H):
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    api = V.OpenVX(lib)
    ctx = api.obj(api.vxCreateContext(), "context")
    img = WL.cfg2_scene(seed=W + H, width=W, height=H, rects=max(3, W * H // 300))
    g = WL.Cfg2Graph(api, ctx, [(W, H)])
    g.run([img])
    (edges, rect, corners, num), = g.results()
    _check(edges, rect, corners, num, img, interior=False)


def test_reference_graph_matches_oracle_full_size_scene():
    """The 3840x2160 configuration-2 scene: the reference library equals the oracle."""
    _reference_run(WL.cfg2_scene(seed=11, width=3840, height=2160, rects=200), 32768)


def test_reference_graph_matches_oracle_full_size_noise():
    """3840x2160 noise: the reference's corner list (sorted and picked from the full
    candidate list) equals the oracle's, all of it."""
    num = _reference_run(noise(3840, 2160, 77), 1 << 19)
    assert num > 100000


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [None, V.OPT_NO_FUSION])
def test_engine_cfg2_noise(cuda, flags):
    """Dense corners through the engine: hundreds of thousands of candidates per frame go to
    the cluster pick; every corner equals the oracle's, in order."""
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    sizes = [(3840, 2160), (1920, 1080)]
    frames = [noise(w, h, 77 + i) for i, (w, h) in enumerate(sizes)]
    g = WL.Cfg2Graph(api, ctx, sizes, flags=flags, capacity=1 << 19)
    for rep in range(2):
        g.run(frames)
        for (edges, rect, corners, num), img in zip(g.results(), frames):
            _check(edges, rect, corners, num, img, interior=True, capacity=1 << 19)


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [None, V.OPT_NO_FUSION])
def test_engine_cfg2(cuda, flags):
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    sizes = [(3840, 2160), (640, 480), (64, 48), (200, 120)]
    frames = [WL.cfg2_scene(seed=i + 11, width=w, height=h, rects=min(200, max(3, w * h // 300)))
              for i, (w, h) in enumerate(sizes)]
    g = WL.Cfg2Graph(api, ctx, sizes, flags=flags)
    plan = api.plan_text(g.graph)
    if flags is None:
        assert "fused_CannyEdgeDetector x4" in plan and "fused_HarrisCorners x4" in plan, plan
    else:
        assert "CannyEdgeTrace_U8_U8XY" in plan and "HarrisMergeSortAndPick_XY_XYS" in plan, plan
    for rep in range(2):
        g.run(frames)
        for (edges, rect, corners, num), img in zip(g.results(), frames):
            _check(edges, rect, corners, num, img, interior=True)
