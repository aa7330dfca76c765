"""Pyramid + optical-flow graph (configuration 4) through the OpenVX API.

CPU: the reference AGO library runs the graph (two GaussianPyramid nodes and one
OpticalFlowPyrLK node per frame pair) and must equal the oracle composition keypoint for
keypoint over two executions (the LK node's scratch state carries from one to the next).
GPU: this package's engine, batched and plain, must equal the oracle the same way."""
import numpy as np
import pytest

import oracle as O
import test_oracle_pin_flow as PF
from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL

KP = WL.KEYPOINT_DTYPE


class OracleGraph:
    """The oracle composition of Cfg4Graph, with per-node state kept across executions."""

    def __init__(self, sizes, n, levels, window, iterations, epsilon, term):
        self.levels, self.window, self.iters, self.eps, self.term = levels, window, iterations, epsilon, term
        self.scratch = [PF.lk_scratch(w, h, n) for (w, h) in sizes]
        self.out = [np.zeros(n, KP) for _ in sizes]        # AGO arrays start zeroed

    def run(self, pairs, points):
        res = []
        for i, ((f1, f2), kp) in enumerate(zip(pairs, points)):
            old_lv, od = PF.build_pyramid(f1, self.levels)
            new_lv, nd = PF.build_pyramid(f2, self.levels)
            out = self.out[i][: len(kp)]
            PF.lk_call("oracle", out, od, nd, self.levels, kp, kp, self.term, self.eps, self.iters, 0, f1.shape[1],
                       self.scratch[i], self.window)
            res.append(out.copy())
        return res


def inputs(sizes, execution, n):
    pairs, points = [], []
    for i, (w, h) in enumerate(sizes):
        f1, f2, _ = WL.cfg4_pair(seed=1000 * execution + i, width=w, height=h)
        pairs.append((f1, f2))
        points.append(WL.cfg4_points(seed=1000 * execution + i, width=w, height=h, n=n))
    return pairs, points


def run_and_compare(api, ctx, sizes, n, flags=None, levels=5, window=9, executions=3, virtual=True, host=False):
    """host: frames in page-locked application buffers (images from handles), which the
    CUDA graph uploads itself."""
    keep = []
    if host:
        import torch
        keep = [torch.zeros((h, w), dtype=torch.uint8).pin_memory() for w, h in sizes for _ in range(2)]
    host_io = {"old": [t.numpy() for t in keep[0::2]], "new": [t.numpy() for t in keep[1::2]]} if host else None
    g = WL.Cfg4Graph(api, ctx, sizes, levels=levels, window=window, capacity=n, flags=flags, virtual_pyramids=virtual,
                     host_io=host_io)
    orc = OracleGraph(sizes, n, levels, window, 20, 0.01, V.VX_TERM_CRITERIA_BOTH)
    for e in range(executions):
        pairs, points = inputs(sizes, e, n)
        if host:
            for i, ((f1, f2), kp) in enumerate(zip(pairs, points)):
                keep[2 * i].numpy()[:] = f1
                keep[2 * i + 1].numpy()[:] = f2
                api.array_set(g.pts[i], kp)
        else:
            g.set_inputs(pairs, points)
        g.run()
        got = g.results()
        want = orc.run(pairs, points)
        for i, (a, b) in enumerate(zip(got, want)):
            assert len(a) == len(b) == n
            bad = np.nonzero(a != b)[0]
            assert bad.size == 0, f"execution {e} pair {i} {sizes[i]}: {bad.size} keypoints differ: {a[bad[:3]]} vs {b[bad[:3]]}"
            assert (a["tracking_status"] != 0).sum() > n // 2
    return g


@pytest.mark.parametrize("virtual", [True, False])
def test_reference_graph_matches_oracle(virtual):
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    api = V.OpenVX(lib)
    ctx = api.obj(api.vxCreateContext(), "context")
    run_and_compare(api, ctx, [(320, 240), (160, 120), (256, 200)], 400, levels=4, virtual=virtual)


def test_reference_graph_matches_oracle_full_size():
    """Configuration-4 pairs at 1920x1080 and 3840x2160, 5 levels, 2000 points, two
    executions: the reference library equals the oracle keypoint for keypoint."""
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    api = V.OpenVX(lib)
    ctx = api.obj(api.vxCreateContext(), "context")
    run_and_compare(api, ctx, [(1920, 1080), (3840, 2160)], 2000, executions=2)


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [None, V.OPT_NO_FUSION])
def test_engine_cfg4_full_size(cuda, flags):
    """The engine at the configuration's full frame sizes, 2000 points per pair, three
    executions: every keypoint record equals the oracle's (positions exactly, which is
    inside the 0.01 px bound)."""
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    run_and_compare(api, ctx, [(1920, 1080), (3840, 2160), (1280, 720), (640, 480)], 2000, flags=flags)


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [None, V.OPT_NO_FUSION, V.OPT_NO_GRAPH_CAPTURE])
def test_engine_cfg4(cuda, flags):
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    g = run_and_compare(api, ctx, [(640, 480), (1280, 720), (320, 240), (640, 480)], 2000, flags=flags)
    plan = api.plan_text(g.graph)
    if flags is None:
        # one launch per pyramid level over all frames, one LK batch (prep + track)
        assert "batch_ScaleGaussianHalf x8" in plan and "batch_OpticalFlowPyrLK x4" in plan, plan
        assert "CHANNEL_COPY" not in plan, plan                # level 0 aliases the input frame


@pytest.mark.gpu
def test_engine_cfg4_non_virtual_pyramids(cuda):
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    run_and_compare(api, ctx, [(640, 480), (320, 240)], 1000, virtual=False)


@pytest.mark.gpu
@pytest.mark.parametrize("host", [False, True])
def test_engine_cfg4_launch_groups(cuda, host):
    """11 pairs: the batched pyramid and LK steps launch over groups of 8 pairs, and with
    page-locked frame buffers each group starts as soon as its frames are uploaded."""
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    # sizes with levels of width % 8 >= 3 (320 -> 20, 160 -> 20 / 10): their derivative
    # columns come from the previous execution's level 0 (carried between executions)
    sizes = [[(320, 240), (160, 120), (256, 200)][i % 3] for i in range(11)]
    g = run_and_compare(api, ctx, sizes, 300, host=host)
    plan = dict(api.plan(g.graph))
    assert plan["batch_ScaleGaussianHalf x22"] == 2 and plan["batch_OpticalFlowPyrLK x11"] == 6, plan
