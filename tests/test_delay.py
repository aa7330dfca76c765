"""Delay objects and graph auto-ageing (vxCreateDelay, vxGetReferenceFromDelay, vxAgeDelay,
vxRegisterAutoAging): the streaming form of the pyramid + LK path.

Two graphs run over several executions:
* an image accumulator: delay[0] = Add(input, delay[-1]) with WRAP, aged after each run;
* a feature tracker: GaussianPyramid(frame t) -> pyramid delay[0];
  OpticalFlowPyrLK(pyramid delay[-1], pyramid delay[0], points delay[-1]) -> points delay[0].
CPU: the reference AGO library must equal the oracle composition execution by execution
(pyramids restated, LK with its node scratch carried across executions).  GPU: the engine
must equal the same oracle; ageing moves device storage, so each execution re-plans."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import test_oracle_pin_flow as PF
from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL

KP = WL.KEYPOINT_DTYPE
U8 = V.VX_DF_IMAGE_U8


def _ref_api():
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    return V.OpenVX(lib)


def accumulate(api, frames):
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        h, w = frames[0].shape
        inp = api.obj(api.vxCreateImage(ctx, w, h, U8), "image")
        ex = api.obj(api.vxCreateImage(ctx, w, h, U8), "image")
        d = api.obj(api.vxCreateDelay(ctx, ex, 3), "delay")
        n = C.c_size_t()
        api.ok(api.vxQueryDelay(d, V._attr_base(0, 0x806) + 1, C.byref(n), C.sizeof(n)), "slots")
        assert n.value == 3
        g = api.obj(api.vxCreateGraph(ctx), "graph")
        api.obj(api.vxAddNode(g, inp, api.vxGetReferenceFromDelay(d, -1), V.VX_CONVERT_POLICY_WRAP,
                              api.vxGetReferenceFromDelay(d, 0)), "node")
        api.ok(api.vxRegisterAutoAging(g, d), "auto ageing")
        api.ok(api.vxVerifyGraph(g), "verify")
        outs = []
        for f in frames:
            api.write_plane(inp, f)
            api.ok(api.vxProcessGraph(g), "process")
            # after ageing the result just written sits at index -1
            outs.append([api.read_plane(api.vxGetReferenceFromDelay(d, -k)) for k in range(3)])
        return outs
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def _check_accumulate(api):
    r = np.random.default_rng(5)
    frames = [r.integers(0, 256, (30, 44), dtype=np.int32).astype(np.uint8) for _ in range(5)]
    outs = accumulate(api, frames)
    acc = [np.zeros_like(frames[0])] * 3          # slots 0, -1, -2 start zeroed
    for f, got in zip(frames, outs):
        new = (f.astype(np.int32) + acc[1]).astype(np.uint8)   # written into slot 0 from slot -1
        acc = [acc[2], new, acc[1]]                              # then aged: 0 <- -2, -1 <- 0, -2 <- -1
        for k in range(3):
            np.testing.assert_array_equal(got[k], acc[k], err_msg=f"slot {-k}")


def test_reference_accumulate():
    _check_accumulate(_ref_api())


@pytest.mark.gpu
def test_engine_accumulate(cuda):
    _check_accumulate(V.OpenVX())


def tracker(api, frames, kp0, levels=4, window=9):
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        h, w = frames[0].shape
        frame = api.obj(api.vxCreateImage(ctx, w, h, U8), "image")
        pex = api.obj(api.vxCreatePyramid(ctx, levels, 0.5, w, h, U8), "pyramid")
        aex = api.obj(api.vxCreateArray(ctx, V.VX_TYPE_KEYPOINT, len(kp0)), "array")
        pd = api.obj(api.vxCreateDelay(ctx, pex, 2), "pyramid delay")
        ad = api.obj(api.vxCreateDelay(ctx, aex, 2), "points delay")
        api.array_set(api.vxGetReferenceFromDelay(ad, -1), kp0)
        g = api.obj(api.vxCreateGraph(ctx), "graph")
        p0, p1 = api.vxGetReferenceFromDelay(pd, -1), api.vxGetReferenceFromDelay(pd, 0)
        a0, a1 = api.vxGetReferenceFromDelay(ad, -1), api.vxGetReferenceFromDelay(ad, 0)
        api.obj(api.vxGaussianPyramidNode(g, frame, p1), "pyramid node")
        api.obj(api.vxOpticalFlowPyrLKNode(g, p0, p1, a0, a0, a1, V.VX_TERM_CRITERIA_BOTH,
                                           api.scalar(ctx, V.VX_TYPE_FLOAT32, 0.01), api.scalar(ctx, V.VX_TYPE_UINT32, 20),
                                           api.scalar(ctx, V.VX_TYPE_BOOL, 0), window), "lk node")
        for dl in (pd, ad):
            api.ok(api.vxRegisterAutoAging(g, dl), "auto ageing")
        api.ok(api.vxVerifyGraph(g), "verify")
        res = []
        for f in frames:
            api.write_plane(frame, f)
            api.ok(api.vxProcessGraph(g), "process")
            res.append(api.array_items(api.vxGetReferenceFromDelay(ad, -1)))   # aged: the new points
        return res
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def oracle_tracker(frames, kp0, levels=4, window=9):
    h, w = frames[0].shape
    scratch = PF.lk_scratch(w, h, len(kp0))
    prev_lv, prev_desc = PF.build_pyramid(np.zeros_like(frames[0]), levels)   # slot -1 starts zeroed
    pts, res = kp0.copy(), []
    for f in frames:
        lv, desc = PF.build_pyramid(f, levels)
        out = np.zeros(len(kp0), KP)
        PF.lk_call("oracle", out, prev_desc, desc, levels, pts, pts, V.VX_TERM_CRITERIA_BOTH, 0.01, 20, 0, w, scratch,
                   window)
        res.append(out.copy())
        pts, prev_lv, prev_desc = out, lv, desc
    return res


def _track_inputs(w, h, n, seed):
    f0, _, _ = WL.cfg4_pair(seed=seed, width=w, height=h)
    frames = [f0]
    for k in range(4):   # a drifting scene: each frame a shifted copy of the previous, plus noise
        f1, f2, _ = WL.cfg4_pair(seed=seed + k + 1, width=w, height=h)
        frames.append(f2)
    return frames, WL.cfg4_points(seed=seed, width=w, height=h, n=n)


def _check_tracker(api, w, h, n, seed):
    frames, kp0 = _track_inputs(w, h, n, seed)
    got = tracker(api, frames, kp0)
    want = oracle_tracker(frames, kp0)
    for t, (a, b) in enumerate(zip(got, want)):
        assert len(a) == len(b)
        np.testing.assert_array_equal(a.view(np.uint8), b.view(np.uint8), err_msg=f"execution {t}")


@pytest.mark.parametrize("W,H", [(160, 120), (331, 217)])
def test_reference_tracker(W, H):
    _check_tracker(_ref_api(), W, H, 300, seed=W)


@pytest.mark.gpu
@pytest.mark.parametrize("W,H", [(160, 120), (331, 217), (1280, 720)])
def test_engine_tracker(cuda, W, H):
    _check_tracker(V.OpenVX(), W, H, 300 if W < 1000 else 2000, seed=W)
