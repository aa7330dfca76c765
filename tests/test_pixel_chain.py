"""Chains of U8 pixel kernels through virtual images (fused into one pixel-chain kernel on
this target) must equal the kernels applied one by one.

CPU: the reference AGO library runs each chain graph through its own OpenVX API and must
equal the numpy composition (oracle/pixelwise.py) inside the valid rectangle, with the same
rectangle.  GPU: the engine, fused and with fusion off, must equal the composition; the plan
shows which nodes were fused."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from oracle import pixelwise as P
from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL

U8 = V.VX_DF_IMAGE_U8
WRAP, SAT = V.VX_CONVERT_POLICY_WRAP, V.VX_CONVERT_POLICY_SATURATE


def _ref_api():
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    return V.OpenVX(lib)


# Each chain: a list of ops applied to the running value.  ("side", k) operands are extra
# input images; "first" puts the side image first (minuend of a subtraction).
CHAINS = {
    "filters": [("gauss",), ("box",), ("median",), ("dilate",)],
    "elementwise": [("absdiff", 0), ("thr", 40), ("not",), ("and", 1), ("or", 0)],
    "mixed": [("sub", 0, SAT, "first"), ("erode",), ("add", 1, WRAP), ("range", 30, 180), ("median",),
              ("xor", 1), ("sub", 0, WRAP), ("box",)],
    "five_stencils": [("box",), ("dilate",), ("erode",), ("median",), ("gauss",), ("not",)],
    "self_operand": [("box",), ("absdiff", "self"), ("add", 0, SAT)],
}


def _oracle_chain(spec, src, sides):
    v = src
    for op in spec:
        k = op[0]
        if k in ("gauss", "box", "median", "dilate", "erode"):
            v = {"gauss": P.gaussian3x3, "box": P.box3x3, "median": P.median3x3, "dilate": P.dilate3x3,
                 "erode": P.erode3x3}[k](v)
        elif k == "not":
            v = P.logical("not", v)
        elif k == "thr":
            v = P.threshold_binary(v, op[1])
        elif k == "range":
            v = P.threshold_range(v, op[1], op[2])
        elif k in ("and", "or", "xor"):
            v = P.logical(k, v, sides[op[1]])
        elif k == "absdiff":
            v = P.absdiff(v, v if op[1] == "self" else sides[op[1]])
        else:   # add / sub
            o = sides[op[1]]
            a, b = (o, v) if len(op) > 3 and op[3] == "first" else (v, o)
            v = (P.add if k == "add" else P.sub)(a, b, np.uint8, op[2] == SAT)
    return v


def _margin(spec):
    return sum(op[0] in ("gauss", "box", "median", "dilate", "erode") for op in spec)


def build_chain(api, ctx, g, spec, src, sides, dst):
    """Nodes of `spec` from image `src` to image `dst` through virtual images."""
    w, h, _ = api.query_image(src)
    cur = src
    for i, op in enumerate(spec):
        out = dst if i == len(spec) - 1 else api.vxCreateVirtualImage(g, w, h, U8)
        k = op[0]
        if k in ("gauss", "box", "median", "dilate", "erode", "not"):
            f = {"gauss": api.vxGaussian3x3Node, "box": api.vxBox3x3Node, "median": api.vxMedian3x3Node,
                 "dilate": api.vxDilate3x3Node, "erode": api.vxErode3x3Node, "not": api.vxNotNode}[k]
            n = f(g, cur, out)
        elif k == "thr":
            n = api.vxThresholdNode(g, cur, api.threshold_binary(ctx, op[1]), out)
        elif k == "range":
            n = api.vxThresholdNode(g, cur, api.threshold_range(ctx, op[1], op[2]), out)
        elif k in ("and", "or", "xor"):
            f = {"and": api.vxAndNode, "or": api.vxOrNode, "xor": api.vxXorNode}[k]
            n = f(g, cur, sides[op[1]], out)
        elif k == "absdiff":
            n = api.vxAbsDiffNode(g, cur, cur if op[1] == "self" else sides[op[1]], out)
        else:
            f = api.vxAddNode if k == "add" else api.vxSubtractNode
            o = sides[op[1]]
            a, b = (o, cur) if len(op) > 3 and op[3] == "first" else (cur, o)
            n = f(g, a, b, op[2], out)
        api.obj(n, f"node {k}")
        cur = out


def run_chains(api, spec, frames, flags=None):
    """One graph holding the chain once per frame (src, side0, side1); returns the outputs,
    their valid rectangles and the plan (when the library reports one)."""
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        g = api.obj(api.vxCreateGraph(ctx), "graph")
        if flags is not None:
            api.set_optimizer_flags(g, flags)
        outs = []
        for src_a, s0, s1 in frames:
            h, w = src_a.shape
            imgs = []
            for a in (src_a, s0, s1):
                im = api.obj(api.vxCreateImage(ctx, w, h, U8), "image")
                api.write_plane(im, a)
                imgs.append(im)
            dst = api.obj(api.vxCreateImage(ctx, w, h, U8), "image")
            build_chain(api, ctx, g, spec, imgs[0], imgs[1:], dst)
            outs.append(dst)
        api.ok(api.vxVerifyGraph(g), "vxVerifyGraph")
        api.ok(api.vxProcessGraph(g), "vxProcessGraph")
        plan = api.plan(g) if hasattr(api, "plan") else []
        return [(api.read_plane(o), api.valid_region(o)) for o in outs], plan
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def _frames(sizes, seed):
    r = np.random.default_rng(seed)
    out = []
    for w, h in sizes:
        a, b = WL.motion_pair(seed=int(r.integers(1 << 30)), width=w, height=h, rects=max(2, w * h // 20000))
        c = r.integers(0, 256, (h, w), dtype=np.int32).astype(np.uint8)
        out.append((a, b, c))
    return out


def _check(results, spec, frames, u1_tail=False):
    """Outputs equal the composition inside the valid rectangle.  `u1_tail`: skip the columns
    from W - W % 16 - 1 on, where the reference's U1 kernels differ (see below)."""
    m = _margin(spec)
    for (got, rect), (a, s0, s1) in zip(results, frames):
        h, w = a.shape
        # each 3x3 op: start = min(start + 1, size), end = max(end - 1, 0) (e.g. ago_kernel_api.cpp:15033)
        assert rect == (min(m, w), min(m, h), max(w - m, 0), max(h - m, 0))
        want = _oracle_chain(spec, a, (s0, s1))
        e = min(w - m, w - w % 16 - 1) if (u1_tail and w % 16) else w - m
        np.testing.assert_array_equal(got[m:h - m, m:e], want[m:h - m, m:e])


@pytest.mark.parametrize("name", sorted(CHAINS))
def test_reference_chain_matches_oracle(name):
    """AGO turns a virtual U8 image written and read only by Threshold / Not / And / Or /
    Xor / Dilate / Erode into a 1-bit image and runs the U1 kernel variants
    (agoOptimizeDramaRemoveImageU8toU1, ago_drama_remove.cpp:1321).  Those leave wrong pixels
    in the last partial 16-pixel group of a row when W % 16 != 0; everywhere else (and for
    every W % 16 == 0) the reference equals the U8 composition, which this target computes."""
    api = _ref_api()
    frames = _frames([(64, 48), (37, 21), (640, 360), (100, 40)], seed=len(name))
    res, _ = run_chains(api, CHAINS[name], frames)
    _check(res, CHAINS[name], frames, u1_tail=True)


@pytest.mark.parametrize("W,H", [(64, 48), (37, 21), (1920, 1080)])
def test_reference_motion_graph_matches_oracle(W, H):
    api = _ref_api()
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        prev, cur = WL.motion_pair(seed=W + H, width=W, height=H, rects=max(2, W * H // 20000))
        g = WL.MotionGraph(api, ctx, [(W, H)])
        g.run([prev, cur])
        (got, rect), = g.results()
        assert rect == (4, 4, W - 4, H - 4)
        want = P.motion_mask(prev, cur, 24)
        np.testing.assert_array_equal(got[4:H - 4, 4:W - 4], want[4:H - 4, 4:W - 4])
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


EXPECTED_PLAN = {
    "filters": ["fused_PixelChain x{n}"],
    "elementwise": ["fused_PixelChain x{n}"],
    "mixed": ["fused_PixelChain x{n}"],
    # four 3x3 ops per fused kernel: the fifth starts a second chain
    "five_stencils": ["fused_PixelChain x{n}", "fused_PixelChain x{n}"],
}


FORMS = {"tma": None, "cp_async": V.OPT_NO_TMA, "plain": V.OPT_NO_FUSION}


@pytest.mark.gpu
@pytest.mark.parametrize("form", sorted(FORMS))
@pytest.mark.parametrize("name", sorted(CHAINS))
def test_engine_chain(cuda, name, form):
    """Fused chains with tiles staged by TMA tensor copies (the default) or by cp.async, and
    the one-launch-per-node form, all equal the oracle on the valid rectangle."""
    api = V.OpenVX()
    sizes = [(1920, 1080), (37, 21), (640, 360), (129, 67), (8, 3)]
    frames = _frames(sizes, seed=7 * len(name))
    fuse = form != "plain"
    res, plan = run_chains(api, CHAINS[name], frames, flags=FORMS[form])
    _check(res, CHAINS[name], frames)
    names = [s for s, _ in plan]
    if not fuse:
        assert not any("fused" in s for s in names), names
    elif name != "self_operand":
        assert [s for s in names if s.startswith("fused")] == [p.format(n=len(sizes)) for p in EXPECTED_PLAN[name]], names


@pytest.mark.gpu
def test_engine_self_operand_splits_chain(cuda):
    """Box -> AbsDiff(v, v) -> Add: the AbsDiff reads the Box output twice, so the Box output
    is not a private intermediate: Box runs alone, AbsDiff + Add fuse."""
    api = V.OpenVX()
    frames = _frames([(320, 200)], seed=3)
    res, plan = run_chains(api, CHAINS["self_operand"], frames)
    _check(res, CHAINS["self_operand"], frames)
    assert [s for s, _ in plan] == ["Box_U8_U8_3x3", "fused_PixelChain x1"], plan


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [None, V.OPT_NO_TMA, V.OPT_NO_FUSION])
def test_engine_motion_graph(cuda, flags):
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        sizes = [(3840, 2160), (1920, 1080), (640, 480), (37, 21)] + [(1280, 720)] * 7
        pairs = [WL.motion_pair(seed=i + 1, width=w, height=h, rects=max(2, w * h // 20000)) for i, (w, h) in enumerate(sizes)]
        g = WL.MotionGraph(api, ctx, sizes, flags=flags)
        plan = api.plan(g.graph)
        if flags != V.OPT_NO_FUSION:
            assert plan == [("fused_PixelChain x11", 2)], plan
        for rep in range(2):
            g.run([f for p in pairs for f in p])
            for (got, rect), (prev, cur), (w, h) in zip(g.results(), pairs, sizes):
                assert rect == (4, 4, w - 4, h - 4)
                want = P.motion_mask(prev, cur, 24)
                np.testing.assert_array_equal(got[4:h - 4, 4:w - 4], want[4:h - 4, 4:w - 4])
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))
