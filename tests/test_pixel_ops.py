"""Element-wise kernels (Add, Subtract, AbsDiff, And, Or, Xor, Not, Threshold RANGE) and the
3x3 Box / Median / Dilate / Erode filters, through the OpenVX API.

CPU: the reference AGO library (built from source) runs each one-node graph and must equal
the numpy restatement (oracle/pixelwise.py) inside the valid rectangle, with the same valid
rectangle -- this pins the oracle, including the lowering of every U8/S16 operand mix.
GPU: this package's engine must equal the oracle bit for bit inside the valid rectangle."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from oracle import pixelwise as P
from mivisionx_b200 import vx as V

U8, S16 = V.VX_DF_IMAGE_U8, V.VX_DF_IMAGE_S16
WRAP, SAT = V.VX_CONVERT_POLICY_WRAP, V.VX_CONVERT_POLICY_SATURATE
SIZES = [(64, 48), (37, 21), (1920, 1080)]


def _ref_api():
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    return V.OpenVX(lib)


def _data(fmt, w, h, seed):
    """Random planes with the extremes of the type well represented."""
    r = np.random.default_rng(seed)
    if fmt == U8:
        a = r.integers(0, 256, (h, w), dtype=np.int32)
        a[r.random((h, w)) < 0.05] = 0
        a[r.random((h, w)) < 0.05] = 255
        return a.astype(np.uint8)
    a = r.integers(-32768, 32768, (h, w), dtype=np.int32)
    m = r.random((h, w))
    a[m < 0.05] = -32768
    a[(m >= 0.05) & (m < 0.1)] = 32767
    a[(m >= 0.1) & (m < 0.3)] = r.integers(-300, 300, int(((m >= 0.1) & (m < 0.3)).sum()))
    return a.astype(np.int16)


def _smooth(w, h, seed):
    """U8 scene with flat areas and ties (median / morphology edge cases)."""
    r = np.random.default_rng(seed)
    base = (np.arange(w)[None, :] // 7 * 9 + np.arange(h)[:, None] // 5 * 13) % 256
    noise = r.integers(-2, 3, (h, w))
    img = np.clip(base + noise, 0, 255).astype(np.uint8)
    img[r.random((h, w)) < 0.02] = 255
    return img


# (case id, operation, policy / threshold bounds, input formats, output format, oracle)
def _cases():
    out = []
    for pol, pn in ((WRAP, "wrap"), (SAT, "sat")):
        for fa, fb, fo in ((U8, U8, U8), (U8, U8, S16), (S16, U8, S16), (U8, S16, S16), (S16, S16, S16)):
            dt = np.uint8 if fo == U8 else np.int16
            for op, fn in (("add", P.add), ("sub", P.sub)):
                out.append((f"{op}_{pn}_{fa:x}_{fb:x}_{fo:x}", op, pol, (fa, fb), fo,
                            lambda a, b, fn=fn, dt=dt, s=pol == SAT: fn(a, b, dt, s)))
    out.append(("absdiff_u8", "absdiff", None, (U8, U8), U8, P.absdiff))
    out.append(("absdiff_s16", "absdiff", None, (S16, S16), S16, P.absdiff))
    for op in ("and", "or", "xor"):
        out.append((op, op, None, (U8, U8), U8, lambda a, b, op=op: P.logical(op, a, b)))
    out.append(("not", "not", None, (U8,), U8, lambda a: P.logical("not", a)))
    for op, fn in (("box", P.box3x3), ("median", P.median3x3), ("dilate", P.dilate3x3), ("erode", P.erode3x3)):
        out.append((op, op, None, (U8,), U8, fn))
    for shift in (0, 3, 7):
        out.append((f"depth_wrap_{shift}", "depth", (WRAP, shift), (S16,), U8,
                    lambda a, s=shift: P.convert_depth(a, np.uint8, False, s)))
        out.append((f"depth_sat_{shift}", "depth", (SAT, shift), (S16,), U8,
                    lambda a, s=shift: P.convert_depth(a, np.uint8, True, s)))
        out.append((f"depth_up_{shift}", "depth", (WRAP, shift), (U8,), S16,
                    lambda a, s=shift: P.convert_depth(a, np.int16, False, s)))
    tab8 = np.random.default_rng(11).integers(0, 256, 256).astype(np.uint8)
    tab16 = np.random.default_rng(12).integers(-32768, 32768, 65536).astype(np.int16)
    out.append(("lut_u8", "lut", (V.VX_TYPE_UINT8, tab8), (U8,), U8, lambda a, t=tab8: P.table_lookup(a, t)))
    out.append(("lut_s16", "lut", (V.VX_TYPE_INT16, tab16), (S16,), S16, lambda a, t=tab16: P.table_lookup(a, t, 32768)))
    out.append(("integral", "integral", None, (U8,), V.VX_DF_IMAGE_U32, P.integral_image))
    out.append(("range", "range", (37, 201), (U8,), U8, lambda a: P.threshold_range(a, 37, 201)))
    out.append(("range_empty", "range", (200, 100), (U8,), U8, lambda a: P.threshold_range(a, 200, 100)))
    return out


CASES = _cases()
NEIGHBOUR = {"box", "median", "dilate", "erode"}


def _node(api, ctx, g, op, extra, ins, out):
    if op in ("add", "sub"):
        f = api.vxAddNode if op == "add" else api.vxSubtractNode
        return f(g, ins[0], ins[1], extra, out)
    if op in ("absdiff", "and", "or", "xor"):
        f = {"absdiff": api.vxAbsDiffNode, "and": api.vxAndNode, "or": api.vxOrNode, "xor": api.vxXorNode}[op]
        return f(g, ins[0], ins[1], out)
    if op == "range":
        return api.vxThresholdNode(g, ins[0], api.threshold_range(ctx, *extra), out)
    if op == "integral":
        return api.vxIntegralImageNode(g, ins[0], out)
    if op == "lut":
        lut = api.obj(api.vxCreateLUT(ctx, extra[0], len(extra[1])), "lut")
        tab = np.ascontiguousarray(extra[1])
        api.ok(api.vxCopyLUT(lut, tab.ctypes.data, V.VX_WRITE_ONLY, V.VX_MEMORY_TYPE_HOST), "vxCopyLUT")
        return api.vxTableLookupNode(g, ins[0], lut, out)
    if op == "depth":
        return api.vxConvertDepthNode(g, ins[0], out, extra[0], api.scalar(ctx, V.VX_TYPE_INT32, extra[1]))
    f = {"not": api.vxNotNode, "box": api.vxBox3x3Node, "median": api.vxMedian3x3Node,
         "dilate": api.vxDilate3x3Node, "erode": api.vxErode3x3Node}[op]
    return f(g, ins[0], out)


def run_node(api, op, extra, fmts, fo, arrays):
    """One-node graph over fresh images; returns the output plane and its valid rectangle."""
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        h, w = arrays[0].shape
        ins = []
        for f, a in zip(fmts, arrays):
            im = api.obj(api.vxCreateImage(ctx, w, h, f), "image")
            api.write_plane(im, a)
            ins.append(im)
        out = api.obj(api.vxCreateImage(ctx, w, h, fo), "image")
        g = api.obj(api.vxCreateGraph(ctx), "graph")
        api.obj(_node(api, ctx, g, op, extra, ins, out), "node")
        api.ok(api.vxVerifyGraph(g), "vxVerifyGraph")
        api.ok(api.vxProcessGraph(g), "vxProcessGraph")
        return api.read_plane(out), api.valid_region(out)
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def _inputs(name, fmts, w, h):
    if name in NEIGHBOUR:
        return [_smooth(w, h, w + h)]
    return [_data(f, w, h, 17 * i + w * 3 + h) for i, f in enumerate(fmts)]


def _check(name, got, rect, want, w, h):
    exp_rect = (1, 1, w - 1, h - 1) if name in NEIGHBOUR else (0, 0, w, h)
    assert rect == exp_rect, (name, rect)
    sx, sy, ex, ey = rect
    np.testing.assert_array_equal(got[sy:ey, sx:ex], want[sy:ey, sx:ex], err_msg=name)


@pytest.mark.parametrize("W,H", SIZES)
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_reference_matches_oracle(case, W, H):
    name, op, extra, fmts, fo, fn = case
    if name == "lut_s16" and W % 8:
        # HafCpu_Lut_S16_S16 walks the planes as if rows had no padding (it never applies the
        # strides), so its rows are misplaced unless the 16-byte-aligned stride equals 2 W
        pytest.skip("reference S16 table lookup ignores the row stride when W % 8 != 0")
    api = _ref_api()
    arrays = _inputs(op, fmts, W, H)
    got, rect = run_node(api, op, extra, fmts, fo, arrays)
    _check(op, got, rect, fn(*arrays), W, H)


def test_median_and_box_identities():
    """The device kernels compute the median as med3(max of column minima, med3 of column
    medians, min of column maxima) and the box mean as (sum * 7282) >> 16: both equal the
    definitions (sorted middle, floor(sum / 9)) -- on every 3x3 window over a small
    alphabet (ties everywhere) and on random byte windows."""
    s = np.arange(2296)
    assert np.array_equal((s * 7282) >> 16, s // 9)
    r = np.random.default_rng(3)
    win = np.concatenate([r.integers(0, 4, (200000, 3, 3)), r.integers(0, 256, (200000, 3, 3))])
    col = np.sort(win, axis=1)                     # each column sorted top to bottom
    lo, mid, hi = col[:, 0, :].max(axis=1), np.sort(col[:, 1, :], axis=1)[:, 1], col[:, 2, :].min(axis=1)
    med = np.sort(np.stack([lo, mid, hi], axis=1), axis=1)[:, 1]
    assert np.array_equal(med, np.sort(win.reshape(-1, 9), axis=1)[:, 4])


def _invalid_formats_fail(api):
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        a = api.obj(api.vxCreateImage(ctx, 32, 16, S16), "image")
        b = api.obj(api.vxCreateImage(ctx, 32, 16, U8), "image")
        o = api.obj(api.vxCreateImage(ctx, 32, 16, U8), "image")
        for make in (lambda g: api.vxAndNode(g, a, b, o), lambda g: api.vxAddNode(g, a, b, SAT, o),
                     lambda g: api.vxBox3x3Node(g, a, o)):
            g = api.obj(api.vxCreateGraph(ctx), "graph")
            api.obj(make(g), "node")
            assert api.vxVerifyGraph(g) != V.VX_SUCCESS
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def test_invalid_formats_fail_verification_reference():
    """Format rules of the reference validators (ago_kernel_api.cpp ovxKernel_And :1473,
    ovxKernel_Add :1681, ovxKernel_Box3x3 :1052): logical ops and filters take U8 only;
    S16 + U8 cannot write a U8 image."""
    _invalid_formats_fail(_ref_api())


@pytest.mark.gpu
def test_invalid_formats_fail_verification(cuda):
    _invalid_formats_fail(V.OpenVX())


@pytest.mark.gpu
@pytest.mark.parametrize("W,H", SIZES + [(3840, 2160), (8, 3)])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_engine_matches_oracle(cuda, case, W, H):
    name, op, extra, fmts, fo, fn = case
    api = V.OpenVX()
    arrays = _inputs(op, fmts, W, H)
    got, rect = run_node(api, op, extra, fmts, fo, arrays)
    _check(op, got, rect, fn(*arrays), W, H)


@pytest.mark.gpu
def test_engine_chain_with_virtual_images(cuda):
    """Median -> AbsDiff(with the input) -> Add(S16, virtual) -> Subtract -> Not: virtual
    intermediates take the inferred formats and the valid rectangles compose."""
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        w, h = 640, 360
        src = _smooth(w, h, 9)
        i0 = api.obj(api.vxCreateImage(ctx, w, h, U8), "image")
        api.write_plane(i0, src)
        out = api.obj(api.vxCreateImage(ctx, w, h, U8), "image")
        g = api.obj(api.vxCreateGraph(ctx), "graph")
        m = api.vxCreateVirtualImage(g, 0, 0, V.VX_DF_IMAGE_VIRT)
        d = api.vxCreateVirtualImage(g, 0, 0, V.VX_DF_IMAGE_VIRT)
        s16 = api.vxCreateVirtualImage(g, 0, 0, V.VX_DF_IMAGE_VIRT)
        e = api.vxCreateVirtualImage(g, w, h, U8)
        api.obj(api.vxMedian3x3Node(g, i0, m), "node")
        api.obj(api.vxAbsDiffNode(g, m, i0, d), "node")
        api.obj(api.vxAddNode(g, d, m, WRAP, s16), "node")          # U8 + U8 into an unset virtual: S16
        api.obj(api.vxSubtractNode(g, i0, d, SAT, e), "node")
        api.obj(api.vxNotNode(g, e, out), "node")
        api.ok(api.vxVerifyGraph(g), "verify")
        api.ok(api.vxProcessGraph(g), "process")
        assert api.query_image(s16)[2] == S16
        med = P.median3x3(src)
        diff = P.absdiff(med, src)
        want = P.logical("not", P.sub(src, diff, np.uint8, True))
        got, rect = api.read_plane(out), api.valid_region(out)
        assert rect == (1, 1, w - 1, h - 1)
        np.testing.assert_array_equal(got[1:-1, 1:-1], want[1:-1, 1:-1])
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))
