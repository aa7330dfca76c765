"""ChannelExtract (RGB, RGBX, NV12, NV21, IYUV, YUV4, UYVY, YUYV) and ChannelCombine (RGB,
RGBX, UYVY, YUYV, NV12, NV21, IYUV, YUV4) through the OpenVX API.

CPU: the reference AGO library runs each one-node graph and must equal the numpy
restatement below (plain byte shuffles of ago_haf_cpu_ch_extract_combine.cpp), with the same
valid rectangle.  GPU: the engine must equal it byte for byte."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from mivisionx_b200 import vx as V

F = {"RGB": V.VX_DF_IMAGE_RGB, "RGBX": V.VX_DF_IMAGE_RGBX, "NV12": V.VX_DF_IMAGE_NV12, "NV21": V._df('N', 'V', '2', '1'),
     "IYUV": V.VX_DF_IMAGE_IYUV, "YUV4": V._df('Y', 'U', 'V', '4'), "UYVY": V._df('U', 'Y', 'V', 'Y'),
     "YUYV": V._df('Y', 'U', 'Y', 'V')}
CH = {"R": V._enum_base(0, 0x09) + 0x10, "G": V._enum_base(0, 0x09) + 0x11, "B": V._enum_base(0, 0x09) + 0x12,
      "A": V._enum_base(0, 0x09) + 0x13, "Y": V._enum_base(0, 0x09) + 0x14, "U": V._enum_base(0, 0x09) + 0x15,
      "V": V._enum_base(0, 0x09) + 0x16}
CHANNELS = {"RGB": "RGB", "RGBX": "RGBA", "NV12": "YUV", "NV21": "YUV", "IYUV": "YUV", "YUV4": "YUV", "UYVY": "YUV",
            "YUYV": "YUV"}


def _ref_api():
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    return V.OpenVX(lib)


def planes_of(fmt, w, h, rng):
    """Random pixel planes of a `fmt` image (interleaved formats as (rows, width, bytes))."""
    u = lambda *s: rng.integers(0, 256, s, dtype=np.int32).astype(np.uint8)
    h2, w2 = h // 2, w // 2
    return {"RGB": [u(h, w, 3)], "RGBX": [u(h, w, 4)], "NV12": [u(h, w), u(h2, w2, 2)], "NV21": [u(h, w), u(h2, w2, 2)],
            "IYUV": [u(h, w), u(h2, w2), u(h2, w2)], "YUV4": [u(h, w), u(h, w), u(h, w)], "UYVY": [u(h, w, 2)],
            "YUYV": [u(h, w, 2)]}[fmt]


def extract_oracle(fmt, planes, ch):
    p = planes
    if fmt in ("RGB", "RGBX"):
        return p[0][..., "RGBA".index(ch)]
    if fmt in ("NV12", "NV21"):
        if ch == "Y":
            return p[0]
        return p[1][..., ("UV" if fmt == "NV12" else "VU").index(ch)]
    if fmt in ("IYUV", "YUV4"):
        return p["YUV".index(ch)]
    flat = p[0].reshape(p[0].shape[0], -1)       # UYVY / YUYV bytes of a row
    if fmt == "UYVY":
        return {"Y": flat[:, 1::2], "U": flat[:, 0::4], "V": flat[:, 2::4]}[ch]
    return {"Y": flat[:, 0::2], "U": flat[:, 1::4], "V": flat[:, 3::4]}[ch]


def combine_oracle(fmt, ins):
    """Expected planes of the combined image from the U8 input planes."""
    if fmt in ("RGB", "RGBX"):
        return [np.stack(ins, axis=-1)]
    if fmt in ("NV12", "NV21"):
        uv = np.stack(ins[1:] if fmt == "NV12" else ins[:0:-1], axis=-1)
        return [ins[0], uv]
    if fmt in ("IYUV", "YUV4"):
        return list(ins)
    y, u, v = ins
    h, w = y.shape
    out = np.zeros((h, w, 2), np.uint8)
    flat = out.reshape(h, -1)
    if fmt == "UYVY":
        flat[:, 0::4], flat[:, 1::2], flat[:, 2::4] = u, y, v
    else:
        flat[:, 1::4], flat[:, 0::2], flat[:, 3::4] = u, y, v
    return [out]


def _read(api, img, fmt, plane, w, h):
    if fmt in ("RGB", "RGBX"):
        return api.read_plane(img, 0, np.uint8, 3 if fmt == "RGB" else 4, (h, w))
    if fmt in ("UYVY", "YUYV"):
        return api.read_plane(img, 0, np.uint8, 2, (h, w))
    if fmt in ("NV12", "NV21"):
        return api.read_plane(img, plane, np.uint8, 2 if plane else 1, (h // 2, w // 2) if plane else (h, w))
    if fmt == "IYUV" and plane:
        return api.read_plane(img, plane, np.uint8, 1, (h // 2, w // 2))
    return api.read_plane(img, plane, np.uint8, 1, (h, w))


def run_extract(api, fmt, ch, w, h, planes):
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        src = api.obj(api.vxCreateImage(ctx, w, h, F[fmt]), "image")
        for k, a in enumerate(planes):
            api.write_plane(src, a, k)
        ow = w // 2 if ch in "UV" and fmt in ("NV12", "NV21", "IYUV", "UYVY", "YUYV") else w
        oh = h // 2 if ch in "UV" and fmt in ("NV12", "NV21", "IYUV") else h
        dst = api.obj(api.vxCreateImage(ctx, ow, oh, V.VX_DF_IMAGE_U8), "image")
        g = api.obj(api.vxCreateGraph(ctx), "graph")
        api.obj(api.vxChannelExtractNode(g, src, CH[ch], dst), "node")
        api.ok(api.vxVerifyGraph(g), "verify")
        api.ok(api.vxProcessGraph(g), "process")
        return api.read_plane(dst), api.valid_region(dst)
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


def run_combine(api, fmt, w, h, ins):
    ctx = api.obj(api.vxCreateContext(), "context")
    try:
        imgs = []
        for a in ins:
            im = api.obj(api.vxCreateImage(ctx, a.shape[1], a.shape[0], V.VX_DF_IMAGE_U8), "image")
            api.write_plane(im, a)
            imgs.append(im)
        while len(imgs) < 4:
            imgs.append(None)
        dst = api.obj(api.vxCreateImage(ctx, w, h, F[fmt]), "image")
        g = api.obj(api.vxCreateGraph(ctx), "graph")
        api.obj(api.vxChannelCombineNode(g, *imgs, dst), "node")
        api.ok(api.vxVerifyGraph(g), "verify")
        api.ok(api.vxProcessGraph(g), "process")
        nplanes = {"NV12": 2, "NV21": 2, "IYUV": 3, "YUV4": 3}.get(fmt, 1)
        return [_read(api, dst, fmt, k, w, h) for k in range(nplanes)], api.valid_region(dst)
    finally:
        api.vxReleaseContext(C.byref(C.c_void_p(ctx)))


EXTRACT = [(f, c) for f, cs in CHANNELS.items() for c in cs]
COMBINE = list(F)
SIZES = [(64, 48), (38, 22), (1920, 1080)]


def _combine_inputs(fmt, w, h, rng):
    u = lambda *s: rng.integers(0, 256, s, dtype=np.int32).astype(np.uint8)
    if fmt in ("RGB",):
        return [u(h, w) for _ in range(3)]
    if fmt == "RGBX":
        return [u(h, w) for _ in range(4)]
    if fmt in ("NV12", "NV21", "IYUV"):
        return [u(h, w), u(h // 2, w // 2), u(h // 2, w // 2)]
    if fmt in ("UYVY", "YUYV"):
        return [u(h, w), u(h, w // 2), u(h, w // 2)]
    return [u(h, w) for _ in range(3)]


def _check_extract(api, fmt, ch, W, H):
    rng = np.random.default_rng(W * 7 + len(fmt) + ord(ch))
    planes = planes_of(fmt, W, H, rng)
    got, rect = run_extract(api, fmt, ch, W, H, planes)
    want = extract_oracle(fmt, planes, ch)
    assert got.shape == want.shape
    np.testing.assert_array_equal(got, want)
    return rect


def _check_combine(api, fmt, W, H):
    rng = np.random.default_rng(W * 5 + len(fmt))
    ins = _combine_inputs(fmt, W, H, rng)
    got, rect = run_combine(api, fmt, W, H, ins)
    for g, wnt in zip(got, combine_oracle(fmt, ins)):
        np.testing.assert_array_equal(g.reshape(wnt.shape), wnt)
    return rect


@pytest.mark.parametrize("W,H", SIZES)
@pytest.mark.parametrize("fmt,ch", EXTRACT)
def test_reference_extract(fmt, ch, W, H):
    rect = _check_extract(_ref_api(), fmt, ch, W, H)
    assert rect[0] == 0 and rect[1] == 0


@pytest.mark.parametrize("W,H", SIZES)
@pytest.mark.parametrize("fmt", COMBINE)
def test_reference_combine(fmt, W, H):
    _check_combine(_ref_api(), fmt, W, H)


def expected_extract_rect(fmt, ch, W, H):
    """The reference's valid rectangle (pinned by test_reference_extract_rect): the input's
    rectangle (ago_kernel_api.cpp:10708, :10868, :11054), i.e. the chroma plane's for
    NV12 / NV21 / IYUV U and V, the whole image otherwise -- also for YUYV / UYVY U and V,
    whose outputs are half as wide."""
    if ch in "UV" and fmt in ("NV12", "NV21", "IYUV"):
        return (0, 0, W // 2, H // 2)
    return (0, 0, W, H)


@pytest.mark.parametrize("fmt,ch", EXTRACT)
def test_reference_extract_rect(fmt, ch):
    W, H = 38, 22
    rect = run_extract(_ref_api(), fmt, ch, W, H, planes_of(fmt, W, H, np.random.default_rng(1)))[1]
    assert rect == expected_extract_rect(fmt, ch, W, H)


@pytest.mark.parametrize("fmt", COMBINE)
def test_reference_combine_rect(fmt):
    W, H = 38, 22
    assert run_combine(_ref_api(), fmt, W, H, _combine_inputs(fmt, W, H, np.random.default_rng(1)))[1] == (0, 0, W, H)


@pytest.mark.gpu
@pytest.mark.parametrize("W,H", SIZES + [(3840, 2160), (6, 4)])
@pytest.mark.parametrize("fmt,ch", EXTRACT)
def test_engine_extract(cuda, fmt, ch, W, H):
    assert _check_extract(V.OpenVX(), fmt, ch, W, H) == expected_extract_rect(fmt, ch, W, H)


@pytest.mark.gpu
@pytest.mark.parametrize("W,H", SIZES + [(3840, 2160), (6, 4)])
@pytest.mark.parametrize("fmt", COMBINE)
def test_engine_combine(cuda, fmt, W, H):
    assert _check_combine(V.OpenVX(), fmt, W, H) == (0, 0, W, H)
