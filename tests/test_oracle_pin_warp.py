"""Pin the WarpPerspective and Remap restatements (oracle/agooracle_geometry.c) to the
reference HAF CPU kernels built from the reference sources, on AGO-layout buffers.

Matrices include projections that send parts of the image outside the source, negative
integer source coordinates (the bilinear kernel's floor is trunc - (x < 0)) and a vanishing
denominator; remap tables come from the oracle's restatement of vxSetRemapPoint's
fixed-point conversion (pinned at graph level in test_graph_warp.py) and include 0xFFFF
border entries and widths with a scalar tail (W % 4 != 0)."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from imgbuf import Img

u32, vp, u8 = C.c_uint32, C.c_void_p, C.c_uint8


def ago_img(h, w):
    return Img(h, w, np.uint8, stride=((w + 15) // 16) * 16, pad=4, align_off=0)


def perspective(kind, W, H, rng):
    """ago_perspective_matrix_t as 9 floats: x' = (m0 x + m3 y + m6) / (m2 x + m5 y + m8)."""
    if kind == "identity":
        m = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1], np.float32)
    elif kind == "mild":
        m = np.array([0.9, 0.05, 1e-4, -0.04, 1.05, 2e-4, 3.5, -2.25, 1.0], np.float32)
    elif kind == "outside":            # shifts part of the output outside the source, negative coordinates
        m = np.array([1.1, -0.2, 5e-4, 0.3, 0.95, -3e-4, -W * 0.3, -H * 0.2, 1.0], np.float32)
    elif kind == "integer_negative":   # integer source coordinates down to -8
        m = np.array([1, 0, 0, 0, 1, 0, -8, -4, 1], np.float32)
    elif kind == "vanishing":          # denominator crosses 0 inside the image
        m = np.array([1.0, 0.0, -2.0 / W, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0], np.float32)
    else:
        m = (rng.standard_normal(9) * [0.2, 0.2, 1e-3, 0.2, 0.2, 1e-3, 10, 10, 0.1] + [1, 0, 0, 0, 1, 0, 0, 0, 1]).astype(np.float32)
    return m


@pytest.mark.parametrize("kind", ["identity", "mild", "outside", "integer_negative", "vanishing", "random"])
@pytest.mark.parametrize("W,H", [(64, 48), (100, 37), (200, 120)])
@pytest.mark.parametrize("interp", ["Nearest", "Bilinear"])
def test_warp_perspective_matches_reference(ref, kind, W, H, interp):
    rng = np.random.default_rng(W * 31 + H)
    src = ago_img(H, W)
    src.set(rng.integers(0, 256, (H, W), dtype=np.uint8))
    m = perspective(kind, W, H, rng)
    for border in (0, 77):
        outs = []
        for impl in ("ref", "oracle"):
            dst = ago_img(H, W)
            local = np.zeros(3 * ((W + 15) // 16) * 16 * 4 + 256, np.uint8)
            lp = local.ctypes.data + (-local.ctypes.data % 64)
            args = [W, H, dst.ptr, dst.stride, W, H, src.ptr, src.stride, m.ctypes.data]
            name = f"WarpPerspective_U8_U8_{interp}_Constant"
            if impl == "ref":
                f = O.ref_haf(f"HafCpu_{name}")
                f.argtypes, f.restype = [u32, u32, vp, u32, u32, u32, vp, u32, vp, u8, vp], C.c_int
                assert f(*args, border, lp) == 0
            else:
                g = getattr(O.oracle_lib(), "oracle_" + name)
                g.argtypes, g.restype = [u32, u32, vp, u32, u32, u32, vp, u32, vp, u8], C.c_int
                assert g(*args, border) == 0
            outs.append(dst.get())
        np.testing.assert_array_equal(outs[1], outs[0], err_msg=f"border {border}")


def remap_table(W, H, sW, sH, rng, spread=5.0):
    """Float source coordinates: a smooth warp plus noise, some outside the source."""
    yy, xx = np.meshgrid(np.arange(H, dtype=np.float32), np.arange(W, dtype=np.float32), indexing="ij")
    sx = xx * (sW / W) + 3.0 * np.sin(yy / 7.0) + rng.uniform(-spread, spread, (H, W)).astype(np.float32)
    sy = yy * (sH / H) + 3.0 * np.cos(xx / 9.0) + rng.uniform(-spread, spread, (H, W)).astype(np.float32)
    xy = np.stack([sx, sy], -1).astype(np.float32)
    fixed = np.zeros((H + 1, W, 2), np.uint16)     # one spare row: the SIMD loop reads 4 entries at a time
    f = O.oracle_lib().oracle_remap_fixed
    f.argtypes, f.restype = [u32, u32, vp, C.c_size_t, vp], None
    f(sW, sH, xy.ctypes.data, W * H, fixed.ctypes.data)
    return xy, fixed


@pytest.mark.parametrize("W,H,sW,sH", [(64, 48, 64, 48), (101, 37, 90, 40), (200, 120, 160, 100), (37, 19, 64, 48)])
@pytest.mark.parametrize("interp", ["Nearest", "Bilinear"])
@pytest.mark.parametrize("border", [None, 0, 7])
def test_remap_matches_reference(ref, W, H, sW, sH, interp, border):
    rng = np.random.default_rng(W + 7 * H + sW)
    src = ago_img(sH, sW)
    src.set(rng.integers(0, 256, (sH, sW), dtype=np.uint8))
    _, fixed = remap_table(W, H, sW, sH, rng)
    assert (fixed[:H] == 0xFFFF).any() and (fixed[:H] != 0xFFFF).any()
    name = f"Remap_U8_U8_{interp}" + ("" if border is None else "_Constant")
    outs = []
    for impl in ("ref", "oracle"):
        dst = ago_img(H, W)
        args = [W, H, dst.ptr, dst.stride, sW, sH, src.ptr, src.stride, fixed.ctypes.data, W * 4]
        types = [u32, u32, vp, u32, u32, u32, vp, u32, vp, u32]
        if border is not None:
            args.append(border)
            types.append(u8)
        f = O.ref_haf(f"HafCpu_{name}") if impl == "ref" else getattr(O.oracle_lib(), "oracle_" + name)
        f.argtypes, f.restype = types, C.c_int
        assert f(*args) == 0
        outs.append(dst.get())
    np.testing.assert_array_equal(outs[1], outs[0])
