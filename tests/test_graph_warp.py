"""WarpPerspective + Remap graph through the OpenVX API (border CONSTANT and UNDEFINED).

CPU: the reference AGO library runs the graph and must equal the oracle composition, which
also pins the oracle's restatement of vxCopyRemapPatch's fixed-point table.  GPU: this
package's engine must equal the oracle bit for bit."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import test_oracle_pin_warp as PW
from mivisionx_b200 import vx as V
from mivisionx_b200 import workloads as WL

u32, vp, u8 = C.c_uint32, C.c_void_p, C.c_uint8


def oracle_graph(img, m, table, border):
    H, W = img.shape
    dH, dW = table.shape[:2]
    src = PW.ago_img(H, W)
    src.set(img)
    out = {}
    for name, interp, bd in (("persp_bilinear_constant", "Bilinear", border), ("persp_nearest", "Nearest", 0)):
        d = PW.ago_img(H, W)
        g = getattr(O.oracle_lib(), f"oracle_WarpPerspective_U8_U8_{interp}_Constant")
        g.argtypes, g.restype = [u32, u32, vp, u32, u32, u32, vp, u32, vp, u8], C.c_int
        assert g(W, H, d.ptr, d.stride, W, H, src.ptr, src.stride, m.ctypes.data, bd) == 0
        out[name] = d.get()
    fixed = np.zeros((dH + 1, dW, 2), np.uint16)
    f = O.oracle_lib().oracle_remap_fixed
    f.argtypes, f.restype = [u32, u32, vp, C.c_size_t, vp], None
    t = np.ascontiguousarray(table, np.float32)
    f(W, H, t.ctypes.data, dW * dH, fixed.ctypes.data)
    for name, fn, args in (("remap_bilinear_constant", "Remap_U8_U8_Bilinear_Constant", [border]),
                           ("remap_nearest", "Remap_U8_U8_Nearest", [])):
        d = PW.ago_img(dH, dW)
        g = getattr(O.oracle_lib(), "oracle_" + fn)
        g.argtypes = [u32, u32, vp, u32, u32, u32, vp, u32, vp, u32] + [u8] * len(args)
        g.restype = C.c_int
        assert g(dW, dH, d.ptr, d.stride, W, H, src.ptr, src.stride, fixed.ctypes.data, dW * 4, *args) == 0
        out[name] = d.get()
    return out


def case(W, H, dW, dH, seed):
    rng = np.random.default_rng(seed)
    img = WL.cfg3_frame(seed=seed, width=W, height=H)[..., 1].copy()
    m = PW.perspective("outside", W, H, rng)
    xy, _ = PW.remap_table(dW, dH, W, H, rng)
    return img, m, xy


def check(g, img, m, xy, border):
    got = g.results()
    want = oracle_graph(img, m, xy, border)
    for k, (a, rect) in got.items():
        np.testing.assert_array_equal(a, want[k], err_msg=k)
        assert rect == (0, 0, a.shape[1], a.shape[0]), (k, rect)


@pytest.mark.parametrize("W,H,dW,dH", [(64, 48, 64, 48), (200, 120, 101, 77)])
def test_reference_graph_matches_oracle(W, H, dW, dH):
    lib = O.ref_lib()
    if lib is None:
        pytest.skip("reference library not built")
    api = V.OpenVX(lib)
    ctx = api.obj(api.vxCreateContext(), "context")
    img, m, xy = case(W, H, dW, dH, W + H)
    g = WL.WarpRemapGraph(api, ctx, (W, H), m, xy, border=9)
    g.run(img)
    check(g, img, m, xy, 9)


@pytest.mark.gpu
@pytest.mark.parametrize("W,H,dW,dH", [(64, 48, 64, 48), (200, 120, 101, 77), (1920, 1080, 1283, 721)])
def test_engine_graph_matches_oracle(cuda, W, H, dW, dH):
    api = V.OpenVX()
    ctx = api.obj(api.vxCreateContext(), "context")
    img, m, xy = case(W, H, dW, dH, W + H)
    g = WL.WarpRemapGraph(api, ctx, (W, H), m, xy, border=9)
    g.run(img)
    check(g, img, m, xy, 9)
