"""GPU parity of the WarpPerspective and Remap kernels (include/agocuda.h) against the oracle
(pinned to the reference in test_oracle_pin_warp.py): bit-exact for every border mode,
interpolation, image size (including W % 4 != 0 remap tails) and device row pitch."""
import ctypes as C

import numpy as np
import pytest

import test_oracle_pin_warp as PW
from mivisionx_b200 import workloads as WL

pytestmark = pytest.mark.gpu

u32, vp, u8 = C.c_uint32, C.c_void_p, C.c_uint8
PERSP = [vp, u32, u32, vp, u32, u32, u32, vp, u32, vp, u8]
REMAP = [vp, u32, u32, vp, u32, u32, u32, vp, u32, vp, u32]


@pytest.fixture(scope="module")
def lib(cuda):
    from mivisionx_b200 import native
    L = native.agocuda()
    for interp in ("Nearest", "Bilinear"):
        getattr(L, f"agocuda_WarpPerspective_U8_U8_{interp}_Constant").argtypes = PERSP
        getattr(L, f"agocuda_Remap_U8_U8_{interp}").argtypes = REMAP
        getattr(L, f"agocuda_Remap_U8_U8_{interp}_Constant").argtypes = REMAP + [u8]
        for n in (f"WarpPerspective_U8_U8_{interp}_Constant", f"Remap_U8_U8_{interp}", f"Remap_U8_U8_{interp}_Constant"):
            getattr(L, "agocuda_" + n).restype = C.c_int
    return L


@pytest.mark.parametrize("kind", ["identity", "mild", "outside", "integer_negative", "vanishing", "random"])
@pytest.mark.parametrize("W,H", [(64, 48), (100, 37), (200, 120), (1920, 1080)])
@pytest.mark.parametrize("interp", ["Nearest", "Bilinear"])
def test_warp_perspective_matches_oracle(lib, kind, W, H, interp):
    import oracle as O

    from devbuf import DevImg, stream_ptr
    rng = np.random.default_rng(W * 31 + H)
    img = rng.integers(0, 256, (H, W), dtype=np.uint8)
    m = PW.perspective(kind, W, H, rng)
    src = PW.ago_img(H, W)
    src.set(img)
    dsrc = DevImg(H, W).upload(img)
    name = f"WarpPerspective_U8_U8_{interp}_Constant"
    for border in (0, 77):
        ref = PW.ago_img(H, W)
        g = getattr(O.oracle_lib(), "oracle_" + name)
        g.argtypes, g.restype = [u32, u32, vp, u32, u32, u32, vp, u32, vp, u8], C.c_int
        assert g(W, H, ref.ptr, ref.stride, W, H, src.ptr, src.stride, m.ctypes.data, border) == 0
        dd = DevImg(H, W)
        assert getattr(lib, "agocuda_" + name)(stream_ptr(), W, H, dd.ptr, dd.stride, W, H, dsrc.ptr, dsrc.stride,
                                               m.ctypes.data, border) == 0
        np.testing.assert_array_equal(dd.download(), ref.get(), err_msg=f"border {border}")


@pytest.mark.parametrize("W,H,sW,sH", [(64, 48, 64, 48), (101, 37, 90, 40), (200, 120, 160, 100), (37, 19, 64, 48),
                                       (1921, 1080, 1920, 1080)])
@pytest.mark.parametrize("interp", ["Nearest", "Bilinear"])
@pytest.mark.parametrize("border", [None, 0, 7])
def test_remap_matches_oracle(lib, W, H, sW, sH, interp, border):
    import oracle as O
    import torch

    from devbuf import DevImg, stream_ptr
    rng = np.random.default_rng(W + 7 * H + sW)
    img = rng.integers(0, 256, (sH, sW), dtype=np.uint8)
    src = PW.ago_img(sH, sW)
    src.set(img)
    _, fixed = PW.remap_table(W, H, sW, sH, rng)
    name = f"Remap_U8_U8_{interp}" + ("" if border is None else "_Constant")
    ref = PW.ago_img(H, W)
    args = [W, H, ref.ptr, ref.stride, sW, sH, src.ptr, src.stride, fixed.ctypes.data, W * 4]
    types = [u32, u32, vp, u32, u32, u32, vp, u32, vp, u32]
    if border is not None:
        args.append(border)
        types.append(u8)
    g = getattr(O.oracle_lib(), "oracle_" + name)
    g.argtypes, g.restype = types, C.c_int
    assert g(*args) == 0
    dsrc = DevImg(sH, sW).upload(img)
    dmap = torch.from_numpy(fixed[:H].view(np.uint32).reshape(-1).copy()).cuda()
    dd = DevImg(H, W)
    dargs = [stream_ptr(), W, H, dd.ptr, dd.stride, sW, sH, dsrc.ptr, dsrc.stride, dmap.data_ptr(), W * 4]
    if border is not None:
        dargs.append(border)
    assert getattr(lib, "agocuda_" + name)(*dargs) == 0
    np.testing.assert_array_equal(dd.download(), ref.get())
