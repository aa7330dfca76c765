"""GPU parity of the config-1 kernels (include/agocuda.h) against the oracle restatement:
bit-exact inside the region each AGO CPU wrapper processes (interior rows/columns for the
3x3 stencils, the whole image for pointwise kernels)."""
import ctypes as C

import numpy as np
import pytest

import oracle_chains as OC
from imgbuf import Img

pytestmark = pytest.mark.gpu

SHAPES = [(16, 5), (17, 7), (37, 11), (130, 33), (256, 70), (1920, 1080)]


@pytest.fixture(scope="module")
def lib():
    from mivisionx_b200 import native
    return native.agocuda()


def _dev():
    import devbuf
    return devbuf


@pytest.mark.parametrize("W,H", SHAPES)
def test_gaussian3x3(lib, cuda, rng, W, H):
    D = _dev()
    img = rng.integers(0, 256, (H, W), dtype=np.uint8)
    src = D.DevImg(H, W).upload(img)
    dst = D.DevImg(H, W)
    assert lib.agocuda_Gaussian_U8_U8_3x3(D.stream_ptr(), W, H, dst.ptr, dst.stride, src.ptr, src.stride) == 0
    s = OC.ago_img(H, W); s.set(img)
    ref = OC.gaussian3x3(s).get()
    np.testing.assert_array_equal(dst.download()[1:H - 1, 1:W - 1], ref[1:H - 1, 1:W - 1])


@pytest.mark.parametrize("W,H", SHAPES)
@pytest.mark.parametrize("dst_off", [0, 8])
def test_sobel_magnitude(lib, cuda, rng, W, H, dst_off):
    D = _dev()
    img = rng.integers(0, 256, (H, W), dtype=np.uint8)
    src = D.DevImg(H, W).upload(img)
    dst = D.DevImg(H, W, np.int16, align_off=dst_off)
    assert lib.agocuda_SobelMagnitude_S16_U8_3x3(D.stream_ptr(), W, H, dst.ptr, dst.stride, src.ptr, src.stride) == 0
    s = Img(H, W); s.set(img)
    out = Img(H, W, np.int16, align_off=dst_off)
    OC.fn("SobelMagnitude_S16_U8_3x3")(W, H - 2, out.row_ptr(1), out.stride, s.row_ptr(1), s.stride)
    np.testing.assert_array_equal(dst.download()[1:H - 1, 1:W - 1], out.get()[1:H - 1, 1:W - 1])


@pytest.mark.parametrize("W,H", SHAPES)
def test_sobel_gxy(lib, cuda, rng, W, H):
    D = _dev()
    img = rng.integers(0, 256, (H, W), dtype=np.uint8)
    src = D.DevImg(H, W).upload(img)
    gx, gy = D.DevImg(H, W, np.int16), D.DevImg(H, W, np.int16)
    assert lib.agocuda_Sobel_S16S16_U8_3x3_GXY(D.stream_ptr(), W, H, gx.ptr, gx.stride, gy.ptr, gy.stride,
                                               src.ptr, src.stride) == 0
    s = OC.ago_img(H, W); s.set(img)
    rx, ry = OC.sobel_gxy(s)
    np.testing.assert_array_equal(gx.download()[1:H - 1, 1:W - 1], rx.get()[1:H - 1, 1:W - 1])
    np.testing.assert_array_equal(gy.download()[1:H - 1, 1:W - 1], ry.get()[1:H - 1, 1:W - 1])


@pytest.mark.parametrize("W,H", SHAPES)
@pytest.mark.parametrize("amp,dst_off", [(1020, 0), (32767, 0), (32767, 8), (500, 8)])
def test_magnitude(lib, cuda, rng, W, H, amp, dst_off):
    D = _dev()
    a = rng.integers(-amp, amp + 1, (H, W)).astype(np.int16)
    b = rng.integers(-amp, amp + 1, (H, W)).astype(np.int16)
    ga, gb = D.DevImg(H, W, np.int16).upload(a), D.DevImg(H, W, np.int16).upload(b)
    dst = D.DevImg(H, W, np.int16, align_off=dst_off)
    assert lib.agocuda_Magnitude_S16_S16S16(D.stream_ptr(), W, H, dst.ptr, dst.stride, ga.ptr, ga.stride,
                                            gb.ptr, gb.stride) == 0
    ha, hb = Img(H, W, np.int16, fill=a), Img(H, W, np.int16, fill=b)
    out = Img(H, W, np.int16, align_off=dst_off)
    OC.fn("Magnitude_S16_S16S16")(W, H, out.ptr, out.stride, ha.ptr, ha.stride, hb.ptr, hb.stride)
    np.testing.assert_array_equal(dst.download(), out.get())


@pytest.mark.parametrize("W,H", SHAPES)
@pytest.mark.parametrize("shift", [0, 2, 7])
def test_colordepth_sat(lib, cuda, rng, W, H, shift):
    D = _dev()
    a = rng.integers(-32768, 32768, (H, W)).astype(np.int16)
    src = D.DevImg(H, W, np.int16).upload(a)
    dst = D.DevImg(H, W)
    assert lib.agocuda_ColorDepth_U8_S16_Sat(D.stream_ptr(), W, H, dst.ptr, dst.stride, src.ptr, src.stride, shift) == 0
    ref = OC.colordepth_sat(Img(H, W, np.int16, fill=a), shift).get()
    np.testing.assert_array_equal(dst.download(), ref)


@pytest.mark.parametrize("W,H", SHAPES)
@pytest.mark.parametrize("thr", [0, 128, 255, 300])
def test_threshold_binary(lib, cuda, rng, W, H, thr):
    D = _dev()
    img = rng.integers(0, 256, (H, W), dtype=np.uint8)
    src = D.DevImg(H, W).upload(img)
    dst = D.DevImg(H, W)
    assert lib.agocuda_Threshold_U8_U8_Binary(D.stream_ptr(), W, H, dst.ptr, dst.stride, src.ptr, src.stride, thr) == 0
    ref = OC.threshold_binary(Img(H, W, fill=img), thr).get()
    np.testing.assert_array_equal(dst.download(), ref)


def _frames_dev(frames):
    import torch
    from mivisionx_b200.native import AgoFrame
    arr = (AgoFrame * len(frames))(*frames)
    raw = np.frombuffer(bytes(arr), dtype=np.uint8).copy()
    return torch.from_numpy(raw).cuda()


@pytest.mark.parametrize("shift,thr", [(0, 128), (1, 40), (0, 0), (0, 255), (2, 10)])
def test_fused_cfg1_batched_uneven(lib, cuda, rng, shift, thr):
    """Several frames of different sizes in one launch; each bit-exact in [2, W-2) x [2, H-2)."""
    from mivisionx_b200.native import AgoFrame
    D = _dev()
    sizes = [(1920, 1080), (37, 11), (640, 480), (20, 9), (130, 66)]
    imgs, srcs, dsts, frames = [], [], [], []
    for (W, H) in sizes:
        img = rng.integers(0, 256, (H, W), dtype=np.uint8)
        s, d = D.DevImg(H, W).upload(img), D.DevImg(H, W)
        imgs.append(img); srcs.append(s); dsts.append(d)
        # AGO's virtual SobelMagnitude output is 16-byte aligned: SIMD body [0, W - W % 16).
        frames.append(AgoFrame(s.ptr, d.ptr, W, H, s.stride, d.stride, 0, W - (W % 16)))
    fd = _frames_dev(frames)
    mw, mh = max(w for w, _ in sizes), max(h for _, h in sizes)
    assert lib.agocuda_fused_GaussSobelMagDepthThresh(D.stream_ptr(), fd.data_ptr(), len(frames), mw, mh, shift, thr) == 0
    for img, d, (W, H) in zip(imgs, dsts, sizes):
        ref, (sx, sy, ex, ey) = OC.cfg1_chain(img, shift, thr)
        got = d.download()
        np.testing.assert_array_equal(got[sy:ey, sx:ex], ref[sy:ey, sx:ex], err_msg=f"{W}x{H}")


@pytest.mark.parametrize("shift,thr", [(0, 128), (1, 40), (0, 0), (0, 255), (2, 10), (4, 127)])
def test_fused_cfg1_tma_batched_uneven(lib, cuda, rng, shift, thr):
    """The TMA-staged chain (tensor maps encoded on the host, fp32 Sobel stage): the same
    uneven batch bit-exact in [2, W-2) x [2, H-2), including high-contrast frames whose
    gradients reach the largest magnitudes, and no timeout status."""
    import ctypes as C
    import torch
    from mivisionx_b200.native import AgoFrame
    D = _dev()
    sizes = [(1920, 1080), (37, 11), (640, 480), (20, 9), (130, 66), (300, 257)]
    imgs, srcs, dsts, frames = [], [], [], []
    for i, (W, H) in enumerate(sizes):
        img = rng.integers(0, 256, (H, W), dtype=np.uint8) if i % 2 == 0 else \
            (rng.integers(0, 2, (H, W)) * 255).astype(np.uint8)
        s, d = D.DevImg(H, W).upload(img), D.DevImg(H, W)
        imgs.append(img); srcs.append(s); dsts.append(d)
        frames.append(AgoFrame(s.ptr, d.ptr, W, H, s.stride, d.stride, 0, W - (W % 16)))
    n = len(frames)
    mb = lib.agocuda_fused_GaussSobelMagDepthThresh_tensor_maps_size(n)
    assert mb == 128 * n
    host = np.zeros(mb + 64, np.uint8)
    off = (-host.ctypes.data) % 64
    arr = (AgoFrame * n)(*frames)
    assert lib.agocuda_fused_GaussSobelMagDepthThresh_tensor_maps(arr, n, host.ctypes.data + off, mb) == 0
    dmaps = torch.from_numpy(host[off:off + mb].copy()).cuda()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    fd = _frames_dev(frames)
    mw, mh = max(w for w, _ in sizes), max(h for _, h in sizes)
    assert lib.agocuda_fused_GaussSobelMagDepthThresh_tma(D.stream_ptr(), fd.data_ptr(), dmaps.data_ptr(), n, mw, mh,
                                                          shift, thr, status.data_ptr()) == 0
    for img, d, (W, H) in zip(imgs, dsts, sizes):
        ref, (sx, sy, ex, ey) = OC.cfg1_chain(img, shift, thr)
        got = d.download()
        np.testing.assert_array_equal(got[sy:ey, sx:ex], ref[sy:ey, sx:ex], err_msg=f"{W}x{H}")
    assert int(status.item()) == 0
    # misaligned maps buffer and unaligned source pitch are refused
    assert lib.agocuda_fused_GaussSobelMagDepthThresh_tma(D.stream_ptr(), fd.data_ptr(), dmaps.data_ptr() + 8, n, mw,
                                                          mh, shift, thr, status.data_ptr()) == -10
    bad = (AgoFrame * 1)(AgoFrame(srcs[0].ptr, dsts[0].ptr, 1920, 1080, 1928, dsts[0].stride, 0, 1920))
    assert lib.agocuda_fused_GaussSobelMagDepthThresh_tensor_maps(bad, 1, host.ctypes.data + off, mb) == -10
    odd = (AgoFrame * 1)(AgoFrame(srcs[0].ptr, dsts[0].ptr, 1920, 1080, srcs[0].stride, dsts[0].stride, 4, 1920))
    assert lib.agocuda_fused_GaussSobelMagDepthThresh_tensor_maps(odd, 1, host.ctypes.data + off, mb) == -10


def test_invalid_params(lib, cuda):
    D = _dev()
    assert lib.agocuda_Gaussian_U8_U8_3x3(D.stream_ptr(), 2, 2, 0, 16, 0, 16) == -10
    d = D.DevImg(8, 8)
    assert lib.agocuda_Gaussian_U8_U8_3x3(D.stream_ptr(), 8, 8, d.ptr + 1, 16, d.ptr, 16) == -10
