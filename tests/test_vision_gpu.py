"""GPU parity of the Canny / Harris kernels of include/agocuda.h against the oracle parts
(bit-exact; lists compared as sets where the device emits them in arbitrary order)."""
import ctypes as C

import numpy as np
import pytest

import oracle_chains as OC
from mivisionx_b200 import workloads as WL

pytestmark = pytest.mark.gpu

SIZES = [(64, 48), (37, 19), (200, 120), (1920, 1080)]

u32, vp, u16, f32, sz = C.c_uint32, C.c_void_p, C.c_uint16, C.c_float, C.c_size_t


@pytest.fixture(scope="module")
def lib():
    from mivisionx_b200 import native
    L = native.agocuda()
    sigs = {
        "agocuda_CannySobel_U16_U8_3x3_L1NORM": [vp, u32, u32, vp, u32, vp, u32],
        "agocuda_CannySuppThreshold_U8XY_U16_3x3": [vp, u32, u32, vp, u32, vp, u32, vp, vp, u32, u16, u16],
        "agocuda_CannyEdgeTrace_U8_U8XY": [vp, u32, u32, vp, u32, vp, vp, u32, vp, sz, vp],
        "agocuda_fused_CannyEdgeDetector_3x3_L1": [vp, u32, u32, vp, u32, vp, u32, u16, u16, vp, sz, vp],
        "agocuda_HarrisSobel_HG3_U8_3x3": [vp, u32, u32, vp, u32, vp, u32],
        "agocuda_HarrisScore_HVC_HG3_3x3": [vp, u32, u32, vp, u32, vp, u32, f32, f32, f32],
        "agocuda_NonMaxSupp_XY_ANY_3x3": [vp, u32, u32, vp, u32, vp, vp, u32],
        "agocuda_HarrisMergeSortAndPick_XY_XYS": [vp, u32, u32, vp, vp, u32, f32, vp, u32, vp, vp, vp, sz, vp],
        "agocuda_fused_HarrisCorners_3x3": [vp, u32, u32, vp, u32, f32, f32, f32, f32, vp, u32, vp, vp, vp, sz, vp],
    }
    for n, a in sigs.items():
        getattr(L, n).argtypes = a
        getattr(L, n).restype = C.c_int
    for n in ("agocuda_CannyEdgeTrace_scratch_size", "agocuda_fused_CannyEdgeDetector_scratch_size"):
        getattr(L, n).argtypes = [u32, u32]
        getattr(L, n).restype = C.c_size_t
    L.agocuda_fused_HarrisCorners_scratch_size.argtypes = [u32, u32, f32]
    L.agocuda_fused_HarrisCorners_scratch_size.restype = C.c_size_t
    L.agocuda_HarrisMergeSortAndPick_scratch_size.argtypes = [u32, u32, u32, f32]
    L.agocuda_HarrisMergeSortAndPick_scratch_size.restype = C.c_size_t
    return L


def _pick(lib, W, H, lst, cnt, list_cap, mind, cap, scratch=True):
    """agocuda_HarrisMergeSortAndPick_XY_XYS -> (corners, corner count, num corners, status)."""
    import torch
    D = _dev()
    corners, ccount, ncorn, status = _buf(28 * cap), _buf(4), _buf(4), _buf(4)
    sb = lib.agocuda_HarrisMergeSortAndPick_scratch_size(W, H, list_cap, mind) if scratch else 0
    scr = _buf(sb) if scratch else None
    base = scr.data_ptr() + (-scr.data_ptr() % 256) if scratch else None
    assert lib.agocuda_HarrisMergeSortAndPick_XY_XYS(D.stream_ptr(), W, H, lst.data_ptr(), cnt.data_ptr(), list_cap, mind,
                                                     corners.data_ptr(), cap, ccount.data_ptr(), ncorn.data_ptr(),
                                                     base, sb, status.data_ptr()) == 0
    torch.cuda.synchronize()
    nk = int(ccount[:4].view(torch.int32).item())
    return (corners[:28 * nk].cpu().numpy().view(OC.KP), nk, int(ncorn[:4].view(torch.int32).item()),
            int(status[:4].view(torch.int32).item()))


def _dev():
    import devbuf
    return devbuf


def _buf(nbytes):
    import torch
    return torch.zeros(nbytes + 256, dtype=torch.uint8, device="cuda")


def _img(W, H, seed):
    return WL.cfg2_scene(seed=seed, width=W, height=H, rects=min(200, max(3, W * H // 300)))


@pytest.mark.parametrize("W,H", SIZES)
def test_canny_kernels(lib, cuda, W, H):
    D = _dev()
    img = _img(W, H, W * 3 + H)
    ref_sob, ref_supp, ref_strong, ref_edges = OC.canny_parts(img)
    src = D.DevImg(H, W).upload(img)
    sob = D.DevImg(H, W, np.uint16)
    assert lib.agocuda_CannySobel_U16_U8_3x3_L1NORM(D.stream_ptr(), W, H, sob.ptr, sob.stride, src.ptr, src.stride) == 0
    got = sob.download()
    np.testing.assert_array_equal(got[1:H - 1], ref_sob[1:H - 1])
    out = D.DevImg(H, W)
    stack, cnt, status = _buf(4 * W * H), _buf(4), _buf(4)
    assert lib.agocuda_CannySuppThreshold_U8XY_U16_3x3(D.stream_ptr(), W, H, out.ptr, out.stride, sob.ptr, sob.stride,
                                                       stack.data_ptr(), cnt.data_ptr(), W * H, 80, 100) == 0
    supp = out.download()
    np.testing.assert_array_equal(supp[1:H - 1, 1:W - 1], ref_supp[1:H - 1, 1:W - 1])
    n = int(cnt[:4].view(dtype=__import__("torch").int32).item())
    got_strong = np.sort(stack[:4 * n].view(dtype=__import__("torch").int32).cpu().numpy().astype(np.uint32))
    np.testing.assert_array_equal(got_strong, np.sort(ref_strong))
    sb = lib.agocuda_CannyEdgeTrace_scratch_size(W, H)
    scr = _buf(sb)
    base = scr.data_ptr() + (-scr.data_ptr() % 256)
    assert lib.agocuda_CannyEdgeTrace_U8_U8XY(D.stream_ptr(), W, H, out.ptr, out.stride, stack.data_ptr(), cnt.data_ptr(),
                                              W * H, base, sb, status.data_ptr()) == 0
    edges = out.download()
    np.testing.assert_array_equal(edges[1:H - 1, 1:W - 1], ref_edges[1:H - 1, 1:W - 1])
    assert int(status[0].item()) == 0


@pytest.mark.parametrize("W,H", SIZES + [(3840, 2160)])
def test_fused_canny(lib, cuda, W, H):
    D = _dev()
    img = _img(W, H, W + 7 * H)
    ref_edges = OC.canny_parts(img)[3]
    src, out = D.DevImg(H, W).upload(img), D.DevImg(H, W)
    sb = lib.agocuda_fused_CannyEdgeDetector_scratch_size(W, H)
    scr, status = _buf(sb), _buf(4)
    base = scr.data_ptr() + (-scr.data_ptr() % 256)
    for _ in range(2):   # twice: scratch state must not leak between runs
        assert lib.agocuda_fused_CannyEdgeDetector_3x3_L1(D.stream_ptr(), W, H, out.ptr, out.stride, src.ptr, src.stride,
                                                          80, 100, base, sb - 256, status.data_ptr()) == 0
        edges = out.download()
        np.testing.assert_array_equal(edges[1:H - 1, 1:W - 1], ref_edges[1:H - 1, 1:W - 1])
    assert int(status[0].item()) == 0


@pytest.mark.parametrize("W,H,lo,hi", [(3, 3, 20, 40), (65, 33, 20, 40), (130, 70, 40, 200), (333, 97, 10, 30),
                                       (1023, 517, 60, 120), (3840, 2160, 30, 90), (64, 40, 20, 40),
                                       (1024, 80, 10, 30)])
@pytest.mark.parametrize("dst_off,src_off", [(0, 0), (1, 0), (0, 4)])
def test_fused_canny_dense(lib, cuda, W, H, lo, hi, dst_off, src_off):
    """Noise with low thresholds: components of every shape cross tile borders, open runs
    without strong pixels wait for the patch pass, tiles hang over the right and bottom
    image edges; an output plane starting off an 8-byte boundary takes the byte stores.  A
    16-byte aligned source is staged by TMA (with W % 16 == 0 the bytes the reference reads
    left of column 0 and at column W come from the neighbouring rows), a source 4 bytes off
    by word loads."""
    D = _dev()
    img = np.random.default_rng(W * H + lo).integers(0, 256, (H, W), dtype=np.int32).astype(np.uint8)
    ref_edges = OC.canny_parts(img, lo, hi)[3]
    src = D.DevImg(H, W, align_off=src_off).upload(img)
    out = D.DevImg(H, W, align_off=dst_off)
    sb = lib.agocuda_fused_CannyEdgeDetector_scratch_size(W, H)
    scr, status = _buf(sb), _buf(4)
    base = scr.data_ptr() + (-scr.data_ptr() % 256)
    for _ in range(2):
        assert lib.agocuda_fused_CannyEdgeDetector_3x3_L1(D.stream_ptr(), W, H, out.ptr, out.stride, src.ptr, src.stride,
                                                          lo, hi, base, sb - 256, status.data_ptr()) == 0
        edges = out.download()
        np.testing.assert_array_equal(edges[1:H - 1, 1:W - 1], ref_edges[1:H - 1, 1:W - 1])
        assert not edges[0].any() and not edges[H - 1].any() and not edges[:, 0].any() and not edges[:, W - 1].any()
    assert int(status[0].item()) == 0
    if W > 100:
        assert (ref_edges == 255).mean() > 0.01


@pytest.mark.parametrize("W,H", [(64, 48), (36, 19), (200, 120), (1920, 1080)])
def test_harris_kernels(lib, cuda, W, H):
    import torch
    D = _dev()
    img = _img(W, H, 5 * W + H)
    ref_hg3, ref_hvc, ref_list = OC.harris_parts(img)
    src = D.DevImg(H, W).upload(img)
    hg3 = D.DevImg(H, W, np.float32, channels=3)
    hvc = D.DevImg(H, W, np.float32)
    assert lib.agocuda_HarrisSobel_HG3_U8_3x3(D.stream_ptr(), W, H, hg3.ptr, hg3.stride, src.ptr, src.stride) == 0
    np.testing.assert_array_equal(hg3.download()[1:H - 1], ref_hg3[1:H - 1])
    norm = OC.harris_norm(3)
    assert lib.agocuda_HarrisScore_HVC_HG3_3x3(D.stream_ptr(), W, H, hvc.ptr, hvc.stride, hg3.ptr, hg3.stride,
                                               0.04, 1e-3, norm) == 0
    np.testing.assert_array_equal(hvc.download(), ref_hvc)
    lst, cnt = _buf(8 * W * H), _buf(4)
    assert lib.agocuda_NonMaxSupp_XY_ANY_3x3(D.stream_ptr(), W, H, hvc.ptr, hvc.stride, lst.data_ptr(), cnt.data_ptr(), W * H) == 0
    n = int(cnt[:4].view(torch.int32).item())
    got = lst[:8 * n].cpu().numpy().view(OC.XYS)
    key = lambda a: np.sort(a.view(np.int64))
    np.testing.assert_array_equal(key(got), key(ref_list))
    for mind, cap in ((5.0, 32768), (5.0, 7), (1.5, 32768)):
        ref_c, ref_n = OC.harris_pick(ref_list, W, H, mind, cap)
        got_c, nk, got_n, status = _pick(lib, W, H, lst, cnt, W * H, mind, cap)
        assert status == 0
        assert got_n == ref_n
        assert nk == min(ref_n, cap)
        np.testing.assert_array_equal(got_c, ref_c)


@pytest.mark.parametrize("W,H,src_off", [(200, 120, 0), (1920, 1080, 0), (3840, 2160, 0), (64, 40, 0), (250, 70, 0),
                                         (1920, 1080, 4), (250, 70, 1)])
def test_fused_harris(lib, cuda, W, H, src_off):
    """A 16-byte aligned source is staged by TMA (with W % 16 == 0 the bytes the reference
    reads left of column 0 and at column W come from the neighbouring rows), a source 4 bytes
    off by word loads, one 1 byte off byte by byte."""
    import torch
    D = _dev()
    img = _img(W, H, 9 * W + H)
    ref_c, ref_n = OC.harris(img, capacity=32768)
    src = D.DevImg(H, W, align_off=src_off).upload(img)
    sb = lib.agocuda_fused_HarrisCorners_scratch_size(W, H, 5.0)
    scr, corners, ccount, ncorn, status = _buf(sb), _buf(28 * 32768), _buf(4), _buf(4), _buf(4)
    base = scr.data_ptr() + (-scr.data_ptr() % 256)
    for _ in range(2):
        assert lib.agocuda_fused_HarrisCorners_3x3(D.stream_ptr(), W, H, src.ptr, src.stride, 0.04, 1e-3, OC.harris_norm(3),
                                                   5.0, corners.data_ptr(), 32768, ccount.data_ptr(), ncorn.data_ptr(),
                                                   base, sb, status.data_ptr()) == 0
        torch.cuda.synchronize()
        assert int(status[0].item()) == 0
        nk = int(ccount[:4].view(torch.int32).item())
        assert int(ncorn[:4].view(torch.int32).item()) == ref_n
        np.testing.assert_array_equal(corners[:28 * nk].cpu().numpy().view(OC.KP), ref_c)


def test_edge_trace_seeds_off_the_map(lib, cuda):
    """Stack entries the suppression never emits: a border pixel and a zero interior pixel
    seed the weak components around them (the reference's trace grows from every entry
    through its 8 neighbours), an entry outside the image is ignored and flagged."""
    import torch
    D = _dev()
    W, H = 200, 120
    img = _img(W, H, 4242)
    _, supp, strong, ref_edges = OC.canny_parts(img)
    supp = supp.copy()
    yb = H // 2
    supp[yb - 1:yb + 2, 0] = 0
    supp[yb, 1:4] = 127                       # a weak run touching column 1, seeded from (0, yb)
    weak_only = (supp == 127) & (ref_edges == 0)
    weak_only[:, :6] = False
    zero_seed = None
    for y, x in zip(*np.nonzero(weak_only[2:H - 2, 2:W - 2])):
        y, x = y + 2, x + 2
        for dy, dx in ((-1, 0), (1, 0), (0, -1), (0, 1)):
            if supp[y + dy, x + dx] == 0:
                zero_seed = (x + dx, y + dy)
                break
        if zero_seed:
            break
    assert zero_seed is not None
    seeds = np.array([(yb << 16) | 0, (zero_seed[1] << 16) | zero_seed[0]], np.uint32)
    stack_in = np.concatenate([strong.astype(np.uint32), seeds])
    # oracle: the same map and stack through the restated reference trace
    o = OC.ago_img(H, W); o.set(supp)
    ost = np.zeros(W * H, np.uint32); ost[:len(stack_in)] = stack_in
    OC.fn("CannyEdgeTrace_U8_U8XY")(W, H, o.ptr, o.stride, W * H, ost.ctypes.data, len(stack_in))
    expected = o.get()
    assert (expected != ref_edges).any(), "the extra seeds must change the result"
    # device: the same stack plus one entry outside the image
    dev_stack = np.concatenate([stack_in, np.array([(5 << 16) | (W + 3)], np.uint32)])
    out = D.DevImg(H, W).upload(supp)
    st = torch.from_numpy(dev_stack.view(np.int32).copy()).cuda()
    cnt = torch.tensor([len(dev_stack)], dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    sb = lib.agocuda_CannyEdgeTrace_scratch_size(W, H)
    scr = _buf(sb)
    base = scr.data_ptr() + (-scr.data_ptr() % 256)
    assert lib.agocuda_CannyEdgeTrace_U8_U8XY(D.stream_ptr(), W, H, out.ptr, out.stride, st.data_ptr(), cnt.data_ptr(),
                                              len(dev_stack), base, sb, status.data_ptr()) == 0
    got = out.download()
    np.testing.assert_array_equal(got[1:H - 1, 1:W - 1], expected[1:H - 1, 1:W - 1])
    assert int(status.item()) == 8            # AGOCUDA_TRACE_STATUS_BAD_ENTRY


@pytest.mark.parametrize("W,H,mind", [(3840, 2160, 5.0), (1920, 1080, 5.0), (640, 480, 10.0), (1920, 1080, 1.5)])
def test_harris_dense_candidates(lib, cuda, W, H, mind):
    """Pure noise: hundreds of thousands of candidates, far above the shared-memory pick's
    8192, so the cluster pick runs; the corner list equals the oracle's in content and order,
    per node and fused.  Without scratch the per-node pick reports the overflow instead."""
    import torch
    D = _dev()
    img = np.random.default_rng(W + H).integers(0, 256, (H, W), dtype=np.int32).astype(np.uint8)
    ref_c, ref_n = OC.harris(img, capacity=1 << 22, min_distance=mind)
    _, _, ref_list = OC.harris_parts(img)
    assert len(ref_list) > 8192
    src = D.DevImg(H, W).upload(img)
    hg3, hvc = D.DevImg(H, W, np.float32, channels=3), D.DevImg(H, W, np.float32)
    assert lib.agocuda_HarrisSobel_HG3_U8_3x3(D.stream_ptr(), W, H, hg3.ptr, hg3.stride, src.ptr, src.stride) == 0
    assert lib.agocuda_HarrisScore_HVC_HG3_3x3(D.stream_ptr(), W, H, hvc.ptr, hvc.stride, hg3.ptr, hg3.stride,
                                               0.04, 1e-3, OC.harris_norm(3)) == 0
    lst, cnt = _buf(8 * W * H), _buf(4)
    assert lib.agocuda_NonMaxSupp_XY_ANY_3x3(D.stream_ptr(), W, H, hvc.ptr, hvc.stride, lst.data_ptr(), cnt.data_ptr(), W * H) == 0
    cap = 1 << 22
    for _ in range(2):   # twice: the scratch left by the first run must not matter
        got_c, nk, got_n, status = _pick(lib, W, H, lst, cnt, W * H, mind, cap)
        assert status == 0
        assert got_n == ref_n and nk == min(ref_n, cap)
        np.testing.assert_array_equal(got_c, ref_c)
    small = 1000   # fewer slots than corners: the first ones in order, the full count
    got_c, nk, got_n, _ = _pick(lib, W, H, lst, cnt, W * H, mind, small)
    assert got_n == ref_n and nk == small
    np.testing.assert_array_equal(got_c, ref_c[:small])
    _, nk, _, status = _pick(lib, W, H, lst, cnt, W * H, mind, cap, scratch=False)
    assert status == 2 and nk == 0
    # fused front end + pick
    sb = lib.agocuda_fused_HarrisCorners_scratch_size(W, H, mind)
    scr, corners, ccount, ncorn, st = _buf(sb), _buf(28 * cap), _buf(4), _buf(4), _buf(4)
    base = scr.data_ptr() + (-scr.data_ptr() % 256)
    assert lib.agocuda_fused_HarrisCorners_3x3(D.stream_ptr(), W, H, src.ptr, src.stride, 0.04, 1e-3, OC.harris_norm(3),
                                               mind, corners.data_ptr(), cap, ccount.data_ptr(), ncorn.data_ptr(),
                                               base, sb, st.data_ptr()) == 0
    torch.cuda.synchronize()
    assert int(st[:4].view(torch.int32).item()) == 0
    nk = int(ccount[:4].view(torch.int32).item())
    assert int(ncorn[:4].view(torch.int32).item()) == ref_n
    np.testing.assert_array_equal(corners[:28 * nk].cpu().numpy().view(OC.KP), ref_c)
