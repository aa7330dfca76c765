"""GPU parity of the pyramid-level and pyramidal-LK kernels (include/agocuda.h) against the
oracle (oracle/agooracle_flow.c, pinned to the reference build): pyramid levels bit-exact,
keypoints identical record for record, over two consecutive calls on one node scratch."""
import ctypes as C

import numpy as np
import pytest

import test_oracle_pin_flow as PF
from mivisionx_b200 import workloads as WL

pytestmark = pytest.mark.gpu

u32, i32, vp, f32, sz = C.c_uint32, C.c_int32, C.c_void_p, C.c_float, C.c_size_t
KP = WL.KEYPOINT_DTYPE


@pytest.fixture(scope="module")
def lib(cuda):
    from mivisionx_b200 import native
    L = native.agocuda()
    L.agocuda_ScaleGaussianHalf_U8_U8_5x5.argtypes = [vp, u32, u32, vp, u32, u32, u32, vp, u32]
    L.agocuda_fused_ScaleGaussianHalf_batch.argtypes = [vp, vp, u32, u32]
    L.agocuda_ScaleGaussianHalf_tiles.argtypes = [u32, u32]
    L.agocuda_ScaleGaussianHalf_tiles.restype = u32
    L.agocuda_OpticalFlowPyrLK_scratch_size.argtypes = [u32]
    L.agocuda_OpticalFlowPyrLK_scratch_size.restype = sz
    L.agocuda_OpticalFlowPyrLK_scharr_rows_size.argtypes = [u32]
    L.agocuda_OpticalFlowPyrLK_scharr_rows_size.restype = sz
    L.agocuda_OpticalFlowPyrLK_scratch_size_carry.argtypes = [u32, u32, u32]
    L.agocuda_OpticalFlowPyrLK_scratch_size_carry.restype = sz
    L.agocuda_OpticalFlowPyrLK_carry_size.argtypes = [u32, u32]
    L.agocuda_OpticalFlowPyrLK_carry_size.restype = sz
    L.agocuda_OpticalFlowPyrLK_XY_XY.argtypes = [vp, vp, u32, vp, f32, u32, vp, vp, vp, vp, vp, vp, i32, f32, u32, i32,
                                                 i32, vp, sz, vp]
    L.agocuda_OpticalFlowPyrLK_batch.argtypes = [vp, vp, u32, u32, vp]
    for n in ("agocuda_ScaleGaussianHalf_U8_U8_5x5", "agocuda_fused_ScaleGaussianHalf_batch",
              "agocuda_OpticalFlowPyrLK_XY_XY", "agocuda_OpticalFlowPyrLK_batch"):
        getattr(L, n).restype = C.c_int
    return L


def dev_bytes(arr: np.ndarray):
    import torch
    return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).reshape(-1).copy()).cuda()


def gpu_pyramid(lib, img: np.ndarray, levels: int):
    from devbuf import DevImg, stream_ptr
    H, W = img.shape
    lv = [DevImg(H, W).upload(img)]
    for (w, h) in WL.pyramid_sizes(W, H, levels)[1:]:
        d = DevImg(h, w)
        s = lv[-1]
        assert lib.agocuda_ScaleGaussianHalf_U8_U8_5x5(stream_ptr(), w, h, d.ptr, d.stride, s.w, s.h, s.ptr, s.stride) == 0
        lv.append(d)
    return lv


@pytest.mark.parametrize("W,H", [(37, 19), (64, 48), (100, 41), (129, 67), (241, 135), (640, 480), (1920, 1080),
                                 (3840, 2160), (1023, 777)])
def test_pyramid_level_matches_oracle(lib, W, H):
    rng = np.random.default_rng(W + 11 * H)
    img = rng.integers(0, 256, (H, W), dtype=np.uint8)
    lv = gpu_pyramid(lib, img, 2)
    ref_lv, _ = PF.build_pyramid(img, 2)
    np.testing.assert_array_equal(lv[1].download(), ref_lv[1].get())


def test_pyramid_batch_of_uneven_images_matches_single_calls(lib):
    import torch

    from devbuf import DevImg, stream_ptr
    from mivisionx_b200 import native
    sizes = [(640, 480), (37, 19), (1920, 1080), (129, 67), (1280, 720)]
    srcs, dsts, jobs, tile = [], [], [], 0
    for i, (W, H) in enumerate(sizes):
        img = WL.cfg2_scene(seed=i, width=W, height=H, rects=20)
        s = DevImg(H, W).upload(img)
        w, h = (W + 1) // 2, (H + 1) // 2
        d = DevImg(h, w)
        jobs.append(native.HalfJob(s.ptr, d.ptr, W, H, s.stride, w, h, d.stride, tile, 0))
        tile += lib.agocuda_ScaleGaussianHalf_tiles(w, h)
        srcs.append((img, s)); dsts.append(d)
    table = (native.HalfJob * len(jobs))(*jobs)
    tdev = dev_bytes(np.frombuffer(bytes(table), np.uint8))
    assert lib.agocuda_fused_ScaleGaussianHalf_batch(stream_ptr(), tdev.data_ptr(), len(jobs), tile) == 0
    torch.cuda.synchronize()
    for (img, _), d in zip(srcs, dsts):
        ref_lv, _ = PF.build_pyramid(img, 2)
        np.testing.assert_array_equal(d.download(), ref_lv[1].get())


@pytest.mark.parametrize("noise", [False, True])
def test_pyramid_batch_tma_matches_oracle(lib, noise):
    """The TMA-staged batch (one source box per 112 x 32 output tile) equals the oracle on
    every output pixel: widths with W % 16 == 0 (the 5x5 reads across row ends reach the
    neighbouring rows), odd and tiny levels, and 4K."""
    import torch

    from devbuf import DevImg, stream_ptr
    from mivisionx_b200 import native
    L = lib
    L.agocuda_ScaleGaussianHalf_tiles_tma.argtypes, L.agocuda_ScaleGaussianHalf_tiles_tma.restype = [u32, u32], u32
    L.agocuda_ScaleGaussianHalf_tensor_maps.argtypes = [vp, u32, vp, sz]
    L.agocuda_ScaleGaussianHalf_tensor_maps.restype = C.c_int
    L.agocuda_fused_ScaleGaussianHalf_tma.argtypes = [vp, vp, vp, u32, u32, vp]
    L.agocuda_fused_ScaleGaussianHalf_tma.restype = C.c_int
    sizes = [(640, 480), (37, 19), (1920, 1080), (129, 67), (1280, 720), (256, 64), (3840, 2160), (241, 136), (8, 7)]
    srcs, dsts, jobs, tile = [], [], [], 0
    for i, (W, H) in enumerate(sizes):
        rng = np.random.default_rng(31 * W + H)
        img = (rng.integers(0, 256, (H, W), dtype=np.int32).astype(np.uint8) if noise
               else WL.cfg2_scene(seed=i, width=W, height=H, rects=20))
        s = DevImg(H, W).upload(img)
        w, h = (W + 1) // 2, (H + 1) // 2
        d = DevImg(h, w)
        jobs.append(native.HalfJob(s.ptr, d.ptr, W, H, s.stride, w, h, d.stride, tile, 0))
        tile += L.agocuda_ScaleGaussianHalf_tiles_tma(w, h)
        srcs.append((img, s)); dsts.append(d)
    n = len(jobs)
    table = (native.HalfJob * n)(*jobs)
    maps = np.zeros(128 * n + 64, np.uint8)
    off = (-maps.ctypes.data) % 64
    assert L.agocuda_ScaleGaussianHalf_tensor_maps(C.addressof(table), n, maps.ctypes.data + off, 128 * n) == 0
    tdev = dev_bytes(np.frombuffer(bytes(table), np.uint8))
    mdev = dev_bytes(maps[off:off + 128 * n])
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    for _ in range(2):
        assert L.agocuda_fused_ScaleGaussianHalf_tma(stream_ptr(), tdev.data_ptr(), mdev.data_ptr(), n, tile,
                                                     status.data_ptr()) == 0
        torch.cuda.synchronize()
        assert int(status[0].item()) == 0
        for (img, _), d in zip(srcs, dsts):
            ref_lv, _ = PF.build_pyramid(img, 2)
            np.testing.assert_array_equal(d.download(), ref_lv[1].get())


def level_descs(lv):
    from mivisionx_b200 import native
    return (native.PyramidLevel * len(lv))(*[native.PyramidLevel(l.ptr, l.w, l.h, l.stride, 0) for l in lv])


def frame_case(W, H, levels, call, n, shift=3.0):
    f1, f2, (dx, dy) = WL.cfg4_pair(seed=100 * W + H + call, width=W, height=H, max_shift=shift)
    old_kp = PF.points(W + H + call, W, H, n, lost_every=17)
    est_kp = old_kp.copy()
    est_kp["x"] = np.clip(old_kp["x"] + int(round(dx)), 0, W - 1)
    est_kp["y"] = np.clip(old_kp["y"] + int(round(dy)), 0, H - 1)
    est_kp["tracking_status"][5::23] = 0
    est_kp["strength"] += 1000
    return f1, f2, old_kp, est_kp


def oracle_lk(f1, f2, levels, old_kp, est_kp, term, eps, iters, use_est, win, scratch):
    n = len(old_kp)
    old_lv, od = PF.build_pyramid(f1, levels)      # the level buffers must outlive the call
    new_lv, nd = PF.build_pyramid(f2, levels)
    kp = np.zeros(n, KP)
    kp.view(np.uint8)[:] = 0xA5
    PF.lk_call("oracle", kp, od, nd, levels, old_kp, est_kp, term, eps, iters, use_est, f1.shape[1], scratch, win)
    return kp


def first_call_only(W, levels):
    """Levels above 0 with width % 8 >= 3 read derivative columns the reference wrote in an
    earlier call; without a carry buffer the kernels reproduce the first call there."""
    return any(w % 8 >= 3 for (w, _) in WL.pyramid_sizes(W, 8, levels)[1:])


@pytest.mark.parametrize("carry", [True, False])
@pytest.mark.parametrize("W,H,levels,win,term,eps,iters,use_est", PF.CASES + [(640, 480, 5, 9, PF.TERM_BOTH, 0.01, 20, 0),
                                                                           (320, 240, 5, 9, PF.TERM_BOTH, 0.01, 20, 0)])
def test_lk_single_node_matches_oracle_over_calls(lib, W, H, levels, win, term, eps, iters, use_est, carry):
    """Three consecutive calls of one node (its scratch state carries over); with the carry
    buffer every call is identical to the oracle, without it the calls after the first only
    where no level above 0 has width % 8 >= 3."""
    import torch

    from devbuf import stream_ptr
    n = 600 if W < 640 else 2000
    size = lib.agocuda_OpticalFlowPyrLK_scratch_size_carry(W, H, levels) if carry else lib.agocuda_OpticalFlowPyrLK_scratch_size(W)
    scratch = torch.zeros(size + 256, dtype=torch.uint8, device="cuda")
    sbase = scratch.data_ptr() + (-scratch.data_ptr() % 256)
    oscratch = PF.lk_scratch(W, H, n)
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    for call in range(3):
        f1, f2, old_kp, est_kp = frame_case(W, H, levels, call, n)
        old_lv, new_lv = gpu_pyramid(lib, f1, levels), gpu_pyramid(lib, f2, levels)
        d_old, d_est = dev_bytes(old_kp), dev_bytes(est_kp)
        out = np.zeros(n, KP)
        out.view(np.uint8)[:] = 0xA5
        d_out = dev_bytes(out)
        cnt = torch.tensor([n, n, 0, 0], dtype=torch.int32, device="cuda")
        rc = lib.agocuda_OpticalFlowPyrLK_XY_XY(
            stream_ptr(), d_out.data_ptr(), n, cnt.data_ptr() + 8, 0.5, levels, level_descs(old_lv), level_descs(new_lv),
            cnt.data_ptr(), d_old.data_ptr(), cnt.data_ptr() + 4, d_est.data_ptr(), term, eps, iters, use_est, win,
            sbase, scratch.numel() - 256, status.data_ptr())
        assert rc == 0
        got = d_out.cpu().numpy().view(KP)
        want = oracle_lk(f1, f2, levels, old_kp, est_kp, term, eps, iters, use_est, win, oscratch)
        assert int(status[0]) == 0 and int(cnt[2]) == n
        if call > 0 and not carry and first_call_only(W, levels):
            continue
        bad = np.nonzero(got != want)[0]
        assert bad.size == 0, f"call {call}: {bad.size} keypoints differ, first {bad[:5]}: {got[bad[:3]]} vs {want[bad[:3]]}"


def test_lk_batch_of_uneven_frames_matches_oracle(lib):
    """Config-4 shape in miniature: frames of different sizes tracked in one batch."""
    import torch

    from devbuf import stream_ptr
    from mivisionx_b200 import native
    sizes = [(640, 480), (1280, 720), (320, 240), (640, 480)]
    levels, win, n = 5, 9, 2000
    frames, keep, wants = [], [], []
    for i, (W, H) in enumerate(sizes):
        f1, f2, old_kp, est_kp = frame_case(W, H, levels, i, n, shift=8.0)
        old_lv, new_lv = gpu_pyramid(lib, f1, levels), gpu_pyramid(lib, f2, levels)
        d_old, d_est = dev_bytes(old_kp), dev_bytes(est_kp)
        out = np.zeros(n, KP)
        d_out = dev_bytes(out)
        cnt = torch.tensor([n, n, 0, 0], dtype=torch.int32, device="cuda")
        rows = torch.zeros(lib.agocuda_OpticalFlowPyrLK_scharr_rows_size(W), dtype=torch.uint8, device="cuda")
        F = native.LkFrame()
        for l in range(levels):
            F.oldPyr[l] = native.PyramidLevel(old_lv[l].ptr, old_lv[l].w, old_lv[l].h, old_lv[l].stride, 0)
            F.newPyr[l] = native.PyramidLevel(new_lv[l].ptr, new_lv[l].w, new_lv[l].h, new_lv[l].stride, 0)
        F.oldPoints, F.estPoints, F.newPoints = d_old.data_ptr(), d_est.data_ptr(), d_out.data_ptr()
        F.pOldCount, F.pEstCount, F.pNewCount = cnt.data_ptr(), cnt.data_ptr() + 4, cnt.data_ptr() + 8
        F.scharrRows = rows.data_ptr()
        F.newCapacity, F.levels, F.termination, F.epsilon = n, levels, PF.TERM_BOTH, 0.01
        F.numIterations, F.useInitialEstimate, F.windowDimension = 20, 0, win
        frames.append(F)
        keep.append((old_lv, new_lv, d_old, d_est, d_out, cnt, rows))
        wants.append(oracle_lk(f1, f2, levels, old_kp, est_kp, PF.TERM_BOTH, 0.01, 20, 0, win, PF.lk_scratch(W, H, n)))
    table = (native.LkFrame * len(frames))(*frames)
    tdev = dev_bytes(np.frombuffer(bytes(table), np.uint8))
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    assert lib.agocuda_OpticalFlowPyrLK_batch(stream_ptr(), tdev.data_ptr(), len(frames), n, status.data_ptr()) == 0
    torch.cuda.synchronize()
    assert int(status[0]) == 0
    for (old_lv, new_lv, d_old, d_est, d_out, cnt, rows), want in zip(keep, wants):
        got = d_out.cpu().numpy().view(KP)
        for f in ("x", "y", "tracking_status", "strength"):
            np.testing.assert_array_equal(got[f], want[f], err_msg=f)
        assert (got["tracking_status"] != 0).sum() > n // 2


def test_lk_rejects_mismatched_counts(lib):
    import torch

    from devbuf import stream_ptr
    W, H, levels, n = 160, 120, 3, 100
    f1, f2, old_kp, est_kp = frame_case(W, H, levels, 0, n)
    old_lv, new_lv = gpu_pyramid(lib, f1, levels), gpu_pyramid(lib, f2, levels)
    d_old, d_est, d_out = dev_bytes(old_kp), dev_bytes(est_kp), dev_bytes(np.zeros(n, KP))
    cnt = torch.tensor([n, n - 1, 0, 0], dtype=torch.int32, device="cuda")
    scratch = torch.zeros(lib.agocuda_OpticalFlowPyrLK_scratch_size(W) + 256, dtype=torch.uint8, device="cuda")
    sbase = scratch.data_ptr() + (-scratch.data_ptr() % 256)
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    assert lib.agocuda_OpticalFlowPyrLK_XY_XY(
        stream_ptr(), d_out.data_ptr(), n, cnt.data_ptr() + 8, 0.5, levels, level_descs(old_lv), level_descs(new_lv),
        cnt.data_ptr(), d_old.data_ptr(), cnt.data_ptr() + 4, d_est.data_ptr(), PF.TERM_BOTH, 0.01, 20, 0, 9, sbase,
        scratch.numel() - 256, status.data_ptr()) == 0
    torch.cuda.synchronize()
    assert int(status[0]) == 16                 # AGOCUDA_LK_STATUS_BAD_COUNT
    # invalid window and scale are refused on the host
    for win, scale in ((2, 0.5), (16, 0.5), (9, 0.8)):
        assert lib.agocuda_OpticalFlowPyrLK_XY_XY(
            stream_ptr(), d_out.data_ptr(), n, cnt.data_ptr() + 8, scale, levels, level_descs(old_lv),
            level_descs(new_lv), cnt.data_ptr(), d_old.data_ptr(), cnt.data_ptr() + 4, d_est.data_ptr(), PF.TERM_BOTH,
            0.01, 20, 0, win, sbase, scratch.numel() - 256, status.data_ptr()) == -10
