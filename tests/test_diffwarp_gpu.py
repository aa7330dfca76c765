"""GPU differentiable warps (mivisionx_b200.diffwarp, CUDA kernels of include/agocuda.h)
against the FP64 CPU reference (oracle/diffwarp_f64.py, itself checked against central
differences in test_diffwarp_ref.py).

Tolerances: forward within 2e-5 absolute (values in [0, 1], float32 arithmetic);
theta gradients within 1e-4 relative; source and field gradients within 1e-4 of the
largest gradient magnitude; losses within 1e-5 relative."""
import numpy as np
import pytest

from oracle import diffwarp_f64 as D
from mivisionx_b200 import workloads as WL

pytestmark = pytest.mark.gpu


def setup(n, size, seed=5):
    import torch
    imgs = WL.cfg5_images(n, seed=seed, size=size)
    gt, init = WL.cfg5_params(n, seed=seed, size=size)
    tgts = np.stack([D.warp_affine(imgs[i].astype(np.float64), gt[i]) for i in range(n)]).astype(np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return imgs, init, tgts, dev(imgs), dev(init.astype(np.float32)), dev(tgts)


def fp64(imgs, theta, tgts, i):
    img = imgs[i].astype(np.float64)
    th = theta[i].astype(np.float32).astype(np.float64)       # the GPU sees float32 theta
    out = D.warp_affine(img, th)
    gsrc, gth = D.warp_affine_adjoint(img, th, 2 * (out - tgts[i].astype(np.float64)))
    return out, D.l2_loss(out, tgts[i].astype(np.float64)), gsrc, gth


def close_grad(got, want, what):
    scale = np.abs(want).max()
    err = np.abs(got - want).max()
    assert err <= 1e-4 * scale, f"{what}: max error {err} vs scale {scale}"


@pytest.mark.parametrize("size", [128, 1024])
def test_l2_step_matches_fp64(cuda, size):
    from mivisionx_b200 import diffwarp
    n = 4
    imgs, theta, tgts, d_img, d_th, d_tgt = setup(n, size)
    loss, gsrc, gth = diffwarp.warp_affine_l2_step(d_img, d_th, d_tgt)
    loss, gsrc, gth = loss.cpu().numpy(), gsrc.cpu().numpy(), gth.cpu().numpy()
    for i in range(n):
        _, l, gs, gt = fp64(imgs, theta, tgts, i)
        assert abs(loss[i] - l) <= 1e-5 * l, (i, loss[i], l)
        np.testing.assert_allclose(gth[i], gt, rtol=1e-4, err_msg=f"image {i}")
        close_grad(gsrc[i], gs, f"gsrc image {i}")


def test_autograd_matches_fp64(cuda):
    import torch

    from mivisionx_b200 import diffwarp
    n, size = 3, 256
    imgs, theta, tgts, d_img, d_th, d_tgt = setup(n, size, seed=11)
    src = d_img.clone().requires_grad_(True)
    th = d_th.clone().requires_grad_(True)
    out = diffwarp.warp_affine(src, th)
    loss = ((out - d_tgt) ** 2).sum()
    loss.backward()
    for i in range(n):
        o, _, gs, gt = fp64(imgs, theta, tgts, i)
        assert np.abs(out[i].detach().cpu().numpy() - o).max() <= 2e-5
        np.testing.assert_allclose(th.grad[i].cpu().numpy().astype(np.float64), gt, rtol=1e-4)
        close_grad(src.grad[i].cpu().numpy(), gs, f"gsrc image {i}")
    # the fused step gives the same gradients as forward + autograd backward
    l2, gs2, gt2 = diffwarp.warp_affine_l2_step(d_img, d_th, d_tgt)
    np.testing.assert_allclose(gt2.cpu().numpy(), th.grad.cpu().numpy().astype(np.float64), rtol=1e-4)
    assert abs(float(l2.sum()) - loss.item()) <= 1e-5 * loss.item()
    assert torch.allclose(gs2, src.grad, rtol=0, atol=1e-4 * float(gs2.abs().max()))


def test_remap_forward_and_adjoint_match_fp64(cuda):
    import torch

    from mivisionx_b200 import diffwarp
    size = 256
    img = WL.cfg5_images(2, seed=21, size=size)
    fields = np.stack([WL.cfg5_field(seed=s, size=size) for s in (1, 2)])
    tgt = np.stack([D.remap(img[i].astype(np.float64), WL.cfg5_field(seed=7 + i, size=size).astype(np.float64))
                    for i in range(2)]).astype(np.float32)
    src = torch.from_numpy(img).cuda().requires_grad_(True)
    fld = torch.from_numpy(fields).cuda().requires_grad_(True)
    out = diffwarp.remap(src, fld)
    ((out - torch.from_numpy(tgt).cuda()) ** 2).sum().backward()
    for i in range(2):
        o = D.remap(img[i].astype(np.float64), fields[i].astype(np.float64))
        assert np.abs(out[i].detach().cpu().numpy() - o).max() <= 2e-5
        gs, gf = D.remap_adjoint(img[i].astype(np.float64), fields[i].astype(np.float64), 2 * (o - tgt[i]))
        close_grad(src.grad[i].cpu().numpy(), gs, "gsrc")
        close_grad(fld.grad[i].cpu().numpy(), gf, "gfield")


def test_border_value_and_far_outside_positions(cuda):
    import torch

    from mivisionx_b200 import diffwarp
    img = WL.cfg5_images(1, seed=3, size=64)
    # shift far outside, a NaN-free but huge scale, and a half-outside shift
    thetas = np.array([[1, 0, 0, 1, 5000.0, -7000.0], [1e6, 0, 0, 1e6, 0, 0], [1, 0, 0, 1, 40.5, -20.25]], np.float32)
    src = torch.from_numpy(np.repeat(img, 3, 0)).cuda()
    out = diffwarp.warp_affine(src, torch.from_numpy(thetas).cuda(), border=0.25).cpu().numpy()
    for i in range(3):
        want = D.warp_affine(img[0].astype(np.float64), thetas[i].astype(np.float64), border=0.25)
        assert np.abs(out[i] - want).max() <= 2e-5, i


def _persp_setup(n, size, seed=6):
    import torch
    imgs = WL.cfg5_images(n, seed=seed, size=size)
    gt, init = WL.cfg5_perspective_params(n, seed=seed, size=size)
    tgts = np.stack([D.warp_perspective(imgs[i].astype(np.float64), gt[i]) for i in range(n)]).astype(np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return imgs, init, tgts, dev(imgs), dev(init.astype(np.float32)), dev(tgts)


def _persp_fp64(imgs, theta, tgts, i):
    img = imgs[i].astype(np.float64)
    th = theta[i].astype(np.float32).astype(np.float64)
    out = D.warp_perspective(img, th)
    gsrc, gth = D.warp_perspective_adjoint(img, th, 2 * (out - tgts[i].astype(np.float64)))
    return out, D.l2_loss(out, tgts[i].astype(np.float64)), gsrc, gth


@pytest.mark.parametrize("size", [128, 1024])
def test_perspective_l2_step_matches_fp64(cuda, size):
    from mivisionx_b200 import diffwarp
    n = 4
    imgs, theta, tgts, d_img, d_th, d_tgt = _persp_setup(n, size)
    loss, gsrc, gth = diffwarp.warp_perspective_l2_step(d_img, d_th, d_tgt)
    loss, gsrc, gth = loss.cpu().numpy(), gsrc.cpu().numpy(), gth.cpu().numpy()
    for i in range(n):
        _, l, gs, gt = _persp_fp64(imgs, theta, tgts, i)
        assert abs(loss[i] - l) <= 1e-5 * l, (i, loss[i], l)
        np.testing.assert_allclose(gth[i], gt, rtol=1e-4, err_msg=f"image {i}")
        close_grad(gsrc[i], gs, f"gsrc image {i}")


def test_perspective_autograd_matches_fp64(cuda):
    from mivisionx_b200 import diffwarp
    n, size = 3, 256
    imgs, theta, tgts, d_img, d_th, d_tgt = _persp_setup(n, size, seed=12)
    src = d_img.clone().requires_grad_(True)
    th = d_th.clone().requires_grad_(True)
    out = diffwarp.warp_perspective(src, th)
    loss = ((out - d_tgt) ** 2).sum()
    loss.backward()
    for i in range(n):
        o, _, gs, gt = _persp_fp64(imgs, theta, tgts, i)
        assert np.abs(out[i].detach().cpu().numpy() - o).max() <= 2e-5
        np.testing.assert_allclose(th.grad[i].cpu().numpy().astype(np.float64), gt, rtol=1e-4)
        close_grad(src.grad[i].cpu().numpy(), gs, f"gsrc image {i}")


def test_perspective_degenerate_rows(cuda):
    """z = 0 on a line through the image and z < 0 beyond it: samples there read the border,
    contribute no theta gradient, and nothing becomes NaN."""
    import torch

    from mivisionx_b200 import diffwarp
    size = 64
    img = WL.cfg5_images(1, seed=4, size=size)
    th = np.array([[1, 0, 1.0 / 32, 0, 1, 0, 0, 0, -1.0]], np.float32)   # z = x/32 - 1: zero at x = 32
    src = torch.from_numpy(img).cuda().requires_grad_(True)
    tht = torch.from_numpy(th).cuda().requires_grad_(True)
    out = diffwarp.warp_perspective(src, tht, border=0.5)
    out.sum().backward()
    o = out.detach().cpu().numpy()[0]
    assert np.isfinite(o).all() and np.all(o[:, 32] == 0.5)
    assert torch.isfinite(tht.grad).all() and torch.isfinite(src.grad).all()
