"""The FP64 reference adjoint of the differentiable warps (oracle/diffwarp_f64.py) is the
derivative of the FP64 forward: checked with central finite differences, h = 1e-3.

* Source-image gradients: the warp is linear in the source, so plain central differences
  are exact; agreement to 1e-6 relative.
* theta and field gradients: central differences of the same bilinear interpolation with
  every pixel's integer cell held at the cell of the evaluation point (the loss is then a
  polynomial in theta); agreement to 1e-6 relative.  Plain central differences of a
  bilinear warp do not converge to its gradient: a 1e-3 step of a matrix entry that
  multiplies pixel coordinates moves samples by up to ~1 px across cell borders, where the
  interpolant's derivative jumps.  That gap is measured in the last tests (percent level for
  the linear entries at h = 1e-3) and is a property of bilinear sampling, not of the adjoint:
  on the translation entries, where a step of h moves every sample by h pixels, plain
  central differences stay within a few percent at h = 1e-3 and converge to the adjoint as
  h shrinks (1e-6 relative at h = 1e-6).
* Perspective theta: the frozen-cell loss is a rational function of the projective row
  (m02, m12, m22), so its central differences are exact only to O(h^2); those entries take
  steps that change z by at most 1e-5 over the image (1e-5 / S for m02 and m12, 1e-5 for
  m22), the others h = 1e-3."""
import numpy as np
import pytest

from oracle import diffwarp_f64 as D
from mivisionx_b200 import workloads as WL

S = 192


@pytest.fixture(scope="module")
def case():
    img = WL.cfg5_images(1, size=S)[0].astype(np.float64)
    gt, init = WL.cfg5_params(1, size=S)
    tgt = D.warp_affine(img, gt[0])
    return img, init[0], tgt


def loss_theta(img, th, tgt, cells=None):
    return D.l2_loss(D.warp_affine(img, th, cells=cells), tgt)


def test_theta_gradient_matches_frozen_cell_central_differences(case):
    img, th, tgt = case
    out = D.warp_affine(img, th)
    _, g = D.warp_affine_adjoint(img, th, 2 * (out - tgt))
    cells = D.affine_cells(th, S, S)
    h = 1e-3
    fd = np.array([(loss_theta(img, th + h * np.eye(6)[k], tgt, cells) - loss_theta(img, th - h * np.eye(6)[k], tgt, cells))
                   / (2 * h) for k in range(6)])
    np.testing.assert_allclose(g, fd, rtol=1e-6)


def test_source_gradient_matches_central_differences(case):
    img, th, tgt = case
    out = D.warp_affine(img, th)
    gsrc, _ = D.warp_affine_adjoint(img, th, 2 * (out - tgt))
    rng = np.random.default_rng(1)
    h = 1e-3
    for _ in range(8):
        y, x = rng.integers(0, S, 2)
        e = np.zeros_like(img)
        e[y, x] = h
        fd = (loss_theta(img + e, th, tgt) - loss_theta(img - e, th, tgt)) / (2 * h)
        assert abs(gsrc[y, x] - fd) <= 1e-6 * max(1.0, abs(fd)), (y, x, gsrc[y, x], fd)


def test_remap_field_gradient_matches_frozen_cell_central_differences():
    img = WL.cfg5_images(1, size=S, seed=9)[0].astype(np.float64)
    field = WL.cfg5_field(seed=3, size=S).astype(np.float64)
    tgt = D.remap(img, WL.cfg5_field(seed=4, size=S).astype(np.float64))
    out = D.remap(img, field)
    gsrc, gf = D.remap_adjoint(img, field, 2 * (out - tgt))
    cells = D.remap_cells(field)
    rng = np.random.default_rng(2)
    h = 1e-3
    for _ in range(8):
        y, x = rng.integers(0, S, 2)
        for c in range(2):
            e = np.zeros_like(field)
            e[y, x, c] = h
            fd = (D.l2_loss(D.remap(img, field + e, cells=cells), tgt) - D.l2_loss(D.remap(img, field - e, cells=cells), tgt)) / (2 * h)
            assert abs(gf[y, x, c] - fd) <= 1e-6 * max(1.0, abs(fd)), (y, x, c, gf[y, x, c], fd)
    y, x = 50, 70
    e = np.zeros_like(img)
    e[y, x] = h
    fd = (D.l2_loss(D.remap(img + e, field), tgt) - D.l2_loss(D.remap(img - e, field), tgt)) / (2 * h)
    assert abs(gsrc[y, x] - fd) <= 1e-6 * max(1.0, abs(fd))


def test_plain_central_differences_differ_by_the_interpolation_kinks(case):
    img, th, tgt = case
    out = D.warp_affine(img, th)
    _, g = D.warp_affine_adjoint(img, th, 2 * (out - tgt))
    h = 1e-3
    fd = np.array([(loss_theta(img, th + h * np.eye(6)[k], tgt) - loss_theta(img, th - h * np.eye(6)[k], tgt)) / (2 * h)
                   for k in range(6)])
    rel = np.abs(g - fd) / np.abs(fd)
    # close (the adjoint is the derivative) but not at 1e-4: samples cross cell borders
    assert rel.max() < 0.3, rel


def _persp_case(S=S, seed=6):
    img = WL.cfg5_images(1, size=S, seed=seed)[0].astype(np.float64)
    gt, init = WL.cfg5_perspective_params(1, seed=seed, size=S)
    return img, init[0], D.warp_perspective(img, gt[0])


def test_perspective_theta_gradient_matches_frozen_cell_central_differences():
    img, th, tgt = _persp_case()
    out = D.warp_perspective(img, th)
    _, g = D.warp_perspective_adjoint(img, th, 2 * (out - tgt))
    cells = D.perspective_cells(th, S, S)
    steps = [1e-3, 1e-3, 1e-5 / S, 1e-3, 1e-3, 1e-5 / S, 1e-3, 1e-3, 1e-5]
    L = lambda t: D.l2_loss(D.warp_perspective(img, t, cells=cells), tgt)
    fd = np.array([(L(th + h * np.eye(9)[k]) - L(th - h * np.eye(9)[k])) / (2 * h) for k, h in enumerate(steps)])
    np.testing.assert_allclose(g, fd, rtol=1e-6)


def test_perspective_source_gradient_matches_central_differences():
    img, th, tgt = _persp_case()
    out = D.warp_perspective(img, th)
    gsrc, _ = D.warp_perspective_adjoint(img, th, 2 * (out - tgt))
    rng = np.random.default_rng(3)
    h = 1e-3
    for _ in range(8):
        y, x = rng.integers(0, S, 2)
        e = np.zeros_like(img)
        e[y, x] = h
        fd = (D.l2_loss(D.warp_perspective(img + e, th), tgt) - D.l2_loss(D.warp_perspective(img - e, th), tgt)) / (2 * h)
        assert abs(gsrc[y, x] - fd) <= 1e-6 * max(1.0, abs(fd)), (y, x, gsrc[y, x], fd)


@pytest.mark.parametrize("kind", ["affine", "perspective"])
def test_translation_entries_match_plain_central_differences(case, kind):
    """m20 and m21 move every sample by the same amount: plain central differences (no
    frozen cells) at h = 1e-3 agree to a few percent, and converge to the adjoint as h
    shrinks -- 1e-6 relative at h = 1e-6."""
    if kind == "affine":
        img, th, tgt = case
        warp, adj, idx = D.warp_affine, D.warp_affine_adjoint, (4, 5)
    else:
        img, th, tgt = _persp_case()
        warp, adj, idx = D.warp_perspective, D.warp_perspective_adjoint, (6, 7)
    out = warp(img, th)
    _, g = adj(img, th, 2 * (out - tgt))
    L = lambda t: D.l2_loss(warp(img, t), tgt)
    n = len(th)
    for h, tol in ((1e-3, 0.05), (1e-6, 1e-6)):
        fd = np.array([(L(th + h * np.eye(n)[k]) - L(th - h * np.eye(n)[k])) / (2 * h) for k in idx])
        np.testing.assert_allclose(g[list(idx)], fd, rtol=tol, err_msg=f"h = {h}")
