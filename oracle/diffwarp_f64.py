"""FP64 CPU reference of the differentiable F32 warps (test infrastructure only: used by the
tests and never by the product path).

There is no F32 warp in the reference (its warps validate U8 only, ago_kernel_api.cpp:19255);
these follow the coordinate convention of its U8 WarpAffine (ago_haf_cpu_geometric.cpp:
679-684, matrix stored as ago_affine_matrix_t m[3][2]):

    xs = m[0][0]*x + m[1][0]*y + m[2][0],   ys = m[0][1]*x + m[1][1]*y + m[2][1]

with bilinear interpolation and a constant border: each of the four taps outside the source
reads the border value.  theta is the 6 matrix entries in storage order
(m00, m01, m10, m11, m20, m21).  The perspective variant follows the reference's U8
WarpPerspective (ago_haf_cpu_geometric.cpp:1594-1602) with its 9 entries in storage order.
The remap variant samples at (x + dx[y, x], y + dy[y, x]).
Loss: sum over pixels of (out - target)^2.

`*_frozen` evaluate the same interpolation with every pixel's integer cell fixed to the cell
of a reference position: the loss is then a polynomial in theta (or the field), whose central
differences converge to the derivative the adjoint computes.  Plain central differences of
a bilinear warp do not, because moving theta moves many samples across cell borders, where
the interpolant's derivative jumps."""
from __future__ import annotations

import numpy as np


def _cells(xs, ys):
    return np.floor(xs).astype(np.int64), np.floor(ys).astype(np.int64)


def _taps(src, x0, y0, border):
    H, W = src.shape

    def at(yy, xx):
        ok = (xx >= 0) & (xx < W) & (yy >= 0) & (yy < H)
        v = np.full(xx.shape, border, np.float64)
        v[ok] = src[yy[ok], xx[ok]]
        return v, ok

    p00, k00 = at(y0, x0)
    p01, k01 = at(y0, x0 + 1)
    p10, k10 = at(y0 + 1, x0)
    p11, k11 = at(y0 + 1, x0 + 1)
    return (p00, p01, p10, p11), (k00, k01, k10, k11)


def _interp(p, fx, fy):
    p00, p01, p10, p11 = p
    return (p00 * (1 - fx) + p01 * fx) * (1 - fy) + (p10 * (1 - fx) + p11 * fx) * fy


def sample(src, xs, ys, border=0.0, cells=None):
    """Bilinear sample at (xs, ys); `cells` = (x0, y0) fixes the integer cell of every pixel."""
    src = np.asarray(src, np.float64)
    x0, y0 = _cells(xs, ys) if cells is None else cells
    p, _ = _taps(src, x0, y0, border)
    return _interp(p, xs - x0, ys - y0)


def affine_coords(theta, H, W):
    yy, xx = np.meshgrid(np.arange(H, dtype=np.float64), np.arange(W, dtype=np.float64), indexing="ij")
    a, d, b, e, c, f = (float(t) for t in theta)
    return a * xx + b * yy + c, d * xx + e * yy + f, xx, yy


def warp_affine(src, theta, border=0.0, cells=None):
    H, W = src.shape
    xs, ys, _, _ = affine_coords(theta, H, W)
    return sample(src, xs, ys, border, cells)


def affine_cells(theta, H, W):
    xs, ys, _, _ = affine_coords(theta, H, W)
    return _cells(xs, ys)


def perspective_coords(theta, H, W):
    """Source positions of the perspective warp (ago_haf_cpu_geometric.cpp:1594-1602,
    ago_perspective_matrix_t m[3][3] in storage order): z = m02 x + m12 y + m22,
    xs = (m00 x + m10 y + m20) / z, ys = (m01 x + m11 y + m21) / z."""
    yy, xx = np.meshgrid(np.arange(H, dtype=np.float64), np.arange(W, dtype=np.float64), indexing="ij")
    a, d, g, b, e, h, c, f, i = (float(t) for t in theta)
    z = g * xx + h * yy + i
    return (a * xx + b * yy + c) / z, (d * xx + e * yy + f) / z, z, xx, yy


def warp_perspective(src, theta, border=0.0, cells=None):
    H, W = src.shape
    xs, ys, _, _, _ = perspective_coords(theta, H, W)
    return sample(src, xs, ys, border, cells)


def perspective_cells(theta, H, W):
    xs, ys, _, _, _ = perspective_coords(theta, H, W)
    return _cells(xs, ys)


def warp_perspective_adjoint(src, theta, gout, border=0.0):
    """(dL/dsrc, dL/dtheta) for L = sum(gout * warp_perspective(src, theta)); theta order as
    perspective_coords: d xs / d(m00, m10, m20) = (x, y, 1) / z, d xs / d(m02, m12, m22) =
    -xs (x, y, 1) / z, and the same for ys with (m01, m11, m21)."""
    H, W = src.shape
    xs, ys, z, xx, yy = perspective_coords(theta, H, W)
    gsrc, gxs, gys = _sample_adjoint(src, xs, ys, gout, border)
    q = -(gxs * xs + gys * ys) / z
    gx, gy = gxs / z, gys / z
    gtheta = np.array([(gx * xx).sum(), (gy * xx).sum(), (q * xx).sum(), (gx * yy).sum(), (gy * yy).sum(),
                       (q * yy).sum(), gx.sum(), gy.sum(), q.sum()])
    return gsrc, gtheta


def remap(src, field, border=0.0, cells=None):
    H, W = src.shape
    yy, xx = np.meshgrid(np.arange(H, dtype=np.float64), np.arange(W, dtype=np.float64), indexing="ij")
    return sample(src, xx + field[..., 0], yy + field[..., 1], border, cells)


def remap_cells(field):
    H, W = field.shape[:2]
    yy, xx = np.meshgrid(np.arange(H, dtype=np.float64), np.arange(W, dtype=np.float64), indexing="ij")
    return _cells(xx + field[..., 0], yy + field[..., 1])


def _sample_adjoint(src, xs, ys, gout, border):
    """d/dsrc (scatter) and d/dxs, d/dys of sum(gout * sample(src, xs, ys))."""
    src = np.asarray(src, np.float64)
    H, W = src.shape
    x0, y0 = _cells(xs, ys)
    fx, fy = xs - x0, ys - y0
    (p00, p01, p10, p11), (k00, k01, k10, k11) = _taps(src, x0, y0, border)
    gsrc = np.zeros((H, W), np.float64)
    for (dy, dx, k, w) in ((0, 0, k00, (1 - fx) * (1 - fy)), (0, 1, k01, fx * (1 - fy)),
                           (1, 0, k10, (1 - fx) * fy), (1, 1, k11, fx * fy)):
        np.add.at(gsrc, ((y0 + dy)[k], (x0 + dx)[k]), (gout * w)[k])
    gxs = gout * ((1 - fy) * (p01 - p00) + fy * (p11 - p10))
    gys = gout * ((1 - fx) * (p10 - p00) + fx * (p11 - p01))
    return gsrc, gxs, gys


def warp_affine_adjoint(src, theta, gout, border=0.0):
    """(dL/dsrc, dL/dtheta) for L = sum(gout * warp_affine(src, theta))."""
    H, W = src.shape
    xs, ys, xx, yy = affine_coords(theta, H, W)
    gsrc, gxs, gys = _sample_adjoint(src, xs, ys, gout, border)
    gtheta = np.array([(gxs * xx).sum(), (gys * xx).sum(), (gxs * yy).sum(), (gys * yy).sum(), gxs.sum(), gys.sum()])
    return gsrc, gtheta


def remap_adjoint(src, field, gout, border=0.0):
    """(dL/dsrc, dL/dfield) for L = sum(gout * remap(src, field))."""
    H, W = src.shape
    yy, xx = np.meshgrid(np.arange(H, dtype=np.float64), np.arange(W, dtype=np.float64), indexing="ij")
    gsrc, gxs, gys = _sample_adjoint(src, xx + field[..., 0], yy + field[..., 1], gout, border)
    return gsrc, np.stack([gxs, gys], -1)


def l2_loss(out, target):
    return float(((out - target) ** 2).sum())
