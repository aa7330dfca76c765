"""Differentiable F32 warps for PyTorch.

`warp_affine(src, theta)`, `warp_perspective(src, theta)` and `remap(src, field)` are
torch.autograd.Functions whose forward and backward passes are the CUDA kernels declared in
include/agocuda.h (bilinear sampling with a constant border; the coordinate conventions of
the reference's U8 warps: affine theta = (m00, m01, m10, m11, m20, m21), xs = m00*x + m10*y
+ m20, ys = m01*x + m11*y + m21; perspective theta = the 3x3 matrix in storage order,
z = m02*x + m12*y + m22, xs = (m00*x + m10*y + m20) / z, ys = (m01*x + m11*y + m21) / z).
`warp_affine_l2_step` / `warp_perspective_l2_step` run warp + L2 loss + adjoint in one
kernel pass.  Tensors are CUDA float32; images are (N, H, W), theta (N, 6) or (N, 9),
fields (N, H, W, 2).  The output has the
source's size.  There is no CPU implementation: without the native library these raise."""
from __future__ import annotations

import ctypes as C

import torch

from . import native

_i, _ll, _vp, _f = C.c_int, C.c_longlong, C.c_void_p, C.c_float
_SIGS = {
    "agocuda_WarpAffine_F32_Bilinear_Constant_batch": [_vp, _i, _i, _i, _vp, _ll, _i, _i, _i, _vp, _ll, _i, _vp, _f],
    "agocuda_WarpAffine_F32_Bilinear_Constant_adjoint_batch": [_vp, _i, _i, _i, _vp, _ll, _i, _i, _i, _vp, _ll, _i, _vp,
                                                               _f, _vp, _vp],
    "agocuda_WarpAffine_F32_L2_step_batch": [_vp, _i, _i, _i, _vp, _ll, _i, _i, _i, _vp, _ll, _i, _vp, _f, _vp, _vp],
    "agocuda_WarpPerspective_F32_Bilinear_Constant_batch": [_vp, _i, _i, _i, _vp, _ll, _i, _i, _i, _vp, _ll, _i, _vp,
                                                            _f],
    "agocuda_WarpPerspective_F32_Bilinear_Constant_adjoint_batch": [_vp, _i, _i, _i, _vp, _ll, _i, _i, _i, _vp, _ll, _i,
                                                                    _vp, _f, _vp, _vp],
    "agocuda_WarpPerspective_F32_L2_step_batch": [_vp, _i, _i, _i, _vp, _ll, _i, _i, _i, _vp, _ll, _i, _vp, _f, _vp, _vp],
    "agocuda_Remap_F32_Bilinear_Constant_batch": [_vp, _i, _i, _i, _vp, _ll, _i, _i, _i, _vp, _ll, _i, _vp, _ll, _i, _f],
    "agocuda_Remap_F32_Bilinear_Constant_adjoint_batch": [_vp, _i, _i, _i, _vp, _ll, _i, _i, _i, _vp, _ll, _i, _vp, _ll,
                                                          _i, _f, _vp, _vp],
}
_lib = None


def _L():
    global _lib
    if _lib is None:
        L = native.agocuda()
        for name, args in _SIGS.items():
            getattr(L, name).argtypes = args
            getattr(L, name).restype = C.c_int
        _lib = L
    return _lib


def _check(rc: int, what: str):
    if rc != 0:
        raise RuntimeError(f"{what} failed with status {rc}")


def _images(t: torch.Tensor, name: str) -> torch.Tensor:
    if not (t.is_cuda and t.dtype == torch.float32 and t.dim() == 3):
        raise ValueError(f"{name} must be a CUDA float32 tensor of shape (N, H, W)")
    return t.contiguous()


def _stream(t: torch.Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


class WarpAffineF32(torch.autograd.Function):
    @staticmethod
    def forward(ctx, src, theta, border=0.0):
        src = _images(src, "src")
        theta = theta.to(device=src.device, dtype=torch.float32).contiguous()
        N, H, W = src.shape
        if theta.shape != (N, 6):
            raise ValueError("theta must have shape (N, 6)")
        out = torch.empty_like(src)
        _check(_L().agocuda_WarpAffine_F32_Bilinear_Constant_batch(_stream(src), N, W, H, out.data_ptr(), H * W, W, W, H,
                                                                  src.data_ptr(), H * W, W, theta.data_ptr(), float(border)),
               "WarpAffine F32")
        ctx.save_for_backward(src, theta)
        ctx.border = float(border)
        return out

    @staticmethod
    def backward(ctx, gout):
        src, theta = ctx.saved_tensors
        N, H, W = src.shape
        gout = gout.to(torch.float32).contiguous()
        gsrc = torch.zeros_like(src)
        gth = torch.zeros((N, 6), dtype=torch.float64, device=src.device)
        _check(_L().agocuda_WarpAffine_F32_Bilinear_Constant_adjoint_batch(
            _stream(src), N, W, H, gout.data_ptr(), H * W, W, W, H, src.data_ptr(), H * W, W, theta.data_ptr(), ctx.border,
            gsrc.data_ptr(), gth.data_ptr()), "WarpAffine F32 adjoint")
        return gsrc, gth.to(torch.float32), None


class WarpPerspectiveF32(torch.autograd.Function):
    @staticmethod
    def forward(ctx, src, theta, border=0.0):
        src = _images(src, "src")
        theta = theta.to(device=src.device, dtype=torch.float32).contiguous()
        N, H, W = src.shape
        if theta.shape != (N, 9):
            raise ValueError("theta must have shape (N, 9)")
        out = torch.empty_like(src)
        _check(_L().agocuda_WarpPerspective_F32_Bilinear_Constant_batch(
            _stream(src), N, W, H, out.data_ptr(), H * W, W, W, H, src.data_ptr(), H * W, W, theta.data_ptr(),
            float(border)), "WarpPerspective F32")
        ctx.save_for_backward(src, theta)
        ctx.border = float(border)
        return out

    @staticmethod
    def backward(ctx, gout):
        src, theta = ctx.saved_tensors
        N, H, W = src.shape
        gout = gout.to(torch.float32).contiguous()
        gsrc = torch.zeros_like(src)
        gth = torch.zeros((N, 9), dtype=torch.float64, device=src.device)
        _check(_L().agocuda_WarpPerspective_F32_Bilinear_Constant_adjoint_batch(
            _stream(src), N, W, H, gout.data_ptr(), H * W, W, W, H, src.data_ptr(), H * W, W, theta.data_ptr(), ctx.border,
            gsrc.data_ptr(), gth.data_ptr()), "WarpPerspective F32 adjoint")
        return gsrc, gth.to(torch.float32), None


class RemapF32(torch.autograd.Function):
    @staticmethod
    def forward(ctx, src, field, border=0.0):
        src = _images(src, "src")
        N, H, W = src.shape
        field = field.to(device=src.device, dtype=torch.float32).contiguous()
        if field.shape != (N, H, W, 2):
            raise ValueError("field must have shape (N, H, W, 2)")
        out = torch.empty_like(src)
        _check(_L().agocuda_Remap_F32_Bilinear_Constant_batch(_stream(src), N, W, H, out.data_ptr(), H * W, W, W, H,
                                                             src.data_ptr(), H * W, W, field.data_ptr(), H * W, W,
                                                             float(border)), "Remap F32")
        ctx.save_for_backward(src, field)
        ctx.border = float(border)
        return out

    @staticmethod
    def backward(ctx, gout):
        src, field = ctx.saved_tensors
        N, H, W = src.shape
        gout = gout.to(torch.float32).contiguous()
        gsrc = torch.zeros_like(src)
        gfield = torch.empty_like(field)
        _check(_L().agocuda_Remap_F32_Bilinear_Constant_adjoint_batch(
            _stream(src), N, W, H, gout.data_ptr(), H * W, W, W, H, src.data_ptr(), H * W, W, field.data_ptr(), H * W, W,
            ctx.border, gsrc.data_ptr(), gfield.data_ptr()), "Remap F32 adjoint")
        return gsrc, gfield, None


def warp_affine(src: torch.Tensor, theta: torch.Tensor, border: float = 0.0) -> torch.Tensor:
    return WarpAffineF32.apply(src, theta, border)


def warp_perspective(src: torch.Tensor, theta: torch.Tensor, border: float = 0.0) -> torch.Tensor:
    return WarpPerspectiveF32.apply(src, theta, border)


def remap(src: torch.Tensor, field: torch.Tensor, border: float = 0.0) -> torch.Tensor:
    return RemapF32.apply(src, field, border)


def warp_affine_l2_step(src: torch.Tensor, theta: torch.Tensor, target: torch.Tensor, border: float = 0.0,
                        gsrc: torch.Tensor | None = None, acc: torch.Tensor | None = None):
    """For each image i: L_i = sum((warp_affine(src, theta)[i] - target[i])^2), dL_i/dsrc and
    dL_i/dtheta from one kernel pass.  Returns (loss (N,) float64, gsrc (N, H, W) float32,
    gtheta (N, 6) float64).  `gsrc` / `acc` may be passed in to reuse buffers (they are
    zeroed here)."""
    src, target = _images(src, "src"), _images(target, "target")
    N, H, W = src.shape
    theta = theta.to(device=src.device, dtype=torch.float32).contiguous()
    if gsrc is None:
        gsrc = torch.zeros_like(src)
    else:
        gsrc.zero_()
    if acc is None:
        acc = torch.zeros((N, 7), dtype=torch.float64, device=src.device)
    else:
        acc.zero_()
    _check(_L().agocuda_WarpAffine_F32_L2_step_batch(_stream(src), N, W, H, target.data_ptr(), H * W, W, W, H,
                                                     src.data_ptr(), H * W, W, theta.data_ptr(), float(border),
                                                     gsrc.data_ptr(), acc.data_ptr()), "WarpAffine F32 L2 step")
    return acc[:, 6], gsrc, acc[:, :6]


def warp_perspective_l2_step(src: torch.Tensor, theta: torch.Tensor, target: torch.Tensor, border: float = 0.0,
                             gsrc: torch.Tensor | None = None, acc: torch.Tensor | None = None):
    """warp_affine_l2_step for the perspective warp: returns (loss (N,) float64, gsrc
    (N, H, W) float32, gtheta (N, 9) float64)."""
    src, target = _images(src, "src"), _images(target, "target")
    N, H, W = src.shape
    theta = theta.to(device=src.device, dtype=torch.float32).contiguous()
    if theta.shape != (N, 9):
        raise ValueError("theta must have shape (N, 9)")
    if gsrc is None:
        gsrc = torch.zeros_like(src)
    else:
        gsrc.zero_()
    if acc is None:
        acc = torch.zeros((N, 10), dtype=torch.float64, device=src.device)
    else:
        acc.zero_()
    _check(_L().agocuda_WarpPerspective_F32_L2_step_batch(_stream(src), N, W, H, target.data_ptr(), H * W, W, W, H,
                                                          src.data_ptr(), H * W, W, theta.data_ptr(), float(border),
                                                          gsrc.data_ptr(), acc.data_ptr()), "WarpPerspective F32 L2 step")
    return acc[:, 9], gsrc, acc[:, :9]
