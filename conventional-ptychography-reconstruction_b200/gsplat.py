"""2-D complex Gaussian splatting on the B200 kernels (``csrc/gsplat.cu``).

Drop-in for the reference's gscp rasteriser bindings
(gscp/cuda/_wrapper.py:18-163): ``GaussianRasterize2D`` (rotation + scaling)
and ``GaussianRasterize2DCholesky`` (L L^T) are autograd Functions with the
same ``apply`` arguments and the same [2, H, W] (real, imaginary) output.

    out = GaussianRasterize2D.apply(xy, scaling, rotation, weight, H, W, max_patch_radius, min_scale)
    out = GaussianRasterize2DCholesky.apply(xy, log_L_diag, L_offdiag, weight, H, W, max_patch_radius, min_scale)

``xy`` [N, 2] pixel positions, ``scaling`` / ``log_L_diag`` [N, 2] in log
space, ``rotation`` [N, 1] or ``L_offdiag`` [N], ``weight`` [N, 2]; all float32
CUDA tensors.  The forward keeps its per-Gaussian geometry and tile masks for
the backward (as the reference keeps its geometry/binning buffers), runs
without a host synchronisation, and the backward is deterministic.
"""
from __future__ import annotations

import torch

from . import _lib

RS, CHOLESKY = 0, 1


def _prep(x, shape, name):
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (there is no CPU path)")
    return x.detach().to(torch.float32).contiguous().reshape(shape)


def _forward(kind, xy, p1, p2, weight, H, W, max_patch_radius, min_scale):
    N = int(xy.shape[0])
    dev = xy.device
    xy_ = _prep(xy, (N, 2), "xy")
    p1_ = _prep(p1, (N, 2), "scaling" if kind == RS else "log_L_diag")
    p2_ = _prep(p2, (N,), "rotation" if kind == RS else "L_offdiag")
    w_ = _prep(weight, (N, 2), "weight")
    H, W = int(H), int(W)
    out = torch.empty((2, H, W), dtype=torch.float32, device=dev)
    radii = torch.empty(N, dtype=torch.int32, device=dev)
    nbytes = int(_lib.lib().ptycho_gs_workspace_size(N, H, W))
    ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=dev)
    _lib.check(_lib.lib().ptycho_gs_forward(kind, xy_.data_ptr(), p1_.data_ptr(), p2_.data_ptr(), w_.data_ptr(),
                                            N, H, W, int(max_patch_radius), float(min_scale), out.data_ptr(),
                                            radii.data_ptr() if N else None, ws.data_ptr(), ws.numel(),
                                            torch.cuda.current_stream(dev).cuda_stream), "ptycho_gs_forward")
    return out, radii, ws, (xy_, p1_, p2_, w_)


def _backward(kind, saved, ws, H, W, max_patch_radius, min_scale, gout):
    xy_, p1_, p2_, w_ = saved
    N = int(xy_.shape[0])
    dev = xy_.device
    g = gout.detach().to(torch.float32).contiguous()
    dxy = torch.empty((N, 2), dtype=torch.float32, device=dev)
    dp1 = torch.empty((N, 2), dtype=torch.float32, device=dev)
    dp2 = torch.empty(N, dtype=torch.float32, device=dev)
    dw = torch.empty((N, 2), dtype=torch.float32, device=dev)
    if N:
        _lib.check(_lib.lib().ptycho_gs_backward(
            kind, xy_.data_ptr(), p1_.data_ptr(), p2_.data_ptr(), w_.data_ptr(), N, H, W, int(max_patch_radius),
            float(min_scale), g.data_ptr(), ws.data_ptr(), ws.numel(), dxy.data_ptr(), dp1.data_ptr(),
            dp2.data_ptr(), dw.data_ptr(), torch.cuda.current_stream(dev).cuda_stream), "ptycho_gs_backward")
    return dxy, dp1, dp2, dw


class GaussianRasterize2D(torch.autograd.Function):
    """(xy, scaling, rotation, weight, H, W, max_patch_radius, min_scale) -> [2, H, W]."""

    @staticmethod
    def forward(ctx, xy, scaling, rotation, weight, H, W, max_patch_radius, min_scale=0.5):
        out, radii, ws, saved = _forward(RS, xy, scaling, rotation, weight, H, W, max_patch_radius, min_scale)
        ctx.save_for_backward(*saved, ws)
        ctx.meta = (int(H), int(W), max_patch_radius, min_scale, tuple(rotation.shape))
        ctx.radii = radii
        return out

    @staticmethod
    def backward(ctx, gout):
        *saved, ws = ctx.saved_tensors
        H, W, R, ms, rshape = ctx.meta
        dxy, dp1, dp2, dw = _backward(RS, saved, ws, H, W, R, ms, gout)
        return dxy, dp1, dp2.reshape(rshape), dw, None, None, None, None


class GaussianRasterize2DCholesky(torch.autograd.Function):
    """(xy, log_L_diag, L_offdiag, weight, H, W, max_patch_radius, min_scale) -> [2, H, W]."""

    @staticmethod
    def forward(ctx, xy, log_L_diag, L_offdiag, weight, H, W, max_patch_radius, min_scale=0.5):
        out, radii, ws, saved = _forward(CHOLESKY, xy, log_L_diag, L_offdiag, weight, H, W, max_patch_radius,
                                         min_scale)
        ctx.save_for_backward(*saved, ws)
        ctx.meta = (int(H), int(W), max_patch_radius, min_scale, tuple(L_offdiag.shape))
        ctx.radii = radii
        return out

    @staticmethod
    def backward(ctx, gout):
        *saved, ws = ctx.saved_tensors
        H, W, R, ms, oshape = ctx.meta
        dxy, dp1, dp2, dw = _backward(CHOLESKY, saved, ws, H, W, R, ms, gout)
        return dxy, dp1, dp2.reshape(oshape), dw, None, None, None, None


def rasterize(kind, xy, p1, p2, weight, H, W, max_patch_radius, min_scale=0.5):
    """Forward only: ([2, H, W] image, int32 radii [N]) -- no autograd."""
    out, radii, _, _ = _forward(kind, xy, p1, p2, weight, H, W, max_patch_radius, min_scale)
    return out, radii
