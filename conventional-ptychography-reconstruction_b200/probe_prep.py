"""Probe centring / energy normalisation and Haar sparsity on the B200 kernels.

``center_and_normalize_probe(P)`` is the per-minibatch probe preparation of
Recovery.py:262-285 -- roll by the centre-of-mass offset, then scale to
sum |P|^2 = M*N -- as one forward kernel and one backward kernel
(``ptycho_probe_center_normalize`` / ``..._backward``), differentiable in P
(the roll amount is an integer and carries no gradient; the scale does).

``haar_sparsity(img)`` is haar_wavelet_sparsity_loss (utils/loss.py:60-83,
added at Recovery.py:309-313) as a deterministic FP64 reduction and an
elementwise backward (``ptycho_haar_sparsity`` / ``..._backward``).
"""
from __future__ import annotations

import torch

from . import _lib


class _ProbePrep(torch.autograd.Function):
    @staticmethod
    def forward(ctx, P):
        M, N = P.shape
        Pc = P.to(torch.complex64).contiguous()
        out = torch.empty((M, N), dtype=torch.complex64, device=P.device)
        state = torch.empty(4, dtype=torch.float64, device=P.device)
        _lib.check(_lib.lib().ptycho_probe_center_normalize(
            Pc.data_ptr(), M, N, out.data_ptr(), state.data_ptr(),
            torch.cuda.current_stream(P.device).cuda_stream), "ptycho_probe_center_normalize")
        ctx.save_for_backward(out, state)
        return out

    @staticmethod
    def backward(ctx, g):
        out, state = ctx.saved_tensors
        M, N = out.shape
        gc = g.to(torch.complex64).contiguous()
        gin = torch.empty((M, N), dtype=torch.complex64, device=g.device)
        _lib.check(_lib.lib().ptycho_probe_center_normalize_backward(
            out.data_ptr(), state.data_ptr(), gc.data_ptr(), M, N, gin.data_ptr(),
            torch.cuda.current_stream(g.device).cuda_stream), "ptycho_probe_center_normalize_backward")
        return gin


def center_and_normalize_probe(P: torch.Tensor) -> torch.Tensor:
    """[M, N] complex CUDA probe -> centred probe with sum |P|^2 = M*N."""
    if not P.is_cuda:
        raise ValueError("the probe must be a CUDA tensor (there is no CPU path)")
    if P.dim() != 2:
        raise ValueError(f"the probe must be 2-D, got shape {tuple(P.shape)}")
    return _ProbePrep.apply(P)


class _Haar(torch.autograd.Function):
    @staticmethod
    def forward(ctx, img):
        H, W = img.shape
        x = img.to(torch.complex64).contiguous()
        loss = torch.empty((), dtype=torch.float64, device=img.device)
        n = int(_lib.lib().ptycho_haar_sparsity_workspace_size(H, W))
        ws = torch.empty(max(n, 8), dtype=torch.uint8, device=img.device)
        _lib.check(_lib.lib().ptycho_haar_sparsity(x.data_ptr(), H, W, loss.data_ptr(), ws.data_ptr(), ws.numel(),
                                                   torch.cuda.current_stream(img.device).cuda_stream),
                   "ptycho_haar_sparsity")
        ctx.save_for_backward(x)
        return loss

    @staticmethod
    def backward(ctx, g):
        (x,) = ctx.saved_tensors
        H, W = x.shape
        gd = g.to(torch.float64).contiguous()
        gin = torch.empty_like(x)
        _lib.check(_lib.lib().ptycho_haar_sparsity_backward(x.data_ptr(), H, W, gd.data_ptr(), gin.data_ptr(),
                                                            torch.cuda.current_stream(x.device).cuda_stream),
                   "ptycho_haar_sparsity_backward")
        return gin


def haar_sparsity(img: torch.Tensor) -> torch.Tensor:
    """[H, W] complex CUDA image (H, W even) -> FP64 0-d Haar L1 sparsity."""
    if not img.is_cuda:
        raise ValueError("the image must be a CUDA tensor (there is no CPU path)")
    if img.dim() != 2 or img.shape[0] % 2 or img.shape[1] % 2:
        raise ValueError(f"the image must be 2-D with even sides, got {tuple(img.shape)}")
    return _Haar.apply(img)
