"""Fourier upsampling of the INR object on the B200 kernels.

``fourier_upsample(x, s)`` computes, for a complex [h, w] tensor, what
models/complex_inr.py:252-271 computes with torch.fft:
``ifft2(ifftshift(pad(fftshift(fft2(x))))) * s**2`` -> [h*s, w*s], with the
backward pass (the operator's conjugate transpose) on the same kernels
(``ptycho_fourier_upsample`` / ``ptycho_fourier_upsample_adjoint``).
Sizes: any h, w >= 1 and integer s >= 1 with h*s, w*s <= 8192 (``supported``).
Power-of-two lines run compile-time radix-8/16 kernels; every other length
(the multiples of 3 that Recovery.py's canvases give, odd lengths, large
prime factors) runs the run-time-planned mixed-radix kernel.  There is no
torch.fft path: other shapes raise.
"""
from __future__ import annotations

import torch

from . import _lib

MAX_LEN = 8192


def supported(h: int, w: int, s) -> bool:
    if int(s) != s or int(s) < 1:
        return False
    s = int(s)
    return 1 <= h and 1 <= w and h * s <= MAX_LEN and w * s <= MAX_LEN


def _workspace(h, w, s, dev):
    n = int(_lib.lib().ptycho_fourier_upsample_workspace_size(h, w, s))
    return torch.empty(n, dtype=torch.uint8, device=dev), n


class _FourierUpsample(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, s: int):
        h, w = x.shape
        xc = x.to(torch.complex64).contiguous()
        y = torch.empty((h * s, w * s), dtype=torch.complex64, device=x.device)
        ws, n = _workspace(h, w, s, x.device)
        _lib.check(_lib.lib().ptycho_fourier_upsample(
            xc.data_ptr(), h, w, s, y.data_ptr(), ws.data_ptr(), n,
            torch.cuda.current_stream(x.device).cuda_stream), "ptycho_fourier_upsample")
        ctx.shape = (h, w, s)
        return y

    @staticmethod
    def backward(ctx, gy):
        h, w, s = ctx.shape
        g = gy.to(torch.complex64).contiguous()
        gx = torch.empty((h, w), dtype=torch.complex64, device=g.device)
        ws, n = _workspace(h, w, s, g.device)
        _lib.check(_lib.lib().ptycho_fourier_upsample_adjoint(
            g.data_ptr(), h, w, s, gx.data_ptr(), ws.data_ptr(), n,
            torch.cuda.current_stream(g.device).cuda_stream), "ptycho_fourier_upsample_adjoint")
        return gx, None


def fourier_upsample(x: torch.Tensor, s: int) -> torch.Tensor:
    """[h, w] complex CUDA tensor -> [h*s, w*s] complex64, differentiable."""
    if not x.is_cuda:
        raise ValueError("x must be a CUDA tensor (there is no CPU path)")
    if x.dim() != 2 or not supported(x.shape[0], x.shape[1], s):
        raise ValueError(f"unsupported shape {tuple(x.shape)} with scale {s}")
    return _FourierUpsample.apply(x, int(s))
