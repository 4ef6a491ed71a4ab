"""Reconstruction accuracy against a ground-truth object, on the B200.

``object_error(recon, truth, box)`` is the global-phase alignment of the
reference's analysis script (resolve_global_phase,
scripts/compare_object_ssim.py:92-98: alpha = arg sum conj(recon) * truth)
followed by the normalised error, as one FP64 device reduction
(``ptycho_object_error``) with fixed-order sums.  It reports the error after
the phase alone and after the least-squares complex factor, which also removes
the probe/object scale ambiguity the script handles by normalising amplitudes
to mean 1 (normalize_amp, :101-103).

``coverage_box(tlY, tlX, probe_shape, canvas_shape, frac)`` is the
high-coverage bounding box of the same script (scan_coverage_mask /
high_coverage_bbox, :42-72): pixels covered by >= ceil(frac * max) probe
footprints.  It is integer bookkeeping on the scan table and stays on the host.

Translation alignment, FP64 on the device: ``align_by_xcorr`` is the script's
integer placement of a recon inside a larger truth (:75-89);
``register_translation`` the sub-pixel shift between two same-size images
(upsampled-DFT cross-correlation, Guizar-Sicairos, Thurman and Fienup, Opt.
Lett. 33, 156, 2008); ``register_in_box`` its windowed, iterated use on the
high-coverage box of two canvases; ``object_error_aligned`` applies that shift
before ``object_error``.  These run once per evaluation, off the training path, on
torch's FP64 FFT and matrix products.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib


def coverage_box(tlY, tlX, probe_shape, canvas_shape, frac: float = 0.5):
    """(y0, y1, x0, x1) of the pixels covered by >= ceil(frac * max) windows."""
    M, N = probe_shape
    Hc, Wc = canvas_shape
    cov = np.zeros((Hc + 1, Wc + 1), dtype=np.int64)  # 2-D difference array
    for y, x in zip(np.asarray(tlY).ravel().tolist(), np.asarray(tlX).ravel().tolist()):
        y0, y1, x0, x1 = max(0, y), min(Hc, y + M), max(0, x), min(Wc, x + N)
        if y1 > y0 and x1 > x0:
            cov[y0, x0] += 1
            cov[y0, x1] -= 1
            cov[y1, x0] -= 1
            cov[y1, x1] += 1
    cov = cov.cumsum(0).cumsum(1)[:Hc, :Wc]
    if cov.max() <= 0:
        return 0, Hc, 0, Wc
    ys, xs = np.nonzero(cov >= max(1, int(math.ceil(frac * cov.max()))))
    return int(ys.min()), int(ys.max()) + 1, int(xs.min()), int(xs.max()) + 1


def object_error(recon: torch.Tensor, truth: torch.Tensor, box=None) -> dict:
    """FP64 error of ``recon`` against ``truth`` ([H, W] complex CUDA tensors)
    over ``box`` = (y0, y1, x0, x1) (default: the whole canvas).

    Returns ``nrmse`` (after the global phase), ``nrmse_scaled`` (after the
    least-squares complex factor), ``phase`` = exp(i alpha) and ``tensor``, the
    7 device doubles [nrmse, cos a, sin a, |c|, sum|recon|^2, sum|truth|^2,
    nrmse_scaled] before they are read back."""
    if not (recon.is_cuda and truth.is_cuda):
        raise ValueError("recon and truth must be CUDA tensors (there is no CPU path)")
    if recon.dim() != 2 or recon.shape != truth.shape:
        raise ValueError(f"recon and truth must be 2-D of one shape, got {tuple(recon.shape)}, {tuple(truth.shape)}")
    H, W = recon.shape
    y0, y1, x0, x1 = box if box is not None else (0, H, 0, W)
    r = recon.detach().to(torch.complex64).contiguous()
    t = truth.detach().to(device=r.device, dtype=torch.complex64).contiguous()
    out = torch.empty(7, dtype=torch.float64, device=r.device)
    n = int(_lib.lib().ptycho_object_error_workspace_size())
    ws = torch.empty(n, dtype=torch.uint8, device=r.device)
    _lib.check(_lib.lib().ptycho_object_error(r.data_ptr(), t.data_ptr(), H, W, int(y0), int(y1), int(x0), int(x1),
                                              out.data_ptr(), ws.data_ptr(), n,
                                              torch.cuda.current_stream(r.device).cuda_stream),
               "ptycho_object_error")
    v = out.tolist()
    return {"nrmse": v[0], "nrmse_scaled": v[6], "phase": complex(v[1], v[2]), "tensor": out}


def _need_cuda(*xs):
    for x in xs:
        if not x.is_cuda:
            raise ValueError("alignment inputs must be CUDA tensors (there is no CPU path)")


def _freqs(n: int, dev) -> torch.Tensor:
    return torch.fft.fftfreq(n, d=1.0 / n, device=dev, dtype=torch.float64)  # signed integer frequencies


def align_by_xcorr(recon_mag: torch.Tensor, truth_mag: torch.Tensor):
    """Integer (row, col) placing ``recon_mag`` inside ``truth_mag`` (at least as
    large): the first maximum, in row-major order over the offsets that keep the
    recon inside, of the circular cross-correlation of the mean-removed
    magnitudes with the recon zero-padded to the truth's size
    (scripts/compare_object_ssim.py:75-89)."""
    _need_cuda(recon_mag, truth_mag)
    r = recon_mag.detach().to(torch.float64)
    g = truth_mag.detach().to(device=r.device, dtype=torch.float64)
    H, W = r.shape
    Hg, Wg = g.shape
    if Hg < H or Wg < W:
        raise ValueError(f"truth ({Hg}x{Wg}) smaller than recon ({H}x{W})")
    rf = torch.fft.fft2(r - r.mean(), s=(Hg, Wg))
    gf = torch.fft.fft2(g - g.mean(), s=(Hg, Wg))
    xc = torch.fft.ifft2(gf * rf.conj()).real[:Hg - H + 1, :Wg - W + 1].contiguous()
    i = int(torch.argmax(xc))
    return divmod(i, xc.shape[1])


def register_translation(recon: torch.Tensor, truth: torch.Tensor, upsample: int = 100):
    """Sub-pixel shift (dy, dx) such that ``fourier_shift(recon, dy, dx)`` best
    matches ``truth`` (same shape): the FFT cross-correlation's peak to the
    pixel, then matrix DFTs of the cross-power spectrum on a 1/upsample grid over
    +-0.75 pixel around it.  FP64 on the device."""
    _need_cuda(recon, truth)
    r = recon.detach().to(torch.complex128)
    g = truth.detach().to(device=r.device, dtype=torch.complex128)
    if r.shape != g.shape or r.dim() != 2:
        raise ValueError("recon and truth must be 2-D of one shape")
    H, W = g.shape
    X = torch.fft.fft2(g) * torch.fft.fft2(r).conj()
    cc = torch.fft.ifft2(X).abs()
    py, px = divmod(int(torch.argmax(cc)), W)
    py = py - H if py > H // 2 else py
    px = px - W if px > W // 2 else px
    if upsample <= 1:
        return float(py), float(px)
    half = int(math.ceil(0.75 * upsample))
    offs = torch.arange(-half, half + 1, device=r.device, dtype=torch.float64) / upsample
    ys, xs = py + offs, px + offs
    Er = torch.exp(2j * math.pi * torch.outer(ys, _freqs(H, r.device)) / H)
    Ec = torch.exp(2j * math.pi * torch.outer(_freqs(W, r.device), xs) / W)
    up = (Er @ X @ Ec).abs()
    iy, ix = divmod(int(torch.argmax(up)), up.shape[1])
    return float(ys[iy]), float(xs[ix])


def fourier_shift(img: torch.Tensor, dy: float, dx: float) -> torch.Tensor:
    """``img`` translated by (dy, dx) pixels, out(y, x) = img(y - dy, x - dx),
    periodic; complex128 on the device."""
    _need_cuda(img)
    a = img.detach().to(torch.complex128)
    H, W = a.shape
    ph = torch.exp(-2j * math.pi * (_freqs(H, a.device)[:, None] * (dy / H) + _freqs(W, a.device)[None, :] * (dx / W)))
    return torch.fft.ifft2(torch.fft.fft2(a) * ph)


def register_in_box(recon: torch.Tensor, truth: torch.Tensor, box, upsample: int = 100, iters: int = 3):
    """Shift aligning the canvas ``recon`` to ``truth`` inside ``box``: the crops'
    mean is removed and a separable Hann window applied (the crops are not
    periodic), ``register_translation`` runs on them, the shift is applied to the
    whole canvas and the registration repeated on the shifted crop until the
    increment is zero (at most ``iters`` times); the increments add up."""
    _need_cuda(recon, truth)
    y0, y1, x0, x1 = box
    dev = recon.device

    def win(a):
        a = a - a.mean()
        wy = torch.hann_window(a.shape[0], periodic=False, dtype=torch.float64, device=dev)
        wx = torch.hann_window(a.shape[1], periodic=False, dtype=torch.float64, device=dev)
        return a * torch.outer(wy, wx)

    g = win(truth.detach().to(device=dev, dtype=torch.complex128)[y0:y1, x0:x1])
    dy = dx = 0.0
    for _ in range(iters):
        rs = fourier_shift(recon, dy, dx)[y0:y1, x0:x1]
        ey, ex = register_translation(win(rs), g, upsample)
        dy, dx = dy + ey, dx + ex
        if ey == 0.0 and ex == 0.0:
            break
    return dy, dx


def object_error_aligned(recon: torch.Tensor, truth: torch.Tensor, box=None, upsample: int = 100) -> dict:
    """``object_error`` after the sub-pixel translation that best aligns recon to
    truth over ``box`` (``register_in_box``; the shift is applied to the whole
    canvas, so the periodic wrap stays at the canvas edges).  Adds ``shift`` =
    (dy, dx)."""
    H, W = recon.shape
    box = box if box is not None else (0, H, 0, W)
    dy, dx = register_in_box(recon, truth, box, upsample)
    out = object_error(fourier_shift(recon, dy, dx).to(torch.complex64), truth, box)
    out["shift"] = (dy, dx)
    return out
