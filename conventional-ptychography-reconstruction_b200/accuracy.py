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
