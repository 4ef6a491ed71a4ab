"""The reference's own torch CPU path for one minibatch -- TEST / BASELINE ONLY.

Restates, in torch on the CPU, what one minibatch of the reference training
loop does for the pixel terms (object and probe as plain complex64 leaves):
the per-frame loop of Recovery.py:288-307 -- crop * probe (:290), fft2 +
fftshift (:291), |.|^2 (:292), the inline losses (:294-305), summed over the
batch (:307) -- followed by ``loss.backward()`` (Recovery.py:316), i.e. torch
autograd (pocketfft + SliceBackward) for the adjoint.

Used as the timed CPU baseline (``bench.py`` cpu_baseline and
``--impl reference``); the reference tree itself is not available on the
measurement host, so this is the oracle port of that path.
"""
from __future__ import annotations

import torch
import torch.nn.functional as F


def frame_loss(oI_sub, oI_cap, loss_type):
    """Per-frame loss exactly as Recovery.py:294-305."""
    if loss_type == "smooth_L1_loss":
        return F.smooth_l1_loss(oI_sub, oI_cap)
    if loss_type == "FD_loss":
        eps = 1e-8
        dW = torch.sqrt(oI_cap + eps) - torch.sqrt(oI_sub + eps)
        RxdW = torch.cat((dW[:, 1:] - dW[:, :-1], dW[:, :1] - dW[:, -1:]), dim=1)
        RydW = torch.cat((dW[1:, :] - dW[:-1, :], dW[:1, :] - dW[-1:, :]), dim=0)
        return torch.sqrt(RxdW ** 2 + RydW ** 2 + eps).mean()
    if loss_type == "Poisson_likelihood_loss":
        eps = 1e-8
        return (oI_sub - oI_cap * torch.log(oI_sub + eps)).mean()
    raise ValueError(loss_type)


def minibatch_fwd_adj(obj, probe, tlY, tlX, stack_mmf, batch_idx, loss_type):
    """One minibatch: per-frame forward + loss, then autograd backward.

    ``obj``/``probe`` are complex64 leaf tensors with requires_grad; their
    ``.grad`` is zeroed first.  ``stack_mmf`` is the measurement stack in the
    reference layout [M, N, F].  Returns the summed loss (float)."""
    if obj.grad is not None:
        obj.grad = None
    if probe.grad is not None:
        probe.grad = None
    M, N = probe.shape
    loss_batch = 0.0
    for i in batch_idx:
        i = int(i)
        y, x = int(tlY[i]), int(tlX[i])
        oI_cap = stack_mmf[:, :, i]
        currentEW = probe * obj[y:y + M, x:x + N]
        fft_EW = torch.fft.fftshift(torch.fft.fft2(currentEW), dim=(-2, -1))
        oI_sub = torch.abs(fft_EW) ** 2
        loss_batch = loss_batch + frame_loss(oI_sub, oI_cap, loss_type)
    loss_batch.backward()
    return float(loss_batch.detach())
