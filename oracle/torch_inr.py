"""The reference's INR training path in plain torch -- BASELINE / TEST ONLY.

Restates, for timing the reference on the same GPU, what Recovery.py runs
with model_type 'inr':

* ``TorchHashGrid`` -- the HashGrid encoding the reference takes from
  tiny-cuda-nn (models/complex_inr.py:130-145).  tiny-cuda-nn cannot be
  installed here, so this is a torch restatement of the same method
  (same indexing as ``oracle.inr``), labelled as such wherever it is timed;
* ``RefComplexMLP`` -- models/complex_inr.py:6-82 (torch complex64 layers,
  exp(1j * omega * linear(x)));
* ``RefINR`` -- models/complex_inr.py:85-306 (coordinate grids, object MLP at
  the downsampled grid, torch.fft Fourier upsampling, probe MLP, residual);
* ``ref_minibatch`` -- Recovery.py:250-321: model(), probe COM roll with host
  syncs, energy normalisation, the per-frame loop of crop * probe ->
  torch.fft.fft2 -> fftshift -> |.|^2 -> loss, backward, Adam step.
"""
from __future__ import annotations

import math

import torch
import torch.nn as nn
import torch.nn.functional as F

from .inr import PRIME_Y, hashgrid_levels
from .torch_cpu_path import frame_loss


class TorchHashGrid(nn.Module):
    def __init__(self, n_levels, log2_hashmap_size, base_resolution, per_level_scale, seed=1337):
        super().__init__()
        self.levels = hashgrid_levels(n_levels, log2_hashmap_size, base_resolution, per_level_scale)
        n = sum(l[2] for l in self.levels)
        g = torch.Generator().manual_seed(seed)
        self.params = nn.Parameter(torch.rand(n * 2, generator=g) * 2e-4 - 1e-4)

    def forward(self, x):
        tab = self.params.view(-1, 2)
        out = []
        for (scale, res, n, off, dense) in self.levels:
            p = x * scale + 0.5
            g = torch.floor(p)
            f = p - g
            gi = g.to(torch.int64)
            acc = 0.0
            for dx, dy in ((0, 0), (1, 0), (0, 1), (1, 1)):
                cx, cy = gi[:, 0] + dx, gi[:, 1] + dy
                if dense:
                    e = cx + cy * res
                else:
                    e = (cx ^ ((cy * PRIME_Y) & 0xFFFFFFFF)) & 0xFFFFFFFF
                e = e % n + off
                wx = f[:, 0] if dx else 1.0 - f[:, 0]
                wy = f[:, 1] if dy else 1.0 - f[:, 1]
                acc = acc + (wx * wy)[:, None] * tab[e]
            out.append(acc)
        return torch.cat(out, dim=1)


class RefGaborLayer(nn.Module):
    def __init__(self, in_f, out_f, is_first=False, omega0=10.0, trainable=False):
        super().__init__()
        self.omega_0 = nn.Parameter(omega0 * torch.ones(1), trainable)
        self.linear = nn.Linear(in_f, out_f, dtype=torch.float if is_first else torch.cfloat)

    def forward(self, x):
        return torch.exp(1j * self.omega_0 * self.linear(x))


class RefComplexMLP(nn.Module):
    def __init__(self, in_f, hidden, layers, out_f, first_omega_0=10.0, hidden_omega_0=10.0, trainable=False):
        super().__init__()
        h = int(hidden / 2)
        net = [RefGaborLayer(in_f, h, True, first_omega_0, trainable)]
        net += [RefGaborLayer(h, h, False, hidden_omega_0, trainable) for _ in range(layers)]
        net.append(nn.Linear(h, out_f, dtype=torch.cfloat))
        self.net = nn.Sequential(*net)


class RefINR(nn.Module):
    def __init__(self, W, ds, pw, n_levels, log2_T, base, pls, w1, wh, hidden=64, layers=2, trainable=True,
                 probe_initial=None):
        super().__init__()
        self.enc = TorchHashGrid(n_levels, log2_T, base, pls)
        self.penc = TorchHashGrid(n_levels, log2_T, base, pls, seed=7331)
        self.omlp = RefComplexMLP(2 * n_levels, hidden, layers, 1, w1, wh, trainable)
        self.pmlp = RefComplexMLP(2 * n_levels, hidden, layers, 1, w1, wh, trainable)
        dw = W // ds
        xs = torch.linspace(0.5 / dw, 1 - 0.5 / dw, dw)
        xv, yv = torch.meshgrid([xs, xs], indexing="ij")
        self.register_buffer("xy", torch.stack((yv.flatten(), xv.flatten())).t().contiguous())
        ps = torch.linspace(0.5 / pw, 1 - 0.5 / pw, pw)
        xv, yv = torch.meshgrid([ps, ps], indexing="ij")
        self.register_buffer("pxy", torch.stack((yv.flatten(), xv.flatten())).t().contiguous())
        self.dw, self.ds, self.pw = dw, ds, pw
        if probe_initial is not None:
            self.register_buffer("probe_initial", probe_initial.clone())
            self.k_probe = nn.Parameter(torch.tensor(1e-8))
        else:
            self.probe_initial = None

    def forward(self):
        o = self.omlp.net(self.enc(self.xy).float()).reshape(self.dw, self.dw)
        X = torch.fft.fftshift(torch.fft.fft2(o), dim=(-2, -1))
        n = self.dw * self.ds
        p0 = (n - self.dw) // 2
        X = F.pad(X, (p0, n - self.dw - p0, p0, n - self.dw - p0))
        o = torch.fft.ifft2(torch.fft.ifftshift(X, dim=(-2, -1))) * (self.ds ** 2)
        p = self.pmlp.net(self.penc(self.pxy).float()).reshape(self.pw, self.pw)
        if self.probe_initial is not None:
            p = self.k_probe * p + self.probe_initial
        return o, p


def ref_minibatch(model, optimizer, stack_mmf, tlY, tlX, batch_idx, loss_type):
    """One reference minibatch (Recovery.py:250-321) on the GPU with torch.fft."""
    model.zero_grad()
    optimizer.zero_grad()
    obj, probe = model()
    with torch.no_grad():
        a = probe.abs() ** 2
        Mp, Np = a.shape
        tot = a.sum()
        cp = None if tot == 0 else torch.trunc(
            torch.tensor([Mp, Np], device=probe.device) / 2
            - torch.tensor([Mp, Np], device=probe.device)
            * torch.stack((a.sum(1).cumsum(0).mean(), a.sum(0).cumsum(0).mean())) / tot + 1).long()
    if cp is not None and cp.any():
        probe = torch.roll(probe, (-cp[0].item(), -cp[1].item()), (0, 1))
    e = (probe.abs() ** 2).sum()
    if e > 0:
        probe = probe * (float(probe.shape[-2] * probe.shape[-1]) / e).sqrt()
    M, N = probe.shape
    loss = 0.0
    for i in batch_idx:
        i = int(i)
        y, x = int(tlY[i]), int(tlX[i])
        I = torch.abs(torch.fft.fftshift(torch.fft.fft2(probe * obj[y:y + M, x:x + N]), dim=(-2, -1))) ** 2
        loss = loss + frame_loss(I, stack_mmf[:, :, i], loss_type)
    loss.backward()
    optimizer.step()
    return float(loss.detach())


def per_level_scale_for(finest, base, n_levels):
    return math.exp(math.log(finest / base) / (n_levels - 1))
