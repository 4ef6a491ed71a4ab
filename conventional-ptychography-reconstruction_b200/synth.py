"""Seeded synthetic ptychography workloads (stand-ins for the reference's
datasets, which are not distributed).

Each workload follows the generation recipe of the benchmark configurations:

* object: amplitude ``0.6 + 0.4 u``, phase ``pi (u' - 0.5)``; ``u``, ``u'`` are
  independent uniform fields (seed 0) smoothed by a sigma = 4 px Gaussian and
  min-max normalised;
* probe: a disk of radius R (22 px for the 64^2 probe, 0.35 N otherwise)
  softened by a sigma = 2 px Gaussian, times ``exp(i 0.002 r^2)``, normalised to
  unit energy;
* scan: an n x n raster with step s plus integer jitter U[-j, j] (seed 2),
  centred so every window lies inside the canvas;
* data: ``I = |fftshift(fft2(P * O_window))|^2`` in FP64, scaled so the
  brightest pixel of the stack is ``peak`` photons, Poisson noise (seed 1),
  stored FP32 as [F, M, M] (frames first).

Generation runs once, outside any timed region; on a CUDA device the FP64
transforms use torch.fft for speed (data preparation, not the measured path).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

try:  # scipy is part of the image; keep the import local to generation
    from scipy.ndimage import gaussian_filter
except Exception:  # pragma: no cover
    gaussian_filter = None


@dataclass(frozen=True)
class Workload:
    name: str
    canvas: int
    probe: int
    n_scan: int
    step: int
    jitter: int
    peak: float
    loss_type: str
    batch: int
    aperture: float  # radius in px (absolute) when > 1, else fraction of N


WORKLOADS = {
    "c0": Workload("c0: 256^2 object, 64^2 probe, 10x10 raster, smooth_L1", 256, 64, 10, 16, 2,
                   1e4, "smooth_L1_loss", 10, 22.0),
    "c1": Workload("c1: 1536^2 object, 128^2 probe, 40x40 raster (1600 positions), Poisson, batch 256",
                   1536, 128, 40, 32, 3, 1e4, "Poisson_likelihood_loss", 256, 0.35),
    "c2": Workload("c2: 1024^2 canvas, 128^2 probe, 28x28 raster, smooth_L1 (INR)", 1024, 128, 28, 32, 0,
                   1e4, "smooth_L1_loss", 10, 0.35),
    "c3": Workload("c3: 2048^2 object, 256^2 probe, 48x48 raster, Poisson, 1e3 photons", 2048, 256, 48,
                   36, 4, 1e3, "Poisson_likelihood_loss", 64, 0.35),
    "c4": Workload("c4: 4096^2 object, 256^2 probe, 96x96 raster (9216 positions), Poisson, batch 512",
                   4096, 256, 96, 40, 0, 1e3, "Poisson_likelihood_loss", 512, 0.35),
}


def _smooth_unit(rng, shape, sigma):
    u = gaussian_filter(rng.random(shape), sigma)
    return (u - u.min()) / (u.max() - u.min())


def make_object(n: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    u = _smooth_unit(rng, (n, n), 4.0)
    u2 = _smooth_unit(rng, (n, n), 4.0)
    return ((0.6 + 0.4 * u) * np.exp(1j * np.pi * (u2 - 0.5))).astype(np.complex128)


def make_probe(n: int, radius: float) -> np.ndarray:
    R = radius if radius > 1 else radius * n
    yy, xx = np.mgrid[:n, :n] - n / 2
    r2 = yy * yy + xx * xx
    disk = gaussian_filter((r2 <= R * R).astype(np.float64), 2.0)
    P = disk * np.exp(1j * 0.002 * r2)
    return P / np.sqrt((np.abs(P) ** 2).sum())


def make_scan(n_scan: int, step: int, jitter: int, canvas: int, probe: int, seed: int = 2):
    rng = np.random.default_rng(seed)
    extent = (n_scan - 1) * step + probe
    off = (canvas - extent) // 2
    iy, ix = np.mgrid[:n_scan, :n_scan]
    tlY = off + iy.ravel() * step + rng.integers(-jitter, jitter + 1, size=n_scan * n_scan)
    tlX = off + ix.ravel() * step + rng.integers(-jitter, jitter + 1, size=n_scan * n_scan)
    tlY = np.clip(tlY, 0, canvas - probe).astype(np.int32)
    tlX = np.clip(tlX, 0, canvas - probe).astype(np.int32)
    return tlY, tlX


def _intensities(O, P, tlY, tlX, device=None, chunk=256):
    M = P.shape[0]
    F = len(tlY)
    try:
        import torch
        use_torch = device is not None and torch.cuda.is_available()
    except Exception:  # pragma: no cover
        use_torch = False
    out = np.empty((F, M, M), np.float64)
    if use_torch:
        Ot = torch.from_numpy(O).to(device)
        Pt = torch.from_numpy(P).to(device)
        ar = torch.arange(M, device=device)
        for s in range(0, F, chunk):
            ty = torch.from_numpy(tlY[s:s + chunk].astype(np.int64)).to(device)
            tx = torch.from_numpy(tlX[s:s + chunk].astype(np.int64)).to(device)
            rows = (ty[:, None] + ar[None, :])[:, :, None]
            cols = (tx[:, None] + ar[None, :])[:, None, :]
            psi = Pt[None] * Ot[rows, cols]
            I = torch.abs(torch.fft.fftshift(torch.fft.fft2(psi), dim=(-2, -1))) ** 2
            out[s:s + chunk] = I.cpu().numpy()
    else:
        for b in range(F):
            y, x = int(tlY[b]), int(tlX[b])
            out[b] = np.abs(np.fft.fftshift(np.fft.fft2(P * O[y:y + M, x:x + M]))) ** 2
    return out


def make_workload(key: str, device=None, n_frames: int | None = None):
    """Return dict(obj, probe, tlY, tlX, Imeas [F,M,M] float32, workload)."""
    w = WORKLOADS[key]
    O = make_object(w.canvas, seed=0)
    P = make_probe(w.probe, w.aperture)
    tlY, tlX = make_scan(w.n_scan, w.step, w.jitter, w.canvas, w.probe, seed=2)
    if n_frames is not None:
        tlY, tlX = tlY[:n_frames], tlX[:n_frames]
    I = _intensities(O, P, tlY, tlX, device=device)
    I *= w.peak / I.max()
    rng = np.random.default_rng(1)
    Imeas = rng.poisson(I).astype(np.float32)
    return {"obj": O, "probe": P, "tlY": tlY, "tlX": tlX, "Imeas": Imeas, "workload": w}
