"""Scan-position sharding for one process per GPU (data parallel).

Scan positions are independent units of the forward model: rank r takes a
contiguous band of the raster (positions ordered by (tlY, tlX), cut into
``world`` blocks of near-equal count), draws its minibatches from that band,
keeps a full replica of the object / probe (or of the INR), and after its
local fused forward + adjoint sums the gradients with the other ranks:

* dP -- one all-reduce of the [M, M] probe gradient;
* dO -- one all-reduce of the canvas rows that any rank's windows touch
  (``scanned_rows``; a contiguous slice of the row-major canvas, so no
  packing), rows outside it are zero on every rank.

With every rank applying the same optimizer step to the same summed
gradients, the replicas stay identical.  This is the exchange step of the
reference's per-minibatch loop (Recovery.py:243-321) when its frames are
split across GPUs; the reference itself runs on one device.
"""
from __future__ import annotations

import numpy as np
import torch


def shard_frames(tlY, tlX, world: int, rank: int) -> np.ndarray:
    """Frame ids of ``rank``: a contiguous block of the raster order
    (sorted by tlY, then tlX), sorted ascending.  Blocks differ in size by at
    most one frame and together cover every frame exactly once."""
    tlY = np.asarray(tlY)
    tlX = np.asarray(tlX)
    if tlY.shape != tlX.shape or tlY.ndim != 1:
        raise ValueError("tlY and tlX must be 1-D arrays of equal length")
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of size {world}")
    F = tlY.shape[0]
    order = np.lexsort((tlX, tlY))
    lo = (F * rank) // world
    hi = (F * (rank + 1)) // world
    return np.sort(order[lo:hi]).astype(np.int64)


def window_bbox(tlY, tlX, frames, M: int):
    """(y0, y1, x0, x1): the canvas box covered by the windows of ``frames``
    (half-open; (0, 0, 0, 0) for no frames)."""
    frames = np.asarray(frames, dtype=np.int64)
    if frames.size == 0:
        return 0, 0, 0, 0
    ty = np.asarray(tlY)[frames]
    tx = np.asarray(tlX)[frames]
    return int(ty.min()), int(ty.max()) + M, int(tx.min()), int(tx.max()) + M


def scanned_rows(tlY, tlX, M: int):
    """(y0, y1): the canvas rows any window touches (all frames, all ranks)."""
    y0, y1, _, _ = window_bbox(tlY, tlX, np.arange(len(tlY)), M)
    return y0, y1


class GradientExchange:
    """Sums dO (over the scanned rows) and dP across the ranks of ``group``.

    ``dO`` [H, W] and ``dP`` [M, M] complex tensors are reduced in place
    through their real views; a world of one does nothing.  Every rank
    issues the same two collectives in the same order."""

    def __init__(self, tlY, tlX, M: int, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
        self.rows = scanned_rows(tlY, tlX, M)

    def all_reduce(self, dO=None, dP=None):
        if self.world == 1:
            return dO, dP
        y0, y1 = self.rows
        if dO is not None:
            band = torch.view_as_real(dO[y0:y1])  # contiguous rows of a row-major canvas
            self.dist.all_reduce(band, group=self.group)
        if dP is not None:
            self.dist.all_reduce(torch.view_as_real(dP), group=self.group)
        return dO, dP


def steps_per_epoch(n_frames: int, world: int, batch_size: int) -> int:
    """Minibatches per epoch on every rank: enough for the largest band, so
    all ranks take the same number of steps (and collectives) per epoch."""
    largest = -(-n_frames // world)
    return max(1, -(-largest // batch_size))


def epoch_minibatches(frames: np.ndarray, batch_size: int, steps: int, rng: np.random.Generator):
    """``steps`` minibatches: permutations of this rank's frames, each cut into
    ``batch_size`` slices (the last one short, as Recovery.py:243-249 cuts its
    epoch); a band that runs out before ``steps`` continues with the next
    permutation."""
    if frames.size == 0:
        raise ValueError("a rank needs at least one frame")
    out = []
    while len(out) < steps:
        perm = frames[rng.permutation(frames.size)]
        out.extend(perm[i:i + batch_size] for i in range(0, perm.size, batch_size))
    return out[:steps]


def all_reduce_grads(params, group=None):
    """Sum the gradients of ``params`` over the ranks (in parameter order; real
    views of complex gradients), as data-parallel training does after each
    local backward pass."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return
    for p in params:
        if p.grad is not None:
            g = torch.view_as_real(p.grad) if p.grad.is_complex() else p.grad
            dist.all_reduce(g, group=group)
