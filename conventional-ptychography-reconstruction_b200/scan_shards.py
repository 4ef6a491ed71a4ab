"""Scan-position sharding for one process per GPU (data parallel).

Scan positions are independent units of the forward model: rank r takes a
contiguous band of the raster (positions ordered by (tlY, tlX), cut into
``world`` blocks of near-equal count), draws its minibatches from that band,
keeps a replica of the object / probe (or of the INR), and after its local
fused forward + adjoint combines the gradients with the other ranks:

* dP -- one all-reduce of the [M, N] probe gradient;
* dO -- a halo exchange.  Rank r's object gradient is non-zero only on the
  canvas rows its windows touch, its band [y0_r, y1_r).  Rows that no other
  band touches already hold the full gradient; on rows shared with other
  bands (the halo, about M - step rows per boundary) the ranks that touch
  them swap their partial gradients point to point and each adds all of
  them in rank order, so every such rank holds bitwise the same sum.  Only
  halo rows cross the link, not the canvas.

Each rank then applies the same optimizer step to the rows it holds; a
rank's object is current on its own band, which is all its windows read.
``gather_object`` assembles the whole object from the ranks' owned rows
(before evaluating it on all frames or saving it).  This is the exchange
step of the reference's per-minibatch loop (Recovery.py:243-321) when its
frames are split across GPUs; the reference itself runs on one device.
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


def window_bbox(tlY, tlX, frames, M: int, N: int | None = None):
    """(y0, y1, x0, x1): the canvas box covered by the M x N windows of
    ``frames`` (half-open; (0, 0, 0, 0) for no frames; N defaults to M)."""
    N = M if N is None else N
    frames = np.asarray(frames, dtype=np.int64)
    if frames.size == 0:
        return 0, 0, 0, 0
    ty = np.asarray(tlY)[frames]
    tx = np.asarray(tlX)[frames]
    return int(ty.min()), int(ty.max()) + M, int(tx.min()), int(tx.max()) + N


def scanned_rows(tlY, tlX, M: int):
    """(y0, y1): the canvas rows any window touches (all frames, all ranks)."""
    y0, y1, _, _ = window_bbox(tlY, tlX, np.arange(len(tlY)), M)
    return y0, y1


def band_rows(tlY, tlX, M: int, world: int):
    """[(y0_r, y1_r)] for every rank: the rows its band's windows touch."""
    out = []
    for r in range(world):
        y0, y1, _, _ = window_bbox(tlY, tlX, shard_frames(tlY, tlX, world, r), M)
        out.append((y0, y1))
    return out


def owned_rows(bands, H: int):
    """A disjoint cover of [0, H) by rank: rank r owns [o_r, o_{r+1}) with
    o_0 = 0, o_r = y0_r (bands start in raster order), o_world = H.  A row
    owned by r lies in r's band or in no band at all (then no rank updates it)."""
    world = len(bands)
    o = [0] + [min(max(bands[r][0], 0), H) for r in range(1, world)] + [H]
    for r in range(1, world + 1):
        o[r] = max(o[r], o[r - 1])
    return [(o[r], o[r + 1]) for r in range(world)]


class GradientExchange:
    """Combines dO (halo exchange over the ranks' bands) and dP (all-reduce)
    across the ranks of ``group``; see the module notes.

    ``dO`` [H, W] and ``dP`` [M, N] complex tensors are combined in place
    through their real views; a world of one does nothing.  After
    ``all_reduce`` a rank's dO holds the full gradient on its band rows
    (outside them, its own zero rows).  ``halo=False`` all-reduces the
    scanned rows instead (every rank then holds the full gradient
    everywhere; used when a term couples rows across band edges, such as the
    Haar sparsity loss).  Every rank issues the same operations in the same
    order; ``bytes_per_step`` is what one rank sends per call."""

    def __init__(self, tlY, tlX, M: int, group=None, halo: bool = True, W: int | None = None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        init = dist.is_available() and dist.is_initialized()
        self.world = dist.get_world_size(group) if init else 1
        self.rank = dist.get_rank(group) if init else 0
        self.rows = scanned_rows(tlY, tlX, M)
        self.halo = halo
        self.bands = band_rows(tlY, tlX, M, self.world)
        y0, y1 = self.bands[self.rank]
        # rows of my band shared with each other rank: [(rank, a, b)] in rank order
        self.shared = []
        for q, (q0, q1) in enumerate(self.bands):
            a, b = max(y0, q0), min(y1, q1)
            if q != self.rank and b > a:
                self.shared.append((q, a, b))
        self._W = W
        self._bufs = None

    def bytes_per_step(self, W: int, N: int | None = None, M: int | None = None) -> int:
        """Bytes one rank sends per call: its halo rows of dO (complex64, W
        wide), or the scanned rows when halo is off, plus the probe gradient."""
        probe = 8 * (M or 0) * (N or M or 0)
        if self.world == 1:
            return 0
        if not self.halo:
            return 8 * (self.rows[1] - self.rows[0]) * W + probe
        return 8 * W * sum(b - a for _, a, b in self.shared) + probe

    def _halo(self, dO: torch.Tensor):
        y0, y1 = self.bands[self.rank]
        if y1 <= y0:
            return
        W = dO.shape[1]
        if self._bufs is None or self._bufs[0] != (dO.device, dO.dtype, W):
            self._bufs = ((dO.device, dO.dtype, W),
                          {q: torch.empty((b - a, W), dtype=dO.dtype, device=dO.device) for q, a, b in self.shared})
        bufs = self._bufs[1]
        ops = []
        for q, a, b in self.shared:
            ops.append(self.dist.P2POp(self.dist.isend, torch.view_as_real(dO[a:b]), q, self.group))
            ops.append(self.dist.P2POp(self.dist.irecv, torch.view_as_real(bufs[q]), q, self.group))
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
        # every covering rank's contribution, added in rank order from zero
        acc = torch.zeros((y1 - y0, W), dtype=dO.dtype, device=dO.device)
        shared = {q: (a, b) for q, a, b in self.shared}
        for q in range(self.world):
            if q == self.rank:
                acc += dO[y0:y1]
            elif q in shared:
                a, b = shared[q]
                acc[a - y0:b - y0] += bufs[q]
        dO[y0:y1] = acc

    def all_reduce(self, dO=None, dP=None):
        if self.world == 1:
            return dO, dP
        if dO is not None:
            if self.halo:
                self._halo(dO)
            else:
                y0, y1 = self.rows
                self.dist.all_reduce(torch.view_as_real(dO[y0:y1]), group=self.group)
        if dP is not None:
            self.dist.all_reduce(torch.view_as_real(dP), group=self.group)
        return dO, dP

    def gather_object(self, O: torch.Tensor) -> torch.Tensor:
        """Overwrite, in place, every row of O that another rank owns with that
        rank's values (the owners' rows are current on their bands), so all
        ranks hold the same whole object."""
        if self.world == 1 or not self.halo:
            return O
        H = O.shape[0]
        for q, (a, b) in enumerate(owned_rows(self.bands, H)):
            if b > a:
                seg = O[a:b]
                self.dist.broadcast(torch.view_as_real(seg) if seg.is_complex() else seg, src=q,
                                    group=self.group)
        return O


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
