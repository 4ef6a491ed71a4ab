"""HashGrid encoding on the B200 kernels -- drop-in for the tiny-cuda-nn class
the reference uses (models/complex_inr.py:4, 130-145, called at :279, :294).

``Encoding(n_input_dims=2, encoding_config={"otype": "HashGrid", ...})`` has
tiny-cuda-nn's constructor and call signature: ``enc(coords [N,2] float32 in
[0,1]) -> [N, n_levels * n_features_per_level]``.  Its single parameter
``params`` is the flat table ([entries * 2] float32, initialised U(-1e-4,
1e-4)).  The forward runs ``ptycho_hashgrid_forward``; the backward is a
deterministic gather (no atomics) in one of two forms, set up once per
coordinate tensor:

* a grid plan, when the coordinates are a tensor-product grid (an INR's
  pixel centres, models/complex_inr.py:179-205): per level, every vertex sums
  the rectangle of coordinates whose cells touch it, with the forward's own
  bilinear weights, then every table entry sums its vertices (hash
  collisions, far-edge aliases) from a vertex list sorted by entry.  Its
  state is a few per-axis tables and one entry per vertex;
* otherwise a CSR of the static (entry, coordinate, weight) contributions.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib
from .optics import device_status  # noqa: F401  (shared status word helpers)


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


class _CSR:
    """Static contributions of one coordinate tensor, sorted by table entry."""

    def __init__(self, coords: torch.Tensor, cfg: tuple, n_entries: int):
        L = _lib.lib()
        N = coords.shape[0]
        n_levels = cfg[0]
        K = N * n_levels * 4
        dev = coords.device
        key = torch.empty(K, dtype=torch.int32, device=dev)
        item = torch.empty(K, dtype=torch.int32, device=dev)
        weight = torch.empty(K, dtype=torch.float32, device=dev)
        _lib.check(L.ptycho_hashgrid_contrib(coords.data_ptr(), N, *cfg, key.data_ptr(), item.data_ptr(),
                                             weight.data_ptr(), _stream(dev)), "ptycho_hashgrid_contrib")
        skey, order = torch.sort(key, stable=True)  # one-time set-up, deterministic order
        self.item = item[order].contiguous()
        self.weight = weight[order].contiguous()
        # the same items addressed into a feature-major [2L][N] gradient (2*l*N + n),
        # for ptycho_hashgrid_backward_planar; the order is unchanged
        self.n = N
        self.item_planar = None
        if 2 * n_levels * N < 2 ** 31:
            it = self.item.long()
            self.item_planar = (2 * (it % n_levels) * N + it // n_levels).to(torch.int32).contiguous()
        self.start = torch.empty(n_entries + 1, dtype=torch.int32, device=dev)
        _lib.check(L.ptycho_hashgrid_segments(skey.data_ptr(), K, n_entries, self.start.data_ptr(),
                                              _stream(dev)), "ptycho_hashgrid_segments")


_PRIME_Y = 2654435761


def level_table(n_levels: int, log2_hashmap_size: int, base_resolution: int, per_level_scale: float):
    """Per level (scale float32, res, entries, offset, dense), as the library
    forms them (csrc/hashgrid.cu make_levels): scale = base * pls^l - 1 in
    double precision, rounded to float32; pls is taken as float32."""
    pls = float(np.float32(per_level_scale))
    T = 1 << log2_hashmap_size
    out, off = [], 0
    for l in range(n_levels):
        scale = float(base_resolution) * math.pow(pls, float(l)) - 1.0
        res = int(math.ceil(scale)) + 1
        dn = (res * res + 7) // 8 * 8
        n = min(dn, T)
        out.append((np.float32(scale), res, n, off, dn <= T))
        off += n
    return out


def _axis_cells(x: np.ndarray, scale: np.float32):
    """Cell corner and fraction of float32 positions x * scale + 0.5 formed with
    one rounding (the forward's fused multiply-add: the float32 product is
    exact in float64, so float64 multiply-add then one rounding is the same)."""
    p = (x.astype(np.float64) * np.float64(scale) + 0.5).astype(np.float32)
    g = np.floor(p)
    return g.astype(np.int64), (p - g).astype(np.float32)


def _entries(cx: np.ndarray, cy: np.ndarray, level) -> np.ndarray:
    """Table entry (within the level) of corners (cx, cy), as corner_entry."""
    scale, res, n, off, dense = level
    cx = cx.astype(np.uint64)
    cy = cy.astype(np.uint64)
    if dense:
        e = (cx + cy * np.uint64(res)) & np.uint64(0xFFFFFFFF)
        return np.where(e >= n, e % np.uint64(n), e).astype(np.int64)
    e = (cx ^ ((cy * np.uint64(_PRIME_Y)) & np.uint64(0xFFFFFFFF))) & np.uint64(0xFFFFFFFF)
    if n & (n - 1) == 0:
        return (e & np.uint64(n - 1)).astype(np.int64)
    return (e % np.uint64(n)).astype(np.int64)


def grid_axes(coords: torch.Tensor):
    """(ax0 [Bj], ax1 [A]) when coordinate n = i * Bj + j is (ax0[j], ax1[i])
    with both axes non-decreasing (a tensor-product grid), else None."""
    c = coords.detach().float().cpu().numpy()
    N = c.shape[0]
    if N < 2 or c.ndim != 2 or c.shape[1] != 2:
        return None
    same = np.flatnonzero(c[:, 1] != c[0, 1])
    Bj = int(same[0]) if same.size else N
    if N % Bj:
        return None
    A = N // Bj
    g = c.reshape(A, Bj, 2)
    ax0, ax1 = g[0, :, 0].copy(), g[:, 0, 1].copy()
    if not (np.array_equal(g[:, :, 0], np.broadcast_to(ax0, (A, Bj)))
            and np.array_equal(g[:, :, 1], np.broadcast_to(ax1[:, None], (A, Bj)))):
        return None
    if np.any(np.diff(ax0) < 0) or np.any(np.diff(ax1) < 0) or c.min() < 0:
        return None
    return ax0, ax1


class GridPlan:
    """Host tables of the grid backward (see the module notes).

    For level l: ix0/fx0 [Bj] (axis 0 corners and fractions), iy1/fy1 [A],
    extents E0 = max ix0 + 2, E1 = max iy1 + 2 (vertex (cx, cy), cx < E0,
    cy < E1, is vertex cy * E0 + cx of the level), lo0 [E0 + 1] with
    lo0[c] = first j whose ix0 >= c (lo1 likewise); then over all levels the
    vertex list sorted by table entry (stable): vorder, vstart [entries + 1]."""

    def __init__(self, ax0, ax1, cfg: tuple, n_entries: int):
        n_levels, log2T, base, pls = cfg
        self.levels = level_table(n_levels, log2T, base, pls)
        self.A, self.Bj = int(ax1.size), int(ax0.size)
        ix0, fx0, iy1, fy1, lo0, lo1, E = [], [], [], [], [], [], []
        ventry, vbase = [], 0
        for lev in self.levels:
            a, fa = _axis_cells(ax0, lev[0])
            b, fb = _axis_cells(ax1, lev[0])
            E0, E1 = int(a.max()) + 2, int(b.max()) + 2
            ix0.append(a); fx0.append(fa); iy1.append(b); fy1.append(fb)
            lo0.append(np.searchsorted(a, np.arange(E0 + 1), side="left"))
            lo1.append(np.searchsorted(b, np.arange(E1 + 1), side="left"))
            cw0 = int(np.diff(lo0[-1]).max()) if E0 > 0 else 1
            cw1 = int(np.diff(lo1[-1]).max()) if E1 > 0 else 1
            E.append((E0, E1, max(cw0, 1), max(cw1, 1)))
            cy, cx = np.divmod(np.arange(E0 * E1, dtype=np.int64), E0)
            ventry.append(lev[3] + _entries(cx, cy, lev))
            vbase += E0 * E1
        self.extents = np.asarray(E, dtype=np.int32)
        self.nvert = vbase
        ventry = np.concatenate(ventry)
        if ventry.max() >= n_entries or self.nvert >= 2 ** 31:
            raise ValueError("grid plan out of range")
        self.vorder = np.argsort(ventry, kind="stable").astype(np.int32)
        self.vstart = np.searchsorted(ventry[self.vorder], np.arange(n_entries + 1), side="left").astype(np.int32)
        self.int_tables = np.concatenate([np.concatenate(ix0), np.concatenate(iy1), np.concatenate(lo0),
                                          np.concatenate(lo1), self.vstart, self.vorder]).astype(np.int32)
        self.frac_tables = np.concatenate([np.concatenate(fx0), np.concatenate(fy1)]).astype(np.float32)

    def to(self, device):
        self.gi = torch.from_numpy(self.int_tables).to(device)
        self.gf = torch.from_numpy(self.frac_tables).to(device)
        self.hl = np.ascontiguousarray(self.extents.reshape(-1))
        return self


class _HashFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, params, enc):
        N = coords.shape[0]
        # features are produced feature-major ([L*F, N], coalesced) and returned as
        # the [N, L*F] transpose view; the MLP kernels read that layout directly
        outT = torch.empty((enc.n_output_dims, N), dtype=torch.float32, device=coords.device)
        _lib.check(_lib.lib().ptycho_hashgrid_forward_planar(coords.data_ptr(), N, params.data_ptr(), *enc.cfg,
                                                             outT.data_ptr(), _stream(coords.device)),
                   "ptycho_hashgrid_forward_planar")
        ctx.enc = enc
        ctx.save_for_backward(coords)
        return outT.t()

    @staticmethod
    def backward(ctx, gout):
        coords, = ctx.saved_tensors  # raises if coords were modified in place after the forward
        enc = ctx.enc
        plan = enc._plan_for(coords)
        N = coords.shape[0]
        dtable = torch.empty(enc.n_entries * 2, dtype=torch.float32, device=coords.device)
        stream = _stream(coords.device)
        planar = gout.dtype == torch.float32 and gout.dim() == 2 and N > 1 and gout.stride() == (1, N)
        if not planar:
            gout = gout.contiguous().float()
        if isinstance(plan, GridPlan):
            ext = plan.hl.ctypes.data
            _lib.check(_lib.lib().ptycho_hashgrid_backward_grid(
                plan.gi.data_ptr(), plan.gf.data_ptr(), ext, plan.A, plan.Bj, gout.data_ptr(), 1 if planar else 0,
                *enc.cfg, dtable.data_ptr(), 0, plan.scratch.data_ptr(), plan.scratch.numel(), stream),
                "ptycho_hashgrid_backward_grid")
            return None, dtable, None
        if planar and plan.item_planar is not None:
            # feature-major gradient (the MLP backward's planar output): coalesced gathers
            _lib.check(_lib.lib().ptycho_hashgrid_backward_planar(
                plan.start.data_ptr(), plan.item_planar.data_ptr(), plan.weight.data_ptr(), gout.data_ptr(), N,
                *enc.cfg, dtable.data_ptr(), 0, stream), "ptycho_hashgrid_backward_planar")
            return None, dtable, None
        gout = gout.contiguous().float()
        _lib.check(_lib.lib().ptycho_hashgrid_backward(
            plan.start.data_ptr(), plan.item.data_ptr(), plan.weight.data_ptr(), gout.data_ptr(),
            N, *enc.cfg, dtable.data_ptr(), 0, stream), "ptycho_hashgrid_backward")
        return None, dtable, None


class Encoding(torch.nn.Module):
    """Multi-resolution hash encoding with tiny-cuda-nn's interface (2-D inputs)."""

    def __init__(self, n_input_dims: int, encoding_config: dict, seed: int = 1337, dtype=None):
        super().__init__()
        if n_input_dims != 2:
            raise NotImplementedError("only 2-D inputs are supported")
        cfg = dict(encoding_config)
        if cfg.get("otype", "HashGrid") != "HashGrid":
            raise NotImplementedError(f"encoding {cfg.get('otype')!r} is not supported")
        if int(cfg.get("n_features_per_level", 2)) != 2:
            raise NotImplementedError("n_features_per_level must be 2")
        self.n_levels = int(cfg.get("n_levels", 16))
        self.log2_hashmap_size = int(cfg.get("log2_hashmap_size", 19))
        self.base_resolution = int(cfg.get("base_resolution", 16))
        self.per_level_scale = float(cfg.get("per_level_scale", 2.0))
        self.n_input_dims = 2
        self.n_output_dims = self.n_levels * 2
        self.cfg = (self.n_levels, self.log2_hashmap_size, self.base_resolution, self.per_level_scale)
        n = int(_lib.lib().ptycho_hashgrid_entries(*self.cfg))
        if n <= 0:
            raise ValueError(f"invalid HashGrid configuration {cfg}")
        self.n_entries = n
        g = torch.Generator().manual_seed(seed)
        self.params = torch.nn.Parameter(torch.rand(n * 2, generator=g) * 2e-4 - 1e-4)
        self._csr = []
        # grid coordinates take the CSR-free backward when it pays ("auto"); True
        # forces it on grid coordinates, False never uses it
        self.use_grid_plan = "auto"

    def _plan_for(self, coords: torch.Tensor):
        """The backward's static set-up for ``coords``, cached per coordinate
        buffer: a GridPlan when the coordinates are a tensor-product grid (an
        INR's pixel centres; a few MB), else the contribution CSR (12 bytes per
        coordinate, level and corner).

        An entry holds a reference to the coordinate tensor, so its memory cannot
        be taken by another tensor while cached, and matches on address, shape,
        strides and version counter (shared by aliases): new coordinates, or the
        same buffer modified in place, get a fresh plan.  Fixed coordinates (an
        INR's pixel grid) build it once."""
        key = (coords.data_ptr(), tuple(coords.shape), tuple(coords.stride()), coords.device)
        for k, t, ver, plan in self._csr:
            if k == key and t._version == ver and coords._version == ver:
                return plan
        plan = None
        axes = grid_axes(coords) if self.use_grid_plan else None
        if axes is not None and (self.use_grid_plan is True or self._grid_pays(axes)):
            try:
                plan = GridPlan(axes[0], axes[1], self.cfg, self.n_entries).to(coords.device)
                nbytes = int(_lib.lib().ptycho_hashgrid_grid_scratch_size(plan.hl.ctypes.data, self.n_levels,
                                                                           plan.A, plan.Bj))
                plan.scratch = torch.empty(max(nbytes, 8), dtype=torch.uint8, device=coords.device)
            except ValueError:
                plan = None
        if plan is None:
            plan = _CSR(coords, self.cfg, self.n_entries)
        self._csr = self._csr[-3:] + [(key, coords, coords._version, plan)]
        return plan

    def _grid_pays(self, axes) -> bool:
        """The vertex-centric grid backward visits every vertex of every level; when
        the vertices far outnumber the coordinates (a small probe grid under the
        object's fine levels) the CSR of the few contributions is the better plan."""
        n = axes[0].size * axes[1].size
        nvert = 0
        for lev in level_table(*self.cfg):
            e0 = int(_axis_cells(axes[0], lev[0])[0].max()) + 2
            e1 = int(_axis_cells(axes[1], lev[0])[0].max()) + 2
            nvert += e0 * e1
        return nvert <= 4 * n

    def _csr_for(self, coords: torch.Tensor) -> _CSR:
        """The contribution CSR of ``coords`` (any coordinates), cached like _plan_for."""
        use = self.use_grid_plan
        self.use_grid_plan = False
        try:
            key = (coords.data_ptr(), tuple(coords.shape), tuple(coords.stride()), coords.device)
            for k, t, ver, plan in self._csr:
                if k == key and t._version == ver and coords._version == ver and isinstance(plan, _CSR):
                    return plan
            csr = _CSR(coords, self.cfg, self.n_entries)
            self._csr = self._csr[-3:] + [(key, coords, coords._version, csr)]
            return csr
        finally:
            self.use_grid_plan = use

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        if not x.is_cuda:
            raise ValueError("coordinates must be a CUDA tensor (there is no CPU path)")
        x = x.float().contiguous()
        return _HashFn.apply(x, self.params, self)
