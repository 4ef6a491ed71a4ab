"""The grid plan of the hash-grid backward, on CPU.

The plan (hashgrid.GridPlan) holds, per level, the cell corner and fraction
of every axis value, the vertex extents, the first coordinate of each cell
along each axis, and the vertex list sorted by table entry.  Emulating the
two kernels from those tables alone -- every vertex sums the rectangle of
coordinates whose cells touch it, with the forward's bilinear weights, then
every entry sums its vertices -- must give the oracle's table gradient (the
scatter of every coordinate's four corner contributions), dense and hashed
levels, far-edge aliases included.
"""
import numpy as np
import pytest
import torch

from conftest import load_pkg
from oracle import inr


def _grid(A, Bj):
    """The INR's pixel-centre coordinates: n = i * Bj + j -> (ys[j], xs[i])."""
    xs = torch.linspace(0.5 / A, 1 - 0.5 / A, A)
    ys = torch.linspace(0.5 / Bj, 1 - 0.5 / Bj, Bj)
    xv, yv = torch.meshgrid([xs, ys], indexing="ij")
    return torch.stack((yv.flatten(), xv.flatten())).t().contiguous()


def _emulate(plan, dfeat, n_entries):
    L = len(plan.levels)
    A, Bj = plan.A, plan.Bj
    gi = plan.int_tables
    gf = plan.frac_tables
    ix0 = gi[:L * Bj].reshape(L, Bj)
    iy1 = gi[L * Bj:L * Bj + L * A].reshape(L, A)
    fx0 = gf[:L * Bj].reshape(L, Bj)
    fy1 = gf[L * Bj:].reshape(L, A)
    pos = L * (Bj + A)
    G = []
    d = dfeat.reshape(A, Bj, L, 2)
    for l, row in enumerate(plan.extents):
        E0, E1 = int(row[0]), int(row[1])
        lo0 = gi[pos:pos + E0 + 1]
        # the cell widths bound every cell (the tile kernel's shared-memory size)
        assert np.diff(lo0).max() <= row[2]
        pos += E0 + 1
        G.append((E0, E1, lo0))
    for l, (E0, E1, lo0) in enumerate(G):
        lo1 = gi[pos:pos + E1 + 1]
        pos += E1 + 1
        G[l] = (E0, E1, lo0, lo1)
    vert = []
    for l, (E0, E1, lo0, lo1) in enumerate(G):
        for cy in range(E1):
            I = range(lo1[max(cy - 1, 0)], lo1[cy + 1])
            for cx in range(E0):
                J = range(lo0[max(cx - 1, 0)], lo0[cx + 1])
                acc = np.zeros(2)
                for i in I:
                    wy = 1.0 - float(fy1[l, i]) if iy1[l, i] == cy else float(fy1[l, i])
                    for j in J:
                        wx = 1.0 - float(fx0[l, j]) if ix0[l, j] == cx else float(fx0[l, j])
                        acc += wx * wy * d[i, j, l]
                vert.append(acc)
    vert = np.asarray(vert)
    assert len(vert) == plan.nvert
    vstart = plan.vstart
    vorder = plan.vorder
    out = np.zeros((n_entries, 2))
    for e in range(n_entries):
        for k in range(vstart[e], vstart[e + 1]):
            out[e] += vert[vorder[k]]
    return out.reshape(-1)


@pytest.mark.parametrize("A,Bj,cfg", [
    (20, 24, (4, 8, 4, 1.7)),     # dense levels, far-edge vertices alias
    (17, 13, (5, 6, 3, 1.9)),     # 2^6-entry table: the finest levels are hashed
    (9, 31, (3, 5, 8, 1.3)),      # hashed from the first level
])
def test_grid_plan_matches_oracle(A, Bj, cfg):
    pkg = load_pkg()
    hg = pkg.hashgrid
    coords = _grid(A, Bj)
    axes = hg.grid_axes(coords)
    assert axes is not None
    levels = inr.hashgrid_levels(cfg[0], cfg[1], cfg[2], float(np.float32(cfg[3])))
    n_entries = sum(lv[2] for lv in levels)
    plan = hg.GridPlan(axes[0], axes[1], cfg, n_entries)
    # the host level table is the library's
    for (s, r, n, off, dense), lv in zip(plan.levels, levels):
        assert (r, n, off, dense) == lv[1:] and s == np.float32(lv[0])
    rng = np.random.default_rng(A * Bj)
    dfeat = rng.standard_normal((A * Bj, 2 * cfg[0]))
    want = inr.hashgrid_backward(coords.numpy().astype(np.float64), dfeat, levels, n_entries, fp32_positions=True)
    got = _emulate(plan, dfeat, n_entries)
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-12 * np.abs(want).max())


def test_grid_axes_rejects_non_grids():
    hg = load_pkg().hashgrid
    assert hg.grid_axes(torch.rand(64, 2)) is None
    c = _grid(8, 8)
    c[5, 0] += 1e-3  # one coordinate off the grid
    assert hg.grid_axes(c) is None
    c = _grid(8, 8).flip(0).contiguous()  # decreasing axes
    assert hg.grid_axes(c) is None
