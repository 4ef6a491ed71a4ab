"""The CSR-free hash-grid backward on grid coordinates (ptycho_hashgrid_backward_grid).

An INR's coordinates are a tensor-product grid, so the encoder's backward
sums per-vertex rectangles and then per-entry vertex lists instead of
streaming a per-contribution CSR.  Checks against the CSR backward (same
mathematics, another summation order) and the FP64 oracle, for feature-major
and row-major gradients, dense and hashed levels, and bitwise repeatability.

Tolerances: against the CSR path max|d| / max|ref| <= 2e-6 (FP32 sums of the
same terms in another order, up to a few thousand terms per entry on the
coarse levels); against the FP64 oracle with float32 positions <= 1e-5.
"""
import numpy as np
import pytest
import torch

from conftest import load_pkg
from oracle import inr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return load_pkg()


def _grid(A, Bj, dev):
    xs = torch.linspace(0.5 / A, 1 - 0.5 / A, A)
    ys = torch.linspace(0.5 / Bj, 1 - 0.5 / Bj, Bj)
    xv, yv = torch.meshgrid([xs, ys], indexing="ij")
    return torch.stack((yv.flatten(), xv.flatten())).t().contiguous().to(dev)


CASES = [(512, 512, (16, 18, 16, 1.2599)),   # the c2 object encoder
         (128, 128, (16, 18, 16, 1.2599)),   # the c2 probe encoder
         (300, 250, (8, 12, 4, 1.6)),        # non-square, hashed fine levels
         (64, 96, (6, 10, 8, 1.5))]


def _backward(pkg, enc, coords, gfeat_planar, use_grid):
    enc.use_grid_plan = use_grid
    enc._csr = []
    x = coords.clone()
    p = enc.params
    p.grad = None
    out = enc(x)
    out.backward(gfeat_planar.t())  # a [N, 2L] view of the feature-major gradient
    g1 = p.grad.clone()
    p.grad = None
    out = enc(x)
    out.backward(gfeat_planar.t().contiguous())  # row-major gradient
    g2 = p.grad.clone()
    return g1, g2, enc._csr[-1][3]


@pytest.mark.parametrize("A,Bj,cfg", CASES)
def test_grid_backward_matches_csr_and_oracle(pkg, A, Bj, cfg):
    dev = torch.device("cuda")
    L, log2T, base, pls = cfg
    enc = pkg.Encoding(2, {"otype": "HashGrid", "n_levels": L, "n_features_per_level": 2,
                           "log2_hashmap_size": log2T, "base_resolution": base, "per_level_scale": pls}).to(dev)
    coords = _grid(A, Bj, dev)
    gen = torch.Generator(device=dev).manual_seed(A + Bj)
    gplanar = torch.randn((2 * L, A * Bj), device=dev, generator=gen)
    ga, gb, plan = _backward(pkg, enc, coords, gplanar, True)
    assert isinstance(plan, pkg.hashgrid.GridPlan)
    ca, cb, csr = _backward(pkg, enc, coords, gplanar, False)
    assert not isinstance(csr, pkg.hashgrid.GridPlan)
    scale = float(ca.abs().max())
    for g in (ga, gb):
        assert float((g - ca).abs().max()) <= 2e-6 * scale
    assert torch.equal(ga, gb)  # planar and row-major gradients read the same values
    levels = inr.hashgrid_levels(L, log2T, base, float(np.float32(pls)))
    ref = inr.hashgrid_backward(coords.cpu().numpy().astype(np.float64), gplanar.t().cpu().numpy(), levels,
                                enc.n_entries, fp32_positions=True)
    assert float(np.abs(ga.cpu().numpy() - ref).max()) <= 1e-5 * np.abs(ref).max()
    # repeatable bit for bit, and the plan holds far less than the CSR
    ga2, _, _ = _backward(pkg, enc, coords, gplanar, True)
    assert torch.equal(ga, ga2)
    plan_bytes = plan.gi.numel() * 4 + plan.gf.numel() * 4 + plan.scratch.numel()
    csr_bytes = csr.item.numel() * 4 * 3 + csr.start.numel() * 4
    assert plan_bytes < csr_bytes


def test_inr_model_trains_on_grid_plan(pkg):
    """ComplexINRModel2D's encoders take the grid plan, and a training step's
    table gradients equal the CSR path's within 2e-6."""
    dev = torch.device("cuda")
    grads = []
    for use in (True, False):
        torch.manual_seed(0)
        m = pkg.ComplexINRModel2D(192, 192, 2, probe_width=64, probe_height=64, n_levels=16, log2_hashmap_size=12,
                                  base_resolution=4, per_level_scale=1.2, first_omega_0=10.0,
                                  hidden_omega_0=1.0).to(dev)
        m.xy_hash_encoder.use_grid_plan = use
        m.probe_hash_encoder.use_grid_plan = use
        obj, probe = m()
        wo = torch.linspace(-1, 1, obj.numel(), device=dev).reshape(obj.shape)
        wp = torch.linspace(1, -1, probe.numel(), device=dev).reshape(probe.shape)
        ((obj * wo).real.sum() + (probe * wp).imag.sum()).backward()
        grads.append((m.xy_hash_encoder.params.grad.clone(), m.probe_hash_encoder.params.grad.clone()))
        if use:
            assert isinstance(m.xy_hash_encoder._csr[-1][3], pkg.hashgrid.GridPlan)
    for a, b in zip(*grads):
        assert torch.isfinite(b).all() and float(b.abs().max()) > 0
        assert float((a - b).abs().max()) <= 2e-6 * float(b.abs().max())
