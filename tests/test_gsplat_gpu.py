"""The Gaussian-splatting kernels (``ptycho_gs_forward`` / ``_backward``)
against the oracle's restatement of the reference rasteriser
(gscp/csrc/gscp_rasterizer/forward.cu, backward.cu).

Tolerances: radii bit-exact except where 3 sqrt(lambda_max) sits on an
integer to within the ulp differences of cos / sin / exp (float32 preprocess
with round-to-nearest steps on both sides); the image within 2e-5 of its max
(float32 sums in the same order against float64); gradients within 5e-4 of
each array's max (float32 warp sums against float64)."""
import importlib

import numpy as np
import pytest
import torch

from conftest import PKG_NAME
from oracle import gsplat as og

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gsm():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return importlib.import_module(PKG_NAME + ".gsplat")


def _scene(seed, kind, N, H, W, smin=0.6, smax=5.0, cluster=None):
    rng = np.random.default_rng(seed)
    if cluster is None:
        xy = np.stack([rng.uniform(-3, W + 2, N), rng.uniform(-3, H + 2, N)], 1)
    else:
        xy = np.asarray(cluster) + rng.normal(0, 2.0, (N, 2))
    p1 = rng.uniform(np.log(smin), np.log(smax), (N, 2))
    p2 = rng.uniform(-np.pi, np.pi, N) if kind == og.RS else rng.uniform(-2, 2, N)
    w = rng.standard_normal((N, 2))
    return [a.astype(np.float32) for a in (xy, p1, p2, w)]


def _cuda(*arrs):
    return [torch.from_numpy(a).cuda() for a in arrs]


def _run(gsm, kind, scene, H, W, R=16, ms=0.5, gout=None):
    xy, p1, p2, w = _cuda(*scene)
    if kind == og.RS:
        p2 = p2[:, None]
    leaves = [t.clone().requires_grad_(True) for t in (xy, p1, p2, w)]
    fn = gsm.GaussianRasterize2D if kind == og.RS else gsm.GaussianRasterize2DCholesky
    out = fn.apply(*leaves, H, W, R, ms)
    grads = None
    if gout is not None:
        (out * torch.from_numpy(gout).float().cuda()).sum().backward()
        grads = [t.grad.detach().cpu().numpy() for t in leaves]
    return out.detach().cpu().numpy(), grads


@pytest.mark.parametrize("kind", [og.RS, og.CHOLESKY])
@pytest.mark.parametrize("N,H,W", [(1, 16, 16), (300, 96, 130), (2000, 257, 200)])
def test_forward_and_backward_match_oracle(gsm, kind, N, H, W):
    scene = _scene(N + kind, kind, N, H, W)
    gout = np.random.default_rng(3).standard_normal((2, H, W))
    out, grads = _run(gsm, kind, scene, H, W, gout=gout)
    ref, g = og.render(kind, *scene, H, W, 16, 0.5)
    assert np.abs(out - ref).max() <= 2e-5 * max(np.abs(ref).max(), 1e-6)
    rg = og.backward(kind, *scene, H, W, 16, 0.5, gout)
    for a, b in zip(grads, rg):
        a = a.reshape(b.shape)
        assert np.abs(a - b).max() <= 5e-4 * max(np.abs(b).max(), 1e-6), (np.abs(a - b).max(), np.abs(b).max())


@pytest.mark.parametrize("kind", [og.RS, og.CHOLESKY])
def test_radii_bit_exact(gsm, kind):
    scene = _scene(7 + kind, kind, 3000, 300, 310, smin=0.3, smax=20.0)
    _, radii = gsm.rasterize(kind, *_cuda(*scene), 300, 310, 16, 0.5)
    g = og.preprocess(kind, *scene[:3], 300, 310, 16, 0.5)
    got = radii.cpu().numpy()
    bad = np.nonzero(got != g["radius"])[0]
    # cos / sin / exp differ by an ulp or two between the device and the
    # oracle: a radius may differ by one only where 3 sqrt(lambda) is an integer
    # to within that rounding (clamped scales make lambda exactly 256, say)
    r3 = g["r3"][bad].astype(np.float64)
    assert np.all(np.abs(got[bad] - g["radius"][bad]) == 1)
    assert np.all(np.abs(r3 - np.round(r3)) <= 1e-5 * r3), r3
    assert bad.size <= 0.02 * got.size


def test_dense_tile_spans_several_mask_chunks(gsm):
    """10,000 Gaussians on one spot: the tile's list is compacted in chunks of
    8192 and must still be summed in ascending index."""
    H = W = 64
    scene = _scene(5, og.CHOLESKY, 10000, H, W, smin=0.6, smax=2.0, cluster=(30.0, 31.0))
    gout = np.random.default_rng(4).standard_normal((2, H, W))
    out, grads = _run(gsm, og.CHOLESKY, scene, H, W, gout=gout)
    ref, _ = og.render(og.CHOLESKY, *scene, H, W, 16, 0.5)
    assert np.abs(out - ref).max() <= 2e-5 * np.abs(ref).max()
    rg = og.backward(og.CHOLESKY, *scene, H, W, 16, 0.5, gout)
    for a, b in zip(grads, rg):
        assert np.abs(a.reshape(b.shape) - b).max() <= 5e-4 * np.abs(b).max()


def test_deterministic_and_culling(gsm):
    H, W = 80, 80
    scene = _scene(9, og.CHOLESKY, 500, H, W)
    scene[1][:10] = -200.0  # exp(-200) = 0 with min_scale 0: det = 0, culled
    gout = np.random.default_rng(5).standard_normal((2, H, W))
    a = _run(gsm, og.CHOLESKY, scene, H, W, ms=0.0, gout=gout)
    b = _run(gsm, og.CHOLESKY, scene, H, W, ms=0.0, gout=gout)
    assert np.array_equal(a[0], b[0])
    for x, y in zip(a[1], b[1]):
        assert np.array_equal(x, y)
    for gr in a[1]:
        assert np.all(gr.reshape(500, -1)[:10] == 0)
    _, radii = gsm.rasterize(og.CHOLESKY, *_cuda(*scene), H, W, 16, 0.0)
    assert np.all(radii.cpu().numpy()[:10] == 0)


def test_empty_and_bad_arguments(gsm):
    z = torch.zeros((0, 2), device="cuda")
    out = gsm.GaussianRasterize2DCholesky.apply(z, z, torch.zeros(0, device="cuda"), z, 20, 30, 16, 0.5)
    assert out.shape == (2, 20, 30) and torch.count_nonzero(out) == 0
    with pytest.raises(ValueError):
        gsm.GaussianRasterize2D.apply(torch.zeros(3, 2), torch.zeros(3, 2), torch.zeros(3, 1), torch.zeros(3, 2),
                                      8, 8, 16, 0.5)
