"""The Gaussian-splatting kernels against the reference's own rasteriser.

oracle/build_ref.py compiles the reference's CUDA sources
(gscp/csrc/gscp_rasterizer/{forward,backward,rasterizer_impl}.cu, with its
-O3 --use_fast_math) and a small C entry point into
oracle/_ref/libgscp_ref.so; these tests run both on the same inputs.

Radii agree except where 3 sqrt(lambda_max) sits on an integer within the
rounding differences (fast-math sqrt and reciprocal on the reference side);
the images and gradients are compared outside the tiles such a Gaussian's
two rectangles could differ on: images within 1e-5 of max (same terms, same
ascending order, __expf on both sides), gradients within 1e-3 of each array's
max (the reference sums them with float atomicAdd in no fixed order)."""
import ctypes
import importlib
import os

import numpy as np
import pytest
import torch

from conftest import PKG_NAME, ROOT
from oracle import gsplat as og

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref", "libgscp_ref.so")


@pytest.fixture(scope="module")
def env():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    if not os.path.exists(REF):
        pytest.skip("the reference rasteriser was not built (oracle/build_ref.py needs the reference tree)")
    L = ctypes.CDLL(REF)
    vp, ci, cf = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    L.gscp_ref_create.restype = vp
    L.gscp_ref_destroy.argtypes = [vp]
    L.gscp_ref_forward.argtypes = [vp, ci, ci, ci, ci, vp, vp, vp, vp, ci, cf, vp, vp]
    L.gscp_ref_backward.argtypes = [vp, ci, ci, ci, ci, vp, vp, vp, vp, ci, cf, vp, vp, vp, vp, vp, vp, vp, vp]
    return L, importlib.import_module(PKG_NAME + ".gsplat")


def _scene(seed, kind, N, H, W):
    rng = np.random.default_rng(seed)
    xy = np.stack([rng.uniform(-3, W + 2, N), rng.uniform(-3, H + 2, N)], 1)
    p1 = rng.uniform(np.log(0.6), np.log(5.0), (N, 2))
    p2 = rng.uniform(-np.pi, np.pi, N) if kind == og.RS else rng.uniform(-2, 2, N)
    w = rng.standard_normal((N, 2))
    return [torch.from_numpy(a.astype(np.float32)).cuda().contiguous() for a in (xy, p1, p2, w)]


def _reference(L, kind, scene, H, W, gout, R=16, ms=0.5):
    xy, p1, p2, w = scene
    N = xy.shape[0]
    out = torch.zeros((2, H, W), device="cuda")
    radii = torch.zeros(N, dtype=torch.int32, device="cuda")
    z = lambda *s: torch.zeros(s, device="cuda")  # noqa: E731
    dmean, dconic, dw, dxy, dp1, dp2 = z(N, 2), z(N, 3), z(N, 2), z(N, 2), z(N, 2), z(N)
    h = L.gscp_ref_create()
    try:
        assert L.gscp_ref_forward(h, kind, N, H, W, xy.data_ptr(), p1.data_ptr(), p2.data_ptr(), w.data_ptr(), R, ms,
                                  out.data_ptr(), radii.data_ptr()) >= 0
        g = gout.contiguous()
        assert L.gscp_ref_backward(h, kind, N, H, W, xy.data_ptr(), p1.data_ptr(), p2.data_ptr(), w.data_ptr(), R,
                                   ms, radii.data_ptr(), g.data_ptr(), dmean.data_ptr(), dconic.data_ptr(),
                                   dw.data_ptr(), dxy.data_ptr(), dp1.data_ptr(), dp2.data_ptr()) == 0
    finally:
        L.gscp_ref_destroy(h)
    return out, radii, (dxy, dp1, dp2, dw)


def _ours(gsm, kind, scene, H, W, gout, R=16, ms=0.5):
    xy, p1, p2, w = scene
    leaves = [t.clone().requires_grad_(True) for t in (xy, p1, p2[:, None] if kind == og.RS else p2, w)]
    fn = gsm.GaussianRasterize2D if kind == og.RS else gsm.GaussianRasterize2DCholesky
    out = fn.apply(*leaves, H, W, R, ms)
    (out * gout).sum().backward()
    _, radii = gsm.rasterize(kind, xy, p1, p2, w, H, W, R, ms)
    return out.detach(), radii, [t.grad.reshape(t.shape[0], -1).squeeze(1) for t in leaves]


@pytest.mark.parametrize("kind", [og.RS, og.CHOLESKY])
@pytest.mark.parametrize("N,H,W", [(500, 96, 130), (4000, 257, 300)])
def test_matches_reference_rasteriser(env, kind, N, H, W):
    L, gsm = env
    scene = _scene(100 + N + kind, kind, N, H, W)
    gout = torch.from_numpy(np.random.default_rng(1).standard_normal((2, H, W)).astype(np.float32)).cuda()
    r_out, r_rad, r_grads = _reference(L, kind, scene, H, W, gout)
    o_out, o_rad, o_grads = _ours(gsm, kind, scene, H, W, gout)
    r_rad, o_rad = r_rad.cpu().numpy(), o_rad.cpu().numpy()
    bad = np.nonzero(r_rad != o_rad)[0]
    assert np.all(np.abs(r_rad[bad] - o_rad[bad]) == 1) and bad.size <= 0.01 * N, bad
    # tiles either rectangle of a Gaussian with a differing radius may cover
    g = og.preprocess(kind, *[t.cpu().numpy() for t in scene[:3]], H, W, 16, 0.5)
    mask = np.ones((H, W), bool)
    for i in bad:
        x0, y0, x1, y1 = g["rect"][i]
        mask[max(0, (y0 - 1) * 16):(y1 + 1) * 16, max(0, (x0 - 1) * 16):(x1 + 1) * 16] = False
    r_out, o_out = r_out.cpu().numpy(), o_out.cpu().numpy()
    assert np.abs(r_out - o_out)[:, mask].max() <= 1e-5 * np.abs(r_out).max()
    keep = np.ones(N, bool)  # a Gaussian's gradients depend only on its own terms and grad_out
    keep[bad] = False
    for a, b in zip(o_grads, r_grads):
        a, b = a.cpu().numpy()[keep], b.cpu().numpy()[keep]
        assert np.abs(a - b).max() <= 1e-3 * max(np.abs(b).max(), 1e-6), (np.abs(a - b).max(), np.abs(b).max())
