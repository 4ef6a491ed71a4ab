"""Probes of any shape (the general path): the reference accepts whatever
probe the data holds (Recovery.py:290, utils/optics.py:102-112), so shapes
other than square 64 / 128 / 256 -- 96^2, 192^2, odd and non-square windows
-- must give the same intensities, losses and gradients as the FP64 oracle.

Tolerances (as test_fwd_adj_gpu.py; FP32 mixed-radix DFTs against FP64):
  intensities  max|I - I_ref| / max|I_ref|   <= 1e-5
  losses       relative                      <= 2e-5
  dO, dP       max|g - g_ref| / max|g_ref|   <= 2e-4 (smooth_L1, Poisson), 1e-3 (FD)
"""
import numpy as np
import pytest
import torch

from conftest import load_pkg
from oracle import forward_model as fm

pytestmark = pytest.mark.gpu
GRAD_TOL = {"smooth_L1_loss": 2e-4, "Poisson_likelihood_loss": 2e-4, "FD_loss": 1e-3}


@pytest.fixture(scope="module")
def pkg():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return load_pkg()


def rel_max(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-30))


def _case(M, N, H, W, B, seed, peak=1e4):
    rng = np.random.default_rng(seed)
    from scipy.ndimage import gaussian_filter
    u = gaussian_filter(rng.random((H, W)), 3)
    ph = gaussian_filter(rng.random((H, W)), 3)
    u = (u - u.min()) / (u.max() - u.min())
    ph = (ph - ph.min()) / (ph.max() - ph.min())
    O = ((0.6 + 0.4 * u) * np.exp(1j * np.pi * (ph - 0.5))).astype(np.complex64)
    yy, xx = np.mgrid[:M, :N]
    r = np.hypot((yy - M / 2) / M, (xx - N / 2) / N)
    P = ((r < 0.35) * np.exp(1j * 2.0 * r * r)).astype(np.complex64)
    P = (P + 0.02 * (rng.standard_normal((M, N)) + 1j * rng.standard_normal((M, N)))).astype(np.complex64)
    tlY = rng.integers(0, H - M + 1, size=B).astype(np.int32)
    tlX = rng.integers(0, W - N + 1, size=B).astype(np.int32)
    Itrue = fm.forward_intensity(O * np.exp(0.2j * u), P, tlY, tlX)
    Imeas = rng.poisson(Itrue / Itrue.max() * peak).astype(np.float32)
    scale = np.float32(np.sqrt(peak / Itrue.max()))
    return (O * scale).astype(np.complex64), P, tlY, tlX, Imeas


def _run(pkg, O, P, tlY, tlX, Imeas, loss_type):
    dev = torch.device("cuda")
    tl = pkg.make_windows(tlY, tlX, dev)
    loss, lp, dO, dP = pkg.fwd_adj_raw(torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev), tl,
                                       torch.from_numpy(Imeas).to(dev), pkg.LOSS_CODES[loss_type],
                                       per_pattern=True)
    torch.cuda.synchronize()
    return float(loss), lp.cpu().numpy(), dO.cpu().numpy(), dP.cpu().numpy()


SHAPES = [(96, 96, 300, 320, 12), (192, 192, 400, 420, 6), (100, 120, 260, 300, 9), (63, 65, 150, 160, 11),
          (7, 10, 40, 41, 5), (128, 96, 300, 280, 8), (81, 81, 200, 200, 7)]


@pytest.mark.parametrize("M,N,H,W,B", SHAPES)
@pytest.mark.parametrize("loss_type", fm.LOSS_TYPES)
def test_general_against_fp64_oracle(pkg, M, N, H, W, B, loss_type):
    O, P, tlY, tlX, Imeas = _case(M, N, H, W, B, seed=M * 7 + N)
    loss, lp, dO, dP = _run(pkg, O, P, tlY, tlX, Imeas, loss_type)
    ref = fm.fwd_adj(O.astype(np.complex128), P.astype(np.complex128), tlY, tlX, Imeas, loss_type)
    assert abs(loss - ref["loss_total"]) <= 2e-5 * abs(ref["loss_total"])
    assert np.all(np.abs(lp - ref["loss"]) <= 2e-5 * np.maximum(np.abs(ref["loss"]), 1e-30))
    assert rel_max(dO, ref["dO"]) <= GRAD_TOL[loss_type], rel_max(dO, ref["dO"])
    assert rel_max(dP, ref["dP"]) <= GRAD_TOL[loss_type], rel_max(dP, ref["dP"])


@pytest.mark.parametrize("M,N,H,W,B", SHAPES)
def test_general_forward_intensity(pkg, M, N, H, W, B):
    O, P, tlY, tlX, _ = _case(M, N, H, W, B, seed=3)
    dev = torch.device("cuda")
    I = pkg.forward_intensity(torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev),
                              pkg.make_windows(tlY, tlX, dev))
    ref = fm.forward_intensity(O.astype(np.complex128), P.astype(np.complex128), tlY, tlX)
    assert I.shape == (B, M, N)
    assert rel_max(I.cpu().numpy(), ref) <= 1e-5


@pytest.mark.parametrize("loss_type", fm.LOSS_TYPES)
def test_general_finite_differences(pkg, loss_type):
    M, N, H, W, B = 30, 27, 64, 70, 4
    O, P, tlY, tlX, Imeas = _case(M, N, H, W, B, seed=21, peak=200.0)
    _, _, dO, dP = _run(pkg, O, P, tlY, tlX, Imeas, loss_type)
    rng = np.random.default_rng(5)
    oi = [(int(tlY[0]) + int(a), int(tlX[0]) + int(b)) for a, b in rng.integers(0, min(M, N), size=(6, 2))]
    pi = [tuple(int(v) for v in x) for x in rng.integers(0, min(M, N), size=(6, 2))]
    O64, P64 = O.astype(np.complex128), P.astype(np.complex128)
    go = np.array(fm.fd_gradient(O64, P64, tlY, tlX, Imeas, loss_type, "O", oi))
    gp = np.array(fm.fd_gradient(O64, P64, tlY, tlX, Imeas, loss_type, "P", pi))
    tol = 1e-3 if loss_type != "FD_loss" else 3e-3
    assert np.abs(np.array([dO[i] for i in oi]) - go).max() <= tol * np.abs(dO).max()
    assert np.abs(np.array([dP[i] for i in pi]) - gp).max() <= tol * np.abs(dP).max()


def test_general_deterministic_and_frame_ids(pkg):
    M, N, H, W, F = 96, 90, 260, 250, 20
    O, P, tlY, tlX, Imeas = _case(M, N, H, W, F, seed=8)
    dev = torch.device("cuda")
    args = (torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev), pkg.make_windows(tlY, tlX, dev),
            torch.from_numpy(Imeas).to(dev), pkg.LOSS_CODES["Poisson_likelihood_loss"])
    ids = torch.tensor([5, 2, 17, 2, 9], dtype=torch.int32, device=dev)
    a = pkg.fwd_adj_raw(*args, batch=ids, per_pattern=True)
    b = pkg.fwd_adj_raw(*args, batch=ids, per_pattern=True)
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    sel = ids.cpu().numpy()
    ref = fm.fwd_adj(O.astype(np.complex128), P.astype(np.complex128), tlY[sel], tlX[sel], Imeas[sel],
                     "Poisson_likelihood_loss")
    assert rel_max(a[2].cpu().numpy(), ref["dO"]) <= 2e-4
    assert rel_max(a[3].cpu().numpy(), ref["dP"]) <= 2e-4


def test_general_window_outside_canvas_and_empty_batch(pkg):
    M, N, H, W = 50, 40, 120, 130
    O, P, tlY, tlX, Imeas = _case(M, N, H, W, 3, seed=9)
    tlY = tlY.copy()
    tlY[1] = H - M + 1  # one row past the canvas
    dev = torch.device("cuda")
    pkg.read_status(dev)
    loss, lp, dO, dP = pkg.fwd_adj_raw(torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev),
                                       pkg.make_windows(tlY, tlX, dev), torch.from_numpy(Imeas).to(dev),
                                       pkg.LOSS_CODES["smooth_L1_loss"], per_pattern=True)
    torch.cuda.synchronize()
    assert pkg.read_status(dev) == 6  # PTYCHO_ERR_WINDOW
    lpn = lp.cpu().numpy()
    assert np.isnan(lpn[1]) and np.isfinite(lpn[[0, 2]]).all()
    keep = np.array([0, 2])
    ref = fm.fwd_adj(O.astype(np.complex128), P.astype(np.complex128), tlY[keep], tlX[keep], Imeas[keep],
                     "smooth_L1_loss")
    assert rel_max(dO.cpu().numpy(), ref["dO"]) <= 2e-4
    assert rel_max(dP.cpu().numpy(), ref["dP"]) <= 2e-4
    e = pkg.fwd_adj_raw(torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev), pkg.make_windows(tlY, tlX, dev),
                        torch.from_numpy(Imeas).to(dev), 0, batch=torch.zeros(0, dtype=torch.int32, device=dev))
    assert float(e[0]) == 0.0 and not e[2].abs().any() and not e[3].abs().any()


def test_general_public_autograd_and_forward_imaging_model(pkg):
    """fused_loss and forward_imaging_model with a non-square probe through autograd."""
    M, N, H, W, B = 72, 60, 160, 170, 5
    O, P, tlY, tlX, Imeas = _case(M, N, H, W, B, seed=12)
    dev = torch.device("cuda")
    Ot = torch.from_numpy(O).to(dev).requires_grad_(True)
    Pt = torch.from_numpy(P).to(dev).requires_grad_(True)
    loss = pkg.fused_loss(Ot, Pt, pkg.make_windows(tlY, tlX, dev), torch.from_numpy(Imeas).to(dev),
                          "Poisson_likelihood_loss")
    (2.0 * loss).backward()
    ref = fm.fwd_adj(O.astype(np.complex128), P.astype(np.complex128), tlY, tlX, Imeas, "Poisson_likelihood_loss")
    assert rel_max(Ot.grad.cpu().numpy(), 2 * ref["dO"]) <= 2e-4
    assert rel_max(Pt.grad.cpu().numpy(), 2 * ref["dP"]) <= 2e-4
    O2 = torch.from_numpy(O).to(dev).requires_grad_(True)
    I = pkg.forward_imaging_model(O2, torch.from_numpy(P).to(dev), int(tlY[0]), int(tlX[0]),
                                  int(tlY[0]) + M, int(tlX[0]) + N)
    refI = fm.forward_intensity(O.astype(np.complex128), P.astype(np.complex128), tlY[:1], tlX[:1])[0]
    assert I.shape == (M, N) and rel_max(I.detach().cpu().numpy(), refI) <= 1e-5
    I.sum().backward()
    assert torch.isfinite(O2.grad).all()


def test_general_plan_graph_replay(pkg):
    """FwdAdjPlan (CUDA-graph replay) on a 96 x 96 probe equals the eager call."""
    M, N, H, W, F = 96, 96, 300, 300, 16
    O, P, tlY, tlX, Imeas = _case(M, N, H, W, F, seed=4)
    dev = torch.device("cuda")
    Ot, Pt = torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev)
    tl, st = pkg.make_windows(tlY, tlX, dev), torch.from_numpy(Imeas).to(dev)
    plan = pkg.optics.FwdAdjPlan(Ot, Pt, tl, st, "smooth_L1_loss", 8)
    ids = torch.arange(3, 11, dtype=torch.int32, device=dev)
    plan.set_batch(ids)
    plan.replay()
    plan.replay()
    torch.cuda.synchronize()
    loss, _, dO, dP = pkg.fwd_adj_raw(Ot, Pt, tl, st, 0, batch=ids)
    assert torch.equal(plan.loss_total, loss) and torch.equal(plan.dO, dO) and torch.equal(plan.dP, dP)
