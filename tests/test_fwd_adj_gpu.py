"""Parity of the fused CUDA forward model / loss / adjoint with the FP64 oracle,
the reference's own golden vectors and torch autograd.

Tolerances (FP32 FFT against an FP64 oracle):
  forward intensities  max|I - I_ref| / max|I_ref|          <= 1e-5
  per-pattern losses   |l - l_ref| / max(|l_ref|, 1e-30)      <= 2e-5
  gradients dO, dP     max|g - g_ref| / max|g_ref|           <= 2e-4 (smooth_L1, Poisson),
                                                              <= 1e-3 (FD)
Scan-window indices are integers and must be bit-exact (checked on the host).
"""
import numpy as np
import pytest
import torch

from conftest import golden, load_pkg
from oracle import forward_model as fm

pytestmark = pytest.mark.gpu
LOSSES = fm.LOSS_TYPES
GRAD_TOL = {"smooth_L1_loss": 2e-4, "Poisson_likelihood_loss": 2e-4, "FD_loss": 1e-3}


@pytest.fixture(scope="module")
def pkg():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return load_pkg()


def rel_max(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-30))


def _case(M, H, B, seed, peak=1e4, W=None):
    """Seeded smooth object, apertured probe, windows and Poisson data."""
    rng = np.random.default_rng(seed)
    W = W or H
    u = rng.random((H, W))
    ph = rng.random((H, W))
    from scipy.ndimage import gaussian_filter
    u = gaussian_filter(u, 3); ph = gaussian_filter(ph, 3)
    u = (u - u.min()) / (u.max() - u.min()); ph = (ph - ph.min()) / (ph.max() - ph.min())
    O = ((0.6 + 0.4 * u) * np.exp(1j * np.pi * (ph - 0.5))).astype(np.complex64)
    yy, xx = np.mgrid[:M, :M] - M / 2
    r = np.hypot(yy, xx)
    P = ((r < 0.35 * M) * np.exp(1j * 0.002 * r * r)).astype(np.complex64)
    P = (P + 0.02 * (rng.standard_normal((M, M)) + 1j * rng.standard_normal((M, M)))).astype(np.complex64)
    tlY = rng.integers(0, H - M + 1, size=B).astype(np.int32)
    tlX = rng.integers(0, W - M + 1, size=B).astype(np.int32)
    Itrue = fm.forward_intensity(O * np.exp(0.2j * u), P, tlY, tlX)
    Imeas = rng.poisson(Itrue / Itrue.max() * peak).astype(np.float32)
    scale = np.float32(np.sqrt(peak / Itrue.max()))
    return (O * scale).astype(np.complex64), P, tlY, tlX, Imeas


def _run(pkg, O, P, tlY, tlX, Imeas, loss_type, per_pattern=True):
    dev = torch.device("cuda")
    Ot = torch.from_numpy(np.ascontiguousarray(O)).to(dev)
    Pt = torch.from_numpy(np.ascontiguousarray(P)).to(dev)
    tl = pkg.make_windows(tlY, tlX, dev)
    Im = torch.from_numpy(np.ascontiguousarray(Imeas)).to(dev)
    loss, lp, dO, dP = pkg.fwd_adj_raw(Ot, Pt, tl, Im, pkg.LOSS_CODES[loss_type], per_pattern=per_pattern)
    torch.cuda.synchronize()
    return (float(loss), lp.cpu().numpy() if lp is not None else None, dO.cpu().numpy(),
            dP.cpu().numpy())


@pytest.mark.parametrize("loss_type", LOSSES)
def test_golden_reference_vectors_m64(pkg, loss_type):
    g = golden("fwd_adj_m64.npz")
    O = g["O"].astype(np.complex64)
    P = g["P"].astype(np.complex64)
    loss, lp, dO, dP = _run(pkg, O, P, g["tlY"], g["tlX"], g["Imeas"], loss_type)
    ref_l = g[f"{loss_type}/loss"]
    assert np.all(np.abs(lp - ref_l) <= 2e-5 * np.abs(ref_l)), (lp, ref_l)
    assert abs(loss - ref_l.sum()) <= 2e-5 * abs(ref_l.sum())
    assert rel_max(dO, g[f"{loss_type}/dO"]) <= GRAD_TOL[loss_type]
    assert rel_max(dP, g[f"{loss_type}/dP"]) <= GRAD_TOL[loss_type]


def test_golden_forward_intensity_m64(pkg):
    g = golden("fwd_adj_m64.npz")
    dev = torch.device("cuda")
    I = pkg.forward_intensity(torch.from_numpy(g["O"].astype(np.complex64)).to(dev),
                              torch.from_numpy(g["P"].astype(np.complex64)).to(dev),
                              pkg.make_windows(g["tlY"], g["tlX"], dev)).cpu().numpy()
    assert rel_max(I, g["I"]) <= 1e-5


@pytest.mark.parametrize("M,H,B", [(64, 160, 7), (128, 300, 9), (128, 256, 300)])
@pytest.mark.parametrize("loss_type", LOSSES)
def test_against_fp64_oracle(pkg, M, H, B, loss_type):
    O, P, tlY, tlX, Imeas = _case(M, H, B, seed=M + B)
    loss, lp, dO, dP = _run(pkg, O, P, tlY, tlX, Imeas, loss_type)
    r = fm.fwd_adj(O, P, tlY, tlX, Imeas, loss_type)
    assert np.all(np.abs(lp - r["loss"]) <= 2e-5 * np.abs(r["loss"]) + 1e-12)
    assert abs(loss - r["loss_total"]) <= 2e-5 * abs(r["loss_total"])
    assert rel_max(dO, r["dO"]) <= GRAD_TOL[loss_type], rel_max(dO, r["dO"])
    assert rel_max(dP, r["dP"]) <= GRAD_TOL[loss_type], rel_max(dP, r["dP"])


@pytest.mark.parametrize("M", [64, 128])
def test_forward_intensity_against_oracle(pkg, M):
    O, P, tlY, tlX, _ = _case(M, 2 * M + 37, 11, seed=5, W=2 * M + 5)
    dev = torch.device("cuda")
    I = pkg.forward_intensity(torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev),
                              pkg.make_windows(tlY, tlX, dev)).cpu().numpy()
    ref = fm.forward_intensity(O, P, tlY, tlX)
    assert rel_max(I, ref) <= 1e-5
    # Parseval: sum I = M*M * sum |psi|^2 per pattern
    psi = fm.exit_waves(O, P, tlY, tlX)
    np.testing.assert_allclose(I.reshape(11, -1).sum(1), M * M * (np.abs(psi) ** 2).reshape(11, -1).sum(1),
                               rtol=1e-5)


def test_known_answers(pkg):
    """Delta object -> |FFT(P)|^2 pattern; constant probe -> |FFT(O_window)|^2."""
    M = 64
    dev = torch.device("cuda")
    rng = np.random.default_rng(1)
    P = (rng.standard_normal((M, M)) + 1j * rng.standard_normal((M, M))).astype(np.complex64)
    O = np.zeros((M + 8, M + 8), np.complex64)
    O[3 + 10, 5 + 20] = 1.0
    I = pkg.forward_intensity(torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev),
                              pkg.make_windows([3], [5], dev)).cpu().numpy()[0]
    # only pixel (10, 20) of the window is lit: |P[10,20]|^2 everywhere
    np.testing.assert_allclose(I, np.full((M, M), abs(P[10, 20]) ** 2), rtol=1e-5)
    Oc = (rng.standard_normal((M + 8, M + 8)) + 1j * rng.standard_normal((M + 8, M + 8))).astype(np.complex64)
    ones = np.ones((M, M), np.complex64)
    I2 = pkg.forward_intensity(torch.from_numpy(Oc).to(dev), torch.from_numpy(ones).to(dev),
                               pkg.make_windows([8], [0], dev)).cpu().numpy()[0]
    ref = np.abs(np.fft.fftshift(np.fft.fft2(Oc[8:8 + M, 0:M].astype(np.complex128)))) ** 2
    assert rel_max(I2, ref) <= 1e-5


@pytest.mark.parametrize("loss_type", LOSSES)
def test_finite_difference_gradient(pkg, loss_type):
    """Kernel gradients against FP64 central differences of the oracle loss."""
    O, P, tlY, tlX, Imeas = _case(64, 96, 4, seed=9, peak=500.0)
    _, _, dO, dP = _run(pkg, O, P, tlY, tlX, Imeas, loss_type)
    rng = np.random.default_rng(2)
    oi = [tuple(x) for x in rng.integers(0, 96, size=(12, 2))]
    pi = [tuple(x) for x in rng.integers(0, 64, size=(6, 2))]
    O64, P64 = O.astype(np.complex128), P.astype(np.complex128)
    fo = fm.fd_gradient(O64, P64, tlY, tlX, Imeas, loss_type, "O", oi, h=1e-5)
    fp = fm.fd_gradient(O64, P64, tlY, tlX, Imeas, loss_type, "P", pi, h=1e-5)
    so, sp = np.abs(dO).max(), np.abs(dP).max()
    tol = 1e-3 if loss_type != "FD_loss" else 3e-3
    assert np.abs(np.array([dO[i] for i in oi]) - fo).max() <= tol * so
    assert np.abs(np.array([dP[i] for i in pi]) - fp).max() <= tol * sp


def test_matches_torch_autograd_of_reference_forward_model(pkg):
    """torch autograd (complex128, GPU) of utils/optics.py:102-112 + Poisson loss."""
    M = 128
    O, P, tlY, tlX, Imeas = _case(M, 200, 5, seed=21)
    dev = torch.device("cuda")
    Ot = torch.tensor(O, dtype=torch.complex128, device=dev, requires_grad=True)
    Pt = torch.tensor(P, dtype=torch.complex128, device=dev, requires_grad=True)
    total = 0.0
    for b in range(5):
        y, x = int(tlY[b]), int(tlX[b])
        I = torch.abs(torch.fft.fftshift(torch.fft.fft2(Pt * Ot[y:y + M, x:x + M]), dim=(-2, -1))) ** 2
        cap = torch.tensor(Imeas[b], dtype=torch.float64, device=dev)
        total = total + (I - cap * torch.log(I + 1e-8)).mean()
    total.backward()
    loss, _, dO, dP = _run(pkg, O, P, tlY, tlX, Imeas, "Poisson_likelihood_loss")
    assert abs(loss - float(total)) <= 2e-5 * abs(float(total))
    assert rel_max(dO, Ot.grad.cpu().numpy()) <= 2e-4
    assert rel_max(dP, Pt.grad.cpu().numpy()) <= 2e-4


def test_forward_imaging_model_dropin_autograd(pkg):
    """pkg.forward_imaging_model has the reference signature and a correct backward."""
    M = 64
    O, P, tlY, tlX, _ = _case(M, 100, 1, seed=3)
    dev = torch.device("cuda")
    Ot = torch.tensor(O, device=dev, requires_grad=True)
    Pt = torch.tensor(P, device=dev, requires_grad=True)
    y, x = int(tlY[0]), int(tlX[0])
    I = pkg.forward_imaging_model(Ot, Pt, y, x, y + M, x + M)
    w = torch.linspace(0, 1, M * M, device=dev).reshape(M, M)
    (I * w).sum().backward()
    O2 = torch.tensor(O, dtype=torch.complex128, device=dev, requires_grad=True)
    P2 = torch.tensor(P, dtype=torch.complex128, device=dev, requires_grad=True)
    I2 = torch.abs(torch.fft.fftshift(torch.fft.fft2(P2 * O2[y:y + M, x:x + M]), dim=(-2, -1))) ** 2
    (I2 * w.double()).sum().backward()
    assert rel_max(I.detach().cpu().numpy(), I2.detach().cpu().numpy()) <= 1e-5
    assert rel_max(Ot.grad.cpu().numpy(), O2.grad.cpu().numpy()) <= 2e-4
    assert rel_max(Pt.grad.cpu().numpy(), P2.grad.cpu().numpy()) <= 2e-4


def test_deterministic_bitwise(pkg):
    O, P, tlY, tlX, Imeas = _case(128, 400, 64, seed=4)
    a = _run(pkg, O, P, tlY, tlX, Imeas, "Poisson_likelihood_loss")
    b = _run(pkg, O, P, tlY, tlX, Imeas, "Poisson_likelihood_loss")
    assert a[0] == b[0]
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])


@pytest.mark.parametrize("M", [64, 128])
def test_probe_alignment_paths_agree_bitwise(pkg, M):
    """A probe that is 8- but not 16-byte aligned takes the one-pixel-per-thread
    dP assembly; a 16-byte aligned one the paired kernel.  Same results, bitwise."""
    O, P, tlY, tlX, Imeas = _case(M, 2 * M + 40, 37, seed=9)
    dev = torch.device("cuda")
    Ot = torch.from_numpy(O).to(dev)
    tl = pkg.make_windows(tlY, tlX, dev)
    Im = torch.from_numpy(Imeas).to(dev)
    buf = torch.zeros(M * M + 1, dtype=torch.complex64, device=dev)
    P_odd = buf[1:].view(M, M)  # starts 8 bytes into an aligned allocation
    P_odd.copy_(torch.from_numpy(P))
    P_al = torch.from_numpy(P).to(dev)
    assert P_odd.data_ptr() % 16 == 8 and P_al.data_ptr() % 16 == 0
    res = []
    for Pt in (P_al, P_odd):
        loss, _, dO, dP = pkg.fwd_adj_raw(Ot, Pt, tl, Im, pkg.LOSS_CODES["Poisson_likelihood_loss"])
        res.append((float(loss), dO.cpu(), dP.cpu()))
    assert res[0][0] == res[1][0]
    assert torch.equal(res[0][1], res[1][1]) and torch.equal(res[0][2], res[1][2])


def test_edge_windows_and_uncovered_canvas(pkg):
    """Windows touching all four canvas edges; a region no window covers gets exactly 0."""
    M = 64
    O, P, _, _, _ = _case(M, 250, 1, seed=8, W=190)
    tlY = np.array([0, 250 - M, 0, 250 - M, 100], np.int32)
    tlX = np.array([0, 190 - M, 190 - M, 0, 60], np.int32)
    Imeas = np.abs(np.random.default_rng(0).standard_normal((5, M, M))).astype(np.float32) * 100
    for lt in LOSSES:
        loss, lp, dO, dP = _run(pkg, O, P, tlY, tlX, Imeas, lt)
        r = fm.fwd_adj(O, P, tlY, tlX, Imeas, lt)
        assert rel_max(dO, r["dO"]) <= GRAD_TOL[lt]
        assert rel_max(dP, r["dP"]) <= GRAD_TOL[lt]
        # rows 64..99 x cols 0..59 lie in no window
        assert np.all(dO[64:100, 0:60] == 0)


def test_empty_batch(pkg):
    dev = torch.device("cuda")
    O = torch.ones((80, 80), dtype=torch.complex64, device=dev)
    P = torch.ones((64, 64), dtype=torch.complex64, device=dev)
    tl = torch.zeros((0, 2), dtype=torch.int32, device=dev)
    Im = torch.zeros((0, 64, 64), dtype=torch.float32, device=dev)
    dO = torch.full((80, 80), 3 + 1j, dtype=torch.complex64, device=dev)
    dP = torch.full((64, 64), 3 + 1j, dtype=torch.complex64, device=dev)
    loss, _, dO, dP = pkg.fwd_adj_raw(O, P, tl, Im, 0, dO=dO, dP=dP)
    assert float(loss) == 0.0
    assert torch.count_nonzero(dO) == 0 and torch.count_nonzero(dP) == 0


def test_window_outside_canvas_sets_status(pkg):
    dev = torch.device("cuda")
    M = 64
    O, P, tlY, tlX, Imeas = _case(M, 100, 3, seed=6)
    pkg.read_status(dev, reset=True)
    tlY = tlY.copy(); tlY[1] = 100 - M + 1  # one row past the edge
    loss, lp, dO, dP = _run(pkg, O, P, tlY, tlX, Imeas, "Poisson_likelihood_loss")
    assert pkg.read_status(dev) == 6
    assert np.isnan(lp[1]) and np.isfinite(lp[0]) and np.isfinite(lp[2])
    # the bad window contributes nothing; the others still match the oracle
    keep = [0, 2]
    r = fm.fwd_adj(O, P, tlY[keep], tlX[keep], Imeas[keep], "Poisson_likelihood_loss")
    assert rel_max(dO, r["dO"]) <= 2e-4 and rel_max(dP, r["dP"]) <= 2e-4
    assert pkg.read_status(dev) == 0


def test_accumulate_flag(pkg):
    dev = torch.device("cuda")
    O, P, tlY, tlX, Imeas = _case(64, 120, 6, seed=12)
    Ot, Pt = torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev)
    tl = pkg.make_windows(tlY, tlX, dev)
    Im = torch.from_numpy(Imeas).to(dev)
    _, _, dO1, dP1 = pkg.fwd_adj_raw(Ot, Pt, tl[:3], Im[:3], 2)
    _, _, dO2, dP2 = pkg.fwd_adj_raw(Ot, Pt, tl[3:], Im[3:], 2, dO=dO1.clone(), dP=dP1.clone(),
                                     accumulate=True)
    _, _, dOa, dPa = pkg.fwd_adj_raw(Ot, Pt, tl, Im, 2)
    assert torch.allclose(dO2, dOa, rtol=1e-5, atol=1e-6 * float(dOa.abs().max()))
    assert torch.allclose(dP2, dPa, rtol=1e-5, atol=1e-6 * float(dPa.abs().max()))


def test_fused_loss_autograd(pkg):
    dev = torch.device("cuda")
    O, P, tlY, tlX, Imeas = _case(64, 120, 6, seed=13)
    Ot = torch.from_numpy(O).to(dev).requires_grad_(True)
    Pt = torch.from_numpy(P).to(dev).requires_grad_(True)
    loss = pkg.fused_loss(Ot, Pt, pkg.make_windows(tlY, tlX, dev), torch.from_numpy(Imeas).to(dev),
                          "smooth_L1_loss")
    (3.0 * loss).backward()
    r = fm.fwd_adj(O, P, tlY, tlX, Imeas, "smooth_L1_loss")
    assert rel_max(Ot.grad.cpu().numpy(), 3 * r["dO"]) <= 2e-4
    assert rel_max(Pt.grad.cpu().numpy(), 3 * r["dP"]) <= 2e-4


@pytest.mark.parametrize("which", ["object", "probe"])
def test_fused_loss_backward_one_input_twice(pkg, which):
    """Only one input needs a gradient; a retained graph backs up twice and the
    scaled copies leave the saved gradients intact (accumulates 2 x 0.5 d)."""
    dev = torch.device("cuda")
    O, P, tlY, tlX, Imeas = _case(64, 120, 5, seed=17)
    Ot = torch.from_numpy(O).to(dev).requires_grad_(which == "object")
    Pt = torch.from_numpy(P).to(dev).requires_grad_(which == "probe")
    loss = pkg.fused_loss(Ot, Pt, pkg.make_windows(tlY, tlX, dev), torch.from_numpy(Imeas).to(dev),
                          "Poisson_likelihood_loss")
    (0.5 * loss).backward(retain_graph=True)
    (0.5 * loss).backward()
    r = fm.fwd_adj(O, P, tlY, tlX, Imeas, "Poisson_likelihood_loss")
    if which == "object":
        assert rel_max(Ot.grad.cpu().numpy(), r["dO"]) <= 2e-4 and Pt.grad is None
    else:
        assert rel_max(Pt.grad.cpu().numpy(), r["dP"]) <= 2e-4 and Ot.grad is None


def test_frame_id_batches(pkg):
    """Frame ids select rows of a resident stack (Recovery.py's perm slice)."""
    dev = torch.device("cuda")
    O, P, tlY, tlX, Imeas = _case(128, 260, 20, seed=14)
    perm = np.random.default_rng(3).permutation(20)[:7].astype(np.int32)
    Ot, Pt = torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev)
    tl = pkg.make_windows(tlY, tlX, dev)
    Im = torch.from_numpy(Imeas).to(dev)
    loss, lp, dO, dP = pkg.fwd_adj_raw(Ot, Pt, tl, Im, 2, batch=torch.from_numpy(perm), per_pattern=True)
    r = fm.fwd_adj(O, P, tlY[perm], tlX[perm], Imeas[perm], "Poisson_likelihood_loss")
    assert np.all(np.abs(lp.cpu().numpy() - r["loss"]) <= 2e-5 * np.abs(r["loss"]))
    assert rel_max(dO.cpu().numpy(), r["dO"]) <= 2e-4 and rel_max(dP.cpu().numpy(), r["dP"]) <= 2e-4
    I = pkg.forward_intensity(Ot, Pt, tl, batch=torch.from_numpy(perm)).cpu().numpy()
    assert rel_max(I, fm.forward_intensity(O, P, tlY[perm], tlX[perm])) <= 1e-5
    # a frame id past the end is skipped and flagged
    pkg.read_status(dev, reset=True)
    bad = perm.copy(); bad[2] = 20
    _, lp2, dO2, _ = pkg.fwd_adj_raw(Ot, Pt, tl, Im, 2, batch=torch.from_numpy(bad), per_pattern=True)
    assert pkg.read_status(dev) == 6 and np.isnan(lp2[2].item())
