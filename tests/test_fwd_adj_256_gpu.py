"""Parity of the 256 x 256 probe paths with the FP64 oracle: the line-DFT
kernels (smooth-L1, Poisson and the intensity gradient; batches above 512
patterns in chunks of 512) and the 4-CTA cluster kernel (FD loss and forward intensities; the
pass-2/pass-3 exchange through distributed shared memory).

Tolerances as for 64 / 128 (FP32 FFT against FP64):
  forward intensities  max|I - I_ref| / max|I_ref|      <= 1e-5
  per-pattern losses   |l - l_ref| / |l_ref|            <= 2e-5
  gradients dO, dP     max|g - g_ref| / max|g_ref|      <= 2e-4 (smooth_L1, Poisson),
                                                         <= 1e-3 (FD)
The FD stencil couples neighbouring frequency rows, which the cluster keeps in
different CTAs: its parity also checks the cross-CTA reads.
"""
import numpy as np
import pytest
import torch

from conftest import load_pkg
from oracle import forward_model as fm
from test_fwd_adj_gpu import GRAD_TOL, _case, _run, rel_max

pytestmark = pytest.mark.gpu
M = 256


@pytest.fixture(scope="module")
def pkg():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return load_pkg()


@pytest.mark.parametrize("loss_type", fm.LOSS_TYPES)
@pytest.mark.parametrize("H,B", [(300, 3), (420, 70)])
def test_against_fp64_oracle_256(pkg, H, B, loss_type):
    # B = 70 exceeds the number of co-resident clusters: the persistent loop runs
    O, P, tlY, tlX, Imeas = _case(M, H, B, seed=256 + B)
    loss, lp, dO, dP = _run(pkg, O, P, tlY, tlX, Imeas, loss_type)
    r = fm.fwd_adj(O, P, tlY, tlX, Imeas, loss_type)
    assert np.all(np.abs(lp - r["loss"]) <= 2e-5 * np.abs(r["loss"]) + 1e-12), np.abs(lp / r["loss"] - 1).max()
    assert abs(loss - r["loss_total"]) <= 2e-5 * abs(r["loss_total"])
    assert rel_max(dO, r["dO"]) <= GRAD_TOL[loss_type], rel_max(dO, r["dO"])
    assert rel_max(dP, r["dP"]) <= GRAD_TOL[loss_type], rel_max(dP, r["dP"])


def test_forward_intensity_256(pkg):
    O, P, tlY, tlX, _ = _case(M, 2 * M + 37, 9, seed=7, W=2 * M + 5)
    dev = torch.device("cuda")
    I = pkg.forward_intensity(torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev),
                              pkg.make_windows(tlY, tlX, dev)).cpu().numpy()
    ref = fm.forward_intensity(O, P, tlY, tlX)
    assert rel_max(I, ref) <= 1e-5, rel_max(I, ref)
    psi = fm.exit_waves(O, P, tlY, tlX)
    np.testing.assert_allclose(I.reshape(9, -1).sum(1), M * M * (np.abs(psi) ** 2).reshape(9, -1).sum(1),
                               rtol=1e-5)


def test_loss_only_256(pkg):
    """No gradient outputs: the loss-only kernel (no adjoint passes)."""
    dev = torch.device("cuda")
    O, P, tlY, tlX, Imeas = _case(M, 320, 5, seed=21)
    loss, lp, _, _ = pkg.fwd_adj_raw(torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev),
                                     pkg.make_windows(tlY, tlX, dev), torch.from_numpy(Imeas).to(dev),
                                     pkg.LOSS_CODES["Poisson_likelihood_loss"], want_grad=False,
                                     per_pattern=True)
    r = fm.fwd_adj(O, P, tlY, tlX, Imeas, "Poisson_likelihood_loss")
    assert np.all(np.abs(lp.cpu().numpy() - r["loss"]) <= 2e-5 * np.abs(r["loss"]))
    assert abs(float(loss) - r["loss_total"]) <= 2e-5 * abs(r["loss_total"])


def test_deterministic_and_edges_256(pkg):
    """Bitwise repeatable; windows on every canvas edge; a skipped window."""
    dev = torch.device("cuda")
    H = 384
    O, P, tlY, tlX, Imeas = _case(M, H, 6, seed=22)
    tlY[:4] = [0, H - M, 0, H - M]
    tlX[:4] = [0, 0, H - M, H - M]
    Imeas = fm.forward_intensity(O * 1.01, P, tlY, tlX).astype(np.float32)
    a = _run(pkg, O, P, tlY, tlX, Imeas, "smooth_L1_loss")
    b = _run(pkg, O, P, tlY, tlX, Imeas, "smooth_L1_loss")
    assert a[0] == b[0] and np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])
    r = fm.fwd_adj(O, P, tlY, tlX, Imeas, "smooth_L1_loss")
    assert rel_max(a[2], r["dO"]) <= 2e-4 and rel_max(a[3], r["dP"]) <= 2e-4
    pkg.read_status(dev, reset=True)
    bad = tlX.copy()
    bad[5] = H - M + 1
    loss, lp, dO, dP = _run(pkg, O, P, tlY, bad, Imeas, "smooth_L1_loss")
    assert pkg.read_status(dev) == 6
    assert np.isnan(lp[5]) and np.all(np.isfinite(lp[:5]))
    keep = list(range(5))
    r = fm.fwd_adj(O, P, tlY[keep], tlX[keep], Imeas[keep], "smooth_L1_loss")
    assert rel_max(dO, r["dO"]) <= 2e-4 and rel_max(dP, r["dP"]) <= 2e-4
    assert pkg.read_status(dev) == 0


def test_fd_loss_only_256(pkg):
    """FD loss without gradients (loss-only kernel, same cross-CTA stencil)."""
    dev = torch.device("cuda")
    O, P, tlY, tlX, Imeas = _case(M, 300, 4, seed=23)
    loss, lp, _, _ = pkg.fwd_adj_raw(torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev),
                                     pkg.make_windows(tlY, tlX, dev), torch.from_numpy(Imeas).to(dev),
                                     pkg.LOSS_CODES["FD_loss"], want_grad=False, per_pattern=True)
    r = fm.fwd_adj(O, P, tlY, tlX, Imeas, "FD_loss")
    assert np.all(np.abs(lp.cpu().numpy() - r["loss"]) <= 2e-5 * np.abs(r["loss"]))


def _intensity_grad_ref(O, P, tlY, tlX, gI):
    """dO, dP of sum(I * gI) in FP64 (the intensity-gradient call's contract)."""
    O, P = O.astype(np.complex128), P.astype(np.complex128)
    F = fm.far_field(fm.exit_waves(O, P, tlY, tlX))
    E = (M * M) * np.fft.ifft2(np.fft.ifftshift(2.0 * gI * F, axes=(-2, -1)), axes=(-2, -1))
    dO, dP = np.zeros_like(O), np.zeros_like(P)
    for b in range(tlY.size):
        y, x = int(tlY[b]), int(tlX[b])
        dP += E[b] * np.conj(O[y:y + M, x:x + M])
        dO[y:y + M, x:x + M] += E[b] * np.conj(P)
    return dO, dP


def _oracle_chunked(O, P, tlY, tlX, Imeas, loss_type, chunk=64):
    loss = np.empty(tlY.size)
    dO = np.zeros(O.shape, np.complex128)
    dP = np.zeros(P.shape, np.complex128)
    for s in range(0, tlY.size, chunk):
        r = fm.fwd_adj(O, P, tlY[s:s + chunk], tlX[s:s + chunk], Imeas[s:s + chunk], loss_type)
        loss[s:s + chunk] = r["loss"]
        dO += r["dO"]
        dP += r["dP"]
    return loss, dO, dP


def test_chunks_repeats_and_a_skipped_window_256(pkg):
    """520 patterns = the line-DFT kernels' chunks of 512 and 8; frame ids
    repeat; one frame's window, drawn in the second chunk, leaves the canvas
    (NaN loss wherever it is drawn, status 6, no contribution); bitwise
    repeatable."""
    dev = torch.device("cuda")
    H, F, B = 460, 40, 520
    O, P, tlY, tlX, Imeas = _case(M, H, F, seed=150)
    ids = np.random.default_rng(3).integers(0, F, B).astype(np.int32)
    bad = tlX.copy()
    bad[ids[515]] = H - M + 3
    Ot, Pt = torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev)
    tl = pkg.make_windows(tlY, bad, dev)
    Im = torch.from_numpy(Imeas).to(dev)
    bt = torch.from_numpy(ids).to(dev)
    pkg.read_status(dev, reset=True)
    runs = [pkg.fwd_adj_raw(Ot, Pt, tl, Im, pkg.LOSS_CODES["Poisson_likelihood_loss"], batch=bt, per_pattern=True)
            for _ in range(2)]
    torch.cuda.synchronize()
    assert pkg.read_status(dev) == 6
    (l0, lp, dO, dP), (l1, lp1, dO1, dP1) = [[x.cpu().numpy() for x in r] for r in runs]
    assert np.array_equal(lp, lp1, equal_nan=True) and np.array_equal(dO, dO1) and np.array_equal(dP, dP1)
    skipped = ids == ids[515]
    assert np.all(np.isnan(lp[skipped])) and np.all(np.isfinite(lp[~skipped]))
    keep = ids[~skipped]
    ref_l, ref_dO, ref_dP = _oracle_chunked(O.astype(np.complex128), P.astype(np.complex128), tlY[keep], tlX[keep],
                                            Imeas[keep], "Poisson_likelihood_loss")
    assert np.all(np.abs(lp[~skipped] - ref_l) <= 2e-5 * np.abs(ref_l))
    assert rel_max(dO, ref_dO) <= 2e-4, rel_max(dO, ref_dO)
    assert rel_max(dP, ref_dP) <= 2e-4, rel_max(dP, ref_dP)
    assert pkg.read_status(dev) == 0
    # accumulate: two calls into the same buffers give twice one call (this
    # batch size takes the probe gradient from the inverse-row kernel)
    gO = torch.zeros_like(Ot)
    gP = torch.zeros_like(Pt)
    for _ in range(2):
        pkg.fwd_adj_raw(Ot, Pt, tl, Im, pkg.LOSS_CODES["Poisson_likelihood_loss"], batch=bt, dO=gO, dP=gP,
                        accumulate=True)
    pkg.read_status(dev, reset=True)
    assert rel_max(gO.cpu().numpy(), 2 * dO) <= 1e-6 and rel_max(gP.cpu().numpy(), 2 * dP) <= 1e-6


def test_intensity_gradient_256(pkg):
    """The intensity-gradient call (autograd of forward_intensity_batched)
    over two chunks, against the FP64 adjoint."""
    dev = torch.device("cuda")
    B = 70
    O, P, tlY, tlX, _ = _case(M, 400, B, seed=31)
    gI = np.random.default_rng(4).standard_normal((B, M, M)).astype(np.float32)
    Ot = torch.from_numpy(O).to(dev).requires_grad_(True)
    Pt = torch.from_numpy(P).to(dev).requires_grad_(True)
    I = pkg.forward_intensity_batched(Ot, Pt, pkg.make_windows(tlY, tlX, dev))
    (I * torch.from_numpy(gI).to(dev)).sum().backward()
    dO, dP = _intensity_grad_ref(O, P, tlY, tlX, gI.astype(np.float64))
    assert rel_max(Ot.grad.cpu().numpy(), dO) <= 2e-4, rel_max(Ot.grad.cpu().numpy(), dO)
    assert rel_max(Pt.grad.cpu().numpy(), dP) <= 2e-4, rel_max(Pt.grad.cpu().numpy(), dP)


def test_one_gradient_output_on_large_batches_256(pkg):
    """B >= 192 takes dP from the inverse-row kernel: asking for dP alone or dO
    alone gives bitwise what the call with both outputs gives."""
    dev = torch.device("cuda")
    B = 200
    O, P, tlY, tlX, Imeas = _case(M, 420, B, seed=41)
    Ot, Pt = torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev)
    tl = pkg.make_windows(tlY, tlX, dev)
    Im = torch.from_numpy(Imeas).to(dev)
    code = pkg.LOSS_CODES["smooth_L1_loss"]
    L = pkg.lib()
    H = W = 420
    ws_n = int(L.ptycho_fwd_adj_workspace_size(H, W, M, M, B))
    st = pkg.optics.device_status(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream

    def call(want_o, want_p):
        ws = torch.empty(ws_n, dtype=torch.uint8, device=dev)
        loss = torch.zeros((), dtype=torch.float64, device=dev)
        dO = torch.full((H, W), float("nan"), dtype=torch.complex64, device=dev) if want_o else None
        dP = torch.full((M, M), float("nan"), dtype=torch.complex64, device=dev) if want_p else None
        rc = L.ptycho_fwd_adj(Ot.data_ptr(), H, W, Pt.data_ptr(), M, M, tl.data_ptr(), Im.data_ptr(), B, None, B,
                              code, None, loss.data_ptr(), dO.data_ptr() if want_o else None,
                              dP.data_ptr() if want_p else None, 0, ws.data_ptr(), ws_n, st.data_ptr(), stream)
        assert rc == 0, L.ptycho_status_string(rc)
        torch.cuda.synchronize()
        return float(loss), (dO.cpu().numpy() if want_o else None), (dP.cpu().numpy() if want_p else None)

    l_both, dO_both, dP_both = call(True, True)
    l_p, _, dP_only = call(False, True)
    l_o, dO_only, _ = call(True, False)
    assert l_both == l_p == l_o
    assert np.array_equal(dP_only, dP_both) and np.array_equal(dO_only, dO_both)
    r = fm.fwd_adj(O, P, tlY, tlX, Imeas, "smooth_L1_loss")
    assert rel_max(dP_both, r["dP"]) <= 2e-4 and rel_max(dO_both, r["dO"]) <= 2e-4


def test_loss_only_over_two_chunks_256(pkg):
    """The loss-only mode (no gradient outputs) over 600 patterns (chunks of
    512 and 88) against the FP64 oracle, pattern by pattern."""
    dev = torch.device("cuda")
    F = 50
    O, P, tlY, tlX, Imeas = _case(M, 360, F, seed=43)
    ids = np.random.default_rng(5).integers(0, F, 600).astype(np.int32)
    loss, lp, _, _ = pkg.fwd_adj_raw(torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev),
                                     pkg.make_windows(tlY, tlX, dev), torch.from_numpy(Imeas).to(dev),
                                     pkg.LOSS_CODES["Poisson_likelihood_loss"], batch=torch.from_numpy(ids).to(dev),
                                     want_grad=False, per_pattern=True)
    lp = lp.cpu().numpy()
    r = fm.fwd_adj(O, P, tlY, tlX, Imeas, "Poisson_likelihood_loss")  # each frame once
    want = r["loss"][ids]
    assert np.all(np.abs(lp - want) <= 2e-5 * np.abs(want))
    assert abs(float(loss) - want.sum()) <= 2e-5 * abs(want.sum())
