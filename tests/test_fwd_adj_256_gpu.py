"""Parity of the 256 x 256 probe path (one 4-CTA cluster per pattern, the
pass-2/pass-3 exchange through distributed shared memory) with the FP64 oracle.

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
