"""Parity of the fused forward / loss / adjoint with the FP64 oracle at the
benchmark workloads' own shapes:

  c1  1536^2 object, 128^2 probe, Poisson, batch 256 (the 1600-position raster)
  c3  2048^2 object, 256^2 probe, Poisson, batch 64  (the 4-CTA cluster path)
  c4  4096^2 object, 256^2 probe, Poisson, batch 512 (9216-position raster)

Objects, probes and scans follow the workload recipes (synth.py); the
measurements are generated for the batch's frames only (same recipe, peak
scaled over those frames), which keeps the test to seconds.  The oracle runs
the whole batch in FP64 (in chunks, summed in FP64); on c4 the intensities
are scored on a 32-pattern sample.  On c1 the gradient is also checked
against FP64 central finite differences at 64 object and 16 probe pixels.

Tolerances (FP32 FFTs against FP64, as in test_fwd_adj_gpu.py):
  intensities   max|I - I_ref| / max|I_ref|     <= 1e-5
  losses        relative                        <= 2e-5
  dO, dP        max|g - g_ref| / max|g_ref|     <= 2e-4
  FD check      |g - g_fd| / max|g_ref|         <= 1e-3
"""
import numpy as np
import pytest
import torch

from conftest import load_pkg
from oracle import forward_model as fm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return load_pkg()


def rel_max(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-30))


def _batch_case(pkg, key, seed=5):
    """Workload `key`'s object, probe and raster; one batch of frame ids with
    Poisson measurements generated for those frames."""
    synth = pkg.synth
    w = synth.WORKLOADS[key]
    O = synth.make_object(w.canvas, seed=0)
    P = synth.make_probe(w.probe, w.aperture)
    tlY, tlX = synth.make_scan(w.n_scan, w.step, w.jitter, w.canvas, w.probe, seed=2)
    rng = np.random.default_rng(seed)
    ids = np.sort(rng.permutation(tlY.size)[:w.batch]).astype(np.int32)
    I = synth._intensities(O, P, tlY[ids], tlX[ids], device=torch.device("cuda"))
    I *= w.peak / I.max()
    Imeas = np.random.default_rng(1).poisson(I).astype(np.float32)
    return w, O.astype(np.complex64), P.astype(np.complex64), tlY[ids], tlX[ids], Imeas


def _oracle_chunked(O, P, tlY, tlX, Imeas, loss_type, chunk=64):
    """fm.fwd_adj over the batch in chunks (bounded host memory), FP64 sums."""
    O64, P64 = O.astype(np.complex128), P.astype(np.complex128)
    loss = np.empty(tlY.size)
    dO = np.zeros(O.shape, np.complex128)
    dP = np.zeros(P.shape, np.complex128)
    for s in range(0, tlY.size, chunk):
        r = fm.fwd_adj(O64, P64, tlY[s:s + chunk], tlX[s:s + chunk], Imeas[s:s + chunk], loss_type)
        loss[s:s + chunk] = r["loss"]
        dO += r["dO"]
        dP += r["dP"]
    return loss, dO, dP


def _gpu(pkg, w, O, P, tlY, tlX, Imeas, sample):
    dev = torch.device("cuda")
    Ot = torch.from_numpy(O).to(dev)
    Pt = torch.from_numpy(P).to(dev)
    tl = pkg.make_windows(tlY, tlX, dev)
    Im = torch.from_numpy(Imeas).to(dev)
    loss, lp, dO, dP = pkg.fwd_adj_raw(Ot, Pt, tl, Im, pkg.LOSS_CODES[w.loss_type], per_pattern=True)
    I = pkg.forward_intensity(Ot, Pt, tl, batch=torch.from_numpy(sample.astype(np.int32)).to(dev))
    torch.cuda.synchronize()
    return float(loss), lp.cpu().numpy(), dO.cpu().numpy(), dP.cpu().numpy(), I.cpu().numpy()


@pytest.mark.parametrize("key", ["c1", "c3", "c4"])
def test_on_config_against_fp64_oracle(pkg, key):
    w, O, P, tlY, tlX, Imeas = _batch_case(pkg, key)
    assert tlY.size == w.batch and O.shape == (w.canvas, w.canvas) and P.shape == (w.probe, w.probe)
    sample = np.arange(tlY.size) if key != "c4" else np.random.default_rng(3).permutation(tlY.size)[:32]
    loss, lp, dO, dP, I = _gpu(pkg, w, O, P, tlY, tlX, Imeas, sample)
    ref_I = fm.forward_intensity(O.astype(np.complex128), P.astype(np.complex128), tlY[sample], tlX[sample])
    assert rel_max(I, ref_I) <= 1e-5, rel_max(I, ref_I)
    ref_lp, ref_dO, ref_dP = _oracle_chunked(O, P, tlY, tlX, Imeas, w.loss_type)
    assert abs(loss - ref_lp.sum()) <= 2e-5 * abs(ref_lp.sum())
    assert np.all(np.abs(lp - ref_lp) <= 2e-5 * np.maximum(np.abs(ref_lp), 1e-30))
    assert rel_max(dO, ref_dO) <= 2e-4, rel_max(dO, ref_dO)
    assert rel_max(dP, ref_dP) <= 2e-4, rel_max(dP, ref_dP)


def test_c1_finite_differences(pkg):
    """FP64 central differences of the batch loss at 64 object and 16 probe
    pixels (the c1 configuration's own check)."""
    w, O, P, tlY, tlX, Imeas = _batch_case(pkg, "c1")
    _, _, dO, dP, _ = _gpu(pkg, w, O, P, tlY, tlX, Imeas, np.arange(4))
    O64, P64 = O.astype(np.complex128), P.astype(np.complex128)
    M = w.probe
    rng = np.random.default_rng(11)
    # object pixels inside the scanned area (each covered by at least one window)
    cov = np.zeros(O.shape, bool)
    for y, x in zip(tlY, tlX):
        cov[y:y + M, x:x + M] = True
    cand = np.argwhere(cov)
    opix = [tuple(c) for c in cand[rng.choice(len(cand), 64, replace=False)]]
    ppix = [tuple(c) for c in rng.integers(M // 4, 3 * M // 4, size=(16, 2))]

    def fd_obj(r, c):  # only the windows holding (r, c) change the loss
        sel = (tlY <= r) & (r < tlY + M) & (tlX <= c) & (c < tlX + M)
        return fm.fd_gradient(O64, P64, tlY[sel], tlX[sel], Imeas[sel], w.loss_type, "O", [(r, c)])[0]

    g_o = np.array([fd_obj(r, c) for r, c in opix])
    g_p = np.array(fm.fd_gradient(O64, P64, tlY, tlX, Imeas, w.loss_type, "P", ppix))
    got_o = np.array([dO[r, c] for r, c in opix])
    got_p = np.array([dP[r, c] for r, c in ppix])
    assert np.abs(got_o - g_o).max() <= 1e-3 * np.abs(dO).max(), np.abs(got_o - g_o).max() / np.abs(dO).max()
    assert np.abs(got_p - g_p).max() <= 1e-3 * np.abs(dP).max(), np.abs(got_p - g_p).max() / np.abs(dP).max()
