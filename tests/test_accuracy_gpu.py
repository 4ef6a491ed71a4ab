"""FP64 object error after global-phase alignment on the device
(``ptycho_object_error``) against the oracle's restatement of
resolve_global_phase (scripts/compare_object_ssim.py:92-98).

Tolerance: the device sums run in FP64 over FP32 inputs, as the oracle does
in complex128, so only summation order differs: 1e-9 relative on the errors
and 1e-9 on the phase factor."""
import importlib

import numpy as np
import pytest
import torch

from conftest import PKG_NAME
from oracle import forward_model as fm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def acc():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return importlib.import_module(PKG_NAME + ".accuracy")


def _pair(rng, H, W, noise):
    g = (rng.standard_normal((H, W)) + 1j * rng.standard_normal((H, W))).astype(np.complex64)
    r = 0.7 * np.exp(-1j * 2.1) * g + noise * (rng.standard_normal((H, W)) + 1j * rng.standard_normal((H, W)))
    return r.astype(np.complex64), g


@pytest.mark.parametrize("H,W,box", [(1, 1, None), (64, 80, (3, 59, 7, 78)), (257, 300, None),
                                     (1024, 1024, (100, 900, 37, 1011)), (3000, 17, (0, 3000, 16, 17))])
def test_object_error_matches_oracle(acc, H, W, box):
    rng = np.random.default_rng(H * 7 + W)
    r, g = _pair(rng, H, W, 0.3)
    dev = torch.device("cuda")
    out = acc.object_error(torch.from_numpy(r).to(dev), torch.from_numpy(g).to(dev), box)
    e_phase, e_scaled = fm.object_error(r, g, box)
    assert abs(out["nrmse"] - e_phase) <= 1e-9 * max(e_phase, 1e-3)
    assert abs(out["nrmse_scaled"] - e_scaled) <= 1e-9 * max(e_scaled, 1e-3)
    y0, y1, x0, x1 = box if box else (0, H, 0, W)
    c = np.vdot(r[y0:y1, x0:x1].astype(np.complex128), g[y0:y1, x0:x1].astype(np.complex128))
    assert abs(out["phase"] - c / abs(c)) <= 1e-9


def test_object_error_exact_cases(acc):
    dev = torch.device("cuda")
    rng = np.random.default_rng(5)
    g = (rng.standard_normal((96, 96)) + 1j * rng.standard_normal((96, 96))).astype(np.complex64)
    gt = torch.from_numpy(g).to(dev)
    same = acc.object_error(gt, gt)
    assert same["nrmse"] < 1e-6 and same["nrmse_scaled"] < 1e-6 and abs(same["phase"] - 1) < 1e-12
    rot = acc.object_error(gt * complex(np.exp(1j * 0.9)), gt)  # a Python complex: torch keeps its phase
    assert rot["nrmse"] < 1e-6 and abs(rot["phase"] - np.exp(-1j * 0.9)) < 1e-6
    zero = acc.object_error(torch.zeros_like(gt), gt)  # nothing to align: error 1, factor 1
    assert zero["nrmse"] == 1.0 and zero["phase"] == 1.0


def test_object_error_rejects_bad_input(acc):
    dev = torch.device("cuda")
    a = torch.zeros(8, 8, dtype=torch.complex64, device=dev)
    with pytest.raises(ValueError):
        acc.object_error(a, torch.zeros(8, 9, dtype=torch.complex64, device=dev))
    with pytest.raises(Exception):
        acc.object_error(a, a, (0, 9, 0, 8))


# ---- translation alignment (FP64 on the device) against the oracle -----------
def _smooth(rng, H, W):
    from scipy.ndimage import gaussian_filter
    return gaussian_filter(rng.random((H, W)), 3) + 1j * gaussian_filter(rng.random((H, W)), 3)


def test_align_by_xcorr_matches_oracle(acc):
    dev = torch.device("cuda")
    rng = np.random.default_rng(21)
    for Hg, Wg, H, W in ((64, 80, 40, 52), (128, 128, 128, 128), (90, 70, 31, 17)):
        g = rng.random((Hg, Wg))
        y, x = rng.integers(0, Hg - H + 1), rng.integers(0, Wg - W + 1)
        r = g[y:y + H, x:x + W] * (1 + 0.05 * rng.random((H, W)))
        got = acc.align_by_xcorr(torch.from_numpy(r).to(dev), torch.from_numpy(g).to(dev))
        assert got == fm.align_by_xcorr(r, g) == (y, x)


@pytest.mark.parametrize("d", [(0.0, 0.0), (0.37, -1.62), (-2.5, 3.01), (6.0, -0.99)])
def test_register_translation_matches_oracle(acc, d):
    """Same peak on the same 1/100 grid as the oracle; the shift found is the one applied."""
    dev = torch.device("cuda")
    g = _smooth(np.random.default_rng(5), 96, 112)
    r = fm.fourier_shift(g, -d[0], -d[1])
    got = acc.register_translation(torch.from_numpy(r).to(dev), torch.from_numpy(g).to(dev))
    assert got == fm.register_translation(r, g, 100)
    assert np.allclose(got, d, atol=1e-9)
    back = acc.fourier_shift(torch.from_numpy(r).to(dev), *got).cpu().numpy()
    assert np.abs(back - fm.fourier_shift(r, *got)).max() <= 1e-12 * np.abs(r).max()


def test_object_error_aligned(acc):
    """A truth shifted by a sub-pixel amount inside the box: the aligned error is
    at FP32 round-off, the unaligned one is not; the box excludes the wrapped edges."""
    dev = torch.device("cuda")
    g = _smooth(np.random.default_rng(8), 160, 160)
    r = (0.8 * np.exp(0.4j) * fm.fourier_shift(g, 1.23, -0.71)).astype(np.complex64)
    box = (20, 140, 24, 136)
    rt, gt = torch.from_numpy(r).to(dev), torch.from_numpy(g.astype(np.complex64)).to(dev)
    e = acc.object_error_aligned(rt, gt, box)
    assert np.allclose(e["shift"], (-1.23, 0.71), atol=1e-9)
    assert np.allclose(e["shift"], fm.register_in_box(r, g, box), atol=1e-9)
    assert e["nrmse_scaled"] < 1e-5, e
    assert acc.object_error(rt, gt, box)["nrmse_scaled"] > 1e-2


def test_alignment_rejects_host_tensors(acc):
    a = torch.zeros(8, 8, dtype=torch.complex64)
    with pytest.raises(ValueError):
        acc.register_translation(a, a)
    with pytest.raises(ValueError):
        acc.align_by_xcorr(a.real, a.real)
