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
