"""Accuracy bookkeeping on the host: the coverage box against the oracle's
restatement of the analysis script, and the oracle's error definitions
against resolve_global_phase directly."""
import importlib

import numpy as np
import pytest

from conftest import PKG_NAME
from oracle import forward_model as fm


@pytest.fixture(scope="module")
def acc():
    return importlib.import_module(PKG_NAME + ".accuracy")


@pytest.mark.parametrize("seed", range(6))
def test_coverage_box_matches_oracle(acc, seed):
    rng = np.random.default_rng(seed)
    H, M, F = int(rng.integers(80, 200)), int(rng.choice([16, 32, 64])), int(rng.integers(1, 40))
    tlY = rng.integers(-M // 2, H - M // 2, F)
    tlX = rng.integers(-M // 2, H - M // 2, F)
    for frac in (0.0, 0.3, 0.5, 1.0):
        assert acc.coverage_box(tlY, tlX, (M, M), (H, H), frac) == fm.coverage_box(tlY, tlX, (M, M), (H, H), frac)


def test_coverage_box_empty_scan(acc):
    assert acc.coverage_box([], [], (8, 8), (20, 30)) == (0, 20, 0, 30)


def test_oracle_object_error_definitions():
    rng = np.random.default_rng(0)
    g = rng.standard_normal((40, 50)) + 1j * rng.standard_normal((40, 50))
    r = 0.5 * np.exp(1j * 1.3) * g
    e_phase, e_scaled = fm.object_error(r, g)
    assert e_scaled < 1e-12
    assert abs(e_phase - 0.5) < 1e-12  # phase removed, the factor 0.5 is left
    noisy = r + 0.1 * (rng.standard_normal(r.shape) + 1j * rng.standard_normal(r.shape))
    a = fm.resolve_global_phase(noisy, g)
    assert abs(fm.object_error(noisy, g)[0] - np.linalg.norm(a - g) / np.linalg.norm(g)) < 1e-12
    box = (5, 30, 7, 41)
    assert fm.object_error(noisy, g, box) == fm.object_error(noisy[5:30, 7:41], g[5:30, 7:41])
