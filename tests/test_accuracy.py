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


def test_oracle_align_by_xcorr_matches_direct_search():
    """The FFT placement of the analysis script equals a direct search over every
    offset that keeps the recon inside the truth (mean-removed magnitudes)."""
    rng = np.random.default_rng(11)
    for Hg, Wg, H, W in ((40, 50, 24, 30), (33, 33, 33, 33), (30, 45, 10, 12)):
        g = rng.random((Hg, Wg))
        y, x = rng.integers(0, Hg - H + 1), rng.integers(0, Wg - W + 1)
        r = g[y:y + H, x:x + W] + 0.01 * rng.random((H, W))
        rm, gm = r - r.mean(), g - g.mean()
        direct = np.array([[np.sum(gm[a:a + H, b:b + W] * rm) for b in range(Wg - W + 1)]
                           for a in range(Hg - H + 1)])
        assert fm.align_by_xcorr(r, g) == tuple(int(v) for v in np.unravel_index(np.argmax(direct), direct.shape))
        assert fm.align_by_xcorr(r, g) == (y, x)


@pytest.mark.parametrize("d", [(0.0, 0.0), (0.37, -1.62), (-2.5, 3.01), (4.0, -0.99)])
def test_oracle_register_translation_recovers_shifts(d):
    """A smooth complex object shifted by d (on the 1/100 grid) is registered
    exactly, and shifting back restores it to round-off."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(3)
    g = gaussian_filter(rng.random((72, 80)), 3) + 1j * gaussian_filter(rng.random((72, 80)), 3)
    r = fm.fourier_shift(g, -d[0], -d[1])
    est = fm.register_translation(r, g, 100)
    assert np.allclose(est, d, atol=1e-9), est
    assert fm.object_error(fm.fourier_shift(r, *est), g)[0] < 1e-12


@pytest.mark.parametrize("seed,d", [(8, (1.23, -0.71)), (10, (-3.3, 2.05))])
def test_oracle_register_in_box(seed, d):
    """Crops are not periodic: windowed registration on the box, iterated on the
    shifted canvas, recovers the shift of the whole canvas exactly."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    g = gaussian_filter(rng.random((160, 160)), 3) + 1j * gaussian_filter(rng.random((160, 160)), 3)
    r = 0.8 * np.exp(0.4j) * fm.fourier_shift(g, *d)
    est = fm.register_in_box(r, g, (20, 140, 24, 136))
    assert np.allclose(est, (-d[0], -d[1]), atol=1e-9), est
