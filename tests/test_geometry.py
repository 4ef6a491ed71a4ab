"""Host geometry of the package matches the reference bit for bit."""
import numpy as np

from conftest import golden, load_pkg


def test_scan_positions_bit_exact_against_reference_fixture():
    pkg = load_pkg()
    g = golden("scan_indices.npz")
    for k in ("c0", "c1", "c2", "c3"):
        lam, L, pitch = g[f"{k}/phys"]
        M = int(g[f"{k}/M"])
        tlX, tlY, brX, brY, dx, canvas = pkg.scan_positions_to_pixels(
            g[f"{k}/x"], g[f"{k}/y"], (M, M), lam, L, pitch)
        assert np.array_equal(np.stack([tlY, tlX]), g[f"{k}/tl"])
        assert np.array_equal(np.stack([brY, brX]), g[f"{k}/br"])
        assert np.array_equal(dx, g[f"{k}/dx"])
        assert canvas == int(g[f"{k}/canvas"])


def test_make_and_check_windows():
    pkg = load_pkg()
    t = pkg.make_windows([0, 5, 36], [1, 2, 36])
    assert t.dtype.is_floating_point is False and tuple(t.shape) == (3, 2)
    assert t[:, 0].tolist() == [0, 5, 36]
    pkg.check_windows(t, (100, 100), 64)
    import pytest
    with pytest.raises(ValueError):
        pkg.check_windows(t, (99, 100), 64)
