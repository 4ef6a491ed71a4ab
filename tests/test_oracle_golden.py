"""Pin the FP64 oracle against golden vectors produced by the reference itself."""
import numpy as np
import pytest

from conftest import golden
from oracle import forward_model as fm

LOSSES = fm.LOSS_TYPES


@pytest.mark.parametrize("case", ["m16", "m64"])
@pytest.mark.parametrize("loss_type", LOSSES)
def test_fwd_adj_matches_reference(case, loss_type):
    g = golden(f"fwd_adj_{case}.npz")
    r = fm.fwd_adj(g["O"], g["P"], g["tlY"], g["tlX"], g["Imeas"], loss_type)
    np.testing.assert_allclose(r["loss"], g[f"{loss_type}/loss"], rtol=1e-11, atol=0)
    for k in ("dO", "dP"):
        ref = g[f"{loss_type}/{k}"]
        err = np.abs(r[k] - ref).max() / np.abs(ref).max()
        assert err < 1e-10, (k, err)
    if loss_type == "Poisson_likelihood_loss":
        np.testing.assert_allclose(r["I"], g["I"], rtol=1e-10, atol=1e-9 * g["I"].max())


@pytest.mark.parametrize("loss_type", LOSSES)
def test_oracle_gradient_matches_finite_differences(loss_type):
    g = golden("fwd_adj_m16.npz")
    r = fm.fwd_adj(g["O"], g["P"], g["tlY"], g["tlX"], g["Imeas"], loss_type)
    rng = np.random.default_rng(3)
    oi = [tuple(x) for x in rng.integers(0, 24, size=(6, 2))]
    pi = [tuple(x) for x in rng.integers(0, 16, size=(4, 2))]
    fo = fm.fd_gradient(g["O"], g["P"], g["tlY"], g["tlX"], g["Imeas"], loss_type, "O", oi, h=1e-6)
    fp = fm.fd_gradient(g["O"], g["P"], g["tlY"], g["tlX"], g["Imeas"], loss_type, "P", pi, h=1e-6)
    ao = np.array([r["dO"][i] for i in oi])
    ap = np.array([r["dP"][i] for i in pi])
    scale_o = np.abs(r["dO"]).max()
    scale_p = np.abs(r["dP"]).max()
    assert np.abs(fo - ao).max() < 1e-5 * scale_o + 1e-9
    assert np.abs(fp - ap).max() < 1e-5 * scale_p + 1e-9


def test_scan_indices_bit_exact():
    g = golden("scan_indices.npz")
    ks = sorted({k.split("/")[0] for k in g.files})
    assert len(ks) == 4
    for k in ks:
        lam, L, pitch = g[f"{k}/phys"]
        M = int(g[f"{k}/M"])
        tlX, tlY, brX, brY, dx, canvas = fm.scan_positions_to_pixels(
            g[f"{k}/x"], g[f"{k}/y"], (M, M), lam, L, pitch)
        assert np.array_equal(np.stack([tlY, tlX]), g[f"{k}/tl"]), k
        assert np.array_equal(np.stack([brY, brX]), g[f"{k}/br"]), k
        assert np.array_equal(dx, g[f"{k}/dx"]), k
        assert canvas == int(g[f"{k}/canvas"]), k


def test_scan_indices_round_half_even_ties_present():
    g = golden("scan_indices.npz")
    lam, L, pitch = g["c0/phys"]
    dx = lam * L / (int(g["c0/M"]) * pitch)
    q = (g["c0/y"] - g["c0/y"].min()) / dx
    assert np.any(np.abs(q - np.floor(q) - 0.5) == 0), "fixture must contain exact .5 ties"


def test_probe_centering_and_haar():
    g = golden("probe_haar.npz")
    for k in range(3):
        P = g[f"p{k}/P"]
        cp = fm.probe_com_shift(P.astype(np.complex128))
        ref = g[f"p{k}/centered"]
        ours = np.roll(P, (-int(cp[0]), -int(cp[1])), axis=(0, 1)) if cp is not None else P
        np.testing.assert_array_equal(ours, ref)
    np.testing.assert_allclose(fm.haar_sparsity(g["haar/img"]), float(g["haar/value"]), rtol=1e-12)
