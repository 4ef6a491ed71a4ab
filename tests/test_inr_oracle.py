"""Pin the INR oracle: ComplexMLP against the reference module's own outputs and
gradients (tests/golden/complex_mlp.npz); HashGrid, Fourier upsample and Adam
against finite differences / their defining identities (HashGrid parity is
unpinned: tiny-cuda-nn is absent and unpinned)."""
import numpy as np
import pytest

from conftest import golden
from oracle import inr


def golden_params(g, k):
    hidden, layers = int(g[f"m{k}/cfg"][0]), int(g[f"m{k}/cfg"][1])
    P = lambda n: g[f"m{k}/param/{n}"]  # noqa: E731
    params = {"W1": P("net.0.linear.weight"), "b1": P("net.0.linear.bias"),
              "w1": float(P("net.0.omega_0")[0]),
              "Wh": [P(f"net.{i + 1}.linear.weight") for i in range(layers)],
              "bh": [P(f"net.{i + 1}.linear.bias") for i in range(layers)],
              "wh": [float(P(f"net.{i + 1}.omega_0")[0]) for i in range(layers)],
              "Wo": P(f"net.{layers + 1}.weight"), "bo": P(f"net.{layers + 1}.bias")}
    return params, layers


@pytest.mark.parametrize("k", [0, 1])
def test_cmlp_matches_reference_module(k):
    g = golden("complex_mlp.npz")
    params, layers = golden_params(g, k)
    y, cache = inr.cmlp_forward(g[f"m{k}/x"], params)
    np.testing.assert_allclose(y, g[f"m{k}/y"][:, 0], rtol=1e-12, atol=1e-12)
    gy = 2 * (y - g[f"m{k}/target"][:, 0])
    gr = inr.cmlp_backward(gy, params, cache)
    G = lambda n: g[f"m{k}/grad/{n}"]  # noqa: E731
    np.testing.assert_allclose(gr["W1"], G("net.0.linear.weight"), rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(gr["b1"], G("net.0.linear.bias"), rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(gr["w1"], G("net.0.omega_0")[0], rtol=1e-10)
    for i in range(layers):
        np.testing.assert_allclose(gr["Wh"][i], G(f"net.{i + 1}.linear.weight"), rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(gr["bh"][i], G(f"net.{i + 1}.linear.bias"), rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(gr["wh"][i], G(f"net.{i + 1}.omega_0")[0], rtol=1e-10)
    np.testing.assert_allclose(gr["Wo"], G(f"net.{layers + 1}.weight"), rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(gr["bo"], G(f"net.{layers + 1}.bias"), rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(gr["x"], g[f"m{k}/dx"], rtol=1e-10, atol=1e-12)


def test_hashgrid_levels_and_gradient():
    levels = inr.hashgrid_levels(8, 10, 4, 1.7)
    assert levels[0][4] and not levels[-1][4]  # coarse dense, fine hashed
    n = sum(l[2] for l in levels)
    rng = np.random.default_rng(0)
    coords = rng.random((300, 2))
    table = rng.uniform(-1, 1, n * 2)
    f = inr.hashgrid_encode(coords, table, levels)
    # bilinear partition of unity: a constant table gives constant features
    np.testing.assert_allclose(inr.hashgrid_encode(coords, np.ones(n * 2), levels), 1.0, rtol=1e-12)
    gfeat = rng.standard_normal(f.shape)
    gt = inr.hashgrid_backward(coords, gfeat, levels, n)
    # linear map: <backward(g), t> == <g, forward(t)>
    np.testing.assert_allclose(np.dot(gt, table), np.sum(gfeat * f), rtol=1e-10)


def test_fourier_upsample_adjoint_identity():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((16, 12)) + 1j * rng.standard_normal((16, 12))
    g = rng.standard_normal((32, 24)) + 1j * rng.standard_normal((32, 24))
    lhs = np.vdot(g, inr.fourier_upsample(x, 2))
    rhs = np.vdot(inr.fourier_upsample_adjoint(g, 2, x.shape), x)
    np.testing.assert_allclose(lhs, rhs, rtol=1e-10)


def test_adam_matches_torch():
    import torch
    rng = np.random.default_rng(2)
    p0 = rng.standard_normal(50)
    grads = [rng.standard_normal(50) for _ in range(4)]
    t = torch.tensor(p0, requires_grad=True)
    opt = torch.optim.Adam([t], lr=1e-2)
    p, m, v = p0.copy(), np.zeros(50), np.zeros(50)
    for s, gr in enumerate(grads, 1):
        t.grad = torch.tensor(gr)
        opt.step()
        p, m, v = inr.adam_step(p, gr, m, v, s, 1e-2)
    np.testing.assert_allclose(p, t.detach().numpy(), rtol=1e-12, atol=1e-14)
