"""Probe centring + energy normalisation kernels (Recovery.py:262-285).

Pinned to the reference's own center_probe output (tests/golden/probe_haar.npz,
integer roll: exact), to the FP64 oracle (values: <= 1e-6 relative to max) and,
for the backward, to torch autograd of the reference formula in complex128
(<= 1e-5 relative to max).
"""
import numpy as np
import pytest
import torch

from conftest import golden, load_pkg
from oracle import forward_model as fm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return load_pkg()


def _run(pkg, P):
    dev = torch.device("cuda")
    Pt = torch.from_numpy(np.ascontiguousarray(P.astype(np.complex64))).to(dev)
    M, N = P.shape
    out = torch.empty_like(Pt)
    state = torch.empty(4, dtype=torch.float64, device=dev)
    pkg._lib.check(pkg.lib().ptycho_probe_center_normalize(Pt.data_ptr(), M, N, out.data_ptr(), state.data_ptr(),
                                                           None), "probe")
    torch.cuda.synchronize()
    return out.cpu().numpy(), state.cpu().numpy()


def _offset_probe(M, N, cy, cx, seed):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[:M, :N]
    r2 = (yy - cy) ** 2 + (xx - cx) ** 2
    P = np.exp(-r2 / (2 * (0.12 * min(M, N)) ** 2)) * np.exp(1j * 0.01 * r2)
    return (P + 0.01 * (rng.standard_normal((M, N)) + 1j * rng.standard_normal((M, N)))).astype(np.complex64)


def test_golden_center_probe(pkg):
    g = golden("probe_haar.npz")
    for k in range(3):
        P = g[f"p{k}/P"]
        out, st = _run(pkg, P)
        cp = fm.probe_com_shift(P.astype(np.complex128))
        assert (int(st[0]), int(st[1])) == (int(cp[0]), int(cp[1]))
        ref = g[f"p{k}/centered"].astype(np.complex128) * st[2]
        np.testing.assert_allclose(out, ref, rtol=1e-6, atol=1e-6 * np.abs(ref).max())


@pytest.mark.parametrize("M,N,cy,cx", [(64, 64, 10, 50), (128, 128, 90, 20), (96, 64, 30, 31),
                                       (256, 256, 200, 128), (128, 128, 64, 64)])
def test_against_oracle(pkg, M, N, cy, cx):
    P = _offset_probe(M, N, cy, cx, M + cy)
    out, st = _run(pkg, P)
    ref = fm.center_and_normalize_probe(P.astype(np.complex128))
    assert np.abs(out - ref).max() <= 1e-6 * np.abs(ref).max()
    assert abs((np.abs(out.astype(np.complex128)) ** 2).sum() - M * N) <= 1e-5 * M * N


def test_zero_probe(pkg):
    out, st = _run(pkg, np.zeros((64, 64), np.complex64))
    assert np.all(out == 0) and st[0] == 0 and st[1] == 0 and st[2] == 1.0 and st[3] == 0.0


def _ref_torch(P):
    """The reference's probe preparation in torch (Recovery.py:262-285)."""
    M, N = P.shape
    with torch.no_grad():
        a = P.abs() ** 2
        tot = a.sum()
        cp = torch.trunc(torch.tensor([M, N], dtype=torch.float64) / 2 - torch.tensor([M, N], dtype=torch.float64)
                         * torch.stack((a.sum(1).cumsum(0).mean(), a.sum(0).cumsum(0).mean())).cpu() / tot.cpu()
                         + 1).long()
    P = torch.roll(P, (-int(cp[0]), -int(cp[1])), (0, 1))
    e = (P.abs() ** 2).sum()
    return P * torch.sqrt(M * N / e)


@pytest.mark.parametrize("M,N", [(64, 64), (128, 96), (256, 256)])
def test_backward_against_autograd(pkg, M, N):
    dev = torch.device("cuda")
    P = _offset_probe(M, N, M // 3, 2 * N // 3, 5)
    W = _offset_probe(M, N, M // 2, N // 2, 6) * 0.3 + 0.1
    a = torch.from_numpy(P.astype(np.complex128)).to(dev).requires_grad_(True)
    (torch.conj(torch.from_numpy(W.astype(np.complex128)).to(dev)) * _ref_torch(a)).real.sum().backward()
    b = torch.from_numpy(P).to(dev).requires_grad_(True)
    out = pkg.probe_prep.center_and_normalize_probe(b)
    (torch.conj(torch.from_numpy(W).to(dev)) * out).real.sum().backward()
    ref = a.grad.cpu().numpy()
    assert np.abs(b.grad.cpu().numpy() - ref).max() <= 1e-5 * np.abs(ref).max()
    assert np.abs(out.detach().cpu().numpy() - _ref_torch(a.detach()).cpu().numpy()).max() <= \
        1e-6 * np.abs(out.detach().cpu().numpy()).max()


def test_validation(pkg):
    L = pkg.lib()
    dev = torch.device("cuda")
    P = torch.zeros(8, 8, dtype=torch.complex64, device=dev)
    st = torch.zeros(4, dtype=torch.float64, device=dev)
    assert L.ptycho_probe_center_normalize(P.data_ptr(), 8, 8, P.data_ptr(), st.data_ptr(), None) == 1
    assert L.ptycho_probe_center_normalize(P.data_ptr(), 2048, 8, P.data_ptr() + 0, st.data_ptr(), None) in (1, 2)


# ---- Haar sparsity (utils/loss.py:60-83) ---------------------------------------
def _haar_torch(img):
    a, b, c, d = img[0::2, 0::2], img[0::2, 1::2], img[1::2, 0::2], img[1::2, 1::2]
    return (a - b + c - d).abs().sum() + (a + b - c - d).abs().sum() + (a - b - c + d).abs().sum()


def test_haar_golden_and_oracle(pkg):
    dev = torch.device("cuda")
    g = golden("probe_haar.npz")
    img = g["haar/img"].astype(np.complex64)
    v = float(pkg.probe_prep.haar_sparsity(torch.from_numpy(img).to(dev)))
    assert abs(v - fm.haar_sparsity(img.astype(np.complex128))) <= 1e-6 * abs(v)
    assert abs(v - float(g["haar/value"])) <= 1e-5 * abs(v)  # golden is on the complex128 image
    big = (np.random.default_rng(3).standard_normal((1536, 1024)) * (1 + 1j)).astype(np.complex64)
    x = torch.from_numpy(big).to(dev)
    v1 = pkg.probe_prep.haar_sparsity(x)
    v2 = pkg.probe_prep.haar_sparsity(x)
    assert float(v1) == float(v2)  # fixed-order reduction
    assert abs(float(v1) - fm.haar_sparsity(big.astype(np.complex128))) <= 1e-6 * float(v1)


def test_haar_backward_against_autograd(pkg):
    dev = torch.device("cuda")
    img = (np.random.default_rng(4).standard_normal((64, 96)) + 1j * np.random.default_rng(5).standard_normal((64, 96)))
    img = img.astype(np.complex64)
    a = torch.from_numpy(img.astype(np.complex128)).to(dev).requires_grad_(True)
    (2.5 * _haar_torch(a.real) + 2.5 * _haar_torch(a.imag)).backward()
    b = torch.from_numpy(img).to(dev).requires_grad_(True)
    (2.5 * pkg.probe_prep.haar_sparsity(b)).backward()
    np.testing.assert_allclose(b.grad.cpu().numpy(), a.grad.cpu().numpy(), rtol=0, atol=1e-6)
