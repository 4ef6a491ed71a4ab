"""Parity of the Fourier-upsampling kernels (models/complex_inr.py:252-271)
with the FP64 oracle: the forward map, its adjoint (the autograd backward)
and the INR model's use of it.

Tolerance (FP32 FFTs of length <= 4096 against FP64):
  max|y - y_ref| / max|y_ref| <= 2e-6, both directions.
"""
import numpy as np
import pytest
import torch

from conftest import load_pkg
from oracle.inr import fourier_upsample, fourier_upsample_adjoint

pytestmark = pytest.mark.gpu
TOL = 2e-6


@pytest.fixture(scope="module")
def pkg():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return load_pkg()


def rel_max(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def _rand(shape, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


# power-of-two lines (compile-time kernels) and every other length the
# reference's geometry gives (run-time mixed-radix plans): canvases are
# multiples of 6, so object grids with downsample_factor 2 are multiples of 3
# (249 -> 498, 498 -> 996, 1536 -> 3072), odd lengths (the reference's
# fftshift / pad / ifftshift then moves the band by one bin), large prime
# factors (83, 97), non-square grids, s = 1 and s = 3, the 8192 maximum
@pytest.mark.parametrize("h,w,s", [(64, 64, 2), (64, 256, 2), (128, 64, 4), (256, 256, 1),
                                   (512, 512, 2), (1024, 512, 2), (2048, 256, 2), (256, 2048, 2),
                                   (249, 249, 2), (498, 498, 2), (500, 500, 2), (1536, 1536, 2),
                                   (333, 333, 3), (250, 125, 2), (83, 97, 2), (96, 96, 2), (91, 1001, 1),
                                   (2048, 60, 4), (15, 6, 3)])
def test_forward_and_adjoint_against_oracle(pkg, h, w, s):
    dev = torch.device("cuda")
    x = _rand((h, w), h + w + s)
    xt = torch.from_numpy(x).to(dev).requires_grad_(True)
    y = pkg.resample.fourier_upsample(xt, s)
    ref = fourier_upsample(x.astype(np.complex128), s)
    assert y.shape == (h * s, w * s)
    assert rel_max(y.detach().cpu().numpy(), ref) <= TOL, rel_max(y.detach().cpu().numpy(), ref)
    g = _rand((h * s, w * s), 7)
    y.backward(torch.from_numpy(g).to(dev))
    ref_g = fourier_upsample_adjoint(g.astype(np.complex128), s, (h, w))
    assert rel_max(xt.grad.cpu().numpy(), ref_g) <= TOL, rel_max(xt.grad.cpu().numpy(), ref_g)


def _reference_formula(x, s):
    """models/complex_inr.py:252-271 verbatim in torch (checker only)."""
    H, W = x.shape[-2:]
    X = torch.fft.fftshift(torch.fft.fft2(x, dim=(-2, -1)), dim=(-2, -1))
    nH, nW = int(H * s), int(W * s)
    ph, pw = (nH - H) // 2, (nW - W) // 2
    X = torch.nn.functional.pad(X, (pw, nW - W - pw, ph, nH - H - ph), mode="constant", value=0)
    return torch.fft.ifft2(torch.fft.ifftshift(X, dim=(-2, -1)), dim=(-2, -1)) * (s ** 2)


@pytest.mark.parametrize("n,s", [(128, 2), (498, 2), (249, 2), (500, 2), (1536, 2)])
def test_matches_torch_fft_formula_and_autograd(pkg, n, s):
    """Same values and gradients as the reference formula run through torch.fft
    (complex64, autograd), at the canvases Recovery.py builds."""
    dev = torch.device("cuda")
    x = torch.from_numpy(_rand((n, n), 3 + n)).to(dev)
    a = x.clone().requires_grad_(True)
    b = x.clone().requires_grad_(True)
    ya = pkg.resample.fourier_upsample(a, s)
    yb = _reference_formula(b, s)
    assert float((ya - yb).abs().max() / yb.abs().max()) <= TOL
    w = torch.from_numpy(_rand((n * s, n * s), 4)).to(dev)
    (ya * w.conj()).real.sum().backward()
    (yb * w.conj()).real.sum().backward()
    assert float((a.grad - b.grad).abs().max() / b.grad.abs().max()) <= TOL


def test_deterministic(pkg):
    dev = torch.device("cuda")
    for n in (512, 498):
        x = torch.from_numpy(_rand((n, n), 9)).to(dev)
        y1 = pkg.resample.fourier_upsample(x, 2)
        y2 = pkg.resample.fourier_upsample(x, 2)
        assert torch.equal(y1, y2)


@pytest.fixture
def no_torch_fft(monkeypatch):
    """Make every torch.fft transform raise: the product path must not use it."""
    def boom(*a, **k):
        raise AssertionError("torch.fft reached on the product path")
    for name in ("fft", "ifft", "fft2", "ifft2", "fftn", "ifftn"):
        monkeypatch.setattr(torch.fft, name, boom)


@pytest.mark.parametrize("canvas,probe,ds", [(256, 64, 2), (498, 64, 2), (996, 128, 2), (498, 96, 3)])
def test_model_uses_kernel_path(pkg, no_torch_fft, canvas, probe, ds):
    """ComplexINRModel2D.fourier_upsample equals the oracle on power-of-two and
    multiple-of-6 canvases, and the model's forward + backward never calls
    torch.fft."""
    dev = torch.device("cuda")
    m = pkg.ComplexINRModel2D(canvas, canvas, ds, probe_width=probe, probe_height=probe).to(dev)
    n = canvas // ds
    x = torch.from_numpy(_rand((n, n), 11)).to(dev)
    y = m.fourier_upsample(x[None, None], ds)[0, 0]
    ref = fourier_upsample(x.cpu().numpy().astype(np.complex128), ds)
    assert rel_max(y.cpu().numpy(), ref) <= TOL
    obj, prb = m()
    assert obj.shape == (canvas, canvas) and prb.shape == (probe, probe)
    (obj.abs().sum() + prb.abs().sum()).backward()
    assert any(p.grad is not None for p in m.parameters() if p.requires_grad)


def test_batched_slices(pkg):
    """[B, C, H, W] inputs run slice by slice on the kernels."""
    dev = torch.device("cuda")
    m = pkg.ComplexINRModel2D(96, 96, 2, probe_width=64, probe_height=64).to(dev)
    x = torch.from_numpy(_rand((2 * 3 * 48, 48), 13)).to(dev).reshape(2, 3, 48, 48)
    y = m.fourier_upsample(x, 2)
    assert y.shape == (2, 3, 96, 96)
    for b in range(2):
        for c in range(3):
            ref = fourier_upsample(x[b, c].cpu().numpy().astype(np.complex128), 2)
            assert rel_max(y[b, c].cpu().numpy(), ref) <= TOL


def test_unsupported_sizes_raise(pkg):
    dev = torch.device("cuda")
    with pytest.raises(ValueError):  # past the 8192-point line maximum
        pkg.resample.fourier_upsample(torch.zeros(4097, 64, dtype=torch.complex64, device=dev), 2)
    with pytest.raises(ValueError):  # not a whole scale
        pkg.resample.fourier_upsample(torch.zeros(64, 64, dtype=torch.complex64, device=dev), 1.5)
    m = pkg.ComplexINRModel2D(96, 96, 2, probe_width=64, probe_height=64).to(dev)
    with pytest.raises(ValueError):
        m.fourier_upsample(torch.zeros(1, 1, 48, 48, dtype=torch.complex64), 2)  # CPU tensor
