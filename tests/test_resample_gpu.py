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


@pytest.mark.parametrize("h,w,s", [(64, 64, 2), (64, 256, 2), (128, 64, 4), (256, 256, 1),
                                   (512, 512, 2), (1024, 512, 2), (2048, 256, 2), (256, 2048, 2)])
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


def test_matches_torch_fft_formula_and_autograd(pkg):
    """Same values and gradients as the reference formula run through torch.fft."""
    dev = torch.device("cuda")
    x = torch.from_numpy(_rand((128, 128), 3)).to(dev)
    a = x.clone().requires_grad_(True)
    b = x.clone().requires_grad_(True)
    ya = pkg.resample.fourier_upsample(a, 2)
    Xf = torch.fft.fftshift(torch.fft.fft2(b), dim=(-2, -1))
    yb = torch.fft.ifft2(torch.fft.ifftshift(torch.nn.functional.pad(Xf, (64, 64, 64, 64)), dim=(-2, -1))) * 4
    assert float((ya - yb).abs().max() / yb.abs().max()) <= TOL
    w = torch.from_numpy(_rand((256, 256), 4)).to(dev)
    (ya * w.conj()).real.sum().backward()
    (yb * w.conj()).real.sum().backward()
    assert float((a.grad - b.grad).abs().max() / b.grad.abs().max()) <= TOL


def test_deterministic(pkg):
    dev = torch.device("cuda")
    x = torch.from_numpy(_rand((512, 512), 9)).to(dev)
    y1 = pkg.resample.fourier_upsample(x, 2)
    y2 = pkg.resample.fourier_upsample(x, 2)
    assert torch.equal(y1, y2)


def test_model_uses_kernel_path(pkg):
    """ComplexINRModel2D.fourier_upsample on a supported shape equals the oracle."""
    dev = torch.device("cuda")
    m = pkg.ComplexINRModel2D(256, 256, 2, probe_width=64, probe_height=64).to(dev)
    x = torch.from_numpy(_rand((128, 128), 11)).to(dev)
    y = m.fourier_upsample(x[None, None], 2)[0, 0]
    ref = fourier_upsample(x.cpu().numpy().astype(np.complex128), 2)
    assert rel_max(y.cpu().numpy(), ref) <= TOL
    # an unsupported shape keeps the torch.fft formula
    z = torch.from_numpy(_rand((96, 96), 12)).to(dev)
    yz = m.fourier_upsample(z[None, None], 2)[0, 0]
    assert rel_max(yz.cpu().numpy(), fourier_upsample(z.cpu().numpy().astype(np.complex128), 2)) <= 1e-5


def test_unsupported_sizes_raise(pkg):
    dev = torch.device("cuda")
    with pytest.raises(ValueError):
        pkg.resample.fourier_upsample(torch.zeros(96, 96, dtype=torch.complex64, device=dev), 2)
    with pytest.raises(ValueError):
        pkg.resample.fourier_upsample(torch.zeros(64, 64, dtype=torch.complex64, device=dev), 3)
