"""End to end through the Recovery.py mirror: YAML config + .mat bundle in,
result.mat and trained_models.pth out (Recovery.py:44-383 contract).

A small seeded dataset is written as a MATLAB v5 bundle (xlocation /
ylocation in metres, probe, imRaw as [M, N, F] like the reference's files);
``recovery.main`` runs a few epochs of the pixel-grid and of the INR model.
Checks: the outputs exist with the reference's names and shapes, are finite,
the saved probe is centred/normalised (sum |P|^2 = M*N), and the pixel-grid
data residual drops below its starting value.
"""
import importlib

import numpy as np
import pytest
import torch

from conftest import PKG_NAME
from oracle import forward_model as fm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rec():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return importlib.import_module(PKG_NAME + ".recovery")


def _dataset(tmp_path, M=64, n=6, step=16, seed=3):
    from scipy.io import savemat
    rng = np.random.default_rng(seed)
    wavelength, camera_length, dx = 1e-9, 1.0, 1e-7
    pitch = wavelength * camera_length / (M * dx)
    iy, ix = np.mgrid[:n, :n]
    # positions in metres, off the .5 rounding ties
    ypix = iy.ravel() * step + rng.integers(-2, 3, n * n) + 0.3
    xpix = ix.ravel() * step + rng.integers(-2, 3, n * n) + 0.3
    yloc, xloc = ypix * dx, xpix * dx
    tlX, tlY, _, _, _, canvas = fm.scan_positions_to_pixels(xloc, yloc, (M, M), wavelength, camera_length, pitch)
    u = rng.random((canvas, canvas))
    O = (0.7 + 0.3 * u) * np.exp(1j * (u - 0.5))
    yy, xx = np.mgrid[:M, :M] - M / 2
    P = (np.hypot(yy, xx) < 0.3 * M) * np.exp(1j * 0.002 * (yy ** 2 + xx ** 2))
    I = fm.forward_intensity(O, P, tlY, tlX)
    I = I / I.max() * 1e4
    stack = rng.poisson(I).astype(np.float64)
    savemat(tmp_path / "bundle.mat", {"xlocation": xloc[None, :], "ylocation": yloc[None, :],
                                      "probe": P.astype(np.complex128), "imRaw": np.moveaxis(stack, 0, -1)})
    return dict(wavelength=wavelength, camera_length=camera_length, pitch=pitch, canvas=canvas, M=M)


def _config(tmp_path, d, model_type, iters, out):
    text = (f"data:\n  data_dir: {tmp_path}\n  bundle_file: bundle.mat\n"
            f"physics:\n  wavelength: {d['wavelength']}\n  camera_length: {d['camera_length']}\n"
            f"  camera_pixel_pitch: {d['pitch']}\n"
            f"model:\n  model_type: {model_type}\n  init_type: initProbe\n  use_residual: true\n"
            f"  log2_hashmap_size: 14\n  downsample_factor: 2\n"
            f"training:\n  iters: {iters}\n  lr: 0.01\n  batch_size: 8\n  loss_type: Poisson_likelihood_loss\n"
            f"  vis_interval: 1\noutput:\n  result_dir: {out}\n")
    p = tmp_path / f"{model_type}.yaml"
    p.write_text(text)
    return str(p)


@pytest.mark.parametrize("model_type,iters", [("pixel_grid", 4), ("inr", 2)])
def test_recovery_main_end_to_end(rec, tmp_path, model_type, iters):
    from scipy.io import loadmat
    d = _dataset(tmp_path)
    out = tmp_path / f"out_{model_type}"
    rec.main(["--config", _config(tmp_path, d, model_type, iters, out)])
    r = loadmat(out / "result.mat")
    obj, probe = r["object_complex"], r["probe_complex"]
    assert obj.shape == (d["canvas"], d["canvas"]) and probe.shape == (d["M"], d["M"])
    assert np.all(np.isfinite(obj)) and np.all(np.isfinite(probe))
    assert abs((np.abs(probe) ** 2).sum() - d["M"] ** 2) <= 1e-3 * d["M"] ** 2
    params = torch.load(out / "trained_models.pth", weights_only=False)
    assert isinstance(params, list) and len(params) >= 2 and all(torch.is_tensor(p) for p in params)


def test_pixel_grid_residual_drops(rec, tmp_path):
    """The driver's training loop on the same data: the FP64 residual falls."""
    d = _dataset(tmp_path)
    cfg = rec.load_config(_config(tmp_path, d, "pixel_grid", 1, tmp_path / "o"))
    data = rec.load_ptychography_data(cfg["data_dir"], cfg.get("bundle_file"))
    dev = torch.device("cuda")
    pkg = importlib.import_module(PKG_NAME)
    tlX, tlY, _, _, _, canvas = pkg.scan_positions_to_pixels(
        data["xlocation"], data["ylocation"], data["probe"].shape, cfg["wavelength"], cfg["camera_length"],
        cfg["camera_pixel_pitch"])
    stack = torch.from_numpy(np.ascontiguousarray(np.moveaxis(data["imRaw"], -1, 0).astype(np.float32))).to(dev)
    P0 = torch.from_numpy(data["probe"].astype(np.complex64)).to(dev)
    model = rec.PixelGrid((canvas, canvas), tuple(data["probe"].shape), probe_init=P0).to(dev)
    tr = rec.Trainer(model, stack, pkg.make_windows(tlY, tlX, dev), "Poisson_likelihood_loss", 8, 1e-2)
    r0 = tr.residual()
    for _ in range(10):
        tr.epoch()
    assert tr.residual() < 0.5 * r0


@pytest.mark.parametrize("model_type,iters", [("pixel_grid", 3), ("inr", 2)])
def test_recovery_main_96_probe_without_torch_fft(rec, tmp_path, monkeypatch, model_type, iters):
    """A 96 x 96 probe (the general forward / adjoint path) on the multiple-of-6
    canvas scan_positions_to_pixels builds (odd INR object grid, mixed-radix
    upsampling): the whole run reaches no torch.fft transform."""
    from scipy.io import loadmat
    d = _dataset(tmp_path, M=96, n=5, step=21)
    assert d["canvas"] == 186  # a multiple of 6 whose half (the INR object grid, 93) is odd

    def boom(*a, **k):
        raise AssertionError("torch.fft reached on the product path")
    for name in ("fft", "ifft", "fft2", "ifft2", "fftn", "ifftn"):
        monkeypatch.setattr(torch.fft, name, boom)
    out = tmp_path / f"out96_{model_type}"
    rec.main(["--config", _config(tmp_path, d, model_type, iters, out)])
    r = loadmat(out / "result.mat")
    obj, probe = r["object_complex"], r["probe_complex"]
    assert obj.shape == (d["canvas"], d["canvas"]) and probe.shape == (96, 96)
    assert np.all(np.isfinite(obj)) and np.all(np.isfinite(probe))
