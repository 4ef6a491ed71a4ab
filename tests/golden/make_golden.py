"""Generate the golden fixtures in this folder by running the reference itself.

Run in a container that holds the reference tree (default
``/root/reference``; override with ``PTYCHO_REFERENCE``)::

    python tests/golden/make_golden.py

Everything is computed by the reference's own code, imported from its tree:

* forward model -- ``utils.optics.forward_imaging_model`` (utils/optics.py:102-112)
  per frame, in complex128;
* losses -- ``utils.loss.calculate_loss`` with ``smoothL1Loss`` / ``GDLoss`` /
  ``PoissonLoss`` (utils/loss.py:9-45), the same formulas as the inline
  losses of Recovery.py:294-305 (``Recovery.py`` itself is a module-level
  script and cannot be imported); per-frame losses are summed as at
  Recovery.py:307;
* adjoint -- torch autograd of the above (what Recovery.py:316 runs);
* scan indices -- ``utils.optics.scan_positions_to_pixels`` (:68-99), with
  positions that hit exact .5 ties of the rounding;
* probe centring -- ``utils.optics.center_probe`` (:151-172);
* Haar sparsity -- ``utils.loss.haar_wavelet_sparsity_loss`` (:60-83);
* ComplexMLP -- ``models/complex_inr.py:6-82`` loaded with a stub
  ``tinycudann`` module (the MLP itself is pure torch).

Inputs are seeded; object/probe values are rounded to complex64 first so the
FP32 CUDA path and the FP64 checker see identical inputs.
"""
from __future__ import annotations

import importlib.util
import os
import sys
import types

import numpy as np
import torch

REF = os.environ.get("PTYCHO_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
LOSSES = {"smooth_L1_loss": "smoothL1Loss", "FD_loss": "GDLoss",
          "Poisson_likelihood_loss": "PoissonLoss"}


def _import_reference():
    sys.path.insert(0, REF)
    from utils import optics, loss  # noqa: E402
    return optics, loss


def _smooth_field(rng, shape, sigma):
    from scipy.ndimage import gaussian_filter
    u = gaussian_filter(rng.random(shape), sigma, mode="wrap")
    return (u - u.min()) / (u.max() - u.min())


def _make_case(rng, H, M, B, peak):
    amp = 0.6 + 0.4 * _smooth_field(rng, (H, H), 2.0)
    ph = np.pi * (_smooth_field(rng, (H, H), 2.0) - 0.5)
    O = (amp * np.exp(1j * ph)).astype(np.complex64).astype(np.complex128)
    yy, xx = np.mgrid[:M, :M] - M / 2 + 0.5
    r = np.hypot(yy, xx)
    P = ((r < 0.35 * M) * np.exp(1j * 0.002 * r * r)
         + 0.05 * (rng.standard_normal((M, M)) + 1j * rng.standard_normal((M, M))))
    P = P.astype(np.complex64).astype(np.complex128)
    tlY = rng.integers(0, H - M + 1, size=B)
    tlX = rng.integers(0, H - M + 1, size=B)
    # measurements from a perturbed "true" object so that the losses and
    # gradients are non-trivial; Poisson counts, stored FP32
    Ot = O * np.exp(0.3j * _smooth_field(rng, (H, H), 3.0))
    Ipure = np.stack([np.abs(np.fft.fftshift(np.fft.fft2(P * Ot[y:y + M, x:x + M]))) ** 2
                      for y, x in zip(tlY, tlX)])
    Imeas = rng.poisson(Ipure / Ipure.max() * peak).astype(np.float32)
    # model object is a scaled copy so smooth_L1 sees both |d|<1 and |d|>1
    scale = np.sqrt(peak / Ipure.max())
    O = (O * scale).astype(np.complex64).astype(np.complex128)
    return O, P, tlY.astype(np.int32), tlX.astype(np.int32), Imeas


def _ref_fwd_adj(optics, lossmod, O, P, tlY, tlX, Imeas, loss_type):
    Ot = torch.tensor(O, dtype=torch.complex128, requires_grad=True)
    Pt = torch.tensor(P, dtype=torch.complex128, requires_grad=True)
    M, N = P.shape
    total = 0.0
    per, Is = [], []
    for b in range(len(tlY)):
        y, x = int(tlY[b]), int(tlX[b])
        I = optics.forward_imaging_model(Ot, Pt, y, x, y + M, x + N)
        cap = torch.tensor(Imeas[b], dtype=torch.float64)
        lb = lossmod.calculate_loss(cap, I, loss_type=LOSSES[loss_type])
        per.append(float(lb.detach()))
        Is.append(I.detach().numpy())
        total = total + lb
    total.backward()
    return {"I": np.stack(Is), "loss": np.array(per), "dO": Ot.grad.numpy(),
            "dP": Pt.grad.numpy()}


def make_fwd_adj(optics, lossmod):
    for name, (H, M, B, peak, seed) in {"m16": (24, 16, 4, 60.0, 11),
                                        "m64": (72, 64, 3, 2000.0, 12)}.items():
        rng = np.random.default_rng(seed)
        O, P, tlY, tlX, Imeas = _make_case(rng, H, M, B, peak)
        out = {"O": O, "P": P, "tlY": tlY, "tlX": tlX, "Imeas": Imeas}
        for lt in LOSSES:
            r = _ref_fwd_adj(optics, lossmod, O, P, tlY, tlX, Imeas, lt)
            if lt == "Poisson_likelihood_loss":
                out["I"] = r["I"]
            out[f"{lt}/loss"] = r["loss"]
            out[f"{lt}/dO"] = r["dO"]
            out[f"{lt}/dP"] = r["dP"]
        np.savez_compressed(os.path.join(HERE, f"fwd_adj_{name}.npz"), **out)


def make_scan(optics):
    cases = {}
    # pitch chosen so dx is exact (0.5 m / px) and positions land on .5 ties
    lam, L, pitch = 1.0, 64.0, 1.0
    for k, (M, n) in enumerate([(128, 40), (64, 10), (256, 12)]):
        rng = np.random.default_rng(100 + k)
        dx = lam * L / (M * pitch)
        q = rng.integers(0, 8 * n * 16, size=n * n)
        ys = (q // (n * 16)) * dx * 2.0 + rng.integers(0, 4, size=n * n) * dx * 0.25
        xs = (q % (n * 16)) * dx * 0.5 + rng.integers(0, 4, size=n * n) * dx * 0.25
        xs = xs + 3.25
        tlX, tlY, brX, brY, dxo, canvas = optics.scan_positions_to_pixels(
            xs, ys, (M, M), lam, L, pitch)
        cases[f"c{k}/x"] = xs
        cases[f"c{k}/y"] = ys
        cases[f"c{k}/M"] = np.array(M)
        cases[f"c{k}/phys"] = np.array([lam, L, pitch])
        cases[f"c{k}/tl"] = np.stack([tlY, tlX]).astype(np.int64)
        cases[f"c{k}/br"] = np.stack([brY, brX]).astype(np.int64)
        cases[f"c{k}/dx"] = np.asarray(dxo)
        cases[f"c{k}/canvas"] = np.array(canvas)
    # a physical case (the simulation.yaml optics) with a jittered raster
    rng = np.random.default_rng(7)
    lam, L, pitch, M = 2.4e-9, 0.5, 2.7e-5, 128
    dx = lam * L / (M * pitch)
    gy, gx = np.mgrid[:20, :20]
    ys = (gy.ravel() * 24 + rng.uniform(-2, 2, 400)) * dx + 1e-6
    xs = (gx.ravel() * 24 + rng.uniform(-2, 2, 400)) * dx - 3e-6
    tlX, tlY, brX, brY, dxo, canvas = optics.scan_positions_to_pixels(xs, ys, (M, M), lam, L, pitch)
    cases.update({"c3/x": xs, "c3/y": ys, "c3/M": np.array(M), "c3/phys": np.array([lam, L, pitch]),
                  "c3/tl": np.stack([tlY, tlX]).astype(np.int64),
                  "c3/br": np.stack([brY, brX]).astype(np.int64),
                  "c3/dx": np.asarray(dxo), "c3/canvas": np.array(canvas)})
    np.savez_compressed(os.path.join(HERE, "scan_indices.npz"), **cases)


def make_probe_and_haar(optics, lossmod):
    rng = np.random.default_rng(21)
    out = {}
    for k, (M, off) in enumerate([(64, (5, -7)), (128, (-13, 9)), (32, (0, 0))]):
        yy, xx = np.mgrid[:M, :M] - M / 2
        r = np.hypot(yy - off[0], xx - off[1])
        P = ((r < 0.3 * M) * np.exp(1j * 0.01 * r * r)
             + 0.01 * rng.standard_normal((M, M))).astype(np.complex64)
        Pt = torch.tensor(P)
        Pc = optics.center_probe(Pt).numpy()
        out[f"p{k}/P"] = P
        out[f"p{k}/centered"] = Pc
    img = (rng.standard_normal((48, 40)) + 1j * rng.standard_normal((48, 40))).astype(np.complex128)
    out["haar/img"] = img
    out["haar/value"] = np.array(float(lossmod.haar_wavelet_sparsity_loss(torch.tensor(img))))
    np.savez_compressed(os.path.join(HERE, "probe_haar.npz"), **out)


def make_complex_mlp():
    stub = types.ModuleType("tinycudann")
    stub.Encoding = object
    sys.modules.setdefault("tinycudann", stub)
    spec = importlib.util.spec_from_file_location(
        "ref_complex_inr", os.path.join(REF, "models", "complex_inr.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    torch.manual_seed(5)
    out = {}
    for k, (hidden, layers, w1, wh) in enumerate([(64, 2, 10.0, 1.0), (32, 1, 3.0, 2.0)]):
        mlp = mod.ComplexMLP(32, hidden, layers, 1, first_omega_0=w1, hidden_omega_0=wh,
                             trainable_omega0=True)
        for p in mlp.parameters():
            p.data = p.data.to(torch.complex128 if p.is_complex() else torch.float64)
        x = torch.rand(50, 32, dtype=torch.float64) * 2e-4 - 1e-4 + 0.05 * torch.randn(50, 32,
                                                                                     dtype=torch.float64)
        y = mlp.net(x)
        tgt = torch.randn(50, 1, dtype=torch.complex128)
        loss = (y - tgt).abs().pow(2).sum()
        xr = x.clone().requires_grad_(True)
        y2 = mlp.net(xr)
        loss2 = (y2 - tgt).abs().pow(2).sum()
        loss2.backward()
        out[f"m{k}/x"] = x.numpy()
        out[f"m{k}/target"] = tgt.numpy()
        out[f"m{k}/y"] = y.detach().numpy()
        out[f"m{k}/loss"] = np.array(float(loss))
        out[f"m{k}/dx"] = xr.grad.numpy()
        out[f"m{k}/cfg"] = np.array([hidden, layers, w1, wh])
        for name, p in mlp.named_parameters():
            out[f"m{k}/param/{name}"] = p.detach().numpy()
            out[f"m{k}/grad/{name}"] = p.grad.numpy()
    np.savez_compressed(os.path.join(HERE, "complex_mlp.npz"), **out)


def main():
    optics, lossmod = _import_reference()
    torch.set_default_dtype(torch.float64)
    make_fwd_adj(optics, lossmod)
    make_scan(optics)
    make_probe_and_haar(optics, lossmod)
    torch.set_default_dtype(torch.float32)
    make_complex_mlp()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
