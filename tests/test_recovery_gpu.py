"""The training loop on the kernels: graph-captured and eager steps agree
bitwise; the INR trained by the hand-written kernels lowers the data residual."""
import importlib

import numpy as np
import pytest
import torch

from conftest import PKG_NAME, load_pkg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    pkg = load_pkg()
    rec = importlib.import_module(PKG_NAME + ".recovery")
    dev = torch.device("cuda")
    rng = np.random.default_rng(0)
    H, M, F = 200, 64, 30
    O = (np.exp(1j * rng.random((H, H)) * 0.5)).astype(np.complex64)
    yy, xx = np.mgrid[:M, :M] - M / 2
    P = ((np.hypot(yy, xx) < 20) * 1.0).astype(np.complex64)
    tlY = rng.integers(0, H - M + 1, F).astype(np.int32)
    tlX = rng.integers(0, H - M + 1, F).astype(np.int32)
    I = np.stack([np.abs(np.fft.fftshift(np.fft.fft2(P * O[y:y + M, x:x + M]))) ** 2 for y, x in zip(tlY, tlX)])
    stack = torch.from_numpy((I / I.max() * 1e3).astype(np.float32)).to(dev)
    tl = pkg.make_windows(tlY, tlX, dev)
    return pkg, rec, dev, stack, tl, H, M


def test_graph_and_eager_training_agree_bitwise(setup):
    pkg, rec, dev, stack, tl, H, M = setup
    res = []
    # eager; graphs captured at first use; graphs captured up front by prepare()
    # (30 frames in minibatches of 8: lengths 8 and 6)
    for use_graph, prep in ((False, False), (True, False), (True, True)):
        torch.manual_seed(0)
        model = rec.PixelGrid((H, H), (M, M)).to(dev)
        tr = rec.Trainer(model, stack, tl, "Poisson_likelihood_loss", 8, 1e-2, lr_decay_step=1, lr_decay_gamma=0.5,
                         seed=3, use_graph=use_graph)
        if prep:
            tr.prepare()
            assert sorted(tr._graphs) == [6, 8]
        for _ in range(3):
            tr.epoch()
        torch.cuda.synchronize()
        res.append([p.detach().clone() for p in model.parameters()])
    for other in res[1:]:
        for a, b in zip(res[0], other):
            assert torch.equal(a, b)


def test_inr_training_lowers_residual(setup):
    pkg, rec, dev, stack, tl, H, M = setup
    cfg = dict(model_type="inr", downsample_factor=2, n_levels=16, log2_hashmap_size=14, base_resolution=8,
               per_level_scale=1.3, first_omega_0=10.0, hidden_omega_0=1.0, trainable_omega0=True)
    model = rec.build_model(cfg, H, (M, M), None, dev)
    tr = rec.Trainer(model, stack, tl, "smooth_L1_loss", 8, 1e-3, seed=1)
    r0 = tr.residual()
    for _ in range(15):
        tr.epoch()
    r1 = tr.residual()
    assert np.isfinite(r1) and r1 < r0, (r0, r1)
