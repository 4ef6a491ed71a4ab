"""The Gaussian-splatting oracle on the CPU: its analytic backward against
torch autograd (float64) of the same per-pixel sum over the same tile
rectangles, for both parameterisations; preprocess bookkeeping (culling,
clamped scales, tile rectangles) against hand-computed cases."""
import numpy as np
import pytest
import torch

from oracle import gsplat as og


def _scene(rng, kind, N, H, W):
    xy = np.stack([rng.uniform(0, W - 1, N), rng.uniform(0, H - 1, N)], 1).astype(np.float32)
    p1 = rng.uniform(np.log(0.8), np.log(4.0), (N, 2)).astype(np.float32)
    p2 = (rng.uniform(-np.pi, np.pi, N) if kind == og.RS else rng.uniform(-1.5, 1.5, N)).astype(np.float32)
    w = rng.standard_normal((N, 2)).astype(np.float32)
    return xy, p1, p2, w


def _torch_render(kind, g, xy, p1, p2, w, H, W, R, ms):
    """float64 torch restatement with the oracle's rectangles held fixed."""
    out = torch.zeros(2, H, W, dtype=torch.float64)
    for i in range(xy.shape[0]):
        if g["radius"][i] <= 0:
            continue
        x0, y0, x1, y1 = (int(v) for v in g["rect"][i])
        px0, py0, px1, py1 = x0 * 16, y0 * 16, min(x1 * 16, W), min(y1 * 16, H)
        if kind == og.RS:
            s = torch.clamp(torch.exp(p1[i]), ms, R)
            ct, st = torch.cos(p2[i]), torch.sin(p2[i])
            a = ct * ct * s[0] ** 2 + st * st * s[1] ** 2
            b = ct * st * (s[0] ** 2 - s[1] ** 2)
            c = st * st * s[0] ** 2 + ct * ct * s[1] ** 2
        else:
            l = torch.clamp(torch.exp(p1[i]), ms, R)
            a, b, c = l[0] ** 2, l[0] * p2[i], p2[i] ** 2 + l[1] ** 2
        det = a * c - b * b
        cx, cy, cz = c / det, -b / det, a / det
        xs = torch.arange(px0, px1, dtype=torch.float64)
        ys = torch.arange(py0, py1, dtype=torch.float64)
        dx = xy[i, 0] - xs[None, :]
        dy = xy[i, 1] - ys[:, None]
        power = -0.5 * (cx * dx * dx + cz * dy * dy) - cy * dx * dy
        G = torch.exp(torch.clamp(power, max=0.0))
        keep = ((power <= 0) & (G >= 1e-7)).double()
        out[0, py0:py1, px0:px1] = out[0, py0:py1, px0:px1] + w[i, 0] * G * keep
        out[1, py0:py1, px0:px1] = out[1, py0:py1, px0:px1] + w[i, 1] * G * keep
    return out


@pytest.mark.parametrize("kind", [og.RS, og.CHOLESKY])
def test_oracle_backward_matches_autograd(kind):
    rng = np.random.default_rng(11 + kind)
    H, W, N, R, ms = 40, 52, 18, 16, 0.5
    xy, p1, p2, w = _scene(rng, kind, N, H, W)
    gout = rng.standard_normal((2, H, W))
    out, g = og.render(kind, xy, p1, p2, w, H, W, R, ms)
    t = [torch.tensor(v.astype(np.float64), requires_grad=True) for v in (xy, p1, p2, w)]
    ref = _torch_render(kind, g, *t, H, W, R, ms)
    assert np.abs(ref.detach().numpy() - out).max() <= 1e-5 * np.abs(out).max()
    (ref * torch.from_numpy(gout)).sum().backward()
    got = og.backward(kind, xy, p1, p2, w, H, W, R, ms, gout)
    for a, b in zip(got, t):
        b = b.grad.numpy().reshape(a.shape)
        assert np.abs(a - b).max() <= 1e-5 * max(np.abs(b).max(), 1e-12), (kind, np.abs(a - b).max())


def test_preprocess_rectangles_and_culling():
    H, W = 64, 80
    xy = np.array([[5.0, 5.0], [79.0, 63.0], [-10.0, 200.0], [40.0, 30.0]], np.float32)
    p1 = np.log(np.array([[1.0, 1.0], [2.0, 2.0], [1.0, 1.0], [100.0, 0.01]], np.float32))
    p2 = np.zeros(4, np.float32)
    g = og.preprocess(og.RS, xy, p1, p2, H, W, 16, 0.5)
    # isotropic sigma 1: lambda = 1 + sqrt(0.1) -> radius ceil(3 sqrt(1.316)) = 4
    assert g["radius"][0] == 4 and tuple(g["rect"][0]) == (0, 0, 1, 1)
    assert tuple(g["mean"][2]) == (0.0, 63.0)  # clamped into the canvas
    assert tuple(g["rect"][1]) == (4, 3, 5, 4)  # tile grid 5 x 4, clamped ends
    # scales clamped to [0.5, 16]: lambda_max = 256 exactly -> radius 3 * 16 = 48
    assert g["radius"][3] == 48
    gc = og.preprocess(og.CHOLESKY, xy[:1], np.full((1, 2), -200.0, np.float32), np.zeros(1, np.float32),
                       H, W, 16, 0.0)
    assert gc["radius"][0] == 0  # exp(-200) = 0: det = 0, culled
