"""TEST / BASELINE ONLY -- CPU restatement of the reference's 2-D complex
Gaussian-splatting rasteriser (gscp/csrc/gscp_rasterizer), the checker for
``ptycho_gs_forward`` / ``ptycho_gs_backward``.  Never imported by the product.

Semantics restated (file:line in the reference):
- preprocess, RS (forward.cu:18-94): mean = clamp(xy, 0, [W-1, H-1]);
  s = clamp(exp(scaling), min_scale, max_patch_radius); Sigma = R diag(s^2) R^T
  with [[a, b], [b, c]], a = cos^2 sx2 + sin^2 sy2, b = cos sin (sx2 - sy2),
  c = sin^2 sx2 + cos^2 sy2; culled if det = ac - b^2 <= 0; conic =
  (c, -b, a) / det; radius = ceil(3 sqrt(mid + sqrt(max(0.1, mid^2 - det)))),
  mid = (a + c) / 2 (the circular bound, USE_SNUGBOX = 0, config.h:17-19);
- preprocess, Cholesky (forward.cu:99-170): l11, l22 = clamp(exp(log_L_diag)),
  l21 = L_offdiag; a = l11^2, b = l11 l21, c = l21^2 + l22^2, det = a l22^2;
- tile rectangle (auxiliary.h:17-30): 16 x 16 tiles, x0 = clamp(int((px - r) / 16)),
  x1 = clamp(int((px + r + 15) / 16)) with C truncation, to [0, tiles];
- render (forward.cu:175-250): a pixel of a tile sums, over the Gaussians whose
  rectangle covers the tile in ascending index order (the stable tile-key sort of
  rasterizer_impl.cu:45-79,253-262), power = -0.5 (cx dx^2 + cz dy^2) - cy dx dy
  with d = mean - pixel; skipped if power > 0 or G = exp(power) < 1e-7;
  out[0] += w_re G, out[1] += w_im G;
- backward (backward.cu:21-275): the same per-pixel terms give dL/dw, dL/dmean,
  dL/dconic; then dL/d(a, b, c) with det2_inv = 1 / (det^2 + 1e-7), the chain
  rule into (scaling, rotation) or (log_L_diag, L_offdiag), zero where the
  activated scale sits outside [min_scale, max_patch_radius]; dL/dxy passes
  dL/dmean through unchanged.

The preprocess runs in float32 one operation at a time, the rounding the
kernel's ``__f*_rn`` sequence reproduces.  cos, sin and exp are correctly
rounded here and within 2 ulp on the device, so a radius can differ by one
where 3 sqrt(lambda_max) lies within a few ulp of an integer (``r3`` is
returned so a test can tell those cases apart); elsewhere radii and tile
rectangles agree bit for bit.  Render and backward run in
float64 on those float32 means and conics.
"""
from __future__ import annotations

import numpy as np

TILE = 16
RS, CHOLESKY = 0, 1

f32 = np.float32


def preprocess(kind, xy, p1, p2, H, W, max_patch_radius, min_scale):
    """-> dict(mean [N,2] f32, conic [N,3] f32, radius [N] int, rect [N,4]
    (x0, y0, x1, y1) tiles, abc [N,3] f32, det [N] f32)."""
    xy = np.asarray(xy, f32).reshape(-1, 2)
    N = xy.shape[0]
    p1 = np.asarray(p1, f32).reshape(N, 2)
    p2 = np.asarray(p2, f32).reshape(N)
    mx = np.minimum(f32(W - 1), np.maximum(f32(0), xy[:, 0]))
    my = np.minimum(f32(H - 1), np.maximum(f32(0), xy[:, 1]))
    mxs = f32(max_patch_radius)
    mns = f32(min_scale)
    if kind == RS:
        sx = np.minimum(mxs, np.maximum(mns, np.exp(p1[:, 0]).astype(f32)))
        sy = np.minimum(mxs, np.maximum(mns, np.exp(p1[:, 1]).astype(f32)))
        sx2, sy2 = sx * sx, sy * sy
        ct = np.cos(p2.astype(np.float64)).astype(f32)
        st = np.sin(p2.astype(np.float64)).astype(f32)
        a = ct * ct * sx2 + st * st * sy2
        b = ct * st * (sx2 - sy2)
        c = st * st * sx2 + ct * ct * sy2
        det = a * c - b * b
    else:
        l11 = np.minimum(mxs, np.maximum(mns, np.exp(p1[:, 0]).astype(f32)))
        l22 = np.minimum(mxs, np.maximum(mns, np.exp(p1[:, 1]).astype(f32)))
        l21 = p2
        a = l11 * l11
        b = l11 * l21
        c = l21 * l21 + l22 * l22
        det = a * l22 * l22
    ok = det > 0
    with np.errstate(divide="ignore", invalid="ignore"):
        dinv = np.where(ok, f32(1) / np.where(ok, det, f32(1)), f32(0)).astype(f32)
    conic = np.stack([c * dinv, -b * dinv, a * dinv], 1).astype(f32)
    mid = f32(0.5) * (a + c)
    lam = mid + np.sqrt(np.maximum(f32(0.1), mid * mid - det))
    r3 = f32(3) * np.sqrt(lam)
    radius = np.ceil(r3).astype(np.int64)
    radius = np.where(ok, radius, 0)
    tx, ty = (W + TILE - 1) // TILE, (H + TILE - 1) // TILE
    r = radius.astype(f32)
    x0 = np.clip(np.trunc((mx - r) / f32(TILE)).astype(np.int64), 0, tx)
    y0 = np.clip(np.trunc((my - r) / f32(TILE)).astype(np.int64), 0, ty)
    x1 = np.clip(np.trunc((mx + r + f32(TILE - 1)) / f32(TILE)).astype(np.int64), 0, tx)
    y1 = np.clip(np.trunc((my + r + f32(TILE - 1)) / f32(TILE)).astype(np.int64), 0, ty)
    radius = np.where(radius > 0, radius, 0)
    rect = np.stack([x0, y0, x1, y1], 1)
    rect[radius <= 0] = 0
    return dict(mean=np.stack([mx, my], 1), conic=conic, radius=radius, rect=rect,
                abc=np.stack([a, b, c], 1), det=det, r3=np.where(ok, r3, f32(0)))


def _terms(g, i, H, W):
    """Pixel box of Gaussian i's tile rectangle and its float64 G (0 where skipped)."""
    x0, y0, x1, y1 = g["rect"][i]
    px0, py0 = x0 * TILE, y0 * TILE
    px1, py1 = min(x1 * TILE, W), min(y1 * TILE, H)
    if px1 <= px0 or py1 <= py0 or g["radius"][i] <= 0:
        return None
    xs = np.arange(px0, px1, dtype=np.float64)
    ys = np.arange(py0, py1, dtype=np.float64)
    dx = g["mean"][i, 0].astype(np.float64) - xs[None, :]
    dy = g["mean"][i, 1].astype(np.float64) - ys[:, None]
    cx, cy, cz = (float(v) for v in g["conic"][i])
    power = -0.5 * (cx * dx * dx + cz * dy * dy) - cy * dx * dy
    G = np.exp(np.minimum(power, 0.0))
    G = np.where((power <= 0) & (G >= 1e-7), G, 0.0)
    return (py0, py1, px0, px1), dx, dy, G


def render(kind, xy, p1, p2, weight, H, W, max_patch_radius, min_scale):
    """-> (out [2, H, W] float64, preprocess dict)."""
    g = preprocess(kind, xy, p1, p2, H, W, max_patch_radius, min_scale)
    weight = np.asarray(weight, f32).reshape(-1, 2).astype(np.float64)
    out = np.zeros((2, H, W))
    for i in range(g["mean"].shape[0]):  # ascending index, as the tile lists
        t = _terms(g, i, H, W)
        if t is None:
            continue
        (y0, y1, x0, x1), _, _, G = t
        out[0, y0:y1, x0:x1] += weight[i, 0] * G
        out[1, y0:y1, x0:x1] += weight[i, 1] * G
    return out, g


def backward(kind, xy, p1, p2, weight, H, W, max_patch_radius, min_scale, grad_out):
    """-> (dxy [N,2], dp1 [N,2], dp2 [N], dweight [N,2]) in float64."""
    g = preprocess(kind, xy, p1, p2, H, W, max_patch_radius, min_scale)
    N = g["mean"].shape[0]
    weight = np.asarray(weight, f32).reshape(N, 2).astype(np.float64)
    p1 = np.asarray(p1, f32).reshape(N, 2).astype(np.float64)
    p2 = np.asarray(p2, f32).reshape(N).astype(np.float64)
    go = np.asarray(grad_out, np.float64).reshape(2, H, W)
    dxy = np.zeros((N, 2))
    dp1 = np.zeros((N, 2))
    dp2 = np.zeros(N)
    dw = np.zeros((N, 2))
    mxs, mns = float(max_patch_radius), float(min_scale)
    for i in range(N):
        t = _terms(g, i, H, W)
        if t is None:
            continue
        (y0, y1, x0, x1), dx, dy, G = t
        g0, g1 = go[0, y0:y1, x0:x1], go[1, y0:y1, x0:x1]
        cx, cy, cz = (float(v) for v in g["conic"][i])
        dLdG = weight[i, 0] * g0 + weight[i, 1] * g1
        dw[i] = (G * g0).sum(), (G * g1).sum()
        gm = np.array([(dLdG * G * (-cx * dx - cy * dy)).sum(), (dLdG * G * (-cz * dy - cy * dx)).sum()])
        gc = np.array([(-0.5 * G * dx * dx * dLdG).sum(), (-G * dx * dy * dLdG).sum(),
                       (-0.5 * G * dy * dy * dLdG).sum()])
        dxy[i] = gm
        if kind == RS:
            th = p2[i]
            ct, st = np.cos(th), np.sin(th)
            sxr, syr = np.exp(p1[i, 0]), np.exp(p1[i, 1])
            sx, sy = min(mxs, max(mns, sxr)), min(mxs, max(mns, syr))
            sx2, sy2 = sx * sx, sy * sy
            a = ct * ct * sx2 + st * st * sy2
            b = ct * st * (sx2 - sy2)
            c = st * st * sx2 + ct * ct * sy2
        else:
            l11r, l22r = np.exp(p1[i, 0]), np.exp(p1[i, 1])
            l11, l22 = min(mxs, max(mns, l11r)), min(mxs, max(mns, l22r))
            l21 = p2[i]
            a, b, c = l11 * l11, l11 * l21, l21 * l21 + l22 * l22
        det = a * c - b * b if kind == RS else a * l22 * l22
        d2 = 1.0 / (det * det + 1e-7)
        da = d2 * (-c * c * gc[0] + b * c * gc[1] + (det - a * c) * gc[2])
        db = d2 * (2 * b * c * gc[0] - (det + 2 * b * b) * gc[1] + 2 * a * b * gc[2])
        dc = d2 * ((det - a * c) * gc[0] + a * b * gc[1] - a * a * gc[2])
        if kind == RS:
            dsx2 = ct * ct * da + ct * st * db + st * st * dc
            dsy2 = st * st * da - ct * st * db + ct * ct * dc
            dth = (2 * ct * st * (sy2 - sx2) * da + (ct * ct - st * st) * (sx2 - sy2) * db
                   + 2 * st * ct * (sx2 - sy2) * dc)
            inx = 1.0 if mns <= sxr <= mxs else 0.0
            iny = 1.0 if mns <= syr <= mxs else 0.0
            dp1[i] = dsx2 * 2 * sx2 * inx, dsy2 * 2 * sy2 * iny
            dp2[i] = dth
        else:
            dl11 = 2 * l11 * da + l21 * db
            dl21 = l11 * db + 2 * l21 * dc
            dl22 = 2 * l22 * dc
            in11 = 1.0 if mns <= l11r <= mxs else 0.0
            in22 = 1.0 if mns <= l22r <= mxs else 0.0
            dp1[i] = dl11 * l11 * in11, dl22 * l22 * in22
            dp2[i] = dl21
    return dxy, dp1, dp2, dw
