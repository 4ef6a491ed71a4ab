"""FP64 NumPy oracle of the complex INR -- TEST INFRASTRUCTURE ONLY.

Restates the representation that feeds the forward model in
zhixuanh0710/conventional-ptychography-reconstruction:

* ``hashgrid_encode`` / ``hashgrid_backward`` -- the multi-resolution hash
  encoding the reference consumes from tiny-cuda-nn as
  ``tcnn.Encoding(n_input_dims=2, {"otype": "HashGrid", ...})``
  (models/complex_inr.py:130-145, called at :279, :294).  tiny-cuda-nn is an
  unpinned third-party dependency absent from the reference tree, so this is a
  restatement of the published Instant-NGP method (Mueller et al. 2022) with
  these choices: level l has scale
  ``s_l = base * per_level_scale**l - 1`` and ``r_l = ceil(s_l) + 1`` vertices
  per axis; a coordinate x in [0,1] maps to ``x * s_l + 0.5``; the cell corner
  is its floor and the bilinear weights the fractional part; a level whose
  ``r_l**2`` (rounded up to a multiple of 8) fits in ``T = 2**log2_hashmap_size``
  entries is indexed densely (``ix + iy * r_l``), otherwise by the spatial hash
  ``(ix * 1) ^ (iy * 2654435761)`` modulo T; entries hold F features.
  Parity for this component is unpinned (no reference output exists).
* ``cmlp_forward`` / ``cmlp_backward`` -- ``ComplexMLP.net``
  (models/complex_inr.py:6-82, used through ``_get_complex_output`` :308-314):
  real Linear(32->H) then exp(i w1 z); ``hidden_layers`` complex
  Linear(H->H) + exp(i w z); complex Linear(H->1).  Gradients in torch's
  complex convention (dL/dRe + i dL/dIm).  Pinned against the reference's
  own module (tests/golden/complex_mlp.npz).
* ``fourier_upsample`` / its adjoint -- models/complex_inr.py:252-271.
* ``adam_step`` -- torch.optim.Adam (Recovery.py:238-241, :321) with complex
  parameters handled as independent real/imaginary parts.
"""
from __future__ import annotations

import math

import numpy as np

PRIME_Y = 2654435761


# --------------------------------------------------------------------------
# HashGrid
# --------------------------------------------------------------------------
def hashgrid_levels(n_levels, log2_hashmap_size, base_resolution, per_level_scale):
    """Per-level (scale, resolution, entries, offset_in_entries, dense)."""
    T = 1 << log2_hashmap_size
    out, off = [], 0
    for l in range(n_levels):
        scale = base_resolution * (per_level_scale ** l) - 1.0
        res = int(math.ceil(scale)) + 1
        dense_n = res * res
        dense_n = (dense_n + 7) // 8 * 8
        n = min(dense_n, T)
        out.append((scale, res, n, off, dense_n <= T))
        off += n
    return out


def hashgrid_corners(coords, levels, fp32_positions=False):
    """For each level: (index [N,4] int64 into the level, weight [N,4]).

    ``fp32_positions`` forms the grid position as a single-rounded float32
    ``x * float32(scale) + 0.5`` (a fused multiply-add), the arithmetic the
    CUDA kernel uses; otherwise positions are FP64."""
    x = np.asarray(coords, dtype=np.float64)
    res_all = []
    for (scale, res, n, off, dense) in levels:
        if fp32_positions:
            s32 = np.float64(np.float32(scale))
            p = (np.float32(x).astype(np.float64) * s32 + 0.5).astype(np.float32).astype(np.float64)
        else:
            p = x * scale + 0.5
        g = np.floor(p)
        f = p - g
        gi = g.astype(np.int64)
        idx = np.empty((x.shape[0], 4), np.int64)
        w = np.empty((x.shape[0], 4), np.float64)
        for k, (dx, dy) in enumerate(((0, 0), (1, 0), (0, 1), (1, 1))):
            cx = gi[:, 0] + dx
            cy = gi[:, 1] + dy
            if dense:
                e = cx + cy * res
            else:
                e = (cx.astype(np.uint64) ^ (cy.astype(np.uint64) * np.uint64(PRIME_Y))).astype(np.uint64)
                e = e & np.uint64(0xFFFFFFFF)
                e = e.astype(np.int64)
            idx[:, k] = e % n
            wx = f[:, 0] if dx else 1.0 - f[:, 0]
            wy = f[:, 1] if dy else 1.0 - f[:, 1]
            w[:, k] = wx * wy
        res_all.append((idx, w))
    return res_all


def hashgrid_encode(coords, table, levels, F=2, fp32_positions=False):
    """Features [N, L*F]: per level the bilinear blend of the 4 corner entries.

    ``table`` is flat: level l occupies entries [off_l, off_l + n_l), F floats each."""
    tab = np.asarray(table, dtype=np.float64).reshape(-1, F)
    corners = hashgrid_corners(coords, levels, fp32_positions)
    N = np.asarray(coords).shape[0]
    out = np.zeros((N, len(levels) * F))
    for l, ((scale, res, n, off, dense), (idx, w)) in enumerate(zip(levels, corners)):
        out[:, l * F:(l + 1) * F] = np.einsum("nk,nkf->nf", w, tab[off + idx])
    return out


def hashgrid_backward(coords, dfeat, levels, n_entries, F=2, fp32_positions=False):
    """d table (flat, [n_entries * F]) from d features [N, L*F]."""
    g = np.zeros((n_entries, F))
    corners = hashgrid_corners(coords, levels, fp32_positions)
    for l, ((scale, res, n, off, dense), (idx, w)) in enumerate(zip(levels, corners)):
        d = np.asarray(dfeat, dtype=np.float64)[:, l * F:(l + 1) * F]
        for k in range(4):
            np.add.at(g, off + idx[:, k], w[:, k:k + 1] * d)
    return g.reshape(-1)


# --------------------------------------------------------------------------
# ComplexMLP
# --------------------------------------------------------------------------
def bf16_round(a):
    """Round float values to bfloat16 (nearest, ties to even); complex: per part."""
    a = np.asarray(a)
    if np.iscomplexobj(a):
        return bf16_round(a.real) + 1j * bf16_round(a.imag)
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_split(a):
    """bf16(a) + bf16(a - bf16(a)): a value as the sum of two BF16 operands."""
    hi = bf16_round(a)
    return hi + bf16_round(np.asarray(a) - hi)


def _ident(a):
    return a


def cmlp_forward(x, params, q=_ident, qh=None):
    """params: dict with W1 [H,32] real, b1 [H] real, w1 (omega), Wh[i] [H,H] complex,
    bh[i] [H] complex, wh[i], Wo [1,H] complex, bo [1] complex.  Returns y [N] and a cache.
    ``q`` rounds every matmul operand and ``qh`` (default ``q``) the hidden
    activations entering layer 2, layer 3 and the output layer in the forward;
    ``q=bf16_round, qh=bf16_split`` mirrors the tensor-core kernel, whose weight
    gradients use the single BF16 rounding of those activations."""
    qh = q if qh is None else qh
    x = np.asarray(x, dtype=np.float64)
    z1 = q(x) @ q(params["W1"]).T + params["b1"]
    h = np.exp(1j * params["w1"] * z1)
    cache = {"x": x, "z": [z1], "h": [h], "q": q}
    for W, b, w in zip(params["Wh"], params["bh"], params["wh"]):
        z = qh(h) @ q(W).T + b
        h = np.exp(1j * w * z)
        cache["z"].append(z)
        cache["h"].append(h)
    y = (qh(h) @ q(params["Wo"]).T + params["bo"])[:, 0]
    return y, cache


def cmlp_backward(gy, params, cache):
    """Gradients (torch complex convention) for upstream gy [N] complex."""
    q = cache.get("q", _ident)
    gy = q(np.asarray(gy, dtype=np.complex128)[:, None])
    hs, zs = cache["h"], cache["z"]
    grads = {"Wo": gy.T @ np.conj(q(hs[-1])), "bo": gy.sum(0)}
    gh = gy @ np.conj(q(params["Wo"]))  # W^H g
    gWh, gbh, gwh = [], [], []
    for li in range(len(params["Wh"]) - 1, -1, -1):
        h_out, z = hs[li + 1], zs[li + 1]
        w = params["wh"][li]
        gz = q(np.conj(1j * w * h_out) * gh)
        gwh.insert(0, float(np.real(np.conj(gh) * (1j * z * h_out)).sum()))
        h_in = hs[li]
        gWh.insert(0, gz.T @ np.conj(q(h_in)))
        gbh.insert(0, gz.sum(0))
        gh = gz @ np.conj(q(params["Wh"][li]))
    h1, z1 = hs[0], zs[0]
    w1 = params["w1"]
    gz1 = np.real(np.conj(gh) * (1j * w1 * h1))
    grads["w1"] = float((np.real(np.conj(gh) * (1j * h1)) * z1).sum())
    gz1 = q(gz1)
    grads["W1"] = gz1.T @ q(cache["x"])
    grads["b1"] = gz1.sum(0)
    grads["x"] = gz1 @ q(params["W1"])
    grads["Wh"], grads["bh"], grads["wh"] = gWh, gbh, gwh
    return grads


# --------------------------------------------------------------------------
# Fourier upsampling (models/complex_inr.py:252-271) and its adjoint
# --------------------------------------------------------------------------
def fourier_upsample(x, s):
    H, W = x.shape
    X = np.fft.fftshift(np.fft.fft2(x))
    nH, nW = int(H * s), int(W * s)
    ph, pw = (nH - H) // 2, (nW - W) // 2
    Xp = np.zeros((nH, nW), np.complex128)
    Xp[ph:ph + H, pw:pw + W] = X
    return np.fft.ifft2(np.fft.ifftshift(Xp)) * (s * s)


def fourier_upsample_adjoint(g, s, shape):
    H, W = shape
    nH, nW = g.shape
    ph, pw = (nH - H) // 2, (nW - W) // 2
    G = np.fft.fftshift(np.fft.fft2(g)) / (nH * nW)
    Gc = G[ph:ph + H, pw:pw + W]
    return np.fft.ifft2(np.fft.ifftshift(Gc)) * (H * W) * (s * s)


# --------------------------------------------------------------------------
# Adam (torch.optim.Adam defaults: betas (0.9, 0.999), eps 1e-8)
# --------------------------------------------------------------------------
def adam_step(p, g, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One step on real arrays (complex parameters: pass their real view)."""
    m = beta1 * m + (1 - beta1) * g
    v = beta2 * v + (1 - beta2) * g * g
    bc1 = 1 - beta1 ** step
    bc2 = 1 - beta2 ** step
    denom = np.sqrt(v) / math.sqrt(bc2) + eps
    p = p - (lr / bc1) * m / denom
    return p, m, v
