"""FP64 NumPy oracle of the far-field ptychography forward model and adjoint.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline legs of ``bench.py`` as the checker; never by the product.

Every function cites the reference lines it restates (paths relative to the
zhixuanh0710/conventional-ptychography-reconstruction tree).  Conventions:

* object ``O`` is [H, W] complex, probe ``P`` is [M, N] complex;
* scan windows are given as top-left corners ``tlY``, ``tlX`` (int arrays
  [B]); the bottom-right corner is ``tl + (M, N)`` (utils/optics.py:93-94);
* measured intensities ``Imeas`` are [B, M, N] (frames first; the reference
  stores [M, N, F], Recovery.py:103-104, 289);
* gradients follow torch's convention for complex leaves:
  ``grad = dL/dRe + 1j * dL/dIm``.
"""
from __future__ import annotations

import math

import numpy as np

LOSS_TYPES = ("smooth_L1_loss", "FD_loss", "Poisson_likelihood_loss")
EPS = 1e-8  # Recovery.py:297, 304


# --------------------------------------------------------------------------
# scan geometry -- utils/optics.py:68-99
# --------------------------------------------------------------------------
def scan_positions_to_pixels(xlocation, ylocation, probe_shape, wavelength,
                             camera_length, camera_pixel_pitch):
    """Physical scan positions (m) -> top-left / bottom-right pixel indices.

    Restates utils/optics.py:68-99: positions are shifted to start at zero
    (:86-87), the sample-plane pitch is ``lambda*L/([M,N]*pitch)`` (:89), the
    top-left index is ``np.round(pos/dx)`` -- NumPy's round-half-to-even --
    cast to the platform int (:91-92), and the canvas is the larger bottom-right
    extent rounded up to a multiple of 6 (:96-97).
    """
    M, N = probe_shape
    xs = np.asarray(xlocation, dtype=np.float64).reshape(-1)
    ys = np.asarray(ylocation, dtype=np.float64).reshape(-1)
    x_pos = xs - xs.min()
    y_pos = ys - ys.min()
    dx = wavelength * camera_length / (np.array([M, N]) * camera_pixel_pitch)
    tlY = np.rint(y_pos / dx[0]).astype(np.int64)
    tlX = np.rint(x_pos / dx[1]).astype(np.int64)
    brY = tlY + M
    brX = tlX + N
    canvas = int(math.ceil(max(int(brY.max()), int(brX.max())) / 6) * 6)
    return tlX, tlY, brX, brY, dx, canvas


# --------------------------------------------------------------------------
# forward model -- utils/optics.py:102-112, Recovery.py:290-292
# --------------------------------------------------------------------------
def exit_waves(O, P, tlY, tlX):
    """psi_b = P * O[tlY_b:tlY_b+M, tlX_b:tlX_b+N]  (Recovery.py:290)."""
    O = np.asarray(O, dtype=np.complex128)
    P = np.asarray(P, dtype=np.complex128)
    M, N = P.shape
    tlY = np.asarray(tlY).reshape(-1)
    tlX = np.asarray(tlX).reshape(-1)
    out = np.empty((tlY.size, M, N), dtype=np.complex128)
    for b in range(tlY.size):
        y, x = int(tlY[b]), int(tlX[b])
        out[b] = P * O[y:y + M, x:x + N]
    return out


def far_field(psi):
    """fftshift(fft2(psi)) over the last two axes (Recovery.py:291)."""
    return np.fft.fftshift(np.fft.fft2(psi, axes=(-2, -1)), axes=(-2, -1))


def forward_intensity(O, P, tlY, tlX):
    """|fftshift(fft2(P * O_window))|^2, [B, M, N] float64 (utils/optics.py:102-112)."""
    return np.abs(far_field(exit_waves(O, P, tlY, tlX))) ** 2


# --------------------------------------------------------------------------
# losses and dloss/dI -- Recovery.py:294-305 (per frame, mean over pixels)
# --------------------------------------------------------------------------
def loss_terms(I, Imeas, loss_type):
    """Per-pattern loss (mean over the M*N pixels) and its gradient dL/dI.

    ``I`` model intensity, ``Imeas`` measurement, both [B, M, N].
    smooth_L1 (beta=1, torch F.smooth_l1_loss, Recovery.py:294-295),
    FD (Recovery.py:296-302), Poisson (Recovery.py:303-305).
    Returns ``(loss [B] float64, g [B, M, N] float64)``.
    """
    I = np.asarray(I, dtype=np.float64)
    Im = np.asarray(Imeas, dtype=np.float64)
    if I.ndim == 2:
        I, Im = I[None], Im[None]
    B, M, N = I.shape
    MN = float(M * N)
    if loss_type == "smooth_L1_loss":
        d = I - Im
        ad = np.abs(d)
        per = np.where(ad < 1.0, 0.5 * d * d, ad - 0.5)
        g = np.where(ad < 1.0, d, np.sign(d)) / MN
    elif loss_type == "Poisson_likelihood_loss":
        per = I - Im * np.log(I + EPS)
        g = (1.0 - Im / (I + EPS)) / MN
    elif loss_type == "FD_loss":
        sI = np.sqrt(I + EPS)
        dW = np.sqrt(Im + EPS) - sI
        Rx = np.roll(dW, -1, axis=2) - dW   # dW[:, j+1] - dW[:, j], circular
        Ry = np.roll(dW, -1, axis=1) - dW   # dW[i+1, :] - dW[i, :], circular
        G = np.sqrt(Rx * Rx + Ry * Ry + EPS)
        per = G
        ax = Rx / G
        ay = Ry / G
        dL_ddW = (np.roll(ax, 1, axis=2) - ax + np.roll(ay, 1, axis=1) - ay) / MN
        g = dL_ddW * (-0.5 / sI)
    else:
        raise ValueError(f"loss_type must be one of {LOSS_TYPES}, got {loss_type!r}")
    loss = per.reshape(B, -1).mean(axis=1)
    return loss, g


# --------------------------------------------------------------------------
# adjoint (what torch autograd computes for Recovery.py:316)
# --------------------------------------------------------------------------
def fwd_adj(O, P, tlY, tlX, Imeas, loss_type):
    """Forward model + loss + adjoint for a batch, all in FP64.

    Returns a dict with ``I`` [B,M,N], ``loss`` [B] (per-pattern means),
    ``loss_total`` (their sum, Recovery.py:307), ``E`` [B,M,N] (gradient of
    the exit waves), ``dO`` [H,W] and ``dP`` [M,N] (torch complex-gradient
    convention).

    Adjoint chain per pattern (torch autograd's formulas):
      G_F   = 2 * g * F                        (|F|^2 backward)
      G_psi = M*N * ifft2(ifftshift(G_F))      (fftshift, then fft2 backward)
      dP   += G_psi * conj(O_window);  dO[window] += G_psi * conj(P).
    """
    O = np.asarray(O, dtype=np.complex128)
    P = np.asarray(P, dtype=np.complex128)
    M, N = P.shape
    tlY = np.asarray(tlY).reshape(-1)
    tlX = np.asarray(tlX).reshape(-1)
    psi = exit_waves(O, P, tlY, tlX)
    F = far_field(psi)
    I = np.abs(F) ** 2
    loss, g = loss_terms(I, Imeas, loss_type)
    GF = 2.0 * g * F
    E = (M * N) * np.fft.ifft2(np.fft.ifftshift(GF, axes=(-2, -1)), axes=(-2, -1))
    dO = np.zeros_like(O)
    dP = np.zeros_like(P)
    Pc = np.conj(P)
    for b in range(tlY.size):
        y, x = int(tlY[b]), int(tlX[b])
        dP += E[b] * np.conj(O[y:y + M, x:x + N])
        dO[y:y + M, x:x + N] += E[b] * Pc
    return {"I": I, "loss": loss, "loss_total": float(loss.sum()), "E": E,
            "dO": dO, "dP": dP}


def total_loss(O, P, tlY, tlX, Imeas, loss_type):
    """Scalar sum of per-pattern losses (for finite-difference checks)."""
    I = forward_intensity(O, P, tlY, tlX)
    return float(loss_terms(I, Imeas, loss_type)[0].sum())


def fd_gradient(O, P, tlY, tlX, Imeas, loss_type, which, idx, h=1e-6):
    """Central finite-difference gradient of the total loss, torch convention.

    ``which`` is "O" or "P", ``idx`` a list of (row, col).  Returns complex
    values dL/dRe + 1j dL/dIm at those pixels.
    """
    out = []
    for (r, c) in idx:
        vals = []
        for unit in (1.0, 1.0j):
            Op = np.array(O, dtype=np.complex128, copy=True)
            Pp = np.array(P, dtype=np.complex128, copy=True)
            Om = Op.copy()
            Pm = Pp.copy()
            if which == "O":
                Op[r, c] += h * unit
                Om[r, c] -= h * unit
            else:
                Pp[r, c] += h * unit
                Pm[r, c] -= h * unit
            lp = total_loss(Op, Pp, tlY, tlX, Imeas, loss_type)
            lm = total_loss(Om, Pm, tlY, tlX, Imeas, loss_type)
            vals.append((lp - lm) / (2 * h))
        out.append(vals[0] + 1j * vals[1])
    return np.array(out)


# --------------------------------------------------------------------------
# probe centring and energy normalisation -- Recovery.py:262-285
# --------------------------------------------------------------------------
def probe_com_shift(P):
    """Centre-of-mass roll amount cp (Recovery.py:262-275), or None if tot==0.

    cp = trunc([M,N]/2 - [M,N] * mean(cumsum(marginal)) / tot + 1)."""
    a = np.abs(np.asarray(P, dtype=np.complex128)) ** 2
    Mp, Np = a.shape
    tot = a.sum()
    if tot == 0:
        return None
    com = np.array([np.cumsum(a.sum(1)).mean(), np.cumsum(a.sum(0)).mean()])
    return np.trunc(np.array([Mp, Np]) / 2 - np.array([Mp, Np]) * com / tot + 1).astype(np.int64)


def center_and_normalize_probe(P):
    """Roll by -cp and scale to sum|P|^2 = M*N (Recovery.py:276-285)."""
    P = np.asarray(P, dtype=np.complex128)
    cp = probe_com_shift(P)
    if cp is not None and np.any(cp):
        P = np.roll(P, (-int(cp[0]), -int(cp[1])), axis=(0, 1))
    e = (np.abs(P) ** 2).sum()
    if e > 0:
        P = P * np.sqrt(P.shape[0] * P.shape[1] / e)
    return P


def haar_sparsity(img):
    """L1 of the LH/HL/HH Haar subbands of Re and Im (utils/loss.py:60-83)."""
    img = np.asarray(img)
    if np.iscomplexobj(img):
        return haar_sparsity(img.real) + haar_sparsity(img.imag)
    a = img[0::2, 0::2]
    b = img[0::2, 1::2]
    c = img[1::2, 0::2]
    d = img[1::2, 1::2]
    return float(np.abs(a - b + c - d).sum() + np.abs(a + b - c - d).sum()
                 + np.abs(a - b - c + d).sum())


# --------------------------------------------------------------------------
# accuracy reporting -- scripts/compare_object_ssim.py:92-98
# --------------------------------------------------------------------------
def resolve_global_phase(recon, gt):
    """recon * exp(i alpha) minimising ||recon e^{i alpha} - gt|| (:92-98)."""
    inner = np.vdot(np.asarray(recon).ravel(), np.asarray(gt).ravel())
    if abs(inner) < 1e-20:
        return recon
    return recon * (inner / abs(inner))


def object_error(recon, gt, box=None):
    """(NRMSE after resolve_global_phase, NRMSE after the least-squares complex
    factor) over box = (y0, y1, x0, x1); FP64 (compare_object_ssim.py:92-98)."""
    r = np.asarray(recon, dtype=np.complex128)
    g = np.asarray(gt, dtype=np.complex128)
    if box is not None:
        y0, y1, x0, x1 = box
        r, g = r[y0:y1, x0:x1], g[y0:y1, x0:x1]
    ng = float(np.vdot(g, g).real)
    a = resolve_global_phase(r, g) - g
    e_phase = float(np.sqrt(np.vdot(a, a).real / ng))
    c = np.vdot(r, g)
    nr = float(np.vdot(r, r).real)
    gfac = c / nr if nr > 0 else 0.0
    d = gfac * r - g
    e_scaled = float(np.sqrt(np.vdot(d, d).real / ng))
    return e_phase, e_scaled


def align_by_xcorr(recon_mag, gt_mag):
    """Integer offset (row, col) of a recon inside a ground truth at least as large
    (compare_object_ssim.py:75-89): the arg-max, over offsets that keep the recon
    inside, of the circular cross-correlation of the mean-removed magnitudes with
    the recon zero-padded to the truth's size; first maximum in row-major order."""
    r = np.asarray(recon_mag, dtype=np.float64)
    g = np.asarray(gt_mag, dtype=np.float64)
    H, W = r.shape
    Hg, Wg = g.shape
    if Hg < H or Wg < W:
        raise ValueError("ground truth smaller than the reconstruction")
    rf = np.fft.fft2(r - r.mean(), s=(Hg, Wg))
    gf = np.fft.fft2(g - g.mean(), s=(Hg, Wg))
    xc = np.fft.ifft2(gf * np.conj(rf)).real[:Hg - H + 1, :Wg - W + 1]
    i = np.unravel_index(int(np.argmax(xc)), xc.shape)
    return int(i[0]), int(i[1])


def _signed_freqs(n):
    return np.fft.fftfreq(n) * n


def register_translation(recon, gt, upsample=100):
    """Sub-pixel shift d = (dy, dx) such that shift(recon, d) best matches gt, by
    the upsampled-DFT cross-correlation of Guizar-Sicairos, Thurman and Fienup
    (Opt. Lett. 33, 156, 2008): the FFT cross-correlation's peak locates d to the
    pixel, then the correlation is evaluated by matrix DFTs on a 1/upsample grid
    over +-0.75 pixel around it.  FP64 throughout."""
    r = np.asarray(recon, dtype=np.complex128)
    g = np.asarray(gt, dtype=np.complex128)
    H, W = g.shape
    X = np.fft.fft2(g) * np.conj(np.fft.fft2(r))
    cc = np.abs(np.fft.ifft2(X))
    py, px = np.unravel_index(int(np.argmax(cc)), cc.shape)
    py = py - H if py > H // 2 else py
    px = px - W if px > W // 2 else px
    if upsample <= 1:
        return float(py), float(px)
    half = int(np.ceil(0.75 * upsample))
    offs = np.arange(-half, half + 1) / upsample
    ys, xs = py + offs, px + offs
    Er = np.exp(2j * np.pi * np.outer(ys, _signed_freqs(H)) / H)
    Ec = np.exp(2j * np.pi * np.outer(_signed_freqs(W), xs) / W)
    up = np.abs(Er @ X @ Ec)
    iy, ix = np.unravel_index(int(np.argmax(up)), up.shape)
    return float(ys[iy]), float(xs[ix])


def fourier_shift(img, dy, dx):
    """img translated by (dy, dx) pixels, out(y, x) = img(y - dy, x - dx), periodic."""
    a = np.asarray(img, dtype=np.complex128)
    H, W = a.shape
    ph = np.exp(-2j * np.pi * (np.outer(_signed_freqs(H) * dy / H, np.ones(W))
                               + np.outer(np.ones(H), _signed_freqs(W) * dx / W)))
    return np.fft.ifft2(np.fft.fft2(a) * ph)


def register_in_box(recon, gt, box, upsample=100, iters=3):
    """Shift aligning a canvas ``recon`` to ``gt`` inside ``box``: the crops'
    mean is removed and a separable Hann window applied (the crops are not
    periodic), ``register_translation`` is run on them, the shift is applied to
    the whole canvas and the registration repeated on the shifted crop until the
    increment is zero (at most ``iters`` times); the increments add up."""
    y0, y1, x0, x1 = box

    def win(a):
        a = a - a.mean()
        return a * np.outer(np.hanning(a.shape[0]), np.hanning(a.shape[1]))

    g = win(np.asarray(gt, dtype=np.complex128)[y0:y1, x0:x1])
    d = np.zeros(2)
    for _ in range(iters):
        rs = fourier_shift(recon, *d)[y0:y1, x0:x1]
        dd = np.array(register_translation(win(rs), g, upsample))
        d = d + dd
        if not dd.any():
            break
    return float(d[0]), float(d[1])


def coverage_box(tlY, tlX, probe_shape, canvas_shape, frac=0.5):
    """scan_coverage_mask + high_coverage_bbox (compare_object_ssim.py:42-72) on
    integer window corners: bbox of pixels covered >= ceil(frac * max) times."""
    M, N = probe_shape
    Hc, Wc = canvas_shape
    cov = np.zeros((Hc, Wc), dtype=np.int32)
    for y, x in zip(np.asarray(tlY).ravel(), np.asarray(tlX).ravel()):
        y0, y1, x0, x1 = max(0, y), min(Hc, y + M), max(0, x), min(Wc, x + N)
        if y1 > y0 and x1 > x0:
            cov[y0:y1, x0:x1] += 1
    thr = max(1, int(np.ceil(frac * cov.max())))
    ys, xs = np.where(cov >= thr)
    if ys.size == 0:
        return 0, Hc, 0, Wc
    return int(ys.min()), int(ys.max()) + 1, int(xs.min()), int(xs.max()) + 1


def data_residual(I_model, Imeas):
    """R = sum (sqrt(I) - sqrt(Imeas))^2 / sum Imeas, FP64 over the stack."""
    I_model = np.asarray(I_model, dtype=np.float64)
    Imeas = np.asarray(Imeas, dtype=np.float64)
    return float(((np.sqrt(I_model) - np.sqrt(Imeas)) ** 2).sum() / Imeas.sum())
