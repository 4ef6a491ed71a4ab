"""Forward model, losses and adjoint on the B200 kernels (drop-in for the
reference's ``utils/optics.py`` forward path and the per-frame loop of
``Recovery.py:288-316``).

Public functions:

* :func:`scan_positions_to_pixels` -- utils/optics.py:68-99, same signature
  and outputs (host NumPy, bit-exact with the reference);
* :func:`forward_imaging_model` -- utils/optics.py:102-112, same signature,
  differentiable w.r.t. object and probe;
* :func:`forward_intensity` -- the batched form: ``I[b] = |fftshift(fft2(P *
  O[window_b]))|^2`` for a stack of windows;
* :func:`fused_loss` -- the fused forward + loss + adjoint used by the
  training loop: returns the FP64 sum over the batch of per-pattern mean
  losses (Recovery.py:294-307) as a differentiable scalar whose backward
  returns the gradients computed in the same kernel pass.

All compute runs in ``libptycho_b200.so``; there is no CPU path.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib

LOSS_CODES = {"smooth_L1_loss": 0, "FD_loss": 1, "Poisson_likelihood_loss": 2}
_INTENSITY_GRAD = 3
FUSED_PROBE_SIZES = (64, 128, 256)  # square probes that run the fused kernels
MAX_PROBE_DIM = 4096                 # any other 1 <= M, N <= 4096 runs the general path


# --------------------------------------------------------------------------
# geometry (host) -- utils/optics.py:68-99
# --------------------------------------------------------------------------
def scan_positions_to_pixels(xlocation, ylocation, probe_shape, wavelength, camera_length,
                             camera_pixel_pitch):
    """Physical scan positions (metres) -> sample-plane pixel windows.

    Same contract as utils/optics.py:68-99: returns ``(tlX, tlY, brX, brY, dx,
    canvas_size)``; indices use NumPy's round-half-to-even of ``pos / dx``
    with ``dx = wavelength * camera_length / ([M, N] * camera_pixel_pitch)``;
    the canvas is the larger bottom-right extent rounded up to a multiple of 6.
    """
    M, N = probe_shape
    x_pos = np.asarray(xlocation).squeeze() - np.min(xlocation)
    y_pos = np.asarray(ylocation).squeeze() - np.min(ylocation)
    dx = wavelength * camera_length / (np.array([M, N]) * camera_pixel_pitch)
    tlY = np.round(y_pos / dx[0]).astype(int)
    tlX = np.round(x_pos / dx[1]).astype(int)
    brY = tlY + M
    brX = tlX + N
    max_size = max(int(np.max(brY)), int(np.max(brX)))
    canvas_size = math.ceil(max_size / 6) * 6
    return tlX, tlY, brX, brY, dx, canvas_size


def make_windows(tlY, tlX, device=None) -> torch.Tensor:
    """Pack top-left corners into the library's [B, 2] int32 (tlY, tlX) layout."""
    tlY = torch.as_tensor(np.asarray(tlY), dtype=torch.int32).reshape(-1)
    tlX = torch.as_tensor(np.asarray(tlX), dtype=torch.int32).reshape(-1)
    t = torch.stack([tlY, tlX], dim=1).contiguous()
    return t.to(device) if device is not None else t


def check_windows(tl: torch.Tensor, canvas_hw, M: int, N: int | None = None) -> None:
    """Host-side bounds check of scan windows of M x N (N defaults to M; raises ``ValueError``)."""
    H, W = canvas_hw
    N = M if N is None else N
    t = tl.detach().to("cpu")
    if t.numel() == 0:
        return
    bad = (t[:, 0] < 0) | (t[:, 1] < 0) | (t[:, 0] > H - M) | (t[:, 1] > W - N)
    if bool(bad.any()):
        i = int(torch.nonzero(bad)[0, 0])
        raise ValueError(f"scan window {i} at {t[i].tolist()} leaves the {H}x{W} canvas (probe {M})")


# --------------------------------------------------------------------------
# raw calls
# --------------------------------------------------------------------------
_raw_stream = getattr(torch._C, "_cuda_getCurrentRawStream", None)


def _stream_handle(device: torch.device) -> int:
    """The current stream of ``device`` as a raw handle (a per-call host cost:
    the direct accessor skips building a Stream object)."""
    if _raw_stream is not None and device.index is not None:
        return _raw_stream(device.index)
    return torch.cuda.current_stream(device).cuda_stream


def _i32(x: torch.Tensor, dev) -> torch.Tensor:
    """x as a contiguous int32 tensor on dev (no conversion call when it already is)."""
    if x.dtype == torch.int32 and x.device == dev and x.is_contiguous():
        return x
    return x.to(device=dev, dtype=torch.int32).contiguous()


def _as_c64(x: torch.Tensor, name: str) -> torch.Tensor:
    if not x.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (there is no CPU path)")
    if x.dtype != torch.complex64:
        x = x.to(torch.complex64)
    return x.contiguous()


def _check_probe(P: torch.Tensor):
    """(M, N) of a probe: square 64 / 128 / 256 run the fused kernels, any
    other 1 <= M, N <= MAX_PROBE_DIM the general path."""
    if P.dim() != 2 or not (1 <= P.shape[0] <= MAX_PROBE_DIM and 1 <= P.shape[1] <= MAX_PROBE_DIM):
        raise ValueError(f"probe must be [M, N] with 1 <= M, N <= {MAX_PROBE_DIM}, got {tuple(P.shape)}")
    return int(P.shape[0]), int(P.shape[1])


_status_cache: dict = {}


def device_status(device) -> torch.Tensor:
    """The per-device int32 status word the kernels raise errors into."""
    st = _status_cache.get(device)
    if st is not None:
        return st
    device = torch.device(device)
    if device.index is None:
        device = torch.device(device.type, torch.cuda.current_device())
    st = _status_cache.get(device)
    if st is None:
        st = torch.zeros(1, dtype=torch.int32, device=device)
        _status_cache[device] = st
    return st


def read_status(device, reset: bool = True) -> int:
    """Synchronously read (and optionally clear) the device status word."""
    st = device_status(device)
    v = int(st.item())
    if reset:
        st.zero_()
    return v


class FwdAdjWorkspace:
    """Reusable device scratch for ``ptycho_fwd_adj`` (grows on demand)."""

    def __init__(self):
        self.buf = None

    def get(self, nbytes: int, device) -> torch.Tensor:
        nbytes = max(int(nbytes), 256)
        buf = self.buf
        if buf is None or buf.numel() < nbytes or buf.device != device:
            buf = self.buf = torch.empty(nbytes, dtype=torch.uint8, device=device)
        return buf


_default_ws: dict = {}
# route fused_loss through the C++ autograd node (csrc/torch_ext.cpp) when it
# is built; False keeps the Python Function (both call the same library)
USE_TORCHEXT = True
_ws_size_cache: dict = {}  # (H, W, M, N, B) -> ptycho_fwd_adj_workspace_size


def _batch_arg(batch, dev):
    if batch is None:
        return None
    return _i32(batch if isinstance(batch, torch.Tensor) else torch.as_tensor(batch), dev)


def forward_intensity(O: torch.Tensor, P: torch.Tensor, tl: torch.Tensor, batch=None) -> torch.Tensor:
    """Far-field intensities ``[B, M, N]`` float32 (no autograd).

    ``tl`` [F, 2] int32 windows of all frames; ``batch`` [B] frame ids (None:
    all F frames in order)."""
    O = _as_c64(O, "object")
    P = _as_c64(P, "probe")
    M, N = _check_probe(P)
    H, W = O.shape
    tl = tl.to(device=O.device, dtype=torch.int32).contiguous()
    F = int(tl.shape[0])
    bt = _batch_arg(batch, O.device)
    B = F if bt is None else int(bt.numel())
    out = torch.empty((B, M, N), dtype=torch.float32, device=O.device)
    st = device_status(O.device)
    L = _lib.lib()
    bp = bt.data_ptr() if bt is not None else None
    if M == N and M in FUSED_PROBE_SIZES:
        _lib.check(L.ptycho_forward_intensity(O.data_ptr(), H, W, P.data_ptr(), M, N, tl.data_ptr(), F, bp, B,
                                              out.data_ptr(), st.data_ptr(), _stream_handle(O.device)),
                   "ptycho_forward_intensity")
    else:
        ws = torch.empty(max(int(L.ptycho_forward_intensity_workspace_size(M, N, B)), 256), dtype=torch.uint8,
                         device=O.device)
        _lib.check(L.ptycho_forward_intensity_ws(O.data_ptr(), H, W, P.data_ptr(), M, N, tl.data_ptr(), F, bp, B,
                                                 out.data_ptr(), ws.data_ptr(), ws.numel(), st.data_ptr(),
                                                 _stream_handle(O.device)), "ptycho_forward_intensity_ws")
    return out


def fwd_adj_raw(O, P, tl, Imeas, loss_code: int, batch=None, want_grad: bool = True,
                per_pattern: bool = False, dO=None, dP=None, accumulate: bool = False,
                workspace: "FwdAdjWorkspace | None" = None):
    """One call of ``ptycho_fwd_adj``.  Returns ``(loss_total, loss_per_pattern|None, dO, dP)``.

    ``tl`` [F, 2] int32 and ``Imeas`` [F, M, N] float32 describe all frames;
    ``batch`` [B] selects the frames of this call (None: all, in order).
    ``loss_total`` is a 0-d float64 CUDA tensor.  Gradient buffers are
    allocated unless given (``accumulate`` adds into given buffers)."""
    O = _as_c64(O, "object")
    P = _as_c64(P, "probe")
    M, N = _check_probe(P)
    H, W = O.shape
    dev = O.device
    tl = _i32(tl, dev)
    F = int(tl.shape[0])
    if Imeas.dtype != torch.float32 or not Imeas.is_contiguous() or Imeas.device != dev:
        Imeas = Imeas.to(device=dev, dtype=torch.float32).contiguous()
    if Imeas.shape != (F, M, N):
        raise ValueError(f"measurements must be [F, M, N] = {(F, M, N)}, got {tuple(Imeas.shape)}")
    bt = _batch_arg(batch, dev)
    B = F if bt is None else int(bt.numel())
    stream = _stream_handle(dev)
    loss_total = torch.empty((), dtype=torch.float64, device=dev)
    lp = torch.empty(B, dtype=torch.float64, device=dev) if per_pattern else None
    if want_grad:
        if dO is None:
            dO = torch.empty((H, W), dtype=torch.complex64, device=dev)
        if dP is None:
            dP = torch.empty((M, N), dtype=torch.complex64, device=dev)
    else:
        dO = dP = None
    key = (H, W, M, N, B)
    ws_bytes = _ws_size_cache.get(key)
    if ws_bytes is None:
        ws_bytes = _ws_size_cache[key] = int(_lib.lib().ptycho_fwd_adj_workspace_size(H, W, M, N, B))
    if workspace is not None:
        ws = workspace.get(ws_bytes, dev)
    elif USE_TORCHEXT and _lib.torchext() is not None:
        # the per-stream workspace the C++ autograd node also uses
        ws = _lib.torchext().workspace(O, ws_bytes)
    else:
        # one default workspace per (device, stream): calls on one stream are
        # ordered, calls on different streams must not share scratch
        workspace = _default_ws.get((dev, stream))
        if workspace is None:
            if len(_default_ws) >= 16:  # a caller creating streams would keep every old workspace
                _default_ws.clear()
            workspace = _default_ws.setdefault((dev, stream), FwdAdjWorkspace())
        ws = workspace.get(ws_bytes, dev)
    st = device_status(dev)
    _lib.check(_lib.fwd_adj(
        O.data_ptr(), H, W, P.data_ptr(), M, N, tl.data_ptr(), Imeas.data_ptr(), F,
        bt.data_ptr() if bt is not None else None, B, int(loss_code),
        lp.data_ptr() if lp is not None else None, loss_total.data_ptr(),
        dO.data_ptr() if dO is not None else None, dP.data_ptr() if dP is not None else None,
        1 if accumulate else 0, ws.data_ptr(), ws.numel(), st.data_ptr(), stream), "ptycho_fwd_adj")
    return loss_total, lp, dO, dP


class FwdAdjPlan:
    """Preallocated ``ptycho_fwd_adj`` call for a fixed problem (the training step).

    Holds the object/probe/windows/measurement tensors by reference (update
    them in place between steps), a static device buffer of ``batch_size``
    frame ids, the gradient outputs and the workspace.  ``run()`` enqueues one
    call with no host-side allocation; ``capture()`` records it into a CUDA
    graph so each step is a single graph launch (``replay()``)."""

    def __init__(self, O, P, tl, Imeas, loss_type: str, batch_size: int, want_dO: bool = True,
                 want_dP: bool = True, per_pattern: bool = False):
        if loss_type not in LOSS_CODES:
            raise ValueError(f"loss_type must be one of {tuple(LOSS_CODES)}")
        for name, x, dt in (("object", O, torch.complex64), ("probe", P, torch.complex64),
                            ("windows", tl, torch.int32), ("measurements", Imeas, torch.float32)):
            if not x.is_cuda or x.dtype != dt or not x.is_contiguous():
                raise ValueError(f"{name} must be a contiguous CUDA {dt} tensor")
        self.M, self.N = _check_probe(P)
        self.O, self.P, self.tl, self.Imeas = O, P, tl, Imeas
        self.dev = O.device
        H, W = O.shape
        F = int(tl.shape[0])
        if Imeas.shape != (F, self.M, self.N):
            raise ValueError("measurements must be [F, M, N]")
        self.B = int(batch_size)
        self.batch = torch.zeros(self.B, dtype=torch.int32, device=self.dev)
        self.loss_total = torch.zeros((), dtype=torch.float64, device=self.dev)
        self.loss_per_pattern = (torch.zeros(self.B, dtype=torch.float64, device=self.dev)
                                 if per_pattern else None)
        self.dO = torch.zeros((H, W), dtype=torch.complex64, device=self.dev) if want_dO else None
        self.dP = torch.zeros((self.M, self.N), dtype=torch.complex64, device=self.dev) if want_dP else None
        nbytes = int(_lib.lib().ptycho_fwd_adj_workspace_size(H, W, self.M, self.N, self.B))
        self.ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.dev)
        self.status = device_status(self.dev)
        ptr = lambda x: x.data_ptr() if x is not None else None  # noqa: E731
        self._args = (O.data_ptr(), H, W, P.data_ptr(), self.M, self.N, tl.data_ptr(), Imeas.data_ptr(), F,
                      self.batch.data_ptr(), self.B, LOSS_CODES[loss_type], ptr(self.loss_per_pattern),
                      self.loss_total.data_ptr(), ptr(self.dO), ptr(self.dP), 0, self.ws.data_ptr(),
                      self.ws.numel(), self.status.data_ptr())
        self.graph = None

    def set_batch(self, frame_ids) -> None:
        """Copy the next minibatch's frame ids into the static buffer (stream-ordered)."""
        self.batch.copy_(torch.as_tensor(frame_ids).to(self.dev, torch.int32), non_blocking=True)

    def run(self) -> None:
        _lib.check(_lib.fwd_adj(*self._args, _stream_handle(self.dev)), "ptycho_fwd_adj")

    def capture(self) -> None:
        self.run()  # warm: sets kernel attributes outside capture
        torch.cuda.synchronize(self.dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run()
        self.graph = g

    def replay(self) -> None:
        if self.graph is None:
            self.capture()
        self.graph.replay()


# --------------------------------------------------------------------------
# autograd
# --------------------------------------------------------------------------
class _FusedLoss(torch.autograd.Function):
    """Loss of a batch with the adjoint fused into the same kernel pass.

    forward: one ``ptycho_fwd_adj`` call computes the FP64 loss and, when any
    input needs a gradient, dO and dP; backward scales them by the incoming
    gradient (exit waves are never stored)."""

    @staticmethod
    def forward(ctx, O, P, tl, Imeas, loss_code, batch):
        need = ctx.needs_input_grad[0] or ctx.needs_input_grad[1]
        loss, _, dO, dP = fwd_adj_raw(O, P, tl, Imeas, loss_code, batch=batch, want_grad=need)
        if need:
            ctx.save_for_backward(dO, dP)
        ctx.need = need
        return loss

    @staticmethod
    def backward(ctx, g):
        if not ctx.need:
            return None, None, None, None, None, None
        dO, dP = ctx.saved_tensors
        s = g if g.dtype == torch.float64 and g.is_contiguous() else g.to(torch.float64).contiguous()
        gO = torch.empty_like(dO) if ctx.needs_input_grad[0] else None
        gP = torch.empty_like(dP) if ctx.needs_input_grad[1] else None
        # one launch scales both gradients by the upstream scalar (out of place:
        # the saved dO/dP stay valid for a second backward)
        ptr = lambda t: t.data_ptr() if t is not None else None  # noqa: E731
        _lib.check(_lib.scale_pair(
            ptr(dO if gO is not None else None), ptr(gO), 2 * dO.numel() if gO is not None else 0,
            ptr(dP if gP is not None else None), ptr(gP), 2 * dP.numel() if gP is not None else 0,
            s.data_ptr(), _stream_handle(s.device)), "ptycho_scale_pair")
        return gO, gP, None, None, None, None


def fused_loss(object_complex: torch.Tensor, probe_complex: torch.Tensor, tl: torch.Tensor,
               Imeas: torch.Tensor, loss_type: str = "smooth_L1_loss", batch=None) -> torch.Tensor:
    """Sum over the batch of the per-pattern mean loss (Recovery.py:288-307).

    ``tl`` [F, 2] int32 (tlY, tlX) and ``Imeas`` [F, M, N] float32 for all
    frames; ``batch`` [B] frame ids of this minibatch (None: all frames).
    Returns a 0-d float64 tensor; ``backward()`` deposits dO / dP (torch's
    complex convention) into the inputs that require grad."""
    code = LOSS_CODES.get(loss_type)
    if code is None:
        raise ValueError(f"loss_type must be one of {tuple(LOSS_CODES)}, got {loss_type!r}")
    if object_complex.dtype != torch.complex64 or probe_complex.dtype != torch.complex64:
        raise TypeError("object and probe must be complex64")
    if not object_complex.is_cuda:
        raise ValueError("object must be a CUDA tensor (there is no CPU path)")
    ext = _lib.torchext() if USE_TORCHEXT else None
    if ext is not None:
        # the C++ autograd node: same library calls, no Python in forward or backward
        if batch is not None and not isinstance(batch, torch.Tensor):
            batch = torch.as_tensor(batch)
        return ext.fused_loss(object_complex, probe_complex, tl, Imeas, code, batch,
                              device_status(object_complex.device))
    return _FusedLoss.apply(object_complex, probe_complex, tl, Imeas, code, batch)


class _ForwardIntensity(torch.autograd.Function):
    @staticmethod
    def forward(ctx, O, P, tl):
        ctx.save_for_backward(O, P, tl)
        return forward_intensity(O, P, tl)

    @staticmethod
    def backward(ctx, gI):
        O, P, tl = ctx.saved_tensors
        _, _, dO, dP = fwd_adj_raw(O.detach(), P.detach(), tl, gI.contiguous(), _INTENSITY_GRAD)
        return (dO if ctx.needs_input_grad[0] else None,
                dP if ctx.needs_input_grad[1] else None, None)


def forward_intensity_batched(O: torch.Tensor, P: torch.Tensor, tl: torch.Tensor) -> torch.Tensor:
    """Differentiable batched intensities [B, M, N] (backward through the adjoint kernel)."""
    return _ForwardIntensity.apply(O, P, tl)


def forward_imaging_model(object_complex, probe_complex, tlY, tlX, brY, brX):
    """Drop-in for utils/optics.py:102-112: ``|fftshift(fft2(P * O[tlY:brY, tlX:brX]))|^2``.

    Scalar window corners as in the reference; differentiable."""
    M = int(brY) - int(tlY)
    N = int(brX) - int(tlX)
    if (M, N) != tuple(probe_complex.shape):
        raise ValueError(f"window {(M, N)} does not match probe {tuple(probe_complex.shape)}")
    tl = torch.tensor([[int(tlY), int(tlX)]], dtype=torch.int32, device=object_complex.device)
    check_windows(tl, object_complex.shape, M, N)
    return forward_intensity_batched(object_complex, probe_complex, tl)[0]
