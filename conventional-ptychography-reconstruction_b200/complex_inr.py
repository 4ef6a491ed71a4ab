"""ComplexINRModel2D on the B200 kernels -- mirrors models/complex_inr.py:85-334.

Same constructor, attributes (``xy_coords``, ``probe_coords``,
``k_object``, ``k_probe``, ``has_*_residual``, ``downsampled_*``) and
``forward() -> (object_complex [W, H], probe_complex [Wp, Hp] or None)``.
The hash encoders are :class:`hashgrid.Encoding` (tiny-cuda-nn's interface),
the MLPs :class:`cmlp.ComplexMLP` (fused tensor-core kernels) and the Fourier
upsampling of the object (models/complex_inr.py:252-271) the shared-memory
FFT resampling kernels of :mod:`resample` (any size the reference's geometry
gives: power-of-two and mixed-radix lines; no torch.fft path).
"""
from __future__ import annotations

import torch
import torch.nn as nn

from . import _lib, resample
from .cmlp import ComplexMLP
from .hashgrid import Encoding


class _Residual(torch.autograd.Function):
    """out = k * m + init on the device (``ptycho_residual``), k a real 0-d
    parameter; the backward gives k * g and sum Re(conj(g) m) in one launch."""

    @staticmethod
    def forward(ctx, k, m, init, ws):
        mm = m.to(torch.complex64).contiguous()
        ii = init.to(device=mm.device, dtype=torch.complex64).contiguous()
        kk = k.detach().to(torch.float32).contiguous()
        out = torch.empty_like(mm)
        _lib.check(_lib.lib().ptycho_residual(kk.data_ptr(), mm.data_ptr(), ii.data_ptr(), mm.numel(),
                                              out.data_ptr(), torch.cuda.current_stream(mm.device).cuda_stream),
                   "ptycho_residual")
        ctx.save_for_backward(kk, mm)
        ctx.ws, ctx.kshape = ws, k.shape
        return out

    @staticmethod
    def backward(ctx, g):
        kk, mm = ctx.saved_tensors
        gc = g.to(torch.complex64).contiguous()
        gm = torch.empty_like(mm) if ctx.needs_input_grad[1] else None
        gk = torch.empty((), dtype=torch.float32, device=mm.device)
        _lib.check(_lib.lib().ptycho_residual_backward(
            kk.data_ptr(), mm.data_ptr(), gc.data_ptr(), mm.numel(), gm.data_ptr() if gm is not None else None,
            gk.data_ptr(), ctx.ws.data_ptr(), ctx.ws.numel(), torch.cuda.current_stream(mm.device).cuda_stream),
            "ptycho_residual_backward")
        return (gk.reshape(ctx.kshape) if ctx.needs_input_grad[0] else None, gm,
                g if ctx.needs_input_grad[2] else None, None)


class ComplexINRModel2D(nn.Module):
    def __init__(self, output_width, output_height, downsample_factor, update_probe=True, probe_width=None,
                 probe_height=None, n_levels=16, n_features_per_level=2, log2_hashmap_size=19,
                 base_resolution=16, per_level_scale=1.5, first_omega_0=10.0, hidden_omega_0=10.0,
                 hidden_features=64, hidden_layers=2, trainable_omega0=False, use_residual=False,
                 object_initial=None, probe_initial=None):
        super().__init__()
        self.update_probe = update_probe
        self.use_residual = use_residual
        self.output_width = output_width
        self.output_height = output_height
        self.probe_width = probe_width if probe_width is not None else output_width
        self.probe_height = probe_height if probe_height is not None else output_height
        self.num_features = n_levels * n_features_per_level
        encoding_config = {"otype": "HashGrid", "n_levels": n_levels, "n_features_per_level": n_features_per_level,
                           "log2_hashmap_size": log2_hashmap_size, "base_resolution": base_resolution,
                           "per_level_scale": per_level_scale}
        self.xy_hash_encoder = Encoding(n_input_dims=2, encoding_config=encoding_config)
        self.probe_hash_encoder = (Encoding(n_input_dims=2, encoding_config=encoding_config.copy(), seed=7331)
                                   if update_probe else None)
        self.object_complex_mlp = ComplexMLP(self.num_features, hidden_features, hidden_layers, 1,
                                             first_omega_0=first_omega_0, hidden_omega_0=hidden_omega_0,
                                             trainable_omega0=trainable_omega0)
        self.probe_complex_mlp = (ComplexMLP(self.num_features, hidden_features, hidden_layers, 1,
                                             first_omega_0=first_omega_0, hidden_omega_0=hidden_omega_0,
                                             trainable_omega0=trainable_omega0) if update_probe else None)
        self.init_scale_grids(downsample_factor)
        if self.use_residual:
            self.init_residual_params(object_initial, probe_initial)

    def init_scale_grids(self, downsample_factor):
        """Pixel-centre coordinates; element [i, j] of the reshaped output gets
        encoder input (dim0 = (j + 0.5) / H, dim1 = (i + 0.5) / W)."""
        dw = self.output_width // downsample_factor
        dh = self.output_height // downsample_factor
        xs = torch.linspace(0.5 / dw, 1 - 0.5 / dw, dw)
        ys = torch.linspace(0.5 / dh, 1 - 0.5 / dh, dh)
        xv, yv = torch.meshgrid([xs, ys], indexing="ij")
        self.downsampled_width = dw
        self.downsampled_height = dh
        self.xy_coords = nn.Parameter(torch.stack((yv.flatten(), xv.flatten())).t().contiguous(),
                                      requires_grad=False)
        if self.update_probe:
            xs = torch.linspace(0.5 / self.probe_width, 1 - 0.5 / self.probe_width, self.probe_width)
            ys = torch.linspace(0.5 / self.probe_height, 1 - 0.5 / self.probe_height, self.probe_height)
            xv, yv = torch.meshgrid([xs, ys], indexing="ij")
            self.probe_coords = nn.Parameter(torch.stack((yv.flatten(), xv.flatten())).t().contiguous(),
                                             requires_grad=False)
        else:
            self.probe_coords = None
        self.downsample_factor = downsample_factor

    def init_residual_params(self, object_initial, probe_initial):
        """output = k * network + initial, k a real parameter initialised to 1e-8
        (models/complex_inr.py:209-250)."""
        if object_initial is not None:
            if not torch.is_complex(object_initial):
                raise ValueError("object_initial must be a complex tensor")
            self.register_buffer("object_initial", object_initial.clone())
            self.k_object = nn.Parameter(torch.tensor(1e-8, dtype=torch.float32))
            self.has_object_residual = True
        else:
            self.has_object_residual = False
        if self.update_probe and probe_initial is not None:
            if not torch.is_complex(probe_initial):
                raise ValueError("probe_initial must be a complex tensor")
            self.register_buffer("probe_initial", probe_initial.clone())
            self.k_probe = nn.Parameter(torch.tensor(1e-8, dtype=torch.float32))
            self.has_probe_residual = True
        else:
            self.has_probe_residual = False

    def fourier_upsample(self, x, scale_factor):
        """fftshift(fft2) -> zero-pad -> ifftshift -> ifft2, times scale^2 (:252-271),
        on the resampling kernels (``resample``) for every [B, C, H, W] slice.
        The scale must be a whole number (Recovery.py coerces downsample_factor
        to int); there is no torch.fft path, so other inputs raise."""
        B, C, H, W = x.shape
        if int(scale_factor) != scale_factor:
            raise ValueError(f"downsample_factor must be a whole number, got {scale_factor}")
        s = int(scale_factor)
        if not x.is_cuda or not resample.supported(H, W, s):
            raise ValueError(f"fourier_upsample: unsupported input {tuple(x.shape)} on {x.device} with scale {s}")
        if B == 1 and C == 1:
            return resample.fourier_upsample(x[0, 0], s)[None, None]
        return torch.stack([resample.fourier_upsample(x[b, c], s) for b in range(B) for c in range(C)]
                           ).reshape(B, C, H * s, W * s)

    def forward(self):
        xy = self.xy_coords if self.xy_coords.is_cuda else self.xy_coords.cuda()
        feats = self.xy_hash_encoder(xy).float()
        obj = self._get_complex_output(self.object_complex_mlp, feats)
        obj = obj.reshape(self.downsampled_width, self.downsampled_height)
        obj = self.fourier_upsample(obj.unsqueeze(0).unsqueeze(0), self.downsample_factor).squeeze(0).squeeze(0)
        if self.update_probe:
            pc = self.probe_coords if self.probe_coords.is_cuda else self.probe_coords.cuda()
            pf = self.probe_hash_encoder(pc).float()
            probe = self._get_complex_output(self.probe_complex_mlp, pf).reshape(self.probe_width,
                                                                                 self.probe_height)
        else:
            probe = None
        if self.use_residual:
            obj = self.apply_residual(obj, is_object=True)
            if self.update_probe and probe is not None:
                probe = self.apply_residual(probe, is_object=False)
        return obj, probe

    def _get_complex_output(self, model, coords):
        return model.net(coords)

    def apply_residual(self, complex_tensor, is_object=True):
        """k * network + initial (models/complex_inr.py:316-334) as one kernel
        forward and one backward (``ptycho_residual``)."""
        if is_object and not self.has_object_residual or not is_object and not self.has_probe_residual:
            return complex_tensor
        k, init = (self.k_object, self.object_initial) if is_object else (self.k_probe, self.probe_initial)
        dev = complex_tensor.device
        ws = getattr(self, "_residual_ws", None)
        if ws is None or ws.device != dev:  # zeroed once; every backward leaves it zeroed
            ws = torch.zeros(int(_lib.lib().ptycho_residual_workspace_size()), dtype=torch.uint8, device=dev)
            self._residual_ws = ws
        return _Residual.apply(k, complex_tensor, init, ws)
