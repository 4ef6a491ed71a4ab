"""Complex-exponential MLP on the tcgen05 kernels -- mirrors ComplexGaborLayer2D
and ComplexMLP of the reference (models/complex_inr.py:6-82).

Constructors, parameter names and shapes match the reference module (so
``named_parameters()`` order and ``trained_models.pth`` lists are the same):
``net.0.omega_0`` / ``net.0.linear.{weight,bias}`` (real first layer),
``net.{i}.omega_0`` / ``net.{i}.linear.{weight,bias}`` (complex hidden
layers), ``net.{L+1}.{weight,bias}`` (complex output).  ``mlp.net(x)`` -- the
call ``_get_complex_output`` makes (models/complex_inr.py:308-314) -- runs
the fused forward kernel and returns the complex [N, 1] output; its backward
is the fused tensor-core backward.  Only the configuration every reference
config uses is supported (32 input features, hidden_features 64,
hidden_layers 2, one output); anything else raises.
"""
from __future__ import annotations

import torch
import torch.nn as nn

from . import _lib
from .optics import device_status


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


class ComplexGaborLayer2D(nn.Module):
    """exp(1j * omega_0 * Linear(x)) -- parameters as models/complex_inr.py:6-40."""

    def __init__(self, in_features, out_features, bias=True, is_first=False, omega0=100.0, trainable=False):
        super().__init__()
        self.is_first = is_first
        self.in_features = in_features
        dtype = torch.float if is_first else torch.cfloat
        self.omega_0 = nn.Parameter(omega0 * torch.ones(1), trainable)
        self.linear = nn.Linear(in_features, out_features, bias=bias, dtype=dtype)


def _params(net):
    layers = list(net)
    return [layers[0].linear.weight, layers[0].linear.bias, layers[0].omega_0,
            layers[1].linear.weight, layers[1].linear.bias, layers[1].omega_0,
            layers[2].linear.weight, layers[2].linear.bias, layers[2].omega_0,
            layers[3].weight, layers[3].bias]


def _f32(t):
    t = t.detach()
    if t.is_complex():
        t = torch.view_as_real(t.contiguous())
    return t.contiguous().float()


def _is_planar(x: torch.Tensor) -> bool:
    """[N, 32] float32 view of a feature-major [32, N] buffer (the encoder's output)."""
    return (x.dim() == 2 and x.shape[1] == 32 and x.shape[0] > 1 and x.stride() == (1, x.shape[0])
            and x.dtype == torch.float32)


class _CmlpFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, *params):
        L = _lib.lib()
        dev = x.device
        flat = [_f32(p) for p in params]
        packed = torch.empty(int(L.ptycho_cmlp_packed_bytes()), dtype=torch.uint8, device=dev)
        _lib.check(L.ptycho_cmlp_pack(*[f.data_ptr() for f in flat], packed.data_ptr(), _stream(dev)),
                   "ptycho_cmlp_pack")
        N = x.shape[0]
        y = torch.empty((N,), dtype=torch.complex64, device=dev)
        st = device_status(dev)
        planar = _is_planar(x)
        fwd = L.ptycho_cmlp_forward_planar if planar else L.ptycho_cmlp_forward
        _lib.check(fwd(packed.data_ptr(), x.data_ptr(), N, y.data_ptr(), st.data_ptr(), _stream(dev)),
                   "ptycho_cmlp_forward")
        ctx.planar = planar
        ctx.save_for_backward(x, packed)
        ctx.shapes = [(p.shape, p.dtype) for p in params]
        return y.unsqueeze(1)

    @staticmethod
    def backward(ctx, gy):
        L = _lib.lib()
        x, packed = ctx.saved_tensors
        dev = x.device
        N = x.shape[0]
        gy = gy.reshape(N).to(torch.complex64).contiguous()
        grad = torch.empty(int(L.ptycho_cmlp_grad_floats()), dtype=torch.float32, device=dev)
        ws = torch.empty(int(L.ptycho_cmlp_backward_workspace_size(N)), dtype=torch.uint8, device=dev)
        st = device_status(dev)
        gx = None
        if ctx.planar:
            # features came feature-major from the encoder: gx goes back the same way
            # ([32, N], handed on as its [N, 32] transpose view, read coalesced there)
            gxT = torch.empty((32, N), dtype=torch.float32, device=dev) if ctx.needs_input_grad[0] else None
            _lib.check(L.ptycho_cmlp_backward_planar(packed.data_ptr(), x.data_ptr(), gy.data_ptr(), N,
                                                     gxT.data_ptr() if gxT is not None else None,
                                                     grad.data_ptr(), None, ws.data_ptr(), ws.numel(),
                                                     st.data_ptr(), _stream(dev)), "ptycho_cmlp_backward_planar")
            gx = gxT.t() if gxT is not None else None
        else:
            gx = torch.empty((N, 32), dtype=torch.float32, device=dev) if ctx.needs_input_grad[0] else None
            _lib.check(L.ptycho_cmlp_backward(packed.data_ptr(), x.data_ptr(), gy.data_ptr(), N,
                                              gx.data_ptr() if gx is not None else None, grad.data_ptr(), None,
                                              ws.data_ptr(), ws.numel(), st.data_ptr(), _stream(dev)),
                       "ptycho_cmlp_backward")
        cplx = lambda o, n: torch.view_as_complex(grad[o:o + 2 * n].view(-1, 2))  # noqa: E731
        g = [grad[0:1024].view(32, 32), grad[1024:1056], grad[1056:1057],
             cplx(1058, 1024).view(32, 32), cplx(3106, 32), grad[3170:3171],
             cplx(3172, 1024).view(32, 32), cplx(5220, 32), grad[5284:5285],
             cplx(5286, 32).view(1, 32), cplx(5350, 1)]
        out = [gx]
        for k, (shape, dtype) in enumerate(ctx.shapes):
            out.append(g[k].reshape(shape).to(dtype) if ctx.needs_input_grad[k + 1] else None)
        return tuple(out)


class _FusedSequential(nn.Sequential):
    """The reference's ``self.net``: same children, forward = fused kernel."""

    def forward(self, x):  # noqa: D401
        if not x.is_cuda:
            raise ValueError("features must be a CUDA tensor (there is no CPU path)")
        x = x.float()
        if not _is_planar(x):
            x = x.contiguous()
        return _CmlpFn.apply(x, *_params(self))


class ComplexMLP(nn.Module):
    """models/complex_inr.py:42-82 with the fused tensor-core forward/backward."""

    def __init__(self, in_features, hidden_features, hidden_layers, out_features, first_omega_0=10,
                 hidden_omega_0=10.0, trainable_omega0=False):
        super().__init__()
        if (in_features, hidden_features, hidden_layers, out_features) != (32, 64, 2, 1):
            raise NotImplementedError(
                "the fused complex MLP supports in_features=32, hidden_features=64, hidden_layers=2, "
                f"out_features=1; got {(in_features, hidden_features, hidden_layers, out_features)}")
        h = int(hidden_features / 2)
        net = [ComplexGaborLayer2D(in_features, h, omega0=first_omega_0, is_first=True,
                                   trainable=trainable_omega0)]
        for _ in range(hidden_layers):
            net.append(ComplexGaborLayer2D(h, h, omega0=hidden_omega_0, trainable=trainable_omega0))
        net.append(nn.Linear(h, out_features, dtype=torch.cfloat))
        self.net = _FusedSequential(*net)

    def forward(self, coords):
        return self.net(coords).real
