"""Fused Adam on the B200 kernel -- drop-in for the torch.optim.Adam of
Recovery.py:238-241 (stepped at :321, scheduled by StepLR at :350).

Same constructor (``params, lr, betas, eps``) and ``step()``; one
``ptycho_adam_step`` launch updates every parameter of a group (up to 48
tensors per launch).  Complex parameters are updated through their real view,
which gives real and imaginary parts independent moments exactly as
torch.optim.Adam does.  weight_decay, amsgrad and maximize are not part of the
reference path and are rejected.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib


def _real(t):
    return torch.view_as_real(t) if t.is_complex() else t


class FusedAdam(torch.optim.Optimizer):
    def __init__(self, params, lr=1e-3, betas=(0.9, 0.999), eps=1e-8, weight_decay=0.0, amsgrad=False):
        if weight_decay != 0.0 or amsgrad:
            raise NotImplementedError("weight_decay and amsgrad are not supported")
        super().__init__(params, dict(lr=lr, betas=betas, eps=eps))

    @torch.no_grad()
    def step(self, closure=None):
        loss = None
        if closure is not None:
            with torch.enable_grad():
                loss = closure()
        L = _lib.lib()
        for group in self.param_groups:
            ps = [p for p in group["params"] if p.grad is not None]
            if not ps:
                continue
            for p in ps:
                if not p.is_cuda or p.dtype not in (torch.float32, torch.complex64):
                    raise TypeError("FusedAdam needs float32 / complex64 CUDA parameters")
                st = self.state[p]
                if not st:
                    st["step"] = 0
                    st["exp_avg"] = torch.zeros_like(p, memory_format=torch.contiguous_format)
                    st["exp_avg_sq"] = torch.zeros_like(p, memory_format=torch.contiguous_format)
                st["step"] += 1
            b1, b2 = group["betas"]
            by_step: dict = {}
            for p in ps:  # parameters with equal step counts share a launch
                by_step.setdefault(self.state[p]["step"], []).append(p)
            chunks = [(st, lst[i:i + 48]) for st, lst in by_step.items() for i in range(0, len(lst), 48)]
            for step, chunk in chunks:
                grads = [_real(p.grad).contiguous() for p in chunk]
                n = len(chunk)
                P = (ctypes.c_void_p * n)(*[_real(p).data_ptr() for p in chunk])
                G = (ctypes.c_void_p * n)(*[g.data_ptr() for g in grads])
                M = (ctypes.c_void_p * n)(*[_real(self.state[p]["exp_avg"]).data_ptr() for p in chunk])
                V = (ctypes.c_void_p * n)(*[_real(self.state[p]["exp_avg_sq"]).data_ptr() for p in chunk])
                N = (ctypes.c_longlong * n)(*[_real(p).numel() for p in chunk])
                dev = chunk[0].device
                _lib.check(L.ptycho_adam_step(ctypes.cast(P, ctypes.POINTER(ctypes.c_void_p)),
                                              ctypes.cast(G, ctypes.POINTER(ctypes.c_void_p)),
                                              ctypes.cast(M, ctypes.POINTER(ctypes.c_void_p)),
                                              ctypes.cast(V, ctypes.POINTER(ctypes.c_void_p)), N, n, step,
                                              float(group["lr"]), float(b1), float(b2), float(group["eps"]),
                                              torch.cuda.current_stream(dev).cuda_stream), "ptycho_adam_step")
        return loss
