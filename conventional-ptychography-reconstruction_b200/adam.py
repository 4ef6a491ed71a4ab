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
    """``capturable=True`` keeps each group's step counter and learning rate in
    device memory (``ptycho_adam_step_dev``) so ``step()`` can be captured in a
    CUDA graph; call ``sync_lr()`` after changing a group's lr (e.g. after
    ``StepLR.step()``).  In that mode every parameter of a group must receive a
    gradient at every step (they share one counter)."""

    def __init__(self, params, lr=1e-3, betas=(0.9, 0.999), eps=1e-8, weight_decay=0.0, amsgrad=False,
                 capturable=False):
        if weight_decay != 0.0 or amsgrad:
            raise NotImplementedError("weight_decay and amsgrad are not supported")
        super().__init__(params, dict(lr=lr, betas=betas, eps=eps))
        self.capturable = capturable
        self._dev = []
        if capturable:
            for g in self.param_groups:
                dev = g["params"][0].device
                self._dev.append({"step": torch.zeros(1, dtype=torch.int32, device=dev),
                                  "lr": torch.tensor([g["lr"]], dtype=torch.float32, device=dev)})

    def sync_lr(self):
        """Copy each group's current lr into its device copy (capturable mode)."""
        for g, d in zip(self.param_groups, self._dev):
            d["lr"].fill_(float(g["lr"]))

    @torch.no_grad()
    def _step_capturable(self):
        L = _lib.lib()
        for group, d in zip(self.param_groups, self._dev):
            ps = [p for p in group["params"] if p.grad is not None]
            if not ps:
                continue
            if len(ps) > 48:
                raise ValueError("capturable FusedAdam handles at most 48 tensors per group")
            for p in ps:
                st = self.state[p]
                if not st:
                    st["exp_avg"] = torch.zeros_like(p, memory_format=torch.contiguous_format)
                    st["exp_avg_sq"] = torch.zeros_like(p, memory_format=torch.contiguous_format)
            grads = [_real(p.grad).contiguous() for p in ps]
            n = len(ps)
            arr = lambda xs: ctypes.cast((ctypes.c_void_p * n)(*xs), ctypes.POINTER(ctypes.c_void_p))  # noqa: E731
            N = (ctypes.c_longlong * n)(*[_real(p).numel() for p in ps])
            b1, b2 = group["betas"]
            _lib.check(L.ptycho_adam_step_dev(
                arr([_real(p).data_ptr() for p in ps]), arr([g.data_ptr() for g in grads]),
                arr([_real(self.state[p]["exp_avg"]).data_ptr() for p in ps]),
                arr([_real(self.state[p]["exp_avg_sq"]).data_ptr() for p in ps]), N, n, d["step"].data_ptr(),
                d["lr"].data_ptr(), float(b1), float(b2), float(group["eps"]),
                torch.cuda.current_stream(ps[0].device).cuda_stream), "ptycho_adam_step_dev")

    @torch.no_grad()
    def step(self, closure=None):
        loss = None
        if closure is not None:
            with torch.enable_grad():
                loss = closure()
        if self.capturable:
            self._step_capturable()
            return loss
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
