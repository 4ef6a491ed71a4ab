"""ctypes binding of the C ABI in ``include/ptycho_b200.h``.

The shared library ``libptycho_b200.so`` is built in-tree by ``csrc/build.py``.
There is no fallback: if the library is missing or a call fails, a
``RuntimeError`` is raised.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libptycho_b200.so")

_c_int, _c_size, _vp = ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p
_c_uint, _c_float, _c_double = ctypes.c_uint, ctypes.c_float, ctypes.c_double
_c_ll = ctypes.c_longlong
_pp = ctypes.POINTER(ctypes.c_void_p)

# name -> (restype, argtypes); every entry is declared in include/ptycho_b200.h
SIGNATURES = {
    "ptycho_status_string": (ctypes.c_char_p, [_c_int]),
    "ptycho_version": (_c_int, []),
    "ptycho_forward_intensity": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int, _c_int, _vp, _c_int, _vp,
                                          _c_int, _vp, _vp, _vp]),
    "ptycho_forward_intensity_workspace_size": (_c_size, [_c_int, _c_int, _c_int]),
    "ptycho_forward_intensity_ws": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int, _c_int, _vp, _c_int, _vp,
                                             _c_int, _vp, _vp, _c_size, _vp, _vp]),
    "ptycho_fwd_adj_workspace_size": (_c_size, [_c_int, _c_int, _c_int, _c_int, _c_int]),
    "ptycho_fwd_adj": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int, _c_int, _vp, _vp, _c_int, _vp, _c_int,
                                _c_int, _vp, _vp, _vp, _vp, _c_uint, _vp, _c_size, _vp, _vp]),
    "ptycho_fourier_upsample_workspace_size": (_c_size, [_c_int, _c_int, _c_int]),
    "ptycho_fourier_upsample": (_c_int, [_vp, _c_int, _c_int, _c_int, _vp, _vp, _c_size, _vp]),
    "ptycho_fourier_upsample_adjoint": (_c_int, [_vp, _c_int, _c_int, _c_int, _vp, _vp, _c_size, _vp]),
    "ptycho_probe_center_normalize": (_c_int, [_vp, _c_int, _c_int, _vp, _vp, _vp]),
    "ptycho_probe_center_normalize_backward": (_c_int, [_vp, _vp, _vp, _c_int, _c_int, _vp, _vp]),
    "ptycho_haar_sparsity_workspace_size": (_c_size, [_c_int, _c_int]),
    "ptycho_haar_sparsity": (_c_int, [_vp, _c_int, _c_int, _vp, _vp, _c_size, _vp]),
    "ptycho_haar_sparsity_backward": (_c_int, [_vp, _c_int, _c_int, _vp, _vp, _vp]),
    "ptycho_object_error_workspace_size": (_c_size, []),
    "ptycho_object_error": (_c_int, [_vp, _vp, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _vp, _vp, _c_size,
                                     _vp]),
    "ptycho_gs_workspace_size": (_c_size, [_c_int, _c_int, _c_int]),
    "ptycho_gs_forward": (_c_int, [_c_int, _vp, _vp, _vp, _vp, _c_int, _c_int, _c_int, _c_int, _c_float, _vp, _vp,
                                   _vp, _c_size, _vp]),
    "ptycho_gs_backward": (_c_int, [_c_int, _vp, _vp, _vp, _vp, _c_int, _c_int, _c_int, _c_int, _c_float, _vp, _vp,
                                    _c_size, _vp, _vp, _vp, _vp, _vp]),
    "ptycho_scale_pair": (_c_int, [_vp, _vp, _c_ll, _vp, _vp, _c_ll, _vp, _vp]),
    "ptycho_residual_workspace_size": (_c_size, []),
    "ptycho_residual": (_c_int, [_vp, _vp, _vp, _c_ll, _vp, _vp]),
    "ptycho_residual_backward": (_c_int, [_vp, _vp, _vp, _c_ll, _vp, _vp, _vp, _c_size, _vp]),
    "ptycho_hashgrid_entries": (_c_int, [_c_int, _c_int, _c_int, _c_float]),
    "ptycho_hashgrid_forward": (_c_int, [_vp, _c_int, _vp, _c_int, _c_int, _c_int, _c_float, _vp, _vp]),
    "ptycho_hashgrid_forward_planar": (_c_int, [_vp, _c_int, _vp, _c_int, _c_int, _c_int, _c_float, _vp, _vp]),
    "ptycho_hashgrid_contrib": (_c_int, [_vp, _c_int, _c_int, _c_int, _c_int, _c_float, _vp, _vp, _vp, _vp]),
    "ptycho_hashgrid_segments": (_c_int, [_vp, _c_ll, _c_int, _vp, _vp]),
    "ptycho_hashgrid_backward": (_c_int, [_vp, _vp, _vp, _vp, _c_int, _c_int, _c_int, _c_int, _c_float, _vp,
                                          _c_int, _vp]),
    "ptycho_hashgrid_backward_planar": (_c_int, [_vp, _vp, _vp, _vp, _c_int, _c_int, _c_int, _c_int, _c_float,
                                                 _vp, _c_int, _vp]),
    "ptycho_hashgrid_grid_scratch_size": (_c_size, [_vp, _c_int, _c_int, _c_int]),
    "ptycho_hashgrid_backward_grid": (_c_int, [_vp, _vp, _vp, _c_int, _c_int, _vp, _c_int, _c_int, _c_int, _c_int,
                                               _c_float, _vp, _c_int, _vp, _c_size, _vp]),
    "ptycho_cmlp_packed_bytes": (_c_size, []),
    "ptycho_cmlp_grad_floats": (_c_int, []),
    "ptycho_cmlp_pack": (_c_int, [_vp] * 12 + [_vp]),
    "ptycho_cmlp_forward": (_c_int, [_vp, _vp, _c_int, _vp, _vp, _vp]),
    "ptycho_cmlp_forward_planar": (_c_int, [_vp, _vp, _c_int, _vp, _vp, _vp]),
    "ptycho_cmlp_backward_workspace_size": (_c_size, [_c_int]),
    "ptycho_cmlp_backward": (_c_int, [_vp, _vp, _vp, _c_int, _vp, _vp, _vp, _vp, _c_size, _vp, _vp]),
    "ptycho_cmlp_backward_planar": (_c_int, [_vp, _vp, _vp, _c_int, _vp, _vp, _vp, _vp, _c_size, _vp, _vp]),
    "ptycho_adam_step": (_c_int, [_pp, _pp, _pp, _pp, ctypes.POINTER(_c_ll), _c_int, _c_int, _c_float, _c_float,
                                  _c_float, _c_float, _vp]),
    "ptycho_adam_step_dev": (_c_int, [_pp, _pp, _pp, _pp, ctypes.POINTER(_c_ll), _c_int, _vp, _vp, _c_float,
                                      _c_float, _c_float, _vp]),
    "ptycho_fwd_adj_noalloc": (_c_int, [_vp, _c_int, _c_int, _vp, _c_int, _c_int, _vp, _vp, _c_int, _vp,
                                        _c_int, _c_int, _vp, _vp, _vp, _vp, _c_uint, _vp, _vp]),
}

_lock = threading.Lock()
_lib = None


def lib() -> ctypes.CDLL:
    """Load (once) and return the library with all signatures declared."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with "
                    "`python conventional-ptychography-reconstruction_b200/csrc/build.py` "
                    "(or __graft_entry__.build()); there is no CPU fallback")
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _bind_fast(L)
            _lib = L
    return _lib


# The per-minibatch entry points through the CPython fast-call module when it
# is built (csrc/fastabi.c: no per-argument ctypes conversion), else through
# ctypes.  Both call the same functions of the one loaded libptycho_b200.so.
_fast = None


def _bind_fast(L) -> None:
    global _fast
    try:
        from . import _fastabi
    except ImportError:
        _fast = None
        return
    addr = lambda f: ctypes.cast(f, ctypes.c_void_p).value  # noqa: E731
    _fastabi.bind(addr(L.ptycho_fwd_adj), addr(L.ptycho_scale_pair))
    _fast = _fastabi


_torchext = None
_torchext_tried = False


def torchext():
    """The fused loss's C++ autograd node (csrc/torch_ext.cpp) bound to this
    process's library, or None when it is not built."""
    global _torchext, _torchext_tried
    if _torchext_tried:
        return _torchext
    L = lib()
    with _lock:
        if not _torchext_tried:
            try:
                from . import _torchext as m
            except ImportError:
                m = None
            if m is not None:
                addr = lambda f: ctypes.cast(f, ctypes.c_void_p).value  # noqa: E731
                m.bind(addr(L.ptycho_fwd_adj), addr(L.ptycho_scale_pair), addr(L.ptycho_fwd_adj_workspace_size),
                       addr(L.ptycho_status_string))
            _torchext = m
            _torchext_tried = True
    return _torchext


def fwd_adj(*args) -> int:
    """ptycho_fwd_adj with the argument list of include/ptycho_b200.h."""
    lib()
    if _fast is not None:
        return _fast.fwd_adj(*args)
    return _lib.ptycho_fwd_adj(*args)


def scale_pair(*args) -> int:
    """ptycho_scale_pair with the argument list of include/ptycho_b200.h."""
    lib()
    if _fast is not None:
        return _fast.scale_pair(*args)
    return _lib.ptycho_scale_pair(*args)


class PtychoError(RuntimeError):
    """A non-zero ptycho_status returned by the library."""

    def __init__(self, code: int, where: str):
        msg = lib().ptycho_status_string(code).decode()
        super().__init__(f"{where}: {msg} (status {code})")
        self.code = code


def check(code: int, where: str) -> None:
    if code != 0:
        raise PtychoError(code, where)


STATUS = {0: "ok", 1: "invalid argument", 2: "unsupported size", 3: "misaligned pointer",
          4: "workspace too small", 5: "CUDA launch failed", 6: "scan window outside the canvas",
          7: "bounded wait timed out"}
