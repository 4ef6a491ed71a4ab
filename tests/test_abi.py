"""The C-ABI library loads without a GPU and exports every declared symbol;
argument validation that happens before any device work returns the
documented status codes."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT, load_pkg


def _declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(ptycho_\w+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    pkg = load_pkg()
    L = pkg.lib()
    declared = _declared_symbols()
    assert declared, "no declarations found"
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    # the ctypes signature table covers exactly the declared functions
    assert set(pkg._lib.SIGNATURES) == declared


def test_status_strings_and_version():
    L = load_pkg().lib()
    assert L.ptycho_version() >= 100
    for code, text in load_pkg()._lib.STATUS.items():
        assert L.ptycho_status_string(code).decode() == text


def test_validation_before_device_work():
    L = load_pkg().lib()
    fake = ctypes.c_void_p(4096)  # never dereferenced: validation fails first
    # probe side past the general path's 4096 maximum
    assert L.ptycho_fwd_adj(fake, 8192, 8192, fake, 5000, 5000, fake, fake, 4, None, 4, 0, None, None, None,
                            None, 0, fake, 1 << 30, None, None) == 2
    assert L.ptycho_fwd_adj_workspace_size(8192, 8192, 5000, 5000, 4) == 0
    # shapes other than square 64 / 128 / 256 need the workspace entry point
    assert L.ptycho_forward_intensity(fake, 256, 256, fake, 64, 128, fake, 1, None, 1, fake, None,
                                      None) == 2
    n = L.ptycho_forward_intensity_workspace_size(96, 80, 3)
    assert n >= 3 * 96 * 80 * 8 and L.ptycho_forward_intensity_workspace_size(96, 80, -1) == 0
    assert L.ptycho_forward_intensity_ws(fake, 256, 256, fake, 96, 80, fake, 3, None, 3, fake, fake, n - 8,
                                         None, None) == 4
    assert L.ptycho_forward_intensity_ws(fake, 256, 256, fake, 96, 80, fake, 3, None, 3, fake,
                                         ctypes.c_void_p(4096 + 16), n, None, None) == 3
    # the general path's workspace holds the FD planes on top of the exit waves
    assert (L.ptycho_fwd_adj_workspace_size(256, 256, 96, 80, 8) >=
            8 * 96 * 80 * (8 + 12) + L.ptycho_fwd_adj_workspace_size(256, 256, 64, 64, 0))
    # null object
    assert L.ptycho_forward_intensity(None, 256, 256, fake, 64, 64, fake, 1, None, 1, fake, None,
                                      None) == 1
    # batch larger than the frame count without explicit frame ids
    assert L.ptycho_forward_intensity(fake, 256, 256, fake, 64, 64, fake, 1, None, 2, fake, None,
                                      None) == 1
    # bad loss type
    assert L.ptycho_fwd_adj(fake, 256, 256, fake, 64, 64, fake, fake, 4, None, 4, 9, None, None, None,
                            None, 0, fake, 1 << 30, None, None) == 1
    # workspace too small
    assert L.ptycho_fwd_adj(fake, 256, 256, fake, 64, 64, fake, fake, 4, None, 4, 0, None, None, None,
                            None, 0, fake, 16, None, None) == 4
    # misaligned object pointer
    assert L.ptycho_forward_intensity(ctypes.c_void_p(4097), 256, 256, fake, 64, 64, fake, 1, None, 1,
                                      fake, None, None) == 3


def test_fourier_upsample_validation_before_device_work():
    L = load_pkg().lib()
    st = {"INVALID_ARG": 1, "UNSUPPORTED_SIZE": 2, "MISALIGNED": 3, "WORKSPACE": 4}  # include/ptycho_b200.h
    fake = ctypes.c_void_p(4096)  # never dereferenced: validation fails first
    n = L.ptycho_fourier_upsample_workspace_size(512, 512, 2)
    assert n == 512 * 512 * 2 * 8 and L.ptycho_fourier_upsample_workspace_size(0, 8, 2) == 0
    for fn in (L.ptycho_fourier_upsample, L.ptycho_fourier_upsample_adjoint):
        assert fn(fake, 4097, 96, 2, fake, fake, n, None) == st["UNSUPPORTED_SIZE"]  # line > 8192
        assert fn(fake, 64, 2048, 8, fake, fake, n, None) == st["UNSUPPORTED_SIZE"]
        assert fn(fake, 96, 96, 0, fake, fake, n, None) == st["INVALID_ARG"]
        assert fn(None, 64, 64, 2, fake, fake, n, None) == st["INVALID_ARG"]
        assert fn(fake, 512, 512, 2, fake, fake, n - 8, None) == st["WORKSPACE"]
        assert fn(ctypes.c_void_p(4100), 512, 512, 2, fake, fake, n, None) == st["MISALIGNED"]


def test_probe_prep_and_haar_validation_before_device_work():
    L = load_pkg().lib()
    fake = ctypes.c_void_p(4096)  # never dereferenced: validation fails first
    other = ctypes.c_void_p(8192)
    assert L.ptycho_probe_center_normalize(None, 64, 64, fake, other, None) == 1
    assert L.ptycho_probe_center_normalize(fake, 64, 64, fake, other, None) == 1  # in place refused
    assert L.ptycho_probe_center_normalize(fake, 2048, 64, other, other, None) == 2
    assert L.ptycho_probe_center_normalize_backward(fake, fake, fake, 64, 64, fake, None) == 1
    assert L.ptycho_haar_sparsity_workspace_size(1536, 1536) == 1184 * 8  # grid capped at 8 CTAs per SM
    assert L.ptycho_haar_sparsity(fake, 63, 64, fake, fake, 4096, None) == 2
    assert L.ptycho_haar_sparsity(fake, 64, 64, fake, fake, 0, None) == 4
    assert L.ptycho_haar_sparsity_backward(fake, 64, 65, fake, fake, None) == 2


def test_object_error_validation_before_device_work():
    L = load_pkg().lib()
    fake = ctypes.c_void_p(4096)
    n = L.ptycho_object_error_workspace_size()
    assert n >= 4 * 8
    assert L.ptycho_object_error(None, fake, 8, 8, 0, 8, 0, 8, fake, fake, n, None) == 1
    assert L.ptycho_object_error(fake, fake, 8, 8, 0, 9, 0, 8, fake, fake, n, None) == 1  # box past the edge
    assert L.ptycho_object_error(fake, fake, 8, 8, 4, 4, 0, 8, fake, fake, n, None) == 1  # empty box
    assert L.ptycho_object_error(fake, fake, 8, 8, 0, 8, 0, 8, fake, fake, n - 8, None) == 4
    assert L.ptycho_object_error(ctypes.c_void_p(4100), fake, 8, 8, 0, 8, 0, 8, fake, fake, n, None) == 3


def test_gsplat_validation_before_device_work():
    L = load_pkg().lib()
    fake = ctypes.c_void_p(4096)
    assert L.ptycho_gs_workspace_size(0, 16, 16) == 0  # nothing to keep for no Gaussians
    assert L.ptycho_gs_workspace_size(10, 0, 16) == 0
    n = L.ptycho_gs_workspace_size(100, 64, 64)
    args = (fake, fake, fake, fake, 100, 64, 64, 16, ctypes.c_float(0.5), fake, None, fake, n, None)
    assert L.ptycho_gs_forward(2, *args) == 1  # unknown parameterisation
    assert L.ptycho_gs_forward(0, fake, fake, fake, fake, 100, 64, 64, 0, ctypes.c_float(0.5), fake, None, fake, n,
                               None) == 1  # max_patch_radius 0
    assert L.ptycho_gs_forward(0, *args[:-3], fake, n - 256, None) == 4
    assert L.ptycho_gs_forward(0, ctypes.c_void_p(4100), *args[1:]) == 3
    assert L.ptycho_gs_backward(0, fake, fake, fake, fake, 100, 64, 64, 16, ctypes.c_float(0.5), None, fake, n,
                                fake, fake, fake, fake, None) == 1


def test_scale_pair_validation_before_device_work():
    L = load_pkg().lib()
    fake = ctypes.c_void_p(4096)
    assert L.ptycho_scale_pair(fake, fake, 8, fake, fake, 8, None, None) == 1  # no scale
    assert L.ptycho_scale_pair(None, fake, 8, fake, fake, 8, fake, None) == 1
    assert L.ptycho_scale_pair(ctypes.c_void_p(4098), fake, 8, fake, fake, 8, fake, None) == 3
    assert L.ptycho_scale_pair(None, None, 0, None, None, 0, fake, None) == 0  # nothing to do


def test_residual_validation_before_device_work():
    L = load_pkg().lib()
    fake = ctypes.c_void_p(4096)
    n = L.ptycho_residual_workspace_size()
    assert L.ptycho_residual(None, fake, fake, 8, fake, None) == 1
    assert L.ptycho_residual(fake, ctypes.c_void_p(4100), fake, 8, fake, None) == 3
    assert L.ptycho_residual_backward(fake, fake, fake, 8, fake, fake, fake, n - 8, None) == 4
    assert L.ptycho_residual_backward(fake, fake, fake, 8, None, None, fake, n, None) == 1  # no gk


def test_workspace_size_monotone():
    L = load_pkg().lib()
    a = L.ptycho_fwd_adj_workspace_size(1536, 1536, 128, 128, 256)
    b = L.ptycho_fwd_adj_workspace_size(1536, 1536, 128, 128, 512)
    assert 0 < a < b
    assert a >= 256 * 128 * 128 * 8
    assert L.ptycho_fwd_adj_workspace_size(-1, 5, 64, 64, 1) == 0


def test_fast_binding_matches_ctypes_validation():
    """The CPython fast-call binding (csrc/fastabi.c) reaches the same library
    functions as ctypes: validation failures return the same status codes."""
    pkg = load_pkg()
    L = pkg.lib()
    lib = pkg._lib
    assert lib._fast is not None, "the _fastabi module was not built"
    fake = 4096
    for args in [(fake, 8192, 8192, fake, 5000, 5000, fake, fake, 4, None, 4, 0, None, None, None, None, 0, fake,
                  1 << 30, None, None),
                 (fake, 256, 256, fake, 64, 64, fake, fake, 4, None, 4, 9, None, None, None, None, 0, fake,
                  1 << 30, None, None),
                 (fake, 256, 256, fake, 64, 64, fake, fake, 4, None, 4, 0, None, None, None, None, 0, fake, 16,
                  None, None)]:
        assert lib.fwd_adj(*args) == L.ptycho_fwd_adj(*args) != 0
    assert lib.scale_pair(None, None, 0, None, None, 0, None, None) == L.ptycho_scale_pair(
        None, None, 0, None, None, 0, None, None) == 1
