"""B200-native (sm_100a) far-field ptychography: fused forward model / loss /
adjoint kernels behind a C ABI (``include/ptycho_b200.h``), with host code
mirroring the reference's ``utils/optics.py`` and ``Recovery.py`` interfaces.

The directory name is not a Python identifier; import it with
``importlib.import_module("conventional-ptychography-reconstruction_b200")``.
"""
from . import _lib, optics, synth
from . import accuracy, adam, cmlp, complex_inr, gsplat, h5mat, hashgrid, probe_prep, resample, scan_shards
from ._lib import PtychoError
from .adam import FusedAdam
from .complex_inr import ComplexINRModel2D
from .hashgrid import Encoding
from .optics import (LOSS_CODES, forward_imaging_model, forward_intensity, forward_intensity_batched,
                     fused_loss, fwd_adj_raw, make_windows, check_windows, read_status,
                     scan_positions_to_pixels)

__all__ = ["PtychoError", "FusedAdam", "ComplexINRModel2D", "Encoding", "LOSS_CODES", "forward_imaging_model", "forward_intensity", "forward_intensity_batched",
           "fused_loss", "fwd_adj_raw", "make_windows", "check_windows", "read_status",
           "scan_positions_to_pixels", "lib"]


def lib():
    """The loaded ``libptycho_b200.so`` (ctypes)."""
    return _lib.lib()
