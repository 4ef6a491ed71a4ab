"""HashGrid encoding on the B200 kernels -- drop-in for the tiny-cuda-nn class
the reference uses (models/complex_inr.py:4, 130-145, called at :279, :294).

``Encoding(n_input_dims=2, encoding_config={"otype": "HashGrid", ...})`` has
tiny-cuda-nn's constructor and call signature: ``enc(coords [N,2] float32 in
[0,1]) -> [N, n_levels * n_features_per_level]``.  Its single parameter
``params`` is the flat table ([entries * 2] float32, initialised U(-1e-4,
1e-4)).  The forward runs ``ptycho_hashgrid_forward``; the backward turns the
table-gradient scatter into a deterministic gather over a CSR of the static
(entry, coordinate, weight) contributions, built once per coordinate tensor.
"""
from __future__ import annotations

import torch

from . import _lib
from .optics import device_status  # noqa: F401  (shared status word helpers)


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


class _CSR:
    """Static contributions of one coordinate tensor, sorted by table entry."""

    def __init__(self, coords: torch.Tensor, cfg: tuple, n_entries: int):
        L = _lib.lib()
        N = coords.shape[0]
        n_levels = cfg[0]
        K = N * n_levels * 4
        dev = coords.device
        key = torch.empty(K, dtype=torch.int32, device=dev)
        item = torch.empty(K, dtype=torch.int32, device=dev)
        weight = torch.empty(K, dtype=torch.float32, device=dev)
        _lib.check(L.ptycho_hashgrid_contrib(coords.data_ptr(), N, *cfg, key.data_ptr(), item.data_ptr(),
                                             weight.data_ptr(), _stream(dev)), "ptycho_hashgrid_contrib")
        skey, order = torch.sort(key, stable=True)  # one-time set-up, deterministic order
        self.item = item[order].contiguous()
        self.weight = weight[order].contiguous()
        # the same items addressed into a feature-major [2L][N] gradient (2*l*N + n),
        # for ptycho_hashgrid_backward_planar; the order is unchanged
        self.n = N
        self.item_planar = None
        if 2 * n_levels * N < 2 ** 31:
            it = self.item.long()
            self.item_planar = (2 * (it % n_levels) * N + it // n_levels).to(torch.int32).contiguous()
        self.start = torch.empty(n_entries + 1, dtype=torch.int32, device=dev)
        _lib.check(L.ptycho_hashgrid_segments(skey.data_ptr(), K, n_entries, self.start.data_ptr(),
                                              _stream(dev)), "ptycho_hashgrid_segments")


class _HashFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, params, enc):
        N = coords.shape[0]
        # features are produced feature-major ([L*F, N], coalesced) and returned as
        # the [N, L*F] transpose view; the MLP kernels read that layout directly
        outT = torch.empty((enc.n_output_dims, N), dtype=torch.float32, device=coords.device)
        _lib.check(_lib.lib().ptycho_hashgrid_forward_planar(coords.data_ptr(), N, params.data_ptr(), *enc.cfg,
                                                             outT.data_ptr(), _stream(coords.device)),
                   "ptycho_hashgrid_forward_planar")
        ctx.enc = enc
        ctx.save_for_backward(coords)
        return outT.t()

    @staticmethod
    def backward(ctx, gout):
        coords, = ctx.saved_tensors  # raises if coords were modified in place after the forward
        enc = ctx.enc
        csr = enc._csr_for(coords)
        N = coords.shape[0]
        dtable = torch.empty(enc.n_entries * 2, dtype=torch.float32, device=coords.device)
        if (csr.item_planar is not None and gout.dtype == torch.float32 and gout.dim() == 2 and N > 1
                and gout.stride() == (1, N)):
            # feature-major gradient (the MLP backward's planar output): coalesced gathers
            _lib.check(_lib.lib().ptycho_hashgrid_backward_planar(
                csr.start.data_ptr(), csr.item_planar.data_ptr(), csr.weight.data_ptr(), gout.data_ptr(), N,
                *enc.cfg, dtable.data_ptr(), 0, _stream(coords.device)), "ptycho_hashgrid_backward_planar")
            return None, dtable, None
        gout = gout.contiguous().float()
        _lib.check(_lib.lib().ptycho_hashgrid_backward(
            csr.start.data_ptr(), csr.item.data_ptr(), csr.weight.data_ptr(), gout.data_ptr(),
            N, *enc.cfg, dtable.data_ptr(), 0, _stream(coords.device)), "ptycho_hashgrid_backward")
        return None, dtable, None


class Encoding(torch.nn.Module):
    """Multi-resolution hash encoding with tiny-cuda-nn's interface (2-D inputs)."""

    def __init__(self, n_input_dims: int, encoding_config: dict, seed: int = 1337, dtype=None):
        super().__init__()
        if n_input_dims != 2:
            raise NotImplementedError("only 2-D inputs are supported")
        cfg = dict(encoding_config)
        if cfg.get("otype", "HashGrid") != "HashGrid":
            raise NotImplementedError(f"encoding {cfg.get('otype')!r} is not supported")
        if int(cfg.get("n_features_per_level", 2)) != 2:
            raise NotImplementedError("n_features_per_level must be 2")
        self.n_levels = int(cfg.get("n_levels", 16))
        self.log2_hashmap_size = int(cfg.get("log2_hashmap_size", 19))
        self.base_resolution = int(cfg.get("base_resolution", 16))
        self.per_level_scale = float(cfg.get("per_level_scale", 2.0))
        self.n_input_dims = 2
        self.n_output_dims = self.n_levels * 2
        self.cfg = (self.n_levels, self.log2_hashmap_size, self.base_resolution, self.per_level_scale)
        n = int(_lib.lib().ptycho_hashgrid_entries(*self.cfg))
        if n <= 0:
            raise ValueError(f"invalid HashGrid configuration {cfg}")
        self.n_entries = n
        g = torch.Generator().manual_seed(seed)
        self.params = torch.nn.Parameter(torch.rand(n * 2, generator=g) * 2e-4 - 1e-4)
        self._csr = []

    def _csr_for(self, coords: torch.Tensor) -> _CSR:
        """The static contribution CSR of ``coords``, cached per coordinate buffer.

        An entry holds a reference to the coordinate tensor, so its memory cannot
        be taken by another tensor while cached, and matches on address, shape,
        strides and version counter (shared by aliases): new coordinates, or the
        same buffer modified in place, get a fresh CSR.  Fixed coordinates (an
        INR's pixel grid) build it once."""
        key = (coords.data_ptr(), tuple(coords.shape), tuple(coords.stride()), coords.device)
        for k, t, ver, csr in self._csr:
            if k == key and t._version == ver and coords._version == ver:
                return csr
        csr = _CSR(coords, self.cfg, self.n_entries)
        self._csr = self._csr[-3:] + [(key, coords, coords._version, csr)]
        return csr

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        if not x.is_cuda:
            raise ValueError("coordinates must be a CUDA tensor (there is no CPU path)")
        x = x.float().contiguous()
        return _HashFn.apply(x, self.params, self)
