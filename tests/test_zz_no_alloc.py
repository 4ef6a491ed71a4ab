"""The allocation-free entry point ptycho_fwd_adj_noalloc.

Some callers of this library cannot allocate device memory when they run a
training step -- an FFI host (Go, Java, a control loop) with no CUDA
allocator of its own, or a step that must not pay an allocation's implicit
device synchronisation.  ptycho_fwd_adj_noalloc serves them from a 48 MiB
static scratch array inside the library.  This test calls it through the C
ABI, twice in a row with different batches (the shared array keeps the first
call's contents), and checks each result against ptycho_fwd_adj with a
caller-provided workspace, within the tolerances the other GPU tests use.
It also checks that a batch needing more than 48 MiB of scratch is refused.
"""
import numpy as np
import pytest
import torch

from conftest import load_pkg

pytestmark = pytest.mark.gpu


def _rel_max(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def test_noalloc_matches_workspace_entry_point_on_two_calls():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    pkg = load_pkg()
    L = pkg.lib()
    dev = torch.device("cuda", torch.cuda.current_device())
    rng = np.random.default_rng(7)
    H, W, M, F = 520, 600, 128, 48
    O = torch.from_numpy(((0.6 + 0.4 * rng.random((H, W))) *
                          np.exp(1j * rng.random((H, W)))).astype(np.complex64)).to(dev)
    P = torch.from_numpy((rng.standard_normal((M, M)) + 1j * rng.standard_normal((M, M)))
                         .astype(np.complex64)).to(dev)
    tl = pkg.make_windows(rng.integers(0, H - M + 1, F), rng.integers(0, W - M + 1, F), dev)
    stack = torch.from_numpy(rng.poisson(50.0, size=(F, M, M)).astype(np.float32)).to(dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call, (loss_code, n) in enumerate([(2, 24), (0, 31)]):
        batch = torch.from_numpy(rng.permutation(F)[:n].astype(np.int32)).to(dev)
        ref_loss, ref_lp, ref_dO, ref_dP = pkg.fwd_adj_raw(O, P, tl, stack, loss_code, batch=batch,
                                                           per_pattern=True)
        loss = torch.zeros((), dtype=torch.float64, device=dev)
        lp = torch.zeros(n, dtype=torch.float64, device=dev)
        dO = torch.zeros((H, W), dtype=torch.complex64, device=dev)
        dP = torch.zeros((M, M), dtype=torch.complex64, device=dev)
        rc = L.ptycho_fwd_adj_noalloc(O.data_ptr(), H, W, P.data_ptr(), M, M, tl.data_ptr(),
                                      stack.data_ptr(), F, batch.data_ptr(), n, loss_code, lp.data_ptr(),
                                      loss.data_ptr(), dO.data_ptr(), dP.data_ptr(), 0, status.data_ptr(),
                                      stream)
        assert rc == 0, (call, L.ptycho_status_string(rc))
        torch.cuda.synchronize(dev)
        assert int(status.item()) == 0
        assert abs(float(loss) - float(ref_loss)) <= 2e-5 * abs(float(ref_loss)), call
        np.testing.assert_allclose(lp.cpu().numpy(), ref_lp.cpu().numpy(), rtol=2e-5)
        assert _rel_max(dO.cpu().numpy(), ref_dO.cpu().numpy()) <= 2e-4, call
        assert _rel_max(dP.cpu().numpy(), ref_dP.cpu().numpy()) <= 2e-4, call

    # a batch whose scratch exceeds the 48 MiB array is refused before any device work
    big = 400
    assert L.ptycho_fwd_adj_workspace_size(H, W, M, M, big) > (48 << 20)
    rc = L.ptycho_fwd_adj_noalloc(O.data_ptr(), H, W, P.data_ptr(), M, M, tl.data_ptr(), stack.data_ptr(),
                                  F, batch.data_ptr(), big, 2, None, loss.data_ptr(), dO.data_ptr(),
                                  dP.data_ptr(), 0, status.data_ptr(), stream)
    assert rc == 4  # PTYCHO_ERR_WORKSPACE
