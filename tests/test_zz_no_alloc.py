"""The allocation-free entry point ptycho_fwd_adj_noalloc.

Some callers of this library cannot allocate device memory when they run a
training step -- an FFI host (Go, Java, a control loop) with no CUDA
allocator of its own, or a step that must not pay an allocation's implicit
device synchronisation.  ptycho_fwd_adj_noalloc serves them from a 48 MiB
static scratch array inside the library.  These tests call it through the C
ABI, for each probe size, twice in a row with different batches (the shared
array keeps the first call's contents), and check each result against
ptycho_fwd_adj with a caller-provided workspace, within the tolerances the
other GPU tests use.  They also check the size limit at each probe size's
own boundary (the largest batch whose scratch fits runs, one more pattern is
refused) and that arguments the workspace entry point refuses get its status.
"""
import numpy as np
import pytest
import torch

from conftest import load_pkg

pytestmark = pytest.mark.gpu

SCRATCH = 48 << 20
WORKSPACE_TOO_SMALL, INVALID_ARG = 4, 1


def _rel_max(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def _largest_batch(L, H, W, M):
    b = 1
    while L.ptycho_fwd_adj_workspace_size(H, W, M, M, b + 1) <= SCRATCH:
        b += 1
    return b


def _call(L, O, H, W, P, M, tl, stack, F, batch, n, loss_code, lp, loss, dO, dP, status, stream):
    return L.ptycho_fwd_adj_noalloc(O.data_ptr(), H, W, P.data_ptr(), M, M, tl.data_ptr(), stack.data_ptr(), F,
                                    batch.data_ptr(), n, loss_code, lp.data_ptr() if lp is not None else None,
                                    loss.data_ptr(), dO.data_ptr(), dP.data_ptr(), 0, status.data_ptr(), stream)


def _check_against_workspace_entry(pkg, L, O, H, W, P, M, tl, stack, F, batch, loss_code, status, stream, tag):
    n = int(batch.numel())
    dev = O.device
    ref_loss, ref_lp, ref_dO, ref_dP = pkg.fwd_adj_raw(O, P, tl, stack, loss_code, batch=batch, per_pattern=True)
    loss = torch.zeros((), dtype=torch.float64, device=dev)
    lp = torch.zeros(n, dtype=torch.float64, device=dev)
    dO = torch.zeros((H, W), dtype=torch.complex64, device=dev)
    dP = torch.zeros((M, M), dtype=torch.complex64, device=dev)
    rc = _call(L, O, H, W, P, M, tl, stack, F, batch, n, loss_code, lp, loss, dO, dP, status, stream)
    assert rc == 0, (tag, L.ptycho_status_string(rc))
    torch.cuda.synchronize(dev)
    assert int(status.item()) == 0, tag
    assert abs(float(loss) - float(ref_loss)) <= 2e-5 * abs(float(ref_loss)), tag
    np.testing.assert_allclose(lp.cpu().numpy(), ref_lp.cpu().numpy(), rtol=2e-5)
    assert _rel_max(dO.cpu().numpy(), ref_dO.cpu().numpy()) <= 2e-4, tag
    assert _rel_max(dP.cpu().numpy(), ref_dP.cpu().numpy()) <= 2e-4, tag


@pytest.mark.parametrize("M, H, W, calls", [
    (64, 300, 340, [(2, 40), (0, 57)]),
    (128, 520, 600, [(2, 24), (0, 31)]),
    (256, 400, 420, [(2, 6), (3, 9)]),
])
def test_noalloc_matches_workspace_entry_point_on_two_calls(M, H, W, calls):
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    pkg = load_pkg()
    L = pkg.lib()
    dev = torch.device("cuda", torch.cuda.current_device())
    rng = np.random.default_rng(7 + M)
    F = 64
    O = torch.from_numpy(((0.6 + 0.4 * rng.random((H, W))) *
                          np.exp(1j * rng.random((H, W)))).astype(np.complex64)).to(dev)
    P = torch.from_numpy((rng.standard_normal((M, M)) + 1j * rng.standard_normal((M, M)))
                         .astype(np.complex64) / M).to(dev)
    tl = pkg.make_windows(rng.integers(0, H - M + 1, F), rng.integers(0, W - M + 1, F), dev)
    stack = torch.from_numpy(rng.poisson(50.0, size=(F, M, M)).astype(np.float32)).to(dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call, (loss_code, n) in enumerate(calls):
        batch = torch.from_numpy(rng.permutation(F)[:n].astype(np.int32)).to(dev)
        _check_against_workspace_entry(pkg, L, O, H, W, P, M, tl, stack, F, batch, loss_code, status, stream,
                                       (M, call))

    # the size limit, at this probe size's own boundary: the largest batch that
    # fits in the 48 MiB array runs (frame ids may repeat), one more is refused
    bmax = _largest_batch(L, H, W, M)
    assert L.ptycho_fwd_adj_workspace_size(H, W, M, M, bmax) <= SCRATCH
    assert L.ptycho_fwd_adj_workspace_size(H, W, M, M, bmax + 1) > SCRATCH
    big = torch.from_numpy(rng.integers(0, F, bmax + 1).astype(np.int32)).to(dev)
    _check_against_workspace_entry(pkg, L, O, H, W, P, M, tl, stack, F, big[:bmax].contiguous(), 2, status,
                                   stream, (M, "boundary"))
    loss = torch.zeros((), dtype=torch.float64, device=dev)
    dO = torch.zeros((H, W), dtype=torch.complex64, device=dev)
    dP = torch.zeros((M, M), dtype=torch.complex64, device=dev)
    rc = _call(L, O, H, W, P, M, tl, stack, F, big, bmax + 1, 2, None, loss, dO, dP, status, stream)
    assert rc == WORKSPACE_TOO_SMALL, (M, bmax, L.ptycho_status_string(rc))


def test_noalloc_refuses_what_the_workspace_entry_point_refuses():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    pkg = load_pkg()
    L = pkg.lib()
    dev = torch.device("cuda", torch.cuda.current_device())
    M, H, W, F = 64, 128, 128, 4
    O = torch.zeros((H, W), dtype=torch.complex64, device=dev)
    P = torch.zeros((M, M), dtype=torch.complex64, device=dev)
    tl = torch.zeros((F, 2), dtype=torch.int32, device=dev)
    stack = torch.zeros((F, M, M), dtype=torch.float32, device=dev)
    batch = torch.zeros(F, dtype=torch.int32, device=dev)
    loss = torch.zeros((), dtype=torch.float64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    args = [(0, W, F), (H, W, -1)]  # empty canvas; negative batch
    for h, w, n in args:
        rc_ws = L.ptycho_fwd_adj(O.data_ptr(), h, w, P.data_ptr(), M, M, tl.data_ptr(), stack.data_ptr(), F,
                                 batch.data_ptr(), n, 2, None, loss.data_ptr(), None, None, 0, None, 0,
                                 status.data_ptr(), stream)
        rc = L.ptycho_fwd_adj_noalloc(O.data_ptr(), h, w, P.data_ptr(), M, M, tl.data_ptr(), stack.data_ptr(), F,
                                      batch.data_ptr(), n, 2, None, loss.data_ptr(), None, None, 0,
                                      status.data_ptr(), stream)
        assert rc == rc_ws == INVALID_ARG, (h, w, n, rc, rc_ws)
    torch.cuda.synchronize(dev)
    assert int(status.item()) == 0
