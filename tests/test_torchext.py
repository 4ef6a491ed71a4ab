"""The fused loss's C++ autograd node (csrc/torch_ext.cpp).

fused_loss runs through a C++ torch::autograd::Function when the extension is
built: its forward calls ptycho_fwd_adj and its backward ptycho_scale_pair,
the same library calls the Python Function makes.  On CPU: the module is
built, loads, binds to the library and exports its entry points.  On the GPU:
both routes give bit-identical losses and gradients (one library, one
kernel sequence), for every loss, with one or both inputs requiring a
gradient, a retained graph backed up twice, frame-id batches given as a list,
and no-grad calls; non-contiguous object / probe views and a side stream give
the same values; argument errors raise the Python route's exception types.
"""
import numpy as np
import pytest
import torch

from conftest import load_pkg


def test_torchext_is_built_and_binds():
    pkg = load_pkg()
    ext = pkg._lib.torchext()
    assert ext is not None, "the C++ autograd node (_torchext) is not built"
    for name in ("bind", "fused_loss", "workspace"):
        assert callable(getattr(ext, name))
    assert pkg.optics.USE_TORCHEXT


def test_torchext_takes_the_shared_cxx_runtime():
    """The module must not carry its own copy of libstdc++'s iostream/locale
    code (a toolchain that links libstdc++ statically): next to the process's
    shared runtime that copy crashes when an error message is formatted."""
    import importlib.util
    import os
    pkg = load_pkg()
    ext = pkg._lib.torchext()
    here = os.path.dirname(pkg.__file__)
    spec = importlib.util.spec_from_file_location("ptycho_build", os.path.join(here, "csrc", "build.py"))
    build = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(build)
    assert build.runtime_copies(ext.__file__) == []


def test_torchext_refuses_host_tensors():
    """No CPU path: host tensors raise ValueError before any library call."""
    pkg = load_pkg()
    assert pkg._lib.torchext() is not None
    O = torch.zeros((80, 80), dtype=torch.complex64, requires_grad=True)
    P = torch.zeros((64, 64), dtype=torch.complex64)
    tl = torch.zeros((2, 2), dtype=torch.int32)
    Im = torch.zeros((2, 64, 64))
    with pytest.raises(ValueError, match="CUDA"):
        pkg.fused_loss(O, P, tl, Im, "smooth_L1_loss", batch=[1, 0])


def _case(M, H, F, seed):
    rng = np.random.default_rng(seed)
    O = ((0.5 + 0.5 * rng.random((H, H))) * np.exp(1j * rng.random((H, H)))).astype(np.complex64)
    P = ((rng.standard_normal((M, M)) + 1j * rng.standard_normal((M, M))) / M).astype(np.complex64)
    tlY = rng.integers(0, H - M + 1, F).astype(np.int32)
    tlX = rng.integers(0, H - M + 1, F).astype(np.int32)
    Imeas = rng.poisson(30.0, size=(F, M, M)).astype(np.float32)
    return O, P, tlY, tlX, Imeas


def _run(pkg, monkeypatch, use_ext, O, P, tl, Im, loss_type, batch, grad_o, grad_p, twice):
    monkeypatch.setattr(pkg.optics, "USE_TORCHEXT", use_ext)
    dev = torch.device("cuda")
    Ot = torch.from_numpy(O).to(dev).requires_grad_(grad_o)
    Pt = torch.from_numpy(P).to(dev).requires_grad_(grad_p)
    loss = pkg.fused_loss(Ot, Pt, tl, Im, loss_type, batch=batch)
    (1.5 * loss).backward(retain_graph=twice)
    if twice:
        (0.25 * loss).backward()
    torch.cuda.synchronize()
    g = lambda t: None if t.grad is None else t.grad.cpu().numpy()  # noqa: E731
    return float(loss.detach()), g(Ot), g(Pt)


@pytest.mark.gpu
@pytest.mark.parametrize("M, loss_type, grad_o, grad_p, twice, batch", [
    (64, "smooth_L1_loss", True, True, False, None),
    (64, "Poisson_likelihood_loss", False, True, True, [5, 1, 1, 7]),
    (128, "FD_loss", True, False, True, None),
    (128, "Poisson_likelihood_loss", True, True, False, [0, 3, 2]),
    (256, "FD_loss", True, True, False, None),
    (96, "smooth_L1_loss", True, True, True, [4, 0]),   # the general path
])
def test_cpp_node_matches_python_function(monkeypatch, M, loss_type, grad_o, grad_p, twice, batch):
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    pkg = load_pkg()
    assert pkg._lib.torchext() is not None
    O, P, tlY, tlX, Imeas = _case(M, M + 70, 8, seed=M)
    dev = torch.device("cuda")
    tl = pkg.make_windows(tlY, tlX, dev)
    Im = torch.from_numpy(Imeas).to(dev)
    a = _run(pkg, monkeypatch, True, O, P, tl, Im, loss_type, batch, grad_o, grad_p, twice)
    b = _run(pkg, monkeypatch, False, O, P, tl, Im, loss_type, batch, grad_o, grad_p, twice)
    assert a[0] == b[0]
    for ga, gb in zip(a[1:], b[1:]):
        assert (ga is None) == (gb is None)
        if ga is not None:
            assert np.array_equal(ga, gb)
    assert (a[1] is None) == (not grad_o) and (a[2] is None) == (not grad_p)


@pytest.mark.gpu
def test_cpp_node_no_grad_and_errors():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    pkg = load_pkg()
    dev = torch.device("cuda")
    O, P, tlY, tlX, Imeas = _case(64, 100, 4, seed=3)
    Ot = torch.from_numpy(O).to(dev).requires_grad_(True)
    Pt = torch.from_numpy(P).to(dev)
    tl = pkg.make_windows(tlY, tlX, dev)
    Im = torch.from_numpy(Imeas).to(dev)
    with torch.no_grad():
        loss = pkg.fused_loss(Ot, Pt, tl, Im, "FD_loss")
    assert loss.grad_fn is None and loss.dtype == torch.float64 and loss.is_cuda
    want = pkg.fwd_adj_raw(Ot.detach(), Pt, tl, Im, pkg.LOSS_CODES["FD_loss"], want_grad=False)[0]
    assert float(loss) == float(want)
    # windows given as int64 on the host are converted as the Python route does
    l2 = pkg.fused_loss(Ot, Pt, tl.cpu().long(), Im, "smooth_L1_loss")
    l3 = pkg.fused_loss(Ot, Pt, tl, Im, "smooth_L1_loss")
    assert float(l2) == float(l3)
    with pytest.raises(ValueError):
        pkg.fused_loss(Ot.detach().cpu(), Pt.cpu(), tl, Im, "smooth_L1_loss")
    with pytest.raises(ValueError):
        pkg.fused_loss(Ot, Pt, tl, Im[:, :32], "smooth_L1_loss")
    with pytest.raises(ValueError):
        pkg.fused_loss(Ot, Pt, tl, Im, "no_such_loss")
    with pytest.raises(TypeError):
        pkg.fused_loss(Ot, Pt.to(torch.complex128), tl, Im, "smooth_L1_loss")
    with pytest.raises(ValueError):
        pkg.fused_loss(Ot, torch.zeros((4097, 4), dtype=torch.complex64, device=dev), tl, Im, "smooth_L1_loss")


@pytest.mark.gpu
def test_cpp_node_views_streams_and_id_types():
    """Non-contiguous object / probe views give the contiguous copies' results
    (gradients shaped like the views); a side stream gets its own workspace and
    the same values; frame ids given as a NumPy array, int64 or on the host."""
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    pkg = load_pkg()
    dev = torch.device("cuda")
    O, P, tlY, tlX, Imeas = _case(128, 300, 10, seed=9)
    tl = pkg.make_windows(tlY, tlX, dev)
    Im = torch.from_numpy(Imeas).to(dev)
    ids = np.array([3, 1, 4, 1, 5, 9], dtype=np.int64)

    def run(Ot, Pt, batch, stream=None):
        with torch.cuda.stream(stream) if stream is not None else torch.cuda.stream(torch.cuda.current_stream()):
            loss = pkg.fused_loss(Ot, Pt, tl, Im, "Poisson_likelihood_loss", batch=batch)
            loss.backward()
        torch.cuda.synchronize()
        return float(loss.detach()), Ot.grad.cpu().numpy(), Pt.grad.cpu().numpy()

    base_O = torch.from_numpy(O).to(dev).requires_grad_(True)
    base_P = torch.from_numpy(P).to(dev).requires_grad_(True)
    ref = run(base_O, base_P, torch.from_numpy(ids.astype(np.int32)).to(dev))

    # views: every other column of a wider buffer, and a transposed-then-transposed probe
    wide = torch.zeros((300, 600), dtype=torch.complex64, device=dev)
    wide[:, ::2] = torch.from_numpy(O).to(dev)
    Ov = wide[:, ::2].detach().requires_grad_(True)
    assert not Ov.is_contiguous()
    Pv = torch.from_numpy(P.T.copy()).to(dev).t().detach().requires_grad_(True)
    assert not Pv.is_contiguous()
    got = run(Ov, Pv, ids)  # ids as a NumPy int64 array
    assert got[0] == ref[0] and np.array_equal(got[1], ref[1]) and np.array_equal(got[2], ref[2])
    assert Ov.grad.shape == Ov.shape and Pv.grad.shape == Pv.shape

    side = torch.cuda.Stream()
    O2 = torch.from_numpy(O).to(dev).requires_grad_(True)
    P2 = torch.from_numpy(P).to(dev).requires_grad_(True)
    got = run(O2, P2, torch.from_numpy(ids), stream=side)  # int64 on the host
    assert got[0] == ref[0] and np.array_equal(got[1], ref[1]) and np.array_equal(got[2], ref[2])


@pytest.mark.gpu
def test_cpp_node_many_streams():
    """More streams than the workspace cache holds (16): entries are dropped,
    results stay the same on every stream."""
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    pkg = load_pkg()
    dev = torch.device("cuda")
    O, P, tlY, tlX, Imeas = _case(64, 120, 6, seed=12)
    tl = pkg.make_windows(tlY, tlX, dev)
    Im = torch.from_numpy(Imeas).to(dev)
    Ot = torch.from_numpy(O).to(dev)
    Pt = torch.from_numpy(P).to(dev)
    want = float(pkg.fused_loss(Ot, Pt, tl, Im, "smooth_L1_loss"))
    streams = [torch.cuda.Stream() for _ in range(20)]
    got = []
    for st in streams:
        with torch.cuda.stream(st):
            got.append(pkg.fused_loss(Ot, Pt, tl, Im, "smooth_L1_loss"))
    torch.cuda.synchronize()
    assert all(float(g) == want for g in got)
