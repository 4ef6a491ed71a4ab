"""Scan sharding and the gradient exchange of the multi-GPU step, on CPU.

The exchange runs as world_size-2 ``gloo`` process groups (127.0.0.1); each
rank's local gradients come from the FP64 oracle, so the test checks the
host logic: every frame is owned by exactly one rank, every rank takes the
same number of steps per epoch, and after the exchange each rank holds the
gradients of the union of the ranks' minibatches (the oracle over that
union), with rows outside the scanned band untouched.
"""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import forward_model as fm


def _shards():
    from conftest import load_pkg
    return load_pkg().scan_shards


def _scan(n=6, step=8, M=16, jitter=2, seed=0):
    rng = np.random.default_rng(seed)
    iy, ix = np.mgrid[:n, :n]
    tlY = (4 + iy.ravel() * step + rng.integers(-jitter, jitter + 1, n * n)).astype(np.int32)
    tlX = (4 + ix.ravel() * step + rng.integers(-jitter, jitter + 1, n * n)).astype(np.int32)
    H = int(max(tlY.max(), tlX.max())) + M + 6
    return tlY, tlX, H


@pytest.mark.parametrize("world", [1, 2, 3, 4, 7])
def test_shard_frames_partition(world):
    ss = _shards()
    tlY, tlX, _ = _scan()
    F = len(tlY)
    parts = [ss.shard_frames(tlY, tlX, world, r) for r in range(world)]
    assert np.array_equal(np.sort(np.concatenate(parts)), np.arange(F))  # each frame exactly once
    sizes = [p.size for p in parts]
    assert max(sizes) - min(sizes) <= 1
    order = np.lexsort((tlX, tlY))
    rank_of = np.empty(F, int)
    for r, p in enumerate(parts):
        rank_of[p] = r
    assert np.all(np.diff(rank_of[order]) >= 0)  # contiguous bands of the raster order


def test_shard_errors_and_bbox():
    ss = _shards()
    tlY, tlX, _ = _scan()
    with pytest.raises(ValueError):
        ss.shard_frames(tlY, tlX, 2, 2)
    with pytest.raises(ValueError):
        ss.shard_frames(tlY, tlX[:-1], 2, 0)
    assert ss.window_bbox(tlY, tlX, [], 16) == (0, 0, 0, 0)
    y0, y1, x0, x1 = ss.window_bbox(tlY, tlX, [0, 1], 16)
    assert (y0, x0) == (min(tlY[:2]), min(tlX[:2])) and (y1, x1) == (max(tlY[:2]) + 16, max(tlX[:2]) + 16)
    with pytest.raises(ValueError):
        ss.epoch_minibatches(np.zeros(0, np.int64), 4, 2, np.random.default_rng(0))


@pytest.mark.parametrize("F,world,bs", [(36, 2, 5), (37, 3, 10), (1600, 8, 256), (5, 4, 2)])
def test_equal_steps_per_epoch(F, world, bs):
    """Every rank takes the same number of steps (collectives) per epoch and a
    band's first permutation is used whole before any frame repeats."""
    ss = _shards()
    rng0 = np.random.default_rng(0)
    tlY = rng0.integers(0, 100, F)
    tlX = rng0.integers(0, 100, F)
    steps = ss.steps_per_epoch(F, world, bs)
    for r in range(world):
        frames = ss.shard_frames(tlY, tlX, world, r)
        mb = ss.epoch_minibatches(frames, bs, steps, np.random.default_rng(r))
        assert len(mb) == steps and all(0 < len(b) <= bs for b in mb)
        assert np.array_equal(np.sort(np.concatenate(mb)[:frames.size]), frames)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem(M=16):
    tlY, tlX, H = _scan(M=M)
    rng = np.random.default_rng(5)
    O = (rng.standard_normal((H, H)) + 1j * rng.standard_normal((H, H))) * 0.3 + 1.0
    P = rng.standard_normal((M, M)) + 1j * rng.standard_normal((M, M))
    Imeas = rng.poisson(5.0, size=(len(tlY), M, M)).astype(np.float64)
    return tlY, tlX, H, O, P, Imeas


def _batches(ss, tlY, tlX, world, rank, nsteps=3, bs=5):
    frames = ss.shard_frames(tlY, tlX, world, rank)
    steps = max(nsteps, ss.steps_per_epoch(len(tlY), world, bs))
    return ss.epoch_minibatches(frames, bs, steps, np.random.default_rng(100 + rank))[:nsteps]


def _rank_main(rank, world, port, out_dir, loss_type):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ss = _shards()
        M = 16
        tlY, tlX, H, O, P, Imeas = _problem(M)
        batches = _batches(ss, tlY, tlX, world, rank)
        ex = ss.GradientExchange(tlY, tlX, M)
        assert ex.world == world and ex.rank == rank
        # one exchange of the first minibatch's gradients
        r = fm.fwd_adj(O, P, tlY[batches[0]], tlX[batches[0]], Imeas[batches[0]], loss_type)
        dO = torch.from_numpy(r["dO"].copy())
        dP = torch.from_numpy(r["dP"].copy())
        ex.all_reduce(dO, dP)
        # the generic parameter-gradient path (used for INR parameters) agrees
        p = torch.nn.Parameter(torch.zeros(M, M, dtype=torch.complex128))
        p.grad = torch.from_numpy(r["dP"].copy())
        ss.all_reduce_grads([p])
        # three Adam steps on the object (probe fixed), then the whole object assembled
        Ot = torch.nn.Parameter(torch.from_numpy(O.copy()))
        opt = torch.optim.Adam([Ot], lr=1e-2)
        for b in batches:
            g = fm.fwd_adj(Ot.detach().numpy(), P, tlY[b], tlX[b], Imeas[b], loss_type)["dO"]
            Ot.grad = torch.from_numpy(g.copy())
            ex.all_reduce(Ot.grad, None)
            opt.step()
        band_O = Ot.detach().numpy().copy()
        with torch.no_grad():
            ex.gather_object(Ot.data)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), dO=dO.numpy(), dP=dP.numpy(), gP=p.grad.numpy(),
                 batch=batches[0], O_band=band_O, O_final=Ot.detach().numpy(),
                 bands=np.array(ex.bands), bytes=ex.bytes_per_step(H, M, M))
    finally:
        dist.destroy_process_group()


def _emulate(ss, world, loss_type):
    """The exchange protocol in one process: every rank's replica, local
    gradients from the oracle, band sums in rank order, Adam per rank."""
    M = 16
    tlY, tlX, H, O, P, Imeas = _problem(M)
    bands = ss.band_rows(tlY, tlX, M, world)
    batches = [_batches(ss, tlY, tlX, world, r) for r in range(world)]
    Os = [torch.nn.Parameter(torch.from_numpy(O.copy())) for _ in range(world)]
    opts = [torch.optim.Adam([o], lr=1e-2) for o in Os]
    for k in range(3):
        local = [torch.from_numpy(fm.fwd_adj(Os[r].detach().numpy(), P, tlY[batches[r][k]], tlX[batches[r][k]],
                                             Imeas[batches[r][k]], loss_type)["dO"].copy()) for r in range(world)]
        for r in range(world):
            y0, y1 = bands[r]
            g = local[r].clone()
            acc = torch.zeros((y1 - y0, H), dtype=g.dtype)
            for q in range(world):
                a, b = max(y0, bands[q][0]), min(y1, bands[q][1])
                if b > a:
                    acc[a - y0:b - y0] += local[q][a:b]
            g[y0:y1] = acc
            Os[r].grad = g
            opts[r].step()
    owned = ss.owned_rows(bands, H)
    final = np.empty_like(O)
    for r, (a, b) in enumerate(owned):
        final[a:b] = Os[r].detach().numpy()[a:b]
    return [o.detach().numpy() for o in Os], final, bands, batches


@pytest.mark.parametrize("world", [2, 4])
@pytest.mark.parametrize("loss_type", ["Poisson_likelihood_loss", "smooth_L1_loss"])
def test_gradient_exchange_gloo(tmp_path, loss_type, world):
    ss = _shards()
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path), loss_type), nprocs=world,
                       join=True, start_method="spawn")
    res = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    M = 16
    tlY, tlX, H, O, P, Imeas = _problem(M)
    bands = [tuple(b) for b in res[0]["bands"]]
    assert bands == ss.band_rows(tlY, tlX, M, world)
    # first exchange: on its band each rank holds the sum of every rank's local
    # gradient, added in rank order (bitwise); outside its band, its own zeros
    locals_ = [fm.fwd_adj(O, P, tlY[x["batch"]], tlX[x["batch"]], Imeas[x["batch"]], loss_type) for x in res]
    union = np.concatenate([x["batch"] for x in res])
    ref = fm.fwd_adj(O, P, tlY[union], tlX[union], Imeas[union], loss_type)
    for r, x in enumerate(res):
        y0, y1 = bands[r]
        want = np.zeros((y1 - y0, H), complex)
        for q in range(world):
            a, b = max(y0, bands[q][0]), min(y1, bands[q][1])
            if b > a:
                want[a - y0:b - y0] += locals_[q]["dO"][a:b]
        np.testing.assert_array_equal(x["dO"][y0:y1], want)
        assert np.all(x["dO"][:y0] == 0) and np.all(x["dO"][y1:] == 0)
        np.testing.assert_allclose(x["dO"][y0:y1], ref["dO"][y0:y1], rtol=1e-12,
                                   atol=1e-12 * np.abs(ref["dO"]).max())
        np.testing.assert_allclose(x["dP"], ref["dP"], rtol=1e-12, atol=1e-12 * np.abs(ref["dP"]).max())
        np.testing.assert_array_equal(x["gP"], x["dP"])
        # only the halo rows are sent (plus the probe gradient)
        halo = sum(max(0, min(y1, q1) - max(y0, q0)) for q, (q0, q1) in enumerate(bands) if q != r)
        assert int(x["bytes"]) == 8 * H * halo + 8 * M * M
        assert halo < ss.scanned_rows(tlY, tlX, M)[1] - ss.scanned_rows(tlY, tlX, M)[0]
    # three optimizer steps: bitwise the emulated protocol, identical on shared rows,
    # one assembled object on every rank, close to world 1 on the union of batches
    emu_O, emu_final, _, batches = _emulate(ss, world, loss_type)
    for r, x in enumerate(res):
        y0, y1 = bands[r]
        np.testing.assert_array_equal(x["O_band"][y0:y1], emu_O[r][y0:y1])
        np.testing.assert_array_equal(x["O_final"], emu_final)
    for r in range(world):
        for q in range(r + 1, world):
            a, b = max(bands[r][0], bands[q][0]), min(bands[r][1], bands[q][1])
            if b > a:
                np.testing.assert_array_equal(res[r]["O_band"][a:b], res[q]["O_band"][a:b])
    O1 = torch.nn.Parameter(torch.from_numpy(O.copy()))
    opt = torch.optim.Adam([O1], lr=1e-2)
    for k in range(3):
        u = np.concatenate([batches[r][k] for r in range(world)])
        O1.grad = torch.from_numpy(fm.fwd_adj(O1.detach().numpy(), P, tlY[u], tlX[u], Imeas[u], loss_type)["dO"].copy())
        opt.step()
    d = np.abs(res[0]["O_final"] - O1.detach().numpy()).max() / np.abs(O).max()
    assert d <= 1e-6, d
    assert not set(res[0]["batch"]) & set(res[1]["batch"])  # disjoint bands
