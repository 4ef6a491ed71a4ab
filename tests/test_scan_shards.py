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


def _rank_main(rank, world, port, out_dir, loss_type):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ss = _shards()
        M = 16
        tlY, tlX, H = _scan(M=M)
        rng = np.random.default_rng(5)
        O = (rng.standard_normal((H, H)) + 1j * rng.standard_normal((H, H))) * 0.3 + 1.0
        P = rng.standard_normal((M, M)) + 1j * rng.standard_normal((M, M))
        Imeas = rng.poisson(5.0, size=(len(tlY), M, M)).astype(np.float64)
        frames = ss.shard_frames(tlY, tlX, world, rank)
        steps = ss.steps_per_epoch(len(tlY), world, 7)
        batch = ss.epoch_minibatches(frames, 7, steps, np.random.default_rng(100 + rank))[0]
        r = fm.fwd_adj(O, P, tlY[batch], tlX[batch], Imeas[batch], loss_type)
        dO = torch.from_numpy(r["dO"].copy())
        dP = torch.from_numpy(r["dP"].copy())
        ex = ss.GradientExchange(tlY, tlX, M)
        assert ex.world == world
        ex.all_reduce(dO, dP)
        # the generic parameter-gradient path (used for INR parameters) agrees
        p = torch.nn.Parameter(torch.zeros(M, M, dtype=torch.complex128))
        p.grad = torch.from_numpy(r["dP"].copy())
        ss.all_reduce_grads([p])
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), dO=dO.numpy(), dP=dP.numpy(), gP=p.grad.numpy(),
                 batch=batch, O=O, P=P, Imeas=Imeas, tlY=tlY, tlX=tlX, rows=np.array(ex.rows))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("loss_type", ["Poisson_likelihood_loss", "smooth_L1_loss"])
def test_gradient_exchange_gloo_world2(tmp_path, loss_type):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path), loss_type), nprocs=world,
                       join=True, start_method="spawn")
    res = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    g = res[0]
    union = np.concatenate([x["batch"] for x in res])
    ref = fm.fwd_adj(g["O"], g["P"], g["tlY"][union], g["tlX"][union], g["Imeas"][union], loss_type)
    for x in res:
        np.testing.assert_allclose(x["dO"], ref["dO"], rtol=1e-12, atol=1e-12 * np.abs(ref["dO"]).max())
        np.testing.assert_allclose(x["dP"], ref["dP"], rtol=1e-12, atol=1e-12 * np.abs(ref["dP"]).max())
        np.testing.assert_array_equal(x["gP"], x["dP"])
    y0, y1 = g["rows"]  # rows outside the scanned band carry no gradient
    assert np.all(res[0]["dO"][:y0] == 0) and np.all(res[0]["dO"][y1:] == 0)
    assert not set(res[0]["batch"]) & set(res[1]["batch"])  # disjoint bands
