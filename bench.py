"""Benchmark: fused far-field forward + loss + adjoint throughput (patterns/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c1] [--no-cpu-baseline] [--no-ttr]
    python bench.py --time-to-residual | --inr-step

Workload (default ``c1``): 1536^2 complex64 object, 128^2 probe, 40 x 40 raster
(1600 positions, 32 px step, U[-3,3] jitter), Poisson loss at a 1e4-photon
peak, batch 256 patterns per GPU, seeded synthetic data (the reference's
datasets are not distributed).  One step = one minibatch: the fused
forward/loss/adjoint kernel plus the deterministic dO/dP assembly (and, for
N > 1, the NCCL all-reduce of dP and the point-to-point halo exchange of dO --
each rank draws its minibatch from its own band of the raster, so per-GPU
work is fixed: weak scaling).  L2 is flushed (a 256 MiB
write) before every timed step; step times are CUDA events on the launching
stream, summed over K steps, max over ranks.

At N = 1 on c1 the line also carries ``time_to_residual``, the headline
metric's second half: on workload c2 the pixel grid trains 200 epochs and sets
the target 1.1 x its converged FP64 data residual; the INR on this library's
kernels and the reference INR code path in torch (same GPU) train until they
reach it (``--time-to-residual`` prints the full record, ``--no-ttr`` skips it).

``--impl reference`` times the reference's own torch CPU path (per-frame
loop of Recovery.py:288-316 with autograd) on the host cores instead.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PKG = "conventional-ptychography-reconstruction_b200"

METRIC = "fwd+adj patterns/s"
L2_FLUSH_BYTES = 256 << 20
SETTLE_S = 0.6  # untimed steps on either side of the timed ones while clocks are sampled


def algorithmic_bytes_per_pattern(M: int, B: int) -> float:
    """Object window read (8 M^2) + measurement read (4 M^2) + object-gradient
    contribution write (8 M^2), plus probe read and probe-gradient write
    amortised over the batch (16 M^2 / B)."""
    return 20.0 * M * M + 16.0 * M * M / B


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic(kernel_key: str):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f).get(kernel_key)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, note=None):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        out = {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
               "samples": len(sm)}
        if note:
            out["note"] = note
        return out


def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def cpu_reference_rate(work, batch: int, budget_s: float, threads: int | None = None):
    """Time the reference's torch CPU path on a bounded sample (whole minibatches)."""
    from oracle import torch_cpu_path
    if threads:
        torch.set_num_threads(threads)
    M = work["probe"].shape[0]
    obj = torch.from_numpy(work["obj"].astype(np.complex64)).requires_grad_(True)
    probe = torch.from_numpy(work["probe"].astype(np.complex64)).requires_grad_(True)
    stack = torch.from_numpy(np.ascontiguousarray(np.moveaxis(work["Imeas"], 0, -1)))  # [M, M, F]
    F = stack.shape[2]
    rng = np.random.default_rng(5)
    n, t_total, steps = 0, 0.0, 0
    lt = work["workload"].loss_type
    first = None
    while t_total < budget_s or steps == 0:
        idx = rng.permutation(F)[:batch]
        t0 = time.perf_counter()
        loss = torch_cpu_path.minibatch_fwd_adj(obj, probe, work["tlY"], work["tlX"], stack, idx, lt)
        t_total += time.perf_counter() - t0
        if first is None:  # kept to check the GPU path on the same minibatch
            first = {"idx": idx.copy(), "loss": loss, "dO": obj.grad.detach().clone(),
                     "dP": probe.grad.detach().clone()}
        n += len(idx)
        steps += 1
    return n / t_total, n, steps, torch.get_num_threads(), first


def parity_vs_cpu(pkg, work, first, dev):
    """The GPU path on the CPU baseline's first minibatch: relative errors of
    the loss, dO and dP against the reference restatement (torch CPU, complex64)."""
    w = work["workload"]
    idx = first["idx"].astype(np.int32)
    O = torch.from_numpy(work["obj"].astype(np.complex64)).to(dev)
    P = torch.from_numpy(work["probe"].astype(np.complex64)).to(dev)
    tl = pkg.make_windows(work["tlY"], work["tlX"], dev)
    stack = torch.from_numpy(work["Imeas"]).to(dev)
    loss, _, dO, dP = pkg.fwd_adj_raw(O, P, tl, stack, pkg.LOSS_CODES[w.loss_type],
                                      batch=torch.from_numpy(idx).to(dev))
    rel = lambda a, b: float((a - b).abs().max() / b.abs().max())  # noqa: E731
    out = {"vs_torch_cpu_complex64": {
        "loss_rel_err": abs(float(loss) - first["loss"]) / abs(first["loss"]),
        "dO_rel_err": rel(dO.cpu(), first["dO"]), "dP_rel_err": rel(dP.cpu(), first["dP"])}}
    from oracle import forward_model as fm  # the FP64 NumPy oracle, as the checker
    ref = fm.fwd_adj(work["obj"], work["probe"], work["tlY"][idx], work["tlX"][idx], work["Imeas"][idx],
                     w.loss_type)
    rn = lambda a, b: float(np.abs(a - b).max() / np.abs(b).max())  # noqa: E731
    I = pkg.forward_intensity(O, P, tl, batch=torch.from_numpy(idx).to(dev))
    out["vs_fp64_oracle"] = {"intensity_rel_err": rn(I.cpu().numpy(), ref["I"]),
                             "loss_rel_err": abs(float(loss) - ref["loss_total"]) / abs(ref["loss_total"]),
                             "dO_rel_err": rn(dO.cpu().numpy(), ref["dO"]),
                             "dP_rel_err": rn(dP.cpu().numpy(), ref["dP"])}
    out["note"] = "max |GPU - ref| / max |ref| on the CPU baseline's first sampled minibatch"
    return out


def side_workload(pkg, key, dev, steps=30, warmup=5, n_check=8):
    """Throughput and parity of the fused path on another workload's shapes
    (c3 / c4: the 256^2 cluster kernel), run inside the default c1 bench.

    Same object, probe and raster recipe as ``synth.make_workload(key)``; the
    measurements are generated for 2 x batch frames taken at a regular stride
    over the whole raster (so minibatches cover the canvas as random ones from
    the full scan do) and the peak is scaled over those frames.  Steps replay
    the same CUDA graph as the headline (FwdAdjPlan), L2 flushed before each,
    CUDA events per step.  Parity: ``n_check`` frames of the first minibatch
    against the FP64 oracle (intensities, per-pattern losses, dO, dP)."""
    synth = pkg.synth
    w = synth.WORKLOADS[key]
    B, M = w.batch, w.probe
    O = synth.make_object(w.canvas, seed=0)
    P = synth.make_probe(w.probe, w.aperture)
    tlY, tlX = synth.make_scan(w.n_scan, w.step, w.jitter, w.canvas, w.probe, seed=2)
    stride = max(1, tlY.size // (2 * B))
    sel = np.arange(0, tlY.size, stride)[:2 * B]
    tlY, tlX = tlY[sel], tlX[sel]
    I = synth._intensities(O, P, tlY, tlX, device=dev)
    I *= w.peak / I.max()
    Imeas = np.random.default_rng(1).poisson(I).astype(np.float32)
    del I
    O, P = O.astype(np.complex64), P.astype(np.complex64)
    Ot, Pt = torch.from_numpy(O).to(dev), torch.from_numpy(P).to(dev)
    tl = pkg.make_windows(tlY, tlX, dev)
    stack = torch.from_numpy(Imeas).to(dev)
    F = tlY.size
    rng = np.random.default_rng(77)
    batches = [torch.from_numpy(rng.permutation(F)[:B].astype(np.int32)).to(dev) for _ in range(8)]
    plan = pkg.optics.FwdAdjPlan(Ot, Pt, tl, stack, w.loss_type, B)
    plan.capture()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    s = torch.cuda.current_stream(dev)
    for i in range(warmup):
        plan.batch.copy_(batches[i % 8])
        plan.replay()
        flush.zero_()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        plan.batch.copy_(batches[k % 8])
        flush.zero_()
        ev[k][0].record(s)
        plan.replay()
        ev[k][1].record(s)
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in ev) / steps
    ids = batches[0][:n_check].cpu().numpy()
    loss, lp, dO, dP = pkg.fwd_adj_raw(Ot, Pt, tl, stack, pkg.LOSS_CODES[w.loss_type],
                                       batch=batches[0][:n_check].contiguous(), per_pattern=True)
    Ig = pkg.forward_intensity(Ot, Pt, tl, batch=batches[0][:n_check].contiguous())
    from oracle import forward_model as fm  # the FP64 NumPy oracle, as the checker
    ref = fm.fwd_adj(O.astype(np.complex128), P.astype(np.complex128), tlY[ids], tlX[ids], Imeas[ids],
                     w.loss_type)
    rn = lambda a, b: float(np.abs(a - b).max() / np.abs(b).max())  # noqa: E731
    bpp = algorithmic_bytes_per_pattern(M, B)
    return {"workload": f"{key}: {w.canvas}^2 object, {M}^2 probe, batch {B}, {w.loss_type}",
            "patterns_per_s": B / (ms / 1e3), "ms_per_step": ms, "steps": steps,
            "hbm_frac_of_measured": bpp * B / (ms / 1e3) / 1e9 / measured_peak_hbm()[0],
            "frames": f"{F} of the {w.n_scan ** 2} raster positions (every {stride}th)",
            "parity_vs_fp64_oracle": {
                "patterns": int(n_check),
                "intensity_rel_err": rn(Ig.cpu().numpy(), ref["I"]),
                "loss_per_pattern_max_rel_err": float(np.max(np.abs(lp.cpu().numpy() - ref["loss"])
                                                             / np.abs(ref["loss"]))),
                "dO_rel_err": rn(dO.cpu().numpy(), ref["dO"]),
                "dP_rel_err": rn(dP.cpu().numpy(), ref["dP"])},
            "note": "one CUDA-graph launch per minibatch (k_fused256 + k_assemble), L2 flushed before "
                    "each step; clocks not sampled for these steps"}


def run_reference(args):
    """--impl reference: the reference's torch CPU path on this host's cores."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    pkg = importlib.import_module(PKG)
    work = pkg.synth.make_workload(args.workload, device=None)
    w = work["workload"]
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    from oracle import torch_cpu_path
    M = w.probe
    obj = torch.from_numpy(work["obj"].astype(np.complex64)).requires_grad_(True)
    probe = torch.from_numpy(work["probe"].astype(np.complex64)).requires_grad_(True)
    stack = torch.from_numpy(np.ascontiguousarray(np.moveaxis(work["Imeas"], 0, -1)))
    F = stack.shape[2]
    rng = np.random.default_rng(5)
    # per-step sample sized so the whole --steps/--warmup run stays near 40k patterns
    batch = args.ref_batch or min(w.batch, max(1, -(-40000 // (args.steps + args.warmup))))
    for _ in range(args.warmup):
        torch_cpu_path.minibatch_fwd_adj(obj, probe, work["tlY"], work["tlX"], stack,
                                         rng.permutation(F)[:batch], w.loss_type)
    t = 0.0
    for _ in range(args.steps):
        idx = rng.permutation(F)[:batch]
        t0 = time.perf_counter()
        torch_cpu_path.minibatch_fwd_adj(obj, probe, work["tlY"], work["tlX"], stack, idx, w.loss_type)
        t += time.perf_counter() - t0
    rate = batch * args.steps / t
    sample = (f"{args.steps} steps of {batch} of the {F} patterns each (per-frame torch CPU loop "
              f"+ autograd over the sample, reference restatement), {torch.get_num_threads()} threads")
    line = {"metric": METRIC, "value": rate, "unit": "patterns/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "complex64 (fp32)",
            "data": "synthetic (seeded generator)", "impl": "reference",
            "config": _config(w, w.batch, args),
            "cpu_baseline": {"value": rate, "unit": "patterns/s", "cores": torch.get_num_threads(),
                             "kind": "port", "sample": sample},
            "e2e": {"value": rate, "unit": "patterns/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _config(w, batch, args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    return {"workload": w.name, "canvas": w.canvas, "probe": w.probe, "positions": w.n_scan ** 2,
            "batch_per_gpu": batch, "loss": w.loss_type, "peak_photons": w.peak,
            "parallelism": f"dp{world}: scan-row bands per rank, all-reduce of dP and scanned dO rows"
                           if world > 1 else "dp1",
            "l2": "flushed before every timed step (256 MiB write)"}


def run_ours(args):
    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    pkg = importlib.import_module(PKG)
    work = pkg.synth.make_workload(args.workload, device=dev)
    w = work["workload"]
    M, B = w.probe, w.batch
    O = torch.from_numpy(work["obj"].astype(np.complex64)).to(dev)
    P = torch.from_numpy(work["probe"].astype(np.complex64)).to(dev)
    tl = pkg.make_windows(work["tlY"], work["tlX"], dev)
    pkg.check_windows(tl, O.shape, M)
    stack = torch.from_numpy(work["Imeas"]).to(dev)  # [F, M, M], resident
    F = stack.shape[0]
    H, W = O.shape
    # each rank draws its minibatches from its own band of the raster (seeded
    # per rank); a band smaller than B wraps into a second permutation
    frames = pkg.scan_shards.shard_frames(work["tlY"], work["tlX"], world, rank)
    rng = np.random.default_rng(1234 + rank)
    nb = args.warmup + args.steps

    def draw():
        reps = -(-B // frames.size)
        ids = np.concatenate([frames[rng.permutation(frames.size)] for _ in range(reps)])[:B]
        return torch.from_numpy(ids.astype(np.int32)).to(dev)

    batches = [draw() for _ in range(nb)]
    exchange = pkg.scan_shards.GradientExchange(work["tlY"], work["tlX"], M)
    plan = pkg.optics.FwdAdjPlan(O, P, tl, stack, w.loss_type, B)
    dO, dP = plan.dO, plan.dP
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    s = torch.cuda.current_stream(dev)
    plan.capture()  # one CUDA graph launch per step

    def step(i):
        plan.batch.copy_(batches[i])
        plan.replay()
        exchange.all_reduce(dO, dP)  # N > 1: dO halo rows, dP all-reduce (NCCL)
        return plan.loss_total

    w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0.record(s)
    for i in range(args.warmup):
        step(i)
        flush.zero_()
    w1.record(s)
    torch.cuda.synchronize()
    # The K timed steps last ~1 ms, shorter than nvidia-smi's sampling period,
    # so the clock record spans them plus SETTLE_S of identical untimed steps
    # on either side (same kernels, same flushes).  The count is agreed over
    # ranks, so every rank takes the same collective steps.
    n_settle = int(min(20000, max(1, args.settle_s * 1e3 / max(w0.elapsed_time(w1) / max(args.warmup, 1), 1e-3))))
    if world > 1:
        import torch.distributed as dist
        nt = torch.tensor([n_settle], dtype=torch.int64, device=dev)
        dist.all_reduce(nt, op=dist.ReduceOp.MAX)
        n_settle = int(nt)

    def settle():
        for i in range(n_settle):
            step(i % nb)
            flush.zero_()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        settle()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(s)
            step(args.warmup + k)
            ev[k][1].record(s)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        settle()
        torch.cuda.synchronize()
    times = [a.elapsed_time(b) for a, b in ev]  # ms
    t_tot = torch.tensor([sum(times)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_tot, op=dist.ReduceOp.MAX)
    t_max_ms = float(t_tot)
    value = world * B * args.steps / (t_max_ms / 1e3)
    launches = 2 * args.steps  # k_fused, k_assemble per step

    # ---- e2e: public API, host-pinned inputs copied in every step -------------
    e2e = e2e_resident = None
    if True:
        Im_host = [stack.index_select(0, batches[i].long()).cpu().pin_memory() for i in range(min(nb, 4))]
        tl_host = [tl.index_select(0, batches[i].long()).cpu().pin_memory() for i in range(min(nb, 4))]
        Oparam = O.clone().requires_grad_(True)
        Pparam = P.clone().requires_grad_(True)
        out_host = torch.empty((), dtype=torch.float64).pin_memory()

        # double-buffered: step i+2's inputs are copied on a copy stream while
        # step i+1 computes; each step still copies its own inputs in the timed region
        cs = torch.cuda.Stream(dev)
        slots = [(torch.empty_like(Im_host[0], device=dev), torch.empty_like(tl_host[0], device=dev))
                 for _ in range(2)]
        copied = [torch.cuda.Event() for _ in range(2)]
        consumed = [torch.cuda.Event() for _ in range(2)]
        for ev in consumed:
            ev.record(s)

        def issue_copy(i):
            k = i % 2
            cs.wait_event(consumed[k])  # the step that last read this slot is done
            with torch.cuda.stream(cs):
                slots[k][0].copy_(Im_host[i % len(Im_host)], non_blocking=True)
                slots[k][1].copy_(tl_host[i % len(tl_host)], non_blocking=True)
                copied[k].record(cs)

        def e2e_step(i):
            k = i % 2
            s.wait_event(copied[k])
            Oparam.grad = None
            Pparam.grad = None
            loss = pkg.fused_loss(Oparam, Pparam, slots[k][1], slots[k][0], w.loss_type)
            loss.backward()
            exchange.all_reduce(Oparam.grad, Pparam.grad)  # N > 1: the step's gradient exchange
            out_host.copy_(loss.detach(), non_blocking=True)
            consumed[k].record(s)

        def run(n):
            issue_copy(0)
            if n > 1:
                issue_copy(1)
            for i in range(n):
                e2e_step(i)
                if i + 2 < n:
                    issue_copy(i + 2)

        run(args.warmup)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        cs.wait_stream(s)
        run(args.steps)
        s.wait_stream(cs)
        e1.record(s)
        torch.cuda.synchronize()
        et = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(et, op=dist.ReduceOp.MAX)
        e2e = {"value": world * B * args.steps / (float(et) / 1e3), "unit": "patterns/s",
               "h2d_bytes_per_step": int(Im_host[0].numel() * 4 + tl_host[0].numel() * 4),
               "d2h_bytes_per_step": 8,
               "note": "fused_loss + backward through the public API; each step's measurements and "
                       "windows copied from pinned host memory (copy stream, double-buffered against "
                       "the previous step's compute) and its loss read back; one interval over all "
                       "steps, L2 not flushed (the measurements arrive from the host every step)"}

        # the reference's own data flow (Recovery.py:103, 243-249): the stack stays
        # resident on the GPU and a step's host input is its minibatch of frame ids
        ids_host = [batches[i].cpu().pin_memory() for i in range(min(nb, 4))]
        ids_dev = torch.empty_like(batches[0])

        def resident_step(i):
            ids_dev.copy_(ids_host[i % len(ids_host)], non_blocking=True)
            Oparam.grad = None
            Pparam.grad = None
            loss = pkg.fused_loss(Oparam, Pparam, tl, stack, w.loss_type, batch=ids_dev)
            loss.backward()
            exchange.all_reduce(Oparam.grad, Pparam.grad)  # N > 1: the step's gradient exchange
            out_host.copy_(loss.detach(), non_blocking=True)

        for i in range(args.warmup):
            resident_step(i)
        torch.cuda.synchronize()
        r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        r0.record(s)
        for k in range(args.steps):
            resident_step(k)
        r1.record(s)
        torch.cuda.synchronize()
        rt = torch.tensor([r0.elapsed_time(r1)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(rt, op=dist.ReduceOp.MAX)
        e2e_resident = {"value": world * B * args.steps / (float(rt) / 1e3), "unit": "patterns/s",
                        "h2d_bytes_per_step": int(ids_host[0].numel() * 4), "d2h_bytes_per_step": 8,
                        "note": "fused_loss(batch=frame ids) + backward through the public API with the "
                                "measurement stack resident in HBM, as the reference keeps it on the GPU; "
                                "per step the frame ids are copied in and the loss read back"}

    if rank == 0:
        peak, kind = measured_peak_hbm()
        bpp = algorithmic_bytes_per_pattern(M, B)
        step_s = (t_max_ms / 1e3) / args.steps
        achieved = bpp * B / step_s / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": f"of {kind}",
                "kernel": "ptycho_fwd_adj (k_fused + k_assemble), one CUDA-graph launch per minibatch",
                "algorithmic_bytes_per_pattern": bpp, "traffic": load_traffic(f"{args.workload}_fwd_adj")}
        line = {"metric": METRIC, "value": value, "unit": "patterns/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_max_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "complex64 (fp32), fp64 loss reduction",
                "data": "synthetic (seeded generator; reference datasets not distributed)",
                "config": _config(w, B, args), "roofline": roof, "e2e": e2e,
                "e2e_resident_stack": e2e_resident, "gpu_launches": launches,
                "exchange": {"scheme": "dO halo rows point to point, dP all-reduce (NCCL)" if world > 1 else "none (one rank)",
                             "bytes_per_step_per_rank": exchange.bytes_per_step(W, M, M),
                             "full_band_all_reduce_bytes": 8 * (exchange.rows[1] - exchange.rows[0]) * W + 8 * M * M},
                "clocks": clk.summary(note=f"sampled every 50 ms over the {args.steps} timed steps and "
                                           f"{n_settle} identical untimed steps on either side "
                                           f"(~{args.settle_s:.1f} s each)")}
        if world == 1 and not args.no_side and args.workload == "c1":
            # the 256^2 cluster path on the c3 / c4 shapes, recorded beside the headline
            side = {}
            for key in ("c3", "c4"):
                try:
                    side[key] = side_workload(pkg, key, dev)
                except Exception as exc:  # reported, not fatal for the throughput line
                    side[key] = {"error": f"{type(exc).__name__}: {exc}"}
                torch.cuda.empty_cache()
            line["other_workloads"] = side
        if world == 1 and not args.no_ttr and args.workload == "c1":
            # the headline's second half: time-to-residual, INR vs pixel grid (c2); run
            # before the CPU baseline, whose idle OpenMP workers would share the host
            # cores with the timed training loops
            try:
                line["time_to_residual"] = ttr_summary(time_to_residual(args))
            except Exception as exc:  # reported, not fatal for the throughput line
                line["time_to_residual"] = {"error": f"{type(exc).__name__}: {exc}"}
        if not args.no_cpu_baseline and world == 1:
            rate, n, steps, cores, first = cpu_reference_rate(work, B, budget_s=args.cpu_budget)
            line["cpu_baseline"] = {"value": rate, "unit": "patterns/s", "cores": cores, "kind": "port",
                                    "sample": f"{steps} minibatches x {B} patterns ({n} patterns) of the "
                                              f"same workload, per-frame torch CPU loop + autograd "
                                              f"(reference restatement), {cores} threads",
                                    "parity_first_minibatch": parity_vs_cpu(pkg, work, first, dev)}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def time_to_residual(args):
    """Time-to-residual on workload c2 (1024^2 canvas, 128^2 probe, 28x28 raster,
    smooth_L1, batch 10; or --ttr-workload c3 / c4 with the settings of
    TTR_SETTINGS and WORKLOADS_DESC): the pixel grid (object and probe as plain parameters,
    fused kernels, Adam lr 1e-2 decayed x0.3 every pg-epochs/5 epochs) trains
    for --pg-epochs epochs and sets the
    target = 1.1 x its final data residual R = sum (sqrt(I) - sqrt(Imeas))^2 /
    sum Imeas (FP64 over the whole stack).  Then the INR built on the
    hand-written kernels and the reference INR (models/complex_inr.py and the
    per-frame Recovery.py loop in torch with torch.fft; tiny-cuda-nn replaced by
    a torch HashGrid restatement because it cannot be installed) each train
    until R <= target or their wall-time cap.  R is evaluated once per epoch,
    outside the timed wall time."""
    dev = torch.device("cuda")
    pkg = importlib.import_module(PKG)
    rec = importlib.import_module(PKG + ".recovery")
    from oracle import torch_inr
    wl = args.ttr_workload
    cfgw = TTR_SETTINGS[wl]
    work = pkg.synth.make_workload(wl, device=dev)
    w = work["workload"]
    canvas, bsz, grid = w.canvas, cfgw["batch"], cfgw["grid"]
    ds = canvas // grid
    stack = torch.from_numpy(work["Imeas"]).to(dev)
    tl = pkg.make_windows(work["tlY"], work["tlX"], dev)
    F, M = stack.shape[0], stack.shape[1]
    P0 = torch.from_numpy(work["probe"].astype(np.complex64)).to(dev) * float(np.sqrt(M * M))
    pls = torch_inr.per_level_scale_for(grid, 16, 16)
    out = {"metric": "time-to-residual (pixel-grid x1.1)", "workload": WORKLOADS_DESC[wl], "frames": F}
    gt = torch.from_numpy(work["obj"].astype(np.complex64)).to(dev)
    box = pkg.accuracy.coverage_box(work["tlY"], work["tlX"], (M, M), tuple(gt.shape), 0.5)

    @torch.no_grad()
    def object_err(model):  # FP64 on the device, global phase (and complex factor) removed, coverage box
        o = model()[0].reshape(gt.shape).to(torch.complex64)
        e = pkg.accuracy.object_error(o, gt, box)
        ea = pkg.accuracy.object_error_aligned(o, gt, box)  # after the sub-pixel translation as well
        return {"nrmse_phase": round(e["nrmse"], 5), "nrmse_scaled": round(e["nrmse_scaled"], 5),
                "nrmse_scaled_aligned": round(ea["nrmse_scaled"], 5), "shift": [round(v, 2) for v in ea["shift"]]}

    def timed(trainer, max_epochs, max_s, target):
        # garbage left by the previous arm (its CUDA graphs among it) is collected
        # here, outside the timed epochs, not by the cyclic GC during them; the
        # kernel arms capture their CUDA graphs first (one-time set-up, timed apart)
        import gc
        gc.collect()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if hasattr(trainer, "prepare"):
            trainer.prepare()
        torch.cuda.synchronize()
        setup_s[0] = time.perf_counter() - t0
        hist, t_train, reached = [], 0.0, None
        for ep in range(max_epochs):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            trainer.epoch()
            torch.cuda.synchronize()
            t_train += time.perf_counter() - t0
            r = trainer.residual()
            hist.append((ep + 1, round(t_train, 3), r))
            if target is not None and r <= target and reached is None:
                reached = (ep + 1, t_train, r)
                break
            if t_train > max_s:
                break
        return hist, reached, t_train

    setup_s = [0.0]
    pg = rec.PixelGrid((canvas, canvas), (M, M), probe_init=P0).to(dev)
    step = max(1, args.pg_epochs // 5)
    tpg = rec.Trainer(pg, stack, tl, w.loss_type, bsz, 1e-2, lr_decay_step=step, lr_decay_gamma=0.3)
    hist, _, t_pg = timed(tpg, args.pg_epochs, 1e9, None)
    r_pg = hist[-1][2]
    r_pg = min(h[2] for h in hist[-max(1, len(hist) // 10):])  # converged tail
    target = 1.1 * r_pg
    out["pixel_grid"] = {"epochs": len(hist), "seconds": round(t_pg, 3), "setup_seconds": round(setup_s[0], 3),
                         "residual": r_pg,
                         "object_error": object_err(pg), "history": hist[:: max(1, len(hist) // 10)]}
    out["object_error_box"] = list(box)
    out["target_residual"] = target
    cfg = dict(model_type="inr", downsample_factor=ds, n_levels=16, log2_hashmap_size=cfgw["log2T"],
               base_resolution=16,
               per_level_scale=pls, first_omega_0=10.0, hidden_omega_0=1.0, trainable_omega0=True,
               use_residual=True, init_type="initProbe")
    torch.manual_seed(0)  # the MLP initialisations (nn.Linear defaults) draw from torch's RNG
    model = rec.build_model(cfg, canvas, (M, M), P0, dev)
    tin = rec.Trainer(model, stack, tl, w.loss_type, bsz, cfgw["lr"])
    hist, reached, t_in = timed(tin, args.inr_epochs, args.inr_cap_s, target)
    out["inr_b200_kernels"] = {"reached": reached is not None, "seconds_to_target": reached[1] if reached else None,
                               "setup_seconds": round(setup_s[0], 3),
                               "epochs_to_target": reached[0] if reached else None,
                               "seconds": round(t_in, 3), "best_residual": min(h[2] for h in hist),
                               "object_error": object_err(model),
                               "ms_per_minibatch": 1e3 * t_in / (len(hist) * -(-F // bsz)),
                               "history": hist[:: max(1, len(hist) // 10)]}

    class RefTrainer:  # the reference loop, per frame, on this GPU
        def __init__(self):
            torch.manual_seed(0)
            self.model = torch_inr.RefINR(canvas, ds, M, 16, cfgw["log2T"], 16, pls, 10.0, 1.0,
                                          probe_initial=P0).to(dev)
            self.opt = torch.optim.Adam([p for p in self.model.parameters() if p.requires_grad], lr=cfgw["lr"])
            self.mmf = stack.permute(1, 2, 0).contiguous()
            self.rng = np.random.default_rng(0)
            self.t_start = None
            self.minibatches = 0

        def epoch(self):
            if self.t_start is None:
                self.t_start = time.perf_counter()
            perm = self.rng.permutation(F)
            for s0 in range(0, F, bsz):
                torch_inr.ref_minibatch(self.model, self.opt, self.mmf, work["tlY"], work["tlX"],
                                        perm[s0:s0 + bsz], w.loss_type)
                self.minibatches += 1
                if time.perf_counter() - self.t_start > args.ref_cap_s:
                    break  # one reference epoch of c4 runs past the cap

        @torch.no_grad()
        def residual(self):
            obj, probe = self.model()
            probe = rec.center_and_normalize_probe(probe)
            num = den = 0.0
            for s0 in range(0, F, 256):
                ids = torch.arange(s0, min(F, s0 + 256), device=dev, dtype=torch.int32)
                I = pkg.forward_intensity(obj.to(torch.complex64), probe.to(torch.complex64), tl, batch=ids).double()
                Im = stack[ids.long()].double()
                num += float(((I.sqrt() - Im.sqrt()) ** 2).sum())
                den += float(Im.sum())
            return num / den

    ref = RefTrainer()
    hist, reached, t_ref = timed(ref, args.inr_epochs, args.ref_cap_s, target)
    out["inr_reference_torch"] = {"reached": reached is not None, "object_error": object_err(ref.model),
                                  "seconds_to_target": reached[1] if reached else None,
                                  "epochs_to_target": reached[0] if reached else None,
                                  "seconds": round(t_ref, 3), "best_residual": min(h[2] for h in hist),
                                  "ms_per_minibatch": 1e3 * t_ref / max(1, ref.minibatches),
                                  "history": hist,
                                  "note": "reference ComplexINRModel2D/ComplexMLP and per-frame loop in torch "
                                          "(torch.fft); tiny-cuda-nn replaced by a torch HashGrid restatement"}
    return out


def run_time_to_residual(args):
    print(json.dumps(time_to_residual(args)), flush=True)


def ttr_summary(out):
    """The time-to-residual result in a few keys (for the default bench line)."""
    a, b, pg = out["inr_b200_kernels"], out["inr_reference_torch"], out["pixel_grid"]
    return {"metric": out["metric"], "workload": out["workload"],
            "unit": "s", "higher_is_better": False,
            "pixel_grid": {"epochs": pg["epochs"], "seconds": pg["seconds"], "residual": pg["residual"],
                           "object_error": pg["object_error"]},
            "target_residual": out["target_residual"],
            "inr_b200": {"seconds_to_target": a["seconds_to_target"], "epochs": a["epochs_to_target"],
                         "setup_seconds": a.get("setup_seconds"),
                         "ms_per_minibatch": a["ms_per_minibatch"], "object_error": a["object_error"]},
            "inr_reference_torch_same_gpu": {"seconds_to_target": b["seconds_to_target"],
                                             "epochs": b["epochs_to_target"],
                                             "ms_per_minibatch": b["ms_per_minibatch"],
                                             "object_error": b["object_error"],
                                             "note": "tiny-cuda-nn replaced by a torch HashGrid restatement"}}


def run_c0_reconstruction(args):
    """The reference's CPU-runnable case run in full: workload c0 (256^2 object,
    64^2 probe, 10x10 raster, 1e4 photons, smooth_L1 on intensities), object
    and probe both starting flat (ones), Adam lr 1e-2, batch 10, 200 epochs.
    Arm 1: the pixel grid on the B200 kernels (recovery.Trainer: probe centring
    and normalisation, fused loss and adjoint, fused Adam, one CUDA graph per
    minibatch).  Arm 2: the same loop in the reference's own form on this
    host's CPU cores (torch CPU, per-frame crop * probe, fft2, |.|^2, loss,
    autograd, torch.optim.Adam; Recovery.py:250-321).  Both results are scored
    by the same FP64 data residual on the GPU and the object error against the
    ground truth (global phase and scale removed, high-coverage box)."""
    dev = torch.device("cuda")
    pkg = importlib.import_module(PKG)
    rec = importlib.import_module(PKG + ".recovery")
    work = pkg.synth.make_workload("c0", device=None)
    w = work["workload"]
    stack = torch.from_numpy(work["Imeas"]).to(dev)
    tl = pkg.make_windows(work["tlY"], work["tlX"], dev)
    F, M, H = stack.shape[0], w.probe, w.canvas
    epochs, batch, lr = args.c0_epochs, 10, 1e-2
    gt = torch.from_numpy(work["obj"].astype(np.complex64)).to(dev)
    box = pkg.accuracy.coverage_box(work["tlY"], work["tlX"], (M, M), (H, H), 0.5)
    probe_prep = importlib.import_module(PKG + ".probe_prep")

    @torch.no_grad()
    def score(obj, probe):  # FP64 residual over the stack and object error, on the device
        obj = obj.to(dev, torch.complex64).contiguous()
        probe = probe_prep.center_and_normalize_probe(probe.to(dev, torch.complex64).contiguous())
        I = pkg.forward_intensity(obj, probe, tl).double()
        Im = stack.double()
        r = float(((I.sqrt() - Im.sqrt()) ** 2).sum() / Im.sum())
        e = pkg.accuracy.object_error(obj, gt, box)
        ea = pkg.accuracy.object_error_aligned(obj, gt, box)
        return r, {"nrmse_phase": round(e["nrmse"], 5), "nrmse_scaled": round(e["nrmse_scaled"], 5),
                   "nrmse_scaled_aligned": round(ea["nrmse_scaled"], 5), "shift": [round(v, 2) for v in ea["shift"]]}

    pg = rec.PixelGrid((H, H), (M, M)).to(dev)
    tr = rec.Trainer(pg, stack, tl, w.loss_type, batch, lr)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    t_first = None
    for ep in range(epochs):
        tr.epoch()
        if ep == 0:
            torch.cuda.synchronize()
            t_first = time.perf_counter() - t0
    torch.cuda.synchronize()
    t_gpu = time.perf_counter() - t0
    r_gpu, e_gpu = score(*pg())

    from oracle import torch_inr  # the reference minibatch, run here on the CPU
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    cpu = rec.PixelGrid((H, H), (M, M))
    opt = torch.optim.Adam([p for p in cpu.parameters() if p.requires_grad], lr=lr)
    mmf = torch.from_numpy(np.ascontiguousarray(np.moveaxis(work["Imeas"], 0, -1)))  # [M, M, F]
    rng = np.random.default_rng(0)
    cpu_epochs = epochs
    t0 = time.perf_counter()
    for ep in range(epochs):
        perm = rng.permutation(F)
        for s0 in range(0, F, batch):
            torch_inr.ref_minibatch(cpu, opt, mmf, work["tlY"], work["tlX"], perm[s0:s0 + batch], w.loss_type)
        if time.perf_counter() - t0 > args.ref_cap_s:
            cpu_epochs = ep + 1
            break
    t_cpu = time.perf_counter() - t0
    r_cpu, e_cpu = score(*cpu())
    out = {"metric": "c0 pixel-grid reconstruction (flat start, 200 epochs): wall time and final data residual",
           "workload": w.name + f", {F} frames, batch {batch}, Adam lr {lr}",
           "b200_kernels": {"epochs": epochs, "seconds": round(t_gpu, 4),
                            "seconds_first_epoch_incl_graph_capture": round(t_first, 4),
                            "residual": r_gpu, "object_error": e_gpu},
           "reference_loop_cpu": {"epochs": cpu_epochs, "seconds": round(t_cpu, 3),
                                  "seconds_per_epoch": t_cpu / cpu_epochs, "threads": torch.get_num_threads(),
                                  "residual": r_cpu, "object_error": e_cpu,
                                  "note": "the reference loop restated in torch on the CPU "
                                          "(per-frame torch.fft + autograd, torch.optim.Adam)"},
           "residual_definition": "sum (sqrt(I) - sqrt(Imeas))^2 / sum Imeas over the stack, FP64, on the GPU",
           "object_error_box": list(box)}
    print(json.dumps(out), flush=True)


def run_inr_step(args):
    """Throughput of one INR training minibatch on workload c2 (or --ttr-workload
    c3 / c4 with the settings of TTR_SETTINGS), graph-replayed: HashGrid forward,
    tcgen05 MLP forward, Fourier upsample, probe INR, fused loss of one
    minibatch, backward through all of them, fused Adam.  Reports ms per
    minibatch and the MLP's tensor-core FLOP rate (forward 18.6 kflop per
    coordinate, backward with the recomputed forward 3 x that)."""
    dev = torch.device("cuda")
    pkg = importlib.import_module(PKG)
    rec = importlib.import_module(PKG + ".recovery")
    from oracle import torch_inr  # per-level scale formula only
    wl = args.ttr_workload
    cfgw = TTR_SETTINGS[wl]
    work = pkg.synth.make_workload(wl, device=dev)
    w = work["workload"]
    stack = torch.from_numpy(work["Imeas"]).to(dev)
    tl = pkg.make_windows(work["tlY"], work["tlX"], dev)
    M, grid, bsz = stack.shape[1], cfgw["grid"], cfgw["batch"]
    P0 = torch.from_numpy(work["probe"].astype(np.complex64)).to(dev) * float(M)
    cfg = dict(model_type="inr", downsample_factor=w.canvas // grid, n_levels=16, log2_hashmap_size=cfgw["log2T"],
               base_resolution=16, per_level_scale=torch_inr.per_level_scale_for(grid, 16, 16), first_omega_0=10.0,
               hidden_omega_0=1.0, trainable_omega0=True, use_residual=True, init_type="initProbe")
    model = rec.build_model(cfg, w.canvas, (M, M), P0, dev)
    tr = rec.Trainer(model, stack, tl, w.loss_type, bsz, cfgw["lr"])
    g = torch.Generator(device=dev).manual_seed(0)
    batches = [torch.randperm(stack.shape[0], device=dev, generator=g)[:bsz].to(torch.int32)
               for _ in range(args.warmup + args.steps)]
    for i in range(args.warmup):
        tr.run(batches[i])
    torch.cuda.synchronize()
    s = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for i in range(args.steps):
        tr.run(batches[args.warmup + i])
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    coords = grid * grid + M * M
    flops = coords * 18624 * 4  # forward + backward (recomputed forward + 2 GEMM passes)
    print(json.dumps({"metric": f"INR training minibatch ({wl})", "ms_per_minibatch": ms, "steps": args.steps,
                      "workload": WORKLOADS_DESC[wl], "coordinates_per_minibatch": coords,
                      "mlp_tflops_effective": flops / (ms * 1e-3) / 1e12,
                      "note": "one CUDA-graph replay per minibatch; MLP flops counted as 4 x 18.6 kflop/coord"}),
          flush=True)


def run_gs(args):
    """Gaussian-field rasteriser (the alternate object representation): one
    step = forward render + backward of N Cholesky Gaussians onto a 512^2 grid
    (the INR's 512^2 object grid for a 1024^2 canvas at downsample 2) through
    the public autograd Function, sigma in [0.6, 3] px, max_patch_radius 16,
    min_scale 0.5.  L2 flushed before every timed step; CUDA events."""
    dev = torch.device("cuda")
    pkg = importlib.import_module(PKG)
    N, H, W = args.gs_gaussians, 512, 512
    rng = np.random.default_rng(0)
    xy = np.stack([rng.uniform(0, W - 1, N), rng.uniform(0, H - 1, N)], 1).astype(np.float32)
    p1 = rng.uniform(np.log(0.6), np.log(3.0), (N, 2)).astype(np.float32)
    p2 = rng.uniform(-1, 1, N).astype(np.float32)
    wt = (0.05 * rng.standard_normal((N, 2))).astype(np.float32)
    gout = torch.from_numpy(rng.standard_normal((2, H, W)).astype(np.float32)).to(dev)
    leaves = [torch.from_numpy(a).to(dev).requires_grad_(True) for a in (xy, p1, p2, wt)]
    fn = pkg.gsplat.GaussianRasterize2DCholesky
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    impl = "ours"

    def step():
        for t in leaves:
            t.grad = None
        out = fn.apply(*leaves, H, W, 16, 0.5)
        out.backward(gout)

    if args.impl == "reference":
        # the reference's own rasteriser (gscp/csrc/gscp_rasterizer, compiled from
        # its sources with its flags into oracle/_ref), same scene, same GPU
        import ctypes
        so = os.path.join(ROOT, "oracle", "_ref", "libgscp_ref.so")
        if not os.path.exists(so):
            print(json.dumps({"impl": "reference", "metric": "Gaussian-field render fwd+bwd",
                              "unavailable": "oracle/_ref/libgscp_ref.so was not built (needs the reference tree)"}))
            return
        L = ctypes.CDLL(so)
        vp, ci, cf = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.gscp_ref_create.restype = vp
        L.gscp_ref_forward.argtypes = [vp, ci, ci, ci, ci, vp, vp, vp, vp, ci, cf, vp, vp]
        L.gscp_ref_backward.argtypes = [vp, ci, ci, ci, ci, vp, vp, vp, vp, ci, cf, vp, vp, vp, vp, vp, vp, vp, vp]
        L.gscp_ref_destroy.argtypes = [vp]
        xy_d, p1_d, p2_d, w_d = (t.detach() for t in leaves)
        out = torch.empty((2, H, W), device=dev)
        radii = torch.empty(N, dtype=torch.int32, device=dev)
        bufs = [torch.empty(s, device=dev) for s in ((N, 2), (N, 3), (N, 2), (N, 2), (N, 2), (N,))]
        h = L.gscp_ref_create()
        impl = "reference"

        def step():  # noqa: F811 -- the reference arm's step
            for b in bufs:  # the reference accumulates its gradients with atomicAdd
                b.zero_()
            assert L.gscp_ref_forward(h, 1, N, H, W, xy_d.data_ptr(), p1_d.data_ptr(), p2_d.data_ptr(),
                                      w_d.data_ptr(), 16, 0.5, out.data_ptr(), radii.data_ptr()) >= 0
            assert L.gscp_ref_backward(h, 1, N, H, W, xy_d.data_ptr(), p1_d.data_ptr(), p2_d.data_ptr(),
                                       w_d.data_ptr(), 16, 0.5, radii.data_ptr(), gout.data_ptr(),
                                       *[b.data_ptr() for b in bufs]) == 0

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    s = torch.cuda.current_stream(dev)
    times = []
    for _ in range(args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        step()
        b.record(s)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    ms = float(np.mean(times))
    line = {"metric": "Gaussian-field render fwd+bwd", "value": N / (ms * 1e-3), "unit": "Gaussians/s",
            "ms_per_step": ms, "steps": args.steps, "warmup": max(3, args.warmup), "higher_is_better": True,
            "config": {"workload": f"{N} Cholesky Gaussians, 512^2 grid, sigma 0.6-3 px, 16x16 tiles",
                       "l2": "flushed before every timed step"},
            "gpu_launches_per_step": 5, "dtype": "f32", "data": "synthetic (seeded)"}
    if impl == "reference":
        line.update({"impl": "reference", "gpu_launches_per_step": None,
                     "note": "the reference's rasteriser compiled from its CUDA sources (-O3 --use_fast_math), "
                             "with its host read-back of the tile-pair count and its radix sort"})
        L.gscp_ref_destroy(h)
    elif not args.no_cpu_baseline:
        from oracle import gsplat as og  # the CPU restatement, timed as the baseline only
        n = min(N, 40000)
        t0 = time.perf_counter()
        ref_img, _ = og.render(og.CHOLESKY, xy[:n], p1[:n], p2[:n], wt[:n], H, W, 16, 0.5)
        ref_g = og.backward(og.CHOLESKY, xy[:n], p1[:n], p2[:n], wt[:n], H, W, 16, 0.5, gout.cpu().numpy())
        dt = time.perf_counter() - t0
        # the kernels on the same subset, checked against that float64 restatement
        sub = [t.detach()[:n].clone().requires_grad_(True) for t in leaves]
        img = fn.apply(*sub, H, W, 16, 0.5)
        img.backward(gout)
        rn = lambda a, b: float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))  # noqa: E731
        parity = {"image_rel_err": rn(img.detach().cpu().numpy(), ref_img)}
        for name, t, r in zip(("dxy", "dlog_L_diag", "dL_offdiag", "dweight"), sub, ref_g):
            parity[name + "_rel_err"] = rn(t.grad.cpu().numpy().reshape(r.shape), r)
        line["cpu_baseline"] = {"value": n / dt, "unit": "Gaussians/s", "cores": 1, "kind": "port",
                                "sample": f"first {n} Gaussians of the same scene, NumPy restatement, fwd+bwd",
                                "parity_vs_oracle": parity}
    print(json.dumps(line), flush=True)


def run_aux(args):
    """The auxiliary kernels around the two hot loops, each timed alone with CUDA
    events over --steps launches (L2 warm: they run between the hot kernels):
    Haar sparsity and its backward (1024^2 object), the FP64 object error
    (1024^2), probe centring/normalisation and its backward (128^2), and the
    hash-encoder CSR build (262,144 coordinates, 16 levels, log2 T 18)."""
    dev = torch.device("cuda")
    pkg = importlib.import_module(PKG)
    rng = np.random.default_rng(0)
    c = lambda *s: torch.from_numpy((rng.standard_normal(s) + 1j * rng.standard_normal(s)).astype(np.complex64)).to(dev)  # noqa: E731
    obj, gt, probe = c(1024, 1024), c(1024, 1024), c(128, 128)
    s = torch.cuda.current_stream(dev)

    def timed(fn):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for _ in range(args.steps):
            fn()
        b.record(s)
        torch.cuda.synchronize()
        return 1e3 * a.elapsed_time(b) / args.steps  # us

    ops = {}
    leaf = obj.clone().requires_grad_(True)

    def haar():
        leaf.grad = None
        pkg.probe_prep.haar_sparsity(leaf).backward()
    ops["haar_sparsity fwd+bwd (1024^2)"] = (timed(haar), 1024 * 1024 * 8 * 3)
    ops["object_error (1024^2, FP64)"] = (timed(lambda: pkg.accuracy.object_error(obj, gt)), 1024 * 1024 * 16)
    pl = probe.clone().requires_grad_(True)
    gp = c(128, 128)

    def prep():
        pl.grad = None
        pkg.probe_prep.center_and_normalize_probe(pl).backward(gp)
    ops["probe centre+normalise fwd+bwd (128^2)"] = (timed(prep), 128 * 128 * 8 * 5)
    enc = pkg.hashgrid.Encoding(2, {"otype": "HashGrid", "n_levels": 16, "n_features_per_level": 2,
                                    "log2_hashmap_size": 18, "base_resolution": 16,
                                    "per_level_scale": float(np.exp(np.log(32) / 15))}).to(dev)
    yy, xx = torch.meshgrid(torch.linspace(0, 1, 512, device=dev), torch.linspace(0, 1, 512, device=dev),
                            indexing="ij")
    coords = torch.stack([xx.flatten(), yy.flatten()], 1).contiguous()
    ops["hash CSR build (262,144 coords, one-time)"] = (
        timed(lambda: pkg.hashgrid._CSR(coords, enc.cfg, enc.n_entries)), 262144 * 16 * 4 * 12)
    out = {k: {"us": round(v, 2), "GB/s_algorithmic": round(b / (v * 1e-6) / 1e9, 1)} for k, (v, b) in ops.items()}
    print(json.dumps({"metric": "auxiliary kernels", "steps": args.steps, "ops": out,
                      "note": "each op through its public Python call; inputs resident, L2 warm"}), flush=True)


WORKLOADS_DESC = {"c2": "c2: 1024^2 canvas, 128^2 probe, 28x28 raster (784 frames), smooth_L1, batch 10; INR "
                        "16 levels x 2, log2 T 18, base 16, finest 512, 512^2 object grid (ds 2), MLP 64x2, "
                        "omega 10/1, probe initProbe + residual",
                  "c3": "c3: 2048^2 object, 256^2 probe, 48x48 raster (2304 frames), Poisson, 1e3 photons, "
                        "batch 64; INR 16 levels x 2, log2 T 19, base 16, finest 1024, 1024^2 object grid (ds 2), "
                        "MLP 64x2, omega 10/1, probe INR + initProbe residual",
                  "c4": "c4: 4096^2 object, 256^2 probe, 96x96 raster (9216 frames), Poisson, 1e3 photons, "
                        "batch 512; INR 16 levels x 2, log2 T 20, base 16, finest 2048, 2048^2 object grid (ds 2), "
                        "MLP 64x2, omega 10/1, probe INR + initProbe residual"}
# per workload: INR object grid (canvas / ds), log2 hash-table size, minibatch, INR learning rate
TTR_SETTINGS = {"c2": dict(grid=512, log2T=18, batch=10, lr=1e-3),
                "c3": dict(grid=1024, log2T=19, batch=64, lr=1e-3),
                "c4": dict(grid=2048, log2T=20, batch=512, lr=1e-3)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="c1")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--ref-batch", type=int, default=0)
    ap.add_argument("--time-to-residual", action="store_true")
    ap.add_argument("--ttr-workload", choices=sorted(TTR_SETTINGS), default="c2",
                    help="workload of the time-to-residual protocol")
    ap.add_argument("--inr-step", action="store_true")
    ap.add_argument("--pg-epochs", type=int, default=200)
    ap.add_argument("--inr-epochs", type=int, default=2000)
    ap.add_argument("--inr-cap-s", type=float, default=60.0)
    ap.add_argument("--ref-cap-s", type=float, default=90.0)
    ap.add_argument("--no-ttr", action="store_true", help="omit the time-to-residual object from the bench line")
    ap.add_argument("--no-side", action="store_true", help="omit the c3 / c4 records from the c1 bench line")
    ap.add_argument("--settle-s", type=float, default=SETTLE_S,
                    help="seconds of untimed steps on either side of the timed ones (clock sampling)")
    ap.add_argument("--gs", action="store_true", help="time the Gaussian-field rasteriser instead")
    ap.add_argument("--c0-reconstruction", action="store_true",
                    help="run workload c0's full pixel-grid reconstruction on the GPU and the CPU reference loop")
    ap.add_argument("--c0-epochs", type=int, default=200)
    ap.add_argument("--aux", action="store_true", help="time the auxiliary kernels instead")
    ap.add_argument("--gs-gaussians", type=int, default=100000)
    args = ap.parse_args()
    if args.time_to_residual:
        run_time_to_residual(args)
        return
    if args.inr_step:
        run_inr_step(args)
        return
    if args.gs:
        run_gs(args)
        return
    if args.aux:
        run_aux(args)
        return
    if args.c0_reconstruction:
        run_c0_reconstruction(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
