"""Far-field ptychography reconstruction driver -- mirrors Recovery.py.

    python -m <package>.recovery --config config.yaml

Same CLI, YAML keys and outputs as the reference script (Recovery.py:44-383):
the YAML sections are flattened one level and type-coerced (:44-72), the
data are read from .mat files (utils/io.py:72-122), scan positions become
windows (utils/optics.py:68-99), the model is ComplexINRModel2D (or, with
``model_type: pixel_grid``, a plain pixel-grid object/probe), and each epoch
draws a random permutation of the frames and runs minibatches of
``batch_size`` (:243-350).  Per minibatch, as in the reference:

* ``object, probe = model()``;
* the probe is re-centred by its centre of mass and scaled to
  sum|P|^2 = M*N (:262-285) -- here on the device, without host syncs;
* the per-frame losses of the minibatch are summed (:288-307) -- here one
  fused forward/loss/adjoint call on frame ids into the resident stack;
* Haar sparsity (:309-313) is added when ``sparsity_weight`` is non-zero;
* backward, Adam step (FusedAdam), StepLR once per epoch.

Outputs: ``result.mat`` with ``object_complex`` / ``probe_complex`` and
``trained_models.pth`` (the requires_grad tensors in named_parameters order)
every ``vis_interval`` epochs and at the end (:352-383).  The per-epoch PNG
panels need matplotlib, which is not part of this environment; they are
skipped.
"""
from __future__ import annotations

import argparse
import math
import os
import time

import numpy as np
import torch
import yaml

from . import h5mat, optics, probe_prep, scan_shards
from .adam import FusedAdam
from .complex_inr import ComplexINRModel2D

VALID_INIT_TYPES = ("initNone", "initProbe", "initQuadratic")
VALID_LOSS_TYPES = ("smooth_L1_loss", "FD_loss", "Poisson_likelihood_loss")
VALID_MODEL_TYPES = ("inr", "gaussian_field", "pixel_grid")
_FLOAT_KEYS = ("wavelength", "camera_length", "camera_pixel_pitch", "lr", "lr_decay_gamma", "per_level_scale",
               "first_omega_0", "hidden_omega_0", "sparsity_weight", "quadratic_focal_length")
_INT_KEYS = ("gap", "downsample_factor", "iters", "lr_decay_step", "n_levels", "n_features_per_level",
             "log2_hashmap_size", "base_resolution", "hidden_features", "hidden_layers", "vis_interval",
             "batch_size", "zoom_size")


def load_config(path):
    """Flatten YAML sections one level, coerce types, validate enums (Recovery.py:44-72)."""
    with open(path, "r", encoding="utf-8") as f:
        raw = yaml.safe_load(f)
    cfg = {}
    for section in raw.values():
        if isinstance(section, dict):
            cfg.update(section)
    for k in _FLOAT_KEYS:
        if k in cfg and cfg[k] is not None:
            cfg[k] = float(cfg[k])
    for k in _INT_KEYS:
        if k in cfg and cfg[k] is not None:
            cfg[k] = int(cfg[k])
    for key, valid, default in (("init_type", VALID_INIT_TYPES, "initNone"),
                                ("loss_type", VALID_LOSS_TYPES, "smooth_L1_loss"),
                                ("model_type", VALID_MODEL_TYPES, "inr")):
        v = cfg.get(key, default)
        if v not in valid:
            raise ValueError(f"{key} must be one of {valid}, got {v!r}")
    return cfg


def load_ptychography_data(data_dir, bundle_file=None, location_file=None, raw_file=None, probe_file=None,
                           gt_file=None, init_probe_file=None, gap=1):
    """.mat bundle or per-variable files -> dict (utils/io.py:72-122).  Files
    are read as utils/io.py:read_data does: scipy's loadmat (v4 - v7), and
    MATLAB v7.3 (HDF5) files through h5mat.read_mat73 (arrays transposed back
    to MATLAB's dimension order, {real, imag} compounds made complex)."""
    return _load(data_dir, bundle_file, location_file, raw_file, probe_file, gt_file, init_probe_file, gap)


def read_data(file_path, key_name=None):
    """One .mat file -> {name: value} (utils/io.py:25-69): loadmat first, the
    v7.3 (HDF5) reader when loadmat cannot read the file."""
    from scipy.io import loadmat

    try:
        return loadmat(file_path)
    except Exception:
        if not h5mat.is_hdf5(file_path):
            raise
    return h5mat.read_mat73(file_path, key_name)


def _load(data_dir, bundle_file, location_file, raw_file, probe_file, gt_file, init_probe_file, gap):
    def read(name):
        return read_data(os.path.join(data_dir, name))

    out = {}
    if bundle_file is not None:
        b = read(bundle_file)
        for k in ("xlocation", "ylocation", "probe", "imRaw", "obj", "initProbe"):
            if k in b:
                out[k] = b[k]
    if location_file is not None:
        loc = read(location_file)
        out["xlocation"], out["ylocation"] = loc["xlocation"], loc["ylocation"]
    if raw_file is not None:
        out["imRaw"] = read(raw_file)["imRaw"]
    if probe_file is not None:
        out["probe"] = read(probe_file)["probe"]
    for fname, key in ((gt_file, "obj"), (init_probe_file, "initProbe")):
        if fname is not None:
            d = read(fname)
            out[key] = d.get(key, next(v for k, v in d.items() if not k.startswith("__")))
    out["xlocation"] = np.asarray(out["xlocation"]).squeeze()
    out["ylocation"] = np.asarray(out["ylocation"]).squeeze()
    if gap and gap > 1:
        out["xlocation"] = out["xlocation"][::gap]
        out["ylocation"] = out["ylocation"][::gap]
        out["imRaw"] = out["imRaw"][:, :, ::gap]
    return out


class PixelGrid(torch.nn.Module):
    """Object and probe as plain complex64 parameters (the pixel-grid baseline);
    ``forward()`` has the model contract of ComplexINRModel2D."""

    def __init__(self, canvas_hw, probe_hw, object_init=None, probe_init=None):
        super().__init__()
        O = torch.ones(canvas_hw, dtype=torch.complex64) if object_init is None else object_init.clone()
        P = torch.ones(probe_hw, dtype=torch.complex64) if probe_init is None else probe_init.clone()
        self.object = torch.nn.Parameter(O.to(torch.complex64))
        self.probe = torch.nn.Parameter(P.to(torch.complex64))

    def forward(self):
        return self.object, self.probe


def center_and_normalize_probe(P: torch.Tensor) -> torch.Tensor:
    """Centre-of-mass roll (Recovery.py:262-278) and energy scaling to
    sum|P|^2 = M*N (:282-285): one device kernel each way, no host syncs."""
    return probe_prep.center_and_normalize_probe(P)


def haar_sparsity(img: torch.Tensor) -> torch.Tensor:
    """L1 of the LH/HL/HH Haar subbands of Re and Im (utils/loss.py:60-83),
    on the device kernels (FP64 reduction, no host syncs)."""
    return probe_prep.haar_sparsity(img)


class Trainer:
    """The reference training loop on resident data (one object per run).

    Under an initialised ``torch.distributed`` process group of more than one
    rank (one process per GPU), each rank trains on its own band of the
    raster (``scan_shards``), every rank takes the same number of minibatches
    per epoch, and the parameter gradients are summed over the ranks after
    each backward pass.  A pixel-grid object's gradient is combined by the
    halo exchange (only rows shared by neighbouring bands cross the link;
    each rank's object is current on its band and ``current`` / ``residual``
    gather it first), all other gradients by all-reduce, so the replicas that
    the next forward reads stay identical.  That mode runs eagerly (no CUDA
    graph holds a collective)."""

    def __init__(self, model, stack, tl, loss_type, batch_size, lr, lr_decay_step=10000, lr_decay_gamma=0.1,
                 sparsity_weight=0.0, seed=0, use_graph=True):
        import torch.distributed as dist
        self.world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
        self.rank = dist.get_rank() if self.world > 1 else 0
        if self.world > 1:
            use_graph = False
            tl_host = tl.cpu().numpy()
            self.frames = scan_shards.shard_frames(tl_host[:, 0], tl_host[:, 1], self.world, self.rank)
            self.steps = scan_shards.steps_per_epoch(int(stack.shape[0]), self.world, int(batch_size))
            self.np_rng = np.random.default_rng(seed + self.rank)
            # the halo exchange needs a row-local loss: the Haar term couples rows across band edges
            self.halo = isinstance(model, PixelGrid) and float(sparsity_weight) == 0.0
            self.exchange = scan_shards.GradientExchange(tl_host[:, 0], tl_host[:, 1], int(stack.shape[1]),
                                                         halo=self.halo)
        self.model = model
        self.stack = stack  # [F, M, N] float32, device
        self.tl = tl        # [F, 2] int32, device
        self.F = int(stack.shape[0])
        self.loss_type = loss_type
        self.batch_size = int(batch_size)
        self.sparsity_weight = float(sparsity_weight)
        self.opt = FusedAdam([p for p in model.parameters() if p.requires_grad], lr=lr, capturable=use_graph)
        self.sched = torch.optim.lr_scheduler.StepLR(self.opt, step_size=lr_decay_step, gamma=lr_decay_gamma)
        self.gen = torch.Generator(device=stack.device).manual_seed(seed)
        self.last_loss = None
        self.use_graph = use_graph
        self._graphs = {}  # minibatch length -> (graph, static batch buffer, static loss)
        self._pool = None

    def _graph_for(self, n: int):
        """Capture the whole minibatch step (model forward, fused loss, backward,
        Adam) for minibatches of length n; the frame ids live in a static buffer."""
        ent = self._graphs.get(n)
        if ent is not None:
            return ent
        dev = self.stack.device
        buf = torch.arange(n, dtype=torch.int32, device=dev)
        # warm-up outside capture (CSR, workspaces, FFT plans, kernel attributes);
        # parameters and optimizer state are restored afterwards
        # only trainable parameters change; frozen ones (the INR's coordinate grids)
        # are left untouched, so caches keyed on their version stay valid
        params = [p for p in self.model.parameters() if p.requires_grad]
        saved = [p.detach().clone() for p in params]
        saved_opt = {k: (v["exp_avg"].clone(), v["exp_avg_sq"].clone()) for k, v in self.opt.state.items()
                     if "exp_avg" in v}
        saved_dev = [(d["step"].clone(), d["lr"].clone()) for d in self.opt._dev]
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            for _ in range(2):
                self.step(buf)
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize(dev)
        with torch.no_grad():
            for p, v in zip(params, saved):
                p.copy_(v)
            for k, v in self.opt.state.items():
                if "exp_avg" in v:
                    if k in saved_opt:
                        v["exp_avg"].copy_(saved_opt[k][0])
                        v["exp_avg_sq"].copy_(saved_opt[k][1])
                    else:
                        v["exp_avg"].zero_()
                        v["exp_avg_sq"].zero_()
            for d, (st, lr) in zip(self.opt._dev, saved_dev):
                d["step"].copy_(st)
                d["lr"].copy_(lr)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, pool=self._pool):
            loss = self.step(buf)
        self._pool = g.pool()
        ent = (g, buf, loss)
        self._graphs[n] = ent
        return ent

    def prepare(self) -> None:
        """Capture the graphs of an epoch's minibatch lengths now (full and, when
        the frames do not divide evenly, the last one) instead of at their first
        use; parameters and optimizer state are unchanged."""
        if not self.use_graph or self.world > 1:
            return
        for n in {min(self.batch_size, self.F), self.F % self.batch_size} - {0}:
            self._graph_for(n)

    def run(self, batch_ids: torch.Tensor) -> torch.Tensor:
        """One minibatch: replay of the captured step (or an eager step)."""
        if not self.use_graph:
            return self.step(batch_ids)
        g, buf, loss = self._graph_for(int(batch_ids.numel()))
        buf.copy_(batch_ids)
        g.replay()
        self.last_loss = loss
        return loss

    def step(self, batch_ids: torch.Tensor) -> torch.Tensor:
        self.opt.zero_grad(set_to_none=True)
        obj, probe = self.model()
        if probe is None:
            raise RuntimeError("update_probe must be True for conventional ptychography")
        probe = center_and_normalize_probe(probe.squeeze())
        obj = obj.squeeze()
        loss = optics.fused_loss(obj, probe, self.tl, self.stack, self.loss_type, batch=batch_ids)
        if self.sparsity_weight != 0.0:
            loss = loss + self.sparsity_weight * haar_sparsity(obj)
        loss.backward()
        if self.world > 1:
            if self.halo:
                self.exchange.all_reduce(self.model.object.grad, self.model.probe.grad)
            else:
                scan_shards.all_reduce_grads([p for p in self.model.parameters() if p.requires_grad])
        self.opt.step()
        self.last_loss = loss.detach()
        return self.last_loss

    def epoch(self):
        if self.world > 1:
            for b in scan_shards.epoch_minibatches(self.frames, self.batch_size, self.steps, self.np_rng):
                self.run(torch.from_numpy(b.astype(np.int32)).to(self.stack.device))
            self.sched.step()
            return
        perm = torch.randperm(self.F, device=self.stack.device, generator=self.gen).to(torch.int32)
        for s in range(0, self.F, self.batch_size):
            self.run(perm[s:s + self.batch_size])
        self.sched.step()
        if self.use_graph:
            self.opt.sync_lr()

    def _gather(self):
        """World > 1 with the halo exchange: assemble the whole object from the
        ranks' owned rows (every rank calls this at the same point)."""
        if self.world > 1 and self.halo:
            with torch.no_grad():
                self.exchange.gather_object(self.model.object.data)

    @torch.no_grad()
    def current(self):
        self._gather()
        obj, probe = self.model()
        return obj.squeeze(), center_and_normalize_probe(probe.squeeze())

    @torch.no_grad()
    def residual(self) -> float:
        """FP64 data residual sum (sqrt(I) - sqrt(Imeas))^2 / sum Imeas over the stack."""
        obj, probe = self.current()
        num = torch.zeros((), dtype=torch.float64, device=obj.device)
        den = torch.zeros((), dtype=torch.float64, device=obj.device)
        for s in range(0, self.F, 512):
            ids = torch.arange(s, min(self.F, s + 512), device=obj.device, dtype=torch.int32)
            I = optics.forward_intensity(obj, probe, self.tl, batch=ids).double()
            Im = self.stack[ids.long()].double()
            num += ((I.sqrt() - Im.sqrt()) ** 2).sum()
            den += Im.sum()
        return float(num / den)


def build_model(cfg, canvas, probe_hw, probe_initial=None, device="cuda"):
    mt = cfg.get("model_type", "inr")
    if mt == "gaussian_field":
        raise NotImplementedError("the Gaussian-field representation has no model here; its rasteriser is gsplat.GaussianRasterize2D")
    if mt == "pixel_grid":
        return PixelGrid((canvas, canvas), probe_hw).to(device)
    use_res = cfg.get("use_residual", False) and cfg.get("init_type", "initNone") != "initNone"
    return ComplexINRModel2D(
        output_width=canvas, output_height=canvas, downsample_factor=cfg.get("downsample_factor", 2),
        update_probe=True, probe_width=probe_hw[1], probe_height=probe_hw[0], use_residual=use_res,
        object_initial=None, probe_initial=probe_initial if use_res else None,
        n_levels=cfg.get("n_levels", 16), n_features_per_level=cfg.get("n_features_per_level", 2),
        log2_hashmap_size=cfg.get("log2_hashmap_size", 18), base_resolution=cfg.get("base_resolution", 16),
        per_level_scale=cfg.get("per_level_scale", 1.5), first_omega_0=cfg.get("first_omega_0", 10.0),
        hidden_omega_0=cfg.get("hidden_omega_0", 1.0), hidden_features=cfg.get("hidden_features", 64),
        hidden_layers=cfg.get("hidden_layers", 2), trainable_omega0=cfg.get("trainable_omega0", True)).to(device)


def save_outputs(vis_dir, model, obj, probe):
    from scipy.io import savemat
    savemat(os.path.join(vis_dir, "result.mat"), {"object_complex": obj.detach().cpu().numpy(),
                                                  "probe_complex": probe.detach().cpu().numpy()})
    torch.save([p for _, p in model.named_parameters() if p.requires_grad],
               os.path.join(vis_dir, "trained_models.pth"))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=str, default="config/plant.yaml")
    args = ap.parse_args(argv)
    cfg = load_config(args.config)
    dev = torch.device("cuda")
    data = load_ptychography_data(cfg["data_dir"], cfg.get("bundle_file"), cfg.get("location_file"),
                                  cfg.get("raw_file"), cfg.get("probe_file"), cfg.get("gt_file"),
                                  cfg.get("init_probe_file"), cfg.get("gap", 1))
    probe = np.asarray(data["probe"])
    stack = torch.from_numpy(np.ascontiguousarray(np.moveaxis(np.asarray(data["imRaw"], np.float32), -1, 0)))
    tlX, tlY, brX, brY, dx, canvas = optics.scan_positions_to_pixels(
        data["xlocation"], data["ylocation"], probe.shape, cfg["wavelength"], cfg["camera_length"],
        cfg["camera_pixel_pitch"])
    tl = optics.make_windows(tlY, tlX, dev)
    optics.check_windows(tl, (canvas, canvas), probe.shape[0], probe.shape[1])
    init_probe = data.get("initProbe", probe) if cfg.get("init_type", "initNone") == "initProbe" else None
    if cfg.get("init_type") == "initQuadratic":
        M, N = probe.shape
        yp = (np.arange(M, dtype=np.float32) - M / 2) * dx[0]
        xp = (np.arange(N, dtype=np.float32) - N / 2) * dx[1]
        X, Y = np.meshgrid(xp, yp)
        ph = np.pi / (cfg["wavelength"] * cfg.get("quadratic_focal_length", 0.1)) * (X ** 2 + Y ** 2)
        init_probe = (np.exp(1j * ph) * np.asarray(data.get("initProbe", probe))).astype(np.complex64)
    pi_t = torch.from_numpy(np.asarray(init_probe).astype(np.complex64)).to(dev) if init_probe is not None else None
    model = build_model(cfg, canvas, probe.shape, pi_t, dev)
    trainer = Trainer(model, stack.to(dev), tl, cfg.get("loss_type", "smooth_L1_loss"), cfg.get("batch_size", 10),
                      cfg.get("lr", 1e-3), cfg.get("lr_decay_step", 10000), cfg.get("lr_decay_gamma", 0.1),
                      cfg.get("sparsity_weight", 0.0))
    vis_dir = cfg.get("result_dir", "./result")
    os.makedirs(vis_dir, exist_ok=True)
    iters, vis = cfg.get("iters", 2000), cfg.get("vis_interval", 100)
    t0 = time.time()
    for epoch in range(iters):
        trainer.epoch()
        if epoch % vis == 0 or epoch == iters - 1:
            obj, pr = trainer.current()
            save_outputs(vis_dir, model, obj, pr)
            print(f"epoch {epoch}: loss {float(trainer.last_loss):.4e}  {time.time() - t0:.1f}s", flush=True)


if __name__ == "__main__":
    main()
