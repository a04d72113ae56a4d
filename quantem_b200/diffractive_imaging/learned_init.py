"""Learned initial object phase for multislice mixed-probe ptychography.

A CNN2d (the reference's UNet topology, core/ml/cnn.py:17-212) maps the binned
diffraction patterns of a raster scan to the projected object phase around
every scan position, and that phase seeds ``ObjectPixelated`` before the plain
iterative reconstruction (ptychography.py:146-308) refines it.

* Input: each pattern (n x n) is binned ``bin x bin`` and square-rooted on the
  GPU (``ptycho_cnn_bin_features``), giving (n/bin)^2 channels per scan position
  on the (scan rows x scan columns) grid; per-channel mean and a global scale,
  fixed from the first training batch, normalise them.
* Output: sub x sub channels per scan position (sub = scan step in pixels): the
  projected phase sum_s phi_s on the sub x sub object pixels around the position
  (rows p - sub/2 ... p + sub/2 - 1); depth-to-space gives a (sub*rows, sub*cols)
  phase map covering the scanned field of view, split evenly over the slices at
  use.  With ``per_slice=True`` the network predicts S x sub x sub channels, the
  phase of every slice, and each slice gets its own map.
* Training pairs come from the method's own forward model: random
  Gaussian-atom multislice objects (atom density and peak phase drawn per
  object), simulated through ``ptycho_forward_loss`` with the experiment's probe
  modes and propagators, Poisson noise at the experiment's dose.  Each step
  simulates fresh objects (nothing is stored), so N training objects cost N
  forward simulations.  The network trains with the tcgen05 BF16 kernels and the
  fused Adam step.
* Use: ``initial_object`` sets every slice to exp(i phi / S) (exp(i phi_s) with
  per-slice maps).
  The plain reconstruction is the fallback and the judge: the forward
  model's loss on the measured data is evaluated for the learned and the flat
  start, and the flat object is returned when the learned one fits worse.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import torch

from .. import ops, synthetic
from ..core.ml import kernels as kk
from ..core.ml.cnn import CNN2d, mse_loss
from ..engine import FusedAdam


@dataclass
class LearnedInitConfig:
    n: int = 128                     # probe window / pattern size
    bin: int = 4                     # n / bin = 32 -> 32 x 32 binned patterns
    scan_crop: int = 32              # training crops of crop x crop scan positions
    step_px: int = 6
    jitter_px: float = 0.5
    sigma_px: float = 1.5
    density: tuple = (0.002, 0.01)   # atoms / px^2 / slice, drawn per object
    peak: tuple = (0.05, 0.5)        # peak phase per atom [rad], drawn per object
    counts: float = 1e5              # Poisson dose per pattern (<= 0: noiseless)
    start_filters: int = 32
    num_layers: int = 5
    num_per_layer: int = 2
    lr: float = 1e-3
    batch_objects: int = 16
    zero_mean_target: bool = True    # the reconstruction fixes the mean phase: learn the structure only
    # predict every slice's phase instead of the projected phase: at the benchmark geometry
    # (8 slices of 20 A) 20k training objects left it at held-out projected NRMSE 0.99 (the
    # depth split is barely determined by the patterns, and its unpredictable part dominates
    # the per-slice loss), against 0.54 for the projected-phase network, so it is off by default
    per_slice: bool = False


class LearnedInitializer:
    """Trains and applies the phase-initialising CNN for one probe / slice geometry."""

    def __init__(self, probes: torch.Tensor, propagators: torch.Tensor, cfg: LearnedInitConfig | None = None,
                 device="cuda", seed: int = 0):
        self.cfg = cfg or LearnedInitConfig()
        c = self.cfg
        self.device = torch.device(device)
        self.probes = probes.to(self.device, torch.complex64).contiguous()
        if isinstance(propagators, (tuple, list)):  # separable per-axis factors (Kr, Kc)
            self.props = tuple(t.to(self.device, torch.complex64).contiguous() for t in propagators)
            self.S = int(self.props[0].shape[0]) + 1
        else:
            self.props = propagators.to(self.device, torch.complex64).contiguous()
            self.S = int(self.props.shape[0]) + 1
        if probes.shape[-1] != c.n or c.n % c.bin:
            raise ValueError("probe size must equal cfg.n and be divisible by cfg.bin")
        self.C = (c.n // c.bin) ** 2
        self.sub = int(c.step_px)
        self.depth = self.S if c.per_slice else 1  # phase maps predicted per position
        self.net = CNN2d(self.C, self.depth * self.sub * self.sub, start_filters=c.start_filters,
                         num_layers=c.num_layers, num_per_layer=c.num_per_layer, device=self.device, seed=seed)
        self.opt = FusedAdam([self.net.flat], lr=c.lr)
        self.gen = torch.Generator(device=self.device).manual_seed(seed + 1)
        self.feat_mean = None
        self.feat_scale = 1.0
        self.history = []
        self.objects_seen = 0

    # ------------------------------------------------------------------ data
    def _crop_geometry(self, crop):
        c = self.cfg
        pad = c.n // 2 + 3
        ho = (crop - 1) * c.step_px + 2 * pad
        ho += (-ho) % 8
        return pad, ho

    def simulate(self, nobj: int):
        """Fresh training pairs: (BF16 feature rows (nobj*crop^2, C), FP32 targets
        (nobj, depth*sub^2, crop, crop), depth = S per-slice maps or 1 projected map)."""
        c = self.cfg
        crop = c.scan_crop
        pad, ho = self._crop_geometry(crop)
        dev, g = self.device, self.gen
        npos = crop * crop
        rr, cc = torch.meshgrid(torch.arange(crop, device=dev), torch.arange(crop, device=dev), indexing="ij")
        nominal = torch.stack([rr.reshape(-1), cc.reshape(-1)], -1).double() * c.step_px + pad
        idx = torch.arange(npos, device=dev, dtype=torch.int64)
        mask = torch.ones((c.n, c.n), device=dev)
        dummy = torch.zeros((npos, c.n, c.n), device=dev)
        rows = torch.empty((nobj * npos, self.C), dtype=torch.bfloat16, device=dev)
        D = self.depth
        targets = torch.empty((nobj, D * self.sub * self.sub, crop, crop), device=dev)
        off = torch.arange(self.sub, device=dev) - self.sub // 2
        ti = (nominal[:, 0].long().view(crop, crop, 1, 1) + off.view(1, 1, -1, 1))
        tj = (nominal[:, 1].long().view(crop, crop, 1, 1) + off.view(1, 1, 1, -1))
        for b in range(nobj):
            u = torch.rand(3, generator=g, device=dev, dtype=torch.float64)
            dens = c.density[0] + float(u[0]) * (c.density[1] - c.density[0])
            peak = c.peak[0] + float(u[1]) * (c.peak[1] - c.peak[0])
            n_atoms = max(4, int(dens * ho * ho))
            phase = torch.stack([synthetic.gaussian_atom_phase((ho, ho), n_atoms, c.sigma_px, peak, g, dev)
                                 for _ in range(self.S)])
            obj = torch.exp(1j * phase).to(torch.complex64)
            pos = nominal + (torch.rand(nominal.shape, generator=g, device=dev, dtype=torch.float64) * 2 - 1) * \
                c.jitter_px
            pos = pos.float().contiguous()
            inten = ops.batch_forward(obj, self.probes, self.props, pos, idx, dummy, mask, npos, 1.0)["intensity"]
            if c.counts > 0:
                inten = torch.poisson(inten * (c.counts / inten.sum(dim=(-2, -1)).mean()), generator=g)
            else:
                inten = inten * (1e5 / inten.sum(dim=(-2, -1)).mean())
            self._features(inten.contiguous(), rows[b * npos:(b + 1) * npos])
            maps = phase.float() if c.per_slice else phase.sum(0, keepdim=True).float()  # (D, ho, ho)
            t = maps[:, ti, tj]  # (D, crop, crop, sub, sub)
            if c.zero_mean_target:
                t = t - t.mean(dim=(1, 2, 3, 4), keepdim=True)
            targets[b] = t.permute(0, 3, 4, 1, 2).reshape(D * self.sub * self.sub, crop, crop)
        return rows, targets

    def _features(self, patterns: torch.Tensor, out: torch.Tensor, amplitudes: bool = False):
        """Dose-normalised features: intensities divided by the mean pattern total
        (in units of (n/bin)^2 so values stay O(1)), then sqrt, centred and scaled
        with statistics fixed from the first data seen."""
        c = self.cfg
        tot = (patterns.square() if amplitudes else patterns).sum(dim=(-2, -1)).mean()
        norm = float(self.C / max(float(tot), 1e-30))
        if self.feat_mean is None:
            raw = torch.empty_like(out)
            kk.bin_features(patterns, c.bin, raw, amplitudes=amplitudes, norm=norm)
            f = raw.float()
            self.feat_mean = f.mean(0).contiguous()
            self.feat_scale = float(1.0 / max(float((f - self.feat_mean).std()), 1e-6))
        kk.bin_features(patterns, c.bin, out, mean=self.feat_mean, scale=self.feat_scale, amplitudes=amplitudes,
                        norm=norm)
        return out

    # ------------------------------------------------------------------ training
    def train(self, num_objects: int, log_every: int = 0, total_objects: int | None = None):
        """Train on ``num_objects`` freshly simulated objects; returns the loss history.

        The learning rate follows a cosine decay from cfg.lr to 0 over
        ``total_objects`` (default: this call's objects), so training may be split
        over several calls."""
        c = self.cfg
        self.net.train()
        total = max(total_objects or (self.objects_seen + num_objects), 1)
        steps = max(1, math.ceil(num_objects / c.batch_objects))
        for k in range(steps):
            frac = min(self.objects_seen / total, 1.0)
            for grp in self.opt.param_groups:
                grp["lr"] = c.lr * 0.5 * (1.0 + math.cos(math.pi * frac))
            rows, tgt = self.simulate(c.batch_objects)
            self.opt.zero_grad(set_to_none=True)
            pred = self.net(rows, rows=(c.batch_objects, c.scan_crop, c.scan_crop))
            loss = mse_loss(pred, tgt)
            loss.backward()
            self.opt.step()
            self.objects_seen += c.batch_objects
            if log_every and (k % log_every == 0 or k == steps - 1):
                self.history.append((self.objects_seen, float(loss.item())))
        return self.history

    @torch.no_grad()
    def evaluate(self, nobj: int = 8, batch_stats: bool = False, projected: bool = True) -> float:
        """Mean phase NRMSE (mean-removed) of the prediction on fresh simulated crops
        (eval-mode batch norm unless ``batch_stats``): of the projected phase (the sum
        of the per-slice maps) with ``projected``, else of all per-slice maps."""
        c = self.cfg
        rows, tgt = self.simulate(nobj)
        if not batch_stats:
            self.net.eval()
        pred = self.net(rows, rows=(nobj, c.scan_crop, c.scan_crop))
        self.net.train()
        if projected and self.depth > 1:
            shp = (nobj, self.depth, self.sub * self.sub, c.scan_crop, c.scan_crop)
            pred, tgt = pred.reshape(shp).sum(1), tgt.reshape(shp).sum(1)
        p = pred.reshape(nobj, -1).double()
        t = tgt.reshape(nobj, -1).double()
        d = (p - p.mean(1, keepdim=True)) - (t - t.mean(1, keepdim=True))
        return float((d.norm(dim=1) / (t - t.mean(1, keepdim=True)).norm(dim=1)).mean())

    # ------------------------------------------------------------------ inference
    @torch.no_grad()
    def predict_phase_map(self, patterns: torch.Tensor, scan: tuple, amplitudes: bool = True) -> torch.Tensor:
        """(depth, sub*rows, sub*cols) phase maps over the scanned field (per slice, or the
        projected phase) from the measured patterns (npos, n, n) in detector layout,
        raster order."""
        rows_n, cols_n = scan
        f = 2 ** self.cfg.num_layers
        if rows_n % f or cols_n % f:
            raise ValueError(f"scan shape must be divisible by {f}")
        self.net.eval()
        x = torch.empty((rows_n * cols_n, self.C), dtype=torch.bfloat16, device=self.device)
        self._features(patterns.float().contiguous(), x, amplitudes=amplitudes)
        out = self.net(x, rows=(1, rows_n, cols_n))[0]  # (depth*sub^2, rows, cols)
        s, D = self.sub, self.depth
        return out.view(D, s, s, rows_n, cols_n).permute(0, 3, 1, 4, 2).reshape(D, rows_n * s, cols_n * s)

    # scalings of the predicted phase the judge compares (0 = the flat start).  Intermediate
    # scalings (0.75, 0.5, 0.25) were measured on the benchmark problems and never won: the
    # data loss preferred the full prediction at every object and dose, so they only cost time
    JUDGE_SCALES = (1.0, 0.0)

    @torch.no_grad()
    def initial_object(self, patterns: torch.Tensor, scan: tuple, obj_shape: tuple, origin_px: tuple,
                       amplitudes: bool = True, judge: dict | None = None) -> torch.Tensor:
        """Complex (S, Ho, Wo) start: exp(i phi_s) for every slice (exp(i phi / S) from a
        projected-phase network) inside the scanned field (scan position (0, 0) at
        object pixel ``origin_px``), 1 elsewhere.

        ``judge`` (optional dict with positions, targets, probe, prop, mask,
        mean_intensity, batch of indices) makes the plain forward model decide: its data
        loss is evaluated for the prediction scaled by each of ``JUDGE_SCALES`` and the
        best-fitting start is returned, the flat object (scale 0) included.  The chosen
        scale is ``judge_scale``; ``used_learned`` is False when the flat start won."""
        S, Ho, Wo = obj_shape
        ph = self.predict_phase_map(patterns, scan, amplitudes)
        if ph.shape[0] not in (1, S):
            raise ValueError(f"the network predicts {ph.shape[0]} slices, the object has {S}")
        full = torch.zeros((ph.shape[0], Ho, Wo), device=self.device)
        r0 = int(origin_px[0]) - self.sub // 2
        c0 = int(origin_px[1]) - self.sub // 2
        full[:, r0:r0 + ph.shape[1], c0:c0 + ph.shape[2]] = ph
        if ph.shape[0] == 1:
            full = (full / S).expand(S, Ho, Wo)
        self.used_learned = True
        self.judge_scale = 1.0
        if judge is None:
            return torch.exp(1j * full).to(torch.complex64).contiguous()
        losses = []
        for a in self.JUDGE_SCALES:
            cand = torch.exp(1j * (a * full)).to(torch.complex64).contiguous()
            oc = ops.constrained_object(cand)
            out = ops.batch_forward(oc, judge["probe"], judge["prop"], judge["positions"], judge["batch"],
                                    judge["targets"], judge["mask"], judge["positions"].shape[0],
                                    judge["mean_intensity"], want_intensity=False)
            losses.append(out["loss"])
        losses = [float(x) for x in torch.stack(losses).cpu()]  # one read-back for all candidates
        self.judge_losses = tuple(losses)
        best = min(range(len(losses)), key=lambda i: losses[i])
        self.judge_scale = float(self.JUDGE_SCALES[best])
        self.used_learned = self.judge_scale > 0.0
        return torch.exp(1j * (self.judge_scale * full)).to(torch.complex64).contiguous()
