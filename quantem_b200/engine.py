"""Device-resident iteration engine for the multislice mixed-probe gradient path.

One ``BatchStep`` is the reference's per-batch body of ``Ptychography.reconstruct``
(ptychography.py:214-245): probe orthogonalisation, hard-constrained object,
fused forward + loss + adjoint (one persistent CUDA launch), the autograd
object-gradient rescale of ptychography.py:330-332 and the optimiser steps.
The per-batch loss stays on the device; an iteration reads it back once.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import torch

from . import ops
from .diffractive_imaging.ptycho_utils import SimpleBatcher, device_batches, orthogonalize_probes


class FusedAdam(torch.optim.Optimizer):
    """torch.optim.Adam / AdamW semantics with the update in one CUDA kernel per
    parameter (complex parameters are updated on their real view, like torch).
    Works with torch LR schedulers (they only edit ``param_groups``)."""

    def __init__(self, params, lr=1e-3, betas=(0.9, 0.999), eps=1e-8, weight_decay=0.0, decoupled=False,
                 amsgrad=False, **unused):
        super().__init__(params, dict(lr=lr, betas=betas, eps=eps, weight_decay=weight_decay,
                                      decoupled=decoupled, amsgrad=bool(amsgrad)))

    @torch.no_grad()
    def step(self, closure=None):
        loss = closure() if closure is not None else None
        for group in self.param_groups:
            for p in group["params"]:
                if p.grad is None:
                    continue
                st = self.state[p]
                if not st:
                    st["step"] = 0
                    st["exp_avg"] = torch.zeros_like(p)
                    st["exp_avg_sq"] = torch.zeros_like(p)
                    if group.get("amsgrad"):
                        st["max_exp_avg_sq"] = torch.zeros_like(p)
                st["step"] += 1
                ops.adam_step(p.data, p.grad.contiguous(), st["exp_avg"], st["exp_avg_sq"], st["step"],
                              group["lr"], group["betas"], group["eps"], group["weight_decay"],
                              group["decoupled"], max_exp_avg_sq=st.get("max_exp_avg_sq"))
        return loss


class FusedSGD(torch.optim.Optimizer):
    """torch.optim.SGD (momentum, dampening, Nesterov, weight decay), the update in one CUDA
    kernel per parameter."""

    def __init__(self, params, lr=1e-3, weight_decay=0.0, momentum=0.0, dampening=0.0, nesterov=False, **unused):
        if nesterov and (momentum <= 0 or dampening != 0):
            raise ValueError("Nesterov momentum requires a momentum and zero dampening")
        super().__init__(params, dict(lr=lr, weight_decay=weight_decay, momentum=momentum, dampening=dampening,
                                      nesterov=bool(nesterov)))

    @torch.no_grad()
    def step(self, closure=None):
        loss = closure() if closure is not None else None
        for group in self.param_groups:
            for p in group["params"]:
                if p.grad is None:
                    continue
                if not group["momentum"]:
                    ops.sgd_step(p.data, p.grad.contiguous(), group["lr"], group["weight_decay"])
                    continue
                st = self.state[p]
                first = "momentum_buffer" not in st
                if first:
                    st["momentum_buffer"] = torch.empty_like(p)
                ops.sgd_momentum_step(p.data, p.grad.contiguous(), st["momentum_buffer"], first, group["lr"],
                                      group["momentum"], group["dampening"], group["nesterov"],
                                      group["weight_decay"])
        return loss


def make_optimizer(params, opt: dict):
    """Optimiser from a reference-style parameter dict (optimizer_mixin.py:84-126)."""
    opt = dict(opt)
    kind = str(opt.pop("type", "adam")).lower()
    if kind == "adam":
        return FusedAdam(params, **opt)
    if kind == "adamw":
        opt.setdefault("weight_decay", 1e-2)  # torch.optim.AdamW default
        return FusedAdam(params, decoupled=True, **opt)
    if kind == "sgd":
        return FusedSGD(params, **opt)
    raise NotImplementedError(f"Unknown optimizer type: {kind}")


@dataclass
class ProblemTensors:
    """Everything the batch kernels read, resident on one CUDA device."""

    obj: torch.Tensor            # raw object parameter (S, Ho, Wo) complex64
    probe: torch.Tensor          # raw probe parameter (P, n, n) complex64
    prop: torch.Tensor           # (S-1, n, n) complex64
    positions: torch.Tensor      # (N, 2) float32
    targets: torch.Tensor        # (N, n, n) float32
    mask: torch.Tensor           # (n, n) float32
    mean_intensity: float
    upsample_factor: float
    orthogonalize: bool = True
    loss_type: str = "l2_amplitude"
    grid: int | None = None
    recompute_every: int | None = None   # 256 x 256 windows: adjoint checkpoint interval (None/0: keep all)
    extra: dict = field(default_factory=dict)

    @property
    def num_gpts(self) -> int:
        return int(self.positions.shape[0])


def batch_step(pt: ProblemTensors, batch_idx: torch.Tensor, optimizers=(), autograd=True):
    """One reference batch: zero grads, loss, backward, rescale, optimiser steps.

    Returns the batch consistency loss as a 0-d device tensor (no host sync)."""
    for opt in optimizers:
        opt.zero_grad(set_to_none=True)
    probe_o = orthogonalize_probes(pt.probe) if pt.orthogonalize else pt.probe
    loss = ops.batch_loss(pt.obj, probe_o, pt.prop, pt.positions, batch_idx, pt.targets, pt.mask,
                          pt.num_gpts, pt.mean_intensity, pt.loss_type, grid=pt.grid,
                          recompute_every=pt.recompute_every)
    if autograd and (pt.obj.requires_grad or pt.probe.requires_grad):
        loss.backward()
        if pt.obj.grad is not None:
            pt.obj.grad.mul_(pt.upsample_factor ** 2 / 2)  # ptychography.py:330-332
        for opt in optimizers:
            opt.step()
    return loss.detach()


def run_iteration(pt: ProblemTensors, batcher: SimpleBatcher, optimizers=(), device=None):
    """One pass over all training positions; returns the mean batch loss as a
    0-d device tensor."""
    device = pt.obj.device if device is None else device
    total = torch.zeros((), dtype=torch.float32, device=device)
    nb = 0
    for idx in device_batches(batcher, device):
        total += batch_step(pt, idx, optimizers)
        nb += 1
    return total / max(nb, 1)


class GraphedIteration:
    """One full-batch iteration of one dataset (forward, loss, fused adjoint, object-
    gradient rescale, Adam on object and probe, probe orthogonalisation) captured in a
    CUDA graph and replayed: the launch sequence of ``batch_step`` without the host's
    per-launch cost.

    The batch is every position in a fixed order (``batch_idx``, default a seeded
    permutation, so that positions processed at the same time stay far apart); the
    loss and gradients of a full batch do not depend on the order.  The optimisers
    keep their step count and learning rate on the device (``multi.CapturableAdam``,
    same update as torch.optim.Adam), so each replay advances the bias corrections."""

    def __init__(self, pt: ProblemTensors, lr_obj: float = 5e-3, lr_probe: float = 1e-3, batch_idx=None,
                 seed: int = 0):
        from .multi import CapturableAdam

        self.pt = pt
        dev = pt.obj.device
        if batch_idx is None:
            g = torch.Generator().manual_seed(seed)
            batch_idx = torch.randperm(pt.num_gpts, generator=g)
        self.batch_idx = batch_idx.to(dev, torch.int64).contiguous()
        self.opts = [CapturableAdam([pt.obj], lr=lr_obj), CapturableAdam([pt.probe], lr=lr_probe)]
        self.graph = None
        self.static_loss = None

    def _step(self):
        pt = self.pt
        pt.obj.grad = None
        pt.probe.grad = None
        probe_o = orthogonalize_probes(pt.probe) if pt.orthogonalize else pt.probe
        loss = ops.batch_loss(pt.obj, probe_o, pt.prop, pt.positions, self.batch_idx, pt.targets, pt.mask,
                              pt.num_gpts, pt.mean_intensity, pt.loss_type, grid=pt.grid,
                              recompute_every=pt.recompute_every)
        loss.backward()
        pt.obj.grad.mul_(pt.upsample_factor ** 2 / 2)  # ptychography.py:330-332
        for o in self.opts:
            o.step()
        return loss.detach()

    def run_eager(self):
        return self._step()

    def capture(self, warmup: int = 3):
        """Warm up on a side stream (workspaces sized, kernels loaded), then capture."""
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for _ in range(warmup):
                self._step()
        torch.cuda.current_stream().wait_stream(s)
        self.pt.obj.grad = None
        self.pt.probe.grad = None
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.static_loss = self._step()
        return self

    def replay(self):
        """One iteration; returns the batch loss (a device tensor overwritten by the next replay)."""
        self.graph.replay()
        return self.static_loss


class HostTargetStream:
    """Per-iteration host-to-device copies of a host array (the measured targets),
    double-buffered: the copy for iteration k + 1 runs on a copy stream into the second
    device buffer while iteration k computes on the current stream.  The first copy is
    exposed.  ``acquire()`` returns this iteration's buffer (the current stream waits
    for its copy), ``prefetch_next()`` starts the next copy once that buffer is free,
    ``release()`` marks the end of this iteration's use of its buffer."""

    def __init__(self, host: torch.Tensor, device):
        self.host = host if host.is_pinned() else host.pin_memory()
        self.device = torch.device(device)
        self.stream = torch.cuda.Stream(device=self.device)
        self.buf = [torch.empty(host.shape, dtype=host.dtype, device=self.device) for _ in range(2)]
        for b in self.buf:
            b.record_stream(self.stream)
        self.ready = [torch.cuda.Event(), torch.cuda.Event()]
        self.free = [None, None]
        self.k = 0
        self.bytes_per_copy = host.numel() * host.element_size()
        self._issue(0)

    def _issue(self, i, after=None):
        with torch.cuda.stream(self.stream):
            if self.free[i] is not None:
                self.stream.wait_event(self.free[i])
            if after is not None:
                self.stream.wait_event(after)
            self.buf[i].copy_(self.host, non_blocking=True)
            self.ready[i].record(self.stream)

    def acquire(self) -> torch.Tensor:
        i = self.k % 2
        torch.cuda.current_stream(self.device).wait_event(self.ready[i])
        return self.buf[i]

    def prefetch_next(self, after=None):
        """Start the next copy; with ``after`` (an event) it also waits for that event, so a
        small copy the current stream issued before it is not queued behind this transfer."""
        self._issue((self.k + 1) % 2, after)

    def release(self):
        i = self.k % 2
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(self.device))
        self.free[i] = ev
        self.k += 1
