"""Device-resident iteration engine for the multislice mixed-probe gradient path.

One ``BatchStep`` is the reference's per-batch body of ``Ptychography.reconstruct``
(ptychography.py:214-245): probe orthogonalisation, hard-constrained object,
fused forward + loss + adjoint (one persistent CUDA launch), the autograd
object-gradient rescale of ptychography.py:330-332 and the optimiser steps.
The per-batch loss stays on the device; an iteration reads it back once.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from . import ops
from .diffractive_imaging.ptycho_utils import SimpleBatcher, orthogonalize_probes


class FusedAdam(torch.optim.Optimizer):
    """torch.optim.Adam / AdamW semantics with the update in one CUDA kernel per
    parameter (complex parameters are updated on their real view, like torch).
    Works with torch LR schedulers (they only edit ``param_groups``)."""

    def __init__(self, params, lr=1e-3, betas=(0.9, 0.999), eps=1e-8, weight_decay=0.0, decoupled=False,
                 amsgrad=False, **unused):
        if amsgrad:
            raise NotImplementedError("amsgrad is not supported by the fused optimiser")
        super().__init__(params, dict(lr=lr, betas=betas, eps=eps, weight_decay=weight_decay,
                                      decoupled=decoupled))

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
                st["step"] += 1
                ops.adam_step(p.data, p.grad.contiguous(), st["exp_avg"], st["exp_avg_sq"], st["step"],
                              group["lr"], group["betas"], group["eps"], group["weight_decay"],
                              group["decoupled"])
        return loss


class FusedSGD(torch.optim.Optimizer):
    """torch.optim.SGD without momentum, update in one CUDA kernel per parameter."""

    def __init__(self, params, lr=1e-3, weight_decay=0.0, momentum=0.0, **unused):
        if momentum:
            raise NotImplementedError("momentum is not supported by the fused optimiser")
        super().__init__(params, dict(lr=lr, weight_decay=weight_decay))

    @torch.no_grad()
    def step(self, closure=None):
        loss = closure() if closure is not None else None
        for group in self.param_groups:
            for p in group["params"]:
                if p.grad is not None:
                    ops.sgd_step(p.data, p.grad.contiguous(), group["lr"], group["weight_decay"])
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
    for bi in batcher:
        idx = torch.as_tensor(np.asarray(bi, dtype=np.int64)).to(device, non_blocking=True)
        total += batch_step(pt, idx, optimizers)
        nb += 1
    return total / max(nb, 1)
