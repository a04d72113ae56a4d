"""Per-model optimiser / scheduler bookkeeping (quantem core/ml/optimizer_mixin.py:13-287).

Optimisers are the fused CUDA ones of ``quantem_b200.engine`` (Adam, AdamW,
SGD); schedulers are torch.optim.lr_scheduler objects wrapped around them.
"""
from __future__ import annotations

import torch


class OptimizerMixin:
    DEFAULT_OPTIMIZER_TYPE = "adam"

    def __init__(self):
        self._optimizer = None
        self._scheduler = None
        self._optimizer_params = {}
        self._scheduler_params = {}

    @property
    def optimizer(self):
        return self._optimizer

    @property
    def scheduler(self):
        return self._scheduler

    @property
    def optimizer_params(self) -> dict:
        return self._optimizer_params

    @optimizer_params.setter
    def optimizer_params(self, d: dict | None):
        self._optimizer_params = dict(d) if d else {}

    @property
    def scheduler_params(self) -> dict:
        return self._scheduler_params

    @scheduler_params.setter
    def scheduler_params(self, d: dict | None):
        if d:
            t = str(d.get("type", "none")).lower()
            if t not in ("cyclic", "plateau", "exp", "gamma", "linear", "none") and not t.startswith(
                    ("plat", "reducelronplat")):
                raise ValueError(f"Unknown scheduler type: {t}")
            self._scheduler_params = dict(d)
        else:
            self._scheduler_params = {}

    def has_optimizer(self) -> bool:
        return self._optimizer is not None

    def get_optimization_parameters(self):
        raise NotImplementedError

    def set_optimizer(self, opt_params: dict | None = None) -> None:
        from ..engine import make_optimizer

        if opt_params is not None:
            self.optimizer_params = opt_params
        if not self._optimizer_params:
            self._optimizer = None
            return
        params = dict(self._optimizer_params)
        kind = str(params.get("type", self.DEFAULT_OPTIMIZER_TYPE)).lower()
        if kind == "none":
            self.remove_optimizer()
            return
        ps = self.get_optimization_parameters()
        ps = [ps] if isinstance(ps, torch.Tensor) else list(ps)
        for p in ps:
            p.requires_grad_(True)
        self._optimizer = make_optimizer(ps, params)

    def remove_optimizer(self):
        self._optimizer = None
        self._scheduler = None
        self._optimizer_params = {}

    def reset_optimizer(self):
        if self._optimizer_params:
            self.set_optimizer(self._optimizer_params)

    def reconnect_optimizer_to_parameters(self):
        if self._optimizer is not None:
            self.set_optimizer(self._optimizer_params)

    def set_scheduler(self, scheduler_params: dict | None = None, num_iter: int | None = None) -> None:
        if scheduler_params is not None:
            self.scheduler_params = scheduler_params
        if not self._scheduler_params or self._optimizer is None:
            self._scheduler = None
            return
        p = self._scheduler_params
        kind = str(p.get("type", "none")).lower()
        opt = self._optimizer
        base = opt.param_groups[0]["lr"]
        S = torch.optim.lr_scheduler
        if kind == "none":
            self._scheduler = None
        elif kind == "cyclic":
            self._scheduler = S.CyclicLR(opt, base_lr=p.get("base_lr", base / 4), max_lr=p.get("max_lr", base * 4),
                                         step_size_up=p.get("step_size_up", 100),
                                         step_size_down=p.get("step_size_down", p.get("step_size_up", 100)),
                                         mode=p.get("mode", "triangular2"), cycle_momentum=p.get("momentum", False))
        elif kind.startswith(("plat", "reducelronplat")):
            self._scheduler = S.ReduceLROnPlateau(opt, mode="min", factor=p.get("factor", 0.5),
                                                  patience=p.get("patience", 10), threshold=p.get("threshold", 1e-3),
                                                  min_lr=p.get("min_lr", base / 20), cooldown=p.get("cooldown", 50))
        elif kind in ("exp", "gamma", "exponential"):
            if "gamma" in p:
                gamma = p["gamma"]
            elif num_iter is not None:
                gamma = p.get("factor", 0.01) ** (1.0 / num_iter)
            else:
                gamma = 0.9
            self._scheduler = S.ExponentialLR(opt, gamma=gamma)
        elif kind == "linear":
            self._scheduler = S.LinearLR(opt, start_factor=p.get("start_factor", 0.1),
                                         end_factor=p.get("end_factor", 1.0), total_iters=p.get("total_iters", num_iter))
        else:
            raise ValueError(f"Unknown scheduler type: {kind}")

    def step_optimizer(self):
        if self._optimizer is not None:
            self._optimizer.step()

    def zero_optimizer_grad(self):
        if self._optimizer is not None:
            self._optimizer.zero_grad(set_to_none=True)

    def step_scheduler(self, loss: float | None = None):
        if self._scheduler is not None:
            if isinstance(self._scheduler, torch.optim.lr_scheduler.ReduceLROnPlateau):
                if loss is not None:
                    self._scheduler.step(loss)
            else:
                self._scheduler.step()
