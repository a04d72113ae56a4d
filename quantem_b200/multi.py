"""Several independent datasets in one persistent launch, CUDA-graph captured
iterations and the launch autotuner.

A "dataset" is one ptychography problem (object, probe modes, propagators,
positions, measured amplitudes).  Datasets that share a probe window run in one
``ptycho_forward_adjoint_multi`` launch whose CTAs are partitioned between them
(datasets with 96 x 96 and 128 x 128 windows: one launch per window size);
the partition comes from ``autotune_grids`` (timed candidates, cached per
problem signature).  ``GraphedMultiIteration`` captures one full iteration of all
datasets (probe orthogonalisation and its autograd backward, hard constraint,
the multi launch, reductions, constraint VJPs, Adam with device-side step
counts) in a CUDA graph and replays it.
"""
from __future__ import annotations

import ctypes
import time
import warnings

import numpy as np
import torch

from . import _lib, ops
from .diffractive_imaging.ptycho_utils import orthogonalize_probes


class Problem:
    """Device tensors of one dataset (raw parameters are leaf tensors)."""

    def __init__(self, obj, probe, prop, positions, targets, mask, mean_intensity, upsample_factor,
                 orthogonalize=True, loss_type="l2_amplitude", batch_idx=None):
        self.obj, self.probe, self.prop = obj, probe, prop
        self.positions, self.targets, self.mask = positions, targets, mask
        self.mean_intensity, self.upsample_factor = float(mean_intensity), float(upsample_factor)
        self.orthogonalize, self.loss_type = orthogonalize, loss_type
        n = positions.shape[0]
        self.batch_idx = (torch.arange(n, device=obj.device, dtype=torch.int64) if batch_idx is None
                          else batch_idx)
        self.ws = ops.Workspace(obj.device)

    @property
    def num_gpts(self):
        return int(self.positions.shape[0])

    def signature(self):
        S, Ho, Wo = self.obj.shape
        P, n, _ = self.probe.shape
        return (n, S, P, Ho, Wo, int(self.batch_idx.numel()))

    def cost(self):
        n, S, P, _, _, B = self.signature()
        return float(B) * P * (4 * S + 2)  # transforms per position: P(2S + 1) forward + P(2S + 1) adjoint


def _window_groups(problems):
    """Indices of the datasets per probe window (one persistent launch each)."""
    groups = {}
    for i, pr in enumerate(problems):
        groups.setdefault(int(pr.probe.shape[-1]), []).append(i)
    return list(groups.values())


def default_grids(problems, total=None):
    """CTAs per dataset proportional to its transform count (at least one); each
    probe-window group (a launch of its own) splits the whole SM count."""
    total = total or ops.sm_count(problems[0].obj.device)
    groups = _window_groups(problems)
    if len(groups) > 1:
        out = [0] * len(problems)
        for idx in groups:
            for i, g in zip(idx, _split(([problems[i] for i in idx]), total)):
                out[i] = g
        return out
    return _split(problems, total)


def _split(problems, total):
    cost = np.array([p.cost() for p in problems])
    raw = np.maximum(1, np.floor(cost / cost.sum() * total)).astype(int)
    B = np.array([p.signature()[-1] for p in problems])
    raw = np.minimum(raw, B)
    while raw.sum() < total and (raw < B).any():  # hand out the remainder to the most loaded
        load = np.where(raw < B, cost / raw, -1)
        raw[int(np.argmax(load))] += 1
    return [int(x) for x in raw]


def multi_forward_adjoint(problems, obj_cs, probe_os, grids):
    """One persistent launch per probe window for all datasets (typically one);
    returns per dataset (loss, grad obj_c, grad probe_o) in the input order."""
    groups = _window_groups(problems)
    if len(groups) > 1:
        res = [None] * len(problems)
        for idx in groups:
            sub = _multi_launch([problems[i] for i in idx], [obj_cs[i] for i in idx], [probe_os[i] for i in idx],
                                [grids[i] for i in idx])
            for i, r in zip(idx, sub):
                res[i] = r
        return res
    return _multi_launch(problems, obj_cs, probe_os, grids)


def _multi_launch(problems, obj_cs, probe_os, grids):
    n = problems[0].probe.shape[-1]
    args = (_lib.BatchArgs * len(problems))()
    keep, outs = [], []
    for d, (pr, oc, po, g) in enumerate(zip(problems, obj_cs, probe_os, grids)):
        geom = ops._check_batch_inputs(oc, po, pr.prop, pr.positions, pr.batch_idx, pr.targets, pr.mask)
        if geom.n != n:
            raise ValueError("datasets of one multi launch need the same probe window")
        ph = ops.fft2(po)
        gobj = torch.zeros_like(oc)
        B = int(pr.batch_idx.numel())
        a = ops._batch_args(geom, oc, ph, pr.prop, pr.positions, pr.batch_idx, pr.targets, pr.mask, B, pr.loss_type,
                            ops.loss_scale_of(pr.loss_type, B, pr.num_gpts, pr.mean_intensity),
                            1.0 / pr.mean_intensity, grad_obj=gobj, variant="serial")
        nn = geom.n * geom.n
        pr.ws.ensure(g * (geom.P * geom.S + geom.P + 1) * nn, g * geom.P * nn, g)
        a.grid = g
        a.scratch, a.probe_grad_part = pr.ws.scratch.data_ptr(), pr.ws.partials.data_ptr()
        a.loss_part, a.status = pr.ws.loss_part.data_ptr(), pr.ws.status.data_ptr()
        args[d] = a
        keep += [ph]
        outs.append((gobj, geom))
    lib = _lib.lib()
    st = ops._stream()
    _lib.check(lib.ptycho_forward_adjoint_multi(ctypes.cast(args, ctypes.c_void_p), len(problems), st),
               "forward_adjoint_multi")
    res = []
    for pr, (gobj, geom), g, po in zip(problems, outs, grids, probe_os):
        loss = torch.empty((), dtype=torch.float32, device=gobj.device)
        _lib.check(lib.ptycho_reduce_loss(ops._p(pr.ws.loss_part), g, ops._p(loss), st), "reduce_loss")
        gp = torch.empty_like(po)
        nn = geom.P * geom.n * geom.n
        _lib.check(lib.ptycho_reduce_partials(ops._p(pr.ws.partials), ops._p(gp), g, nn, st), "reduce_partials")
        _lib.check(lib.ptycho_fft2(ops._p(gp), ops._p(gp), geom.P, geom.n, 1, 1.0 / (geom.n * geom.n), st), "fft2")
        res.append((loss, gobj, gp))
    del keep
    return res


class _MultiLossFn(torch.autograd.Function):
    """Losses of all datasets (vector) w.r.t. raw objects and orthogonalised probes."""

    @staticmethod
    def forward(ctx, grids, problems, *tensors):
        nd = len(problems)
        objs, probe_os = tensors[:nd], tensors[nd:]
        works, obj_cs = [], []
        for o in objs:
            oc, w = ops.obj_constrain(o.detach().contiguous())
            obj_cs.append(oc)
            works.append(w)
        res = multi_forward_adjoint(problems, obj_cs, [p.detach().contiguous() for p in probe_os], grids)
        ctx.save_for_backward(*[o.detach() for o in objs], *works, *[r[1] for r in res], *[r[2] for r in res])
        ctx.nd = nd
        return torch.stack([r[0] for r in res])

    @staticmethod
    def backward(ctx, gout):
        nd = ctx.nd
        t = ctx.saved_tensors
        objs, works, gcs, gps = t[:nd], t[nd:2 * nd], t[2 * nd:3 * nd], t[3 * nd:]
        gout = ops.dense(gout.detach().to(torch.float32))
        g_objs = [ops.obj_constrain_vjp(o, gc, w, scale=gout[d:d + 1]) for d, (o, gc, w) in
                  enumerate(zip(objs, gcs, works))]
        g_probes = [gp * gout[d] for d, gp in enumerate(gps)]
        return (None, None, *g_objs, *g_probes)


def multi_losses(problems, grids):
    probe_os = [orthogonalize_probes(p.probe) if p.orthogonalize else p.probe for p in problems]
    return _MultiLossFn.apply(grids, problems, *[p.obj for p in problems], *probe_os)


class CapturableAdam:
    """Adam/AdamW over complex or real leaf tensors with the step count and the
    learning rate on the device, so a CUDA-graph replay advances the bias
    corrections (same update as torch.optim.Adam)."""

    def __init__(self, params, lr=1e-3, betas=(0.9, 0.999), eps=1e-8, weight_decay=0.0, decoupled=False):
        self.params = list(params)
        dev = self.params[0].device
        self.lr = torch.full((1,), float(lr), device=dev)
        self.step_t = torch.zeros(1, device=dev)
        self.betas, self.eps, self.wd, self.decoupled = betas, eps, weight_decay, decoupled
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]

    def step(self):
        lib = _lib.lib()
        st = ops._stream()
        _lib.check(lib.ptycho_add_scalar(ops._p(self.step_t), 1.0, st), "add_scalar")
        for p, m, v in zip(self.params, self.m, self.v):
            if p.grad is None:
                continue
            rv = ops._real_view
            _lib.check(lib.ptycho_adam_step_dev(ops._p(rv(p.data)), ops._p(rv(p.grad)), ops._p(rv(m)), ops._p(rv(v)),
                                                rv(p.data).numel(), ops._p(self.lr), ops._p(self.step_t),
                                                self.betas[0], self.betas[1], self.eps, self.wd, int(self.decoupled),
                                                st), "adam_step_dev")


class MultiIteration:
    """One full-batch gradient iteration over several datasets (eager or graphed)."""

    def __init__(self, problems, grids=None, lr_obj=5e-3, lr_probe=1e-3):
        self.problems = problems
        self.grids = grids or default_grids(problems)
        self.opt_obj = CapturableAdam([p.obj for p in problems], lr=lr_obj)
        self.opt_probe = CapturableAdam([p.probe for p in problems], lr=lr_probe)
        self.graph = None
        self.static_losses = None

    def _step(self):
        for p in self.problems:
            p.obj.grad = None
            p.probe.grad = None
        losses = multi_losses(self.problems, self.grids)
        losses.sum().backward()
        for p in self.problems:
            p.obj.grad.mul_(p.upsample_factor ** 2 / 2)  # ptychography.py:330-332
        self.opt_obj.step()
        self.opt_probe.step()
        return losses.detach()

    def run_eager(self):
        return self._step()

    def capture(self, warmup=2):
        """Warm up on a side stream, then capture one iteration in a CUDA graph."""
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for _ in range(warmup):
                self._step()
        torch.cuda.current_stream().wait_stream(s)
        for p in self.problems:
            p.obj.grad = None
            p.probe.grad = None
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.static_losses = self._step()
        return self

    def replay(self):
        self.graph.replay()
        return self.static_losses

    def check_status(self):
        """Read and clear every dataset's status word (one small copy each, which waits for
        the queued work): raise on out-of-range batch indices, warn on non-finite predicted
        intensities, like ``ops.check_status`` for single-dataset launches."""
        # every word is read and cleared before anything is raised, so no dataset's
        # count is left behind for the next check
        out = []
        for p in self.problems:
            v = int(p.ws.status.item())
            if v:
                p.ws.status.zero_()
            out.append(ops.decode_status(v))
        for d, st in enumerate(out):
            if st["nonfinite"]:
                warnings.warn(f"dataset {d}: {st['nonfinite']} predicted intensities were not finite",
                              RuntimeWarning, stacklevel=2)
        bad = [(d, st["invalid_indices"]) for d, st in enumerate(out) if st["invalid_indices"]]
        if bad:
            raise RuntimeError("batch position(s) with an index outside [0, num positions): "
                               + ", ".join(f"dataset {d}: {k}" for d, k in bad))
        return out


def autotune_grids(problems, total=None, trials=2, cache={}):
    """Pick the CTA partition of a multi-dataset launch by timing candidates.

    Candidates: the cost-proportional split of the SM count, the same with one
    extra wave of CTAs, and splits that move CTAs towards the datasets with
    the highest cost per CTA.  Each is timed (CUDA events) on the forward +
    adjoint launch; the fastest is cached per problem signature."""
    key = tuple(p.signature() for p in problems)
    if key in cache:
        return cache[key]
    sms = total or ops.sm_count(problems[0].obj.device)
    cands = [default_grids(problems, sms), default_grids(problems, 2 * sms)]
    base = np.array(cands[0])
    cost = np.array([p.cost() for p in problems])
    for shift in (1, 2):
        g = base.copy()
        hi = int(np.argmax(cost / g))
        lo = int(np.argmin(cost / g))
        if g[lo] > shift:
            g[lo] -= shift
            g[hi] += shift
            cands.append([int(x) for x in g])
    probe_os = [p.probe.detach().contiguous() for p in problems]
    obj_cs = [ops.obj_constrain(p.obj.detach().contiguous())[0] for p in problems]
    best, best_t = None, float("inf")
    for g in cands:
        g = [min(int(x), int(p.batch_idx.numel())) for x, p in zip(g, problems)]
        multi_forward_adjoint(problems, obj_cs, probe_os, g)  # warm-up
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(trials):
            multi_forward_adjoint(problems, obj_cs, probe_os, g)
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / trials
        if t < best_t:
            best, best_t = g, t
    cache[key] = best
    return best
