"""Torch-facing wrappers around the C ABI of libptycho_b200.

PyTorch supplies device memory (caching allocator), the current CUDA stream and
autograd plumbing; every computation on the ptychography path runs in the
hand-written sm_100a kernels of ``csrc/``.  All functions require CUDA tensors
and raise ``RuntimeError`` if the library is unavailable (no CPU fallback).
"""
from __future__ import annotations

import ctypes
import warnings
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib

SUPPORTED_N = (64, 96, 128, 256)

# Adjoint checkpoint interval for 256 x 256 windows (0: keep every slice's wave;
# k > 0: keep every k-th and recompute the rest in the reverse sweep).
RECOMPUTE_EVERY = 0

# When set to a list, every fused forward+adjoint launch appends a pair of CUDA
# events recorded on the launching stream around it (used by bench.py to time
# the dominant kernel inside the timed region).
PROFILE_EVENTS = None


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def dense(t: torch.Tensor) -> torch.Tensor:
    """t with its lazy conjugate / negative bits applied and contiguous: the memory the
    kernels read (autograd hands complex gradients in as lazy conjugate views)."""
    return t.resolve_conj().resolve_neg().contiguous()


def _req(t: torch.Tensor, name: str, dtype: torch.dtype, device=None):
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if t.is_conj() or t.is_neg():
        raise ValueError(f"{name} is a lazy conjugate / negative view; pass ops.dense({name})")
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor (the B200 path has no CPU fallback)")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if device is not None and t.device != device:
        raise ValueError(f"{name} is on {t.device}, expected {device}")
    return t


_SM_COUNT: dict[int, int] = {}


def sm_count(device: torch.device | None = None) -> int:
    dev = torch.cuda.current_device() if device is None else (device.index or 0)
    if dev not in _SM_COUNT:
        with torch.cuda.device(dev):
            v = ctypes.c_int(0)
            _lib.check(_lib.lib().ptycho_sm_count(ctypes.byref(v)), "sm_count")
            _SM_COUNT[dev] = v.value
    return _SM_COUNT[dev]


def reduce_blocks() -> int:
    return int(_lib.lib().ptycho_reduce_blocks())


# ----------------------------------------------------------------------------
# small building blocks
# ----------------------------------------------------------------------------

def fft2(x: torch.Tensor, inverse: bool = False, scale: float = 1.0, out: torch.Tensor | None = None):
    """scale * (i)fft2 of a (..., n, n) complex64 stack, unnormalised transform."""
    _req(x, "x", torch.complex64)
    n = x.shape[-1]
    if x.shape[-2] != n or n not in SUPPORTED_N:
        raise ValueError(f"fft2 supports square {SUPPORTED_N} windows, got {tuple(x.shape[-2:])}")
    out = torch.empty_like(x) if out is None else _req(out, "out", torch.complex64)
    count = x.numel() // (n * n)
    _lib.check(_lib.lib().ptycho_fft2(_p(x), _p(out), count, n, int(inverse), float(scale), _stream()), "fft2")
    return out


def new_constraint_work(device) -> torch.Tensor:
    return torch.empty(2 * reduce_blocks(), dtype=torch.float64, device=device)


def obj_constrain(obj: torch.Tensor, work: torch.Tensor | None = None, out: torch.Tensor | None = None):
    """Complex-object hard constraint (object_models.py:289-300)."""
    _req(obj, "obj", torch.complex64)
    work = new_constraint_work(obj.device) if work is None else work
    out = torch.empty_like(obj) if out is None else out
    _lib.check(_lib.lib().ptycho_obj_constrain(_p(obj), _p(out), obj.numel(), _p(work), work.numel(), _stream()),
               "obj_constrain")
    return out, work


def obj_constrain_vjp(obj: torch.Tensor, grad_c: torch.Tensor, work: torch.Tensor,
                      scale: torch.Tensor | None = None, out: torch.Tensor | None = None):
    _req(obj, "obj", torch.complex64)
    _req(grad_c, "grad_c", torch.complex64)
    out = torch.empty_like(obj) if out is None else out
    if scale is not None:
        scale = scale.detach().to(torch.float32).contiguous()
    _lib.check(_lib.lib().ptycho_obj_constrain_vjp(_p(obj), _p(grad_c), _p(out), obj.numel(), _p(work),
                                                   work.numel(), _p(scale), _stream()), "obj_constrain_vjp")
    return out


class _ObjConstrainFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, obj):
        out, work = obj_constrain(dense(obj.detach()))
        ctx.save_for_backward(obj, work)
        return out

    @staticmethod
    def backward(ctx, g):
        obj, work = ctx.saved_tensors
        return obj_constrain_vjp(dense(obj.detach()), dense(g.to(torch.complex64)), work)


def constrained_object(obj: torch.Tensor) -> torch.Tensor:
    """Differentiable hard-constrained object computed by the CUDA kernels."""
    return _ObjConstrainFn.apply(obj)


OBJ_TYPES = {"complex": 0, "pure_phase": 1, "potential": 2}


@dataclass(frozen=True)
class ObjSpec:
    """How a raw object becomes the transmission the batch kernels multiply by
    (object_models.py:289-339, 252-256): the object type and the potential's
    positivity / baseline constraints."""

    obj_type: str = "complex"
    positivity: bool = True
    fix_baseline: bool = False
    baseline_factor: float = 1.0
    # False: the raw complex object is the transmission as it is (the reference's
    # ObjectDIP.forward feeds the network output to the patches without the hard
    # constraint, object_models.py:990-1008)
    hard_constraint: bool = True

    def __post_init__(self):
        if self.obj_type not in OBJ_TYPES:
            raise ValueError(f"object type must be one of {list(OBJ_TYPES)}, got {self.obj_type!r}")

    @property
    def raw_dtype(self):
        return torch.float32 if self.obj_type == "potential" else torch.complex64


COMPLEX_OBJECT = ObjSpec()


def _spec_args(spec: ObjSpec):
    return (OBJ_TYPES[spec.obj_type], int(bool(spec.positivity)), int(bool(spec.fix_baseline)),
            float(spec.baseline_factor))


def obj_transmission(obj: torch.Tensor, spec: ObjSpec = COMPLEX_OBJECT, work: torch.Tensor | None = None,
                     out: torch.Tensor | None = None):
    """Transmission (complex64) of a raw object of any type; returns (out, work)."""
    _req(obj, "obj", spec.raw_dtype)
    work = new_constraint_work(obj.device) if work is None else work
    if not spec.hard_constraint:
        if spec.obj_type != "complex":
            raise ValueError("an unconstrained transmission is a complex object")
        return (obj if out is None else out.copy_(obj)), work
    out = torch.empty(obj.shape, dtype=torch.complex64, device=obj.device) if out is None else out
    _lib.check(_lib.lib().ptycho_obj_transmission(_p(obj), _p(out), obj.numel(), *_spec_args(spec), _p(work),
                                                  work.numel(), _stream()), "obj_transmission")
    return out, work


def obj_transmission_vjp(obj: torch.Tensor, grad_t: torch.Tensor, work: torch.Tensor, spec: ObjSpec = COMPLEX_OBJECT,
                         scale: torch.Tensor | None = None, out: torch.Tensor | None = None):
    """Gradient w.r.t. the raw object (its own dtype) of a loss whose gradient w.r.t. the
    transmission is ``grad_t``; ``work`` from the matching ``obj_transmission`` call."""
    _req(obj, "obj", spec.raw_dtype)
    _req(grad_t, "grad_t", torch.complex64)
    if not spec.hard_constraint:  # identity transmission
        g = grad_t if scale is None else grad_t * scale.detach().to(torch.float32)
        return g.clone() if out is None else out.copy_(g)
    out = torch.empty_like(obj) if out is None else out
    if scale is not None:
        scale = scale.detach().to(torch.float32).contiguous()
    _lib.check(_lib.lib().ptycho_obj_transmission_vjp(_p(obj), _p(grad_t), _p(out), obj.numel(), *_spec_args(spec),
                                                      _p(work), work.numel(), _p(scale), _stream()),
               "obj_transmission_vjp")
    return out


class _ObjTransmissionFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, obj, spec):
        out, work = obj_transmission(dense(obj.detach()), spec)
        ctx.spec = spec
        ctx.save_for_backward(obj, work)
        return out

    @staticmethod
    def backward(ctx, g):
        obj, work = ctx.saved_tensors
        return obj_transmission_vjp(dense(obj.detach()), dense(g.to(torch.complex64)), work, ctx.spec), None


def object_transmission(obj: torch.Tensor, spec: ObjSpec = COMPLEX_OBJECT) -> torch.Tensor:
    """Differentiable transmission of a raw object of any type (CUDA kernels)."""
    return _ObjTransmissionFn.apply(obj, spec)


# ----------------------------------------------------------------------------
# batch kernels
# ----------------------------------------------------------------------------

@dataclass
class BatchGeometry:
    n: int
    S: int
    P: int
    Ho: int
    Wo: int
    npos: int

    @classmethod
    def of(cls, obj: torch.Tensor, probe: torch.Tensor, npos: int):
        S, Ho, Wo = obj.shape
        P, n, n2 = probe.shape
        if n != n2:
            raise ValueError("probe window must be square")
        if n not in SUPPORTED_N:
            raise ValueError(f"probe window {n} not supported (built: {SUPPORTED_N})")
        return cls(n=n, S=S, P=P, Ho=Ho, Wo=Wo, npos=npos)


class Workspace:
    """Per-device scratch for batch launches, grown on demand and reused."""

    def __init__(self, device):
        self.device = torch.device(device)
        self.scratch = None
        self.partials = None
        self.loss_part = None
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)

    def ensure(self, scratch_elems: int, partial_elems: int, grid: int):
        if scratch_elems and (self.scratch is None or self.scratch.numel() < scratch_elems):
            self.scratch = None
            self.scratch = torch.empty(int(scratch_elems), dtype=torch.complex64, device=self.device)
        if partial_elems and (self.partials is None or self.partials.numel() < partial_elems):
            self.partials = torch.empty(int(partial_elems), dtype=torch.complex64, device=self.device)
        if self.loss_part is None or self.loss_part.numel() < grid:
            self.loss_part = torch.empty(max(grid, 256), dtype=torch.float64, device=self.device)
        return self


_WORKSPACES: dict = {}


def workspace(device) -> Workspace:
    key = str(torch.device(device))
    if key not in _WORKSPACES:
        _WORKSPACES[key] = Workspace(device)
    return _WORKSPACES[key]


# Status word written by the batch kernels (one int32 per device workspace):
# bits 0-19 count non-finite predicted intensities, bits 20-30 count batch indices
# outside [0, npos) (those positions are skipped).  Each field saturates at its
# maximum, so a large non-finite count never reads as bad indices.
STATUS_NONFINITE_MASK = (1 << 20) - 1
STATUS_INVALID_SHIFT = 20
STATUS_INVALID_MASK = (1 << 11) - 1


def decode_status(v: int) -> dict:
    """Split a raw status word into its two counters."""
    return {"nonfinite": v & STATUS_NONFINITE_MASK,
            "invalid_indices": (v >> STATUS_INVALID_SHIFT) & STATUS_INVALID_MASK, "raw": v}


def read_status(device=None, reset: bool = True) -> dict:
    """Read (and by default clear) the batch kernels' status word of ``device``:
    ``{"nonfinite": n, "invalid_indices": k, "raw": v}``.  One 4-byte device-to-host
    copy, which waits for the work queued before it."""
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    ws = workspace(dev)
    v = int(ws.status.item())
    if reset and v:
        ws.status.zero_()
    return decode_status(v)


def check_status(device=None) -> dict:
    """Raise ``RuntimeError`` if a batch index was out of range since the last check
    (the kernels skip such positions); warn when predicted intensities were non-finite
    (the loss is then non-finite too, as in the reference).  Clears the word."""
    st = read_status(device, reset=True)
    if st["invalid_indices"]:
        raise RuntimeError(f"{st['invalid_indices']} batch position(s) had an index outside [0, num positions); "
                           "they were skipped by the batch kernel")
    if st["nonfinite"]:
        warnings.warn(f"{st['nonfinite']} predicted intensities were not finite (NaN / inf in the object or probe)",
                      RuntimeWarning, stacklevel=2)
    return st


def default_grid(B: int, device=None) -> int:
    return max(1, min(B, sm_count(device)))


def _batch_args(geom, obj_c, probe_hat, prop, positions, batch_idx, targets, mask, B, loss_type, loss_scale,
                inv_mean, grad_obj=None, out_intensity=None, out_exit=None, out_waves=None, variant="auto",
                recompute_every=None, descan=None):
    a = _lib.BatchArgs()
    if descan is not None:
        _req(descan, "descan", torch.float32, positions.device)
        if tuple(descan.shape) != tuple(positions.shape):
            raise ValueError(f"descan shifts must be {tuple(positions.shape)} like the positions")
        a.descan = descan.data_ptr()
    a.recompute_every = int(RECOMPUTE_EVERY if recompute_every is None else recompute_every)
    a.obj = obj_c.data_ptr()
    a.probe_hat = probe_hat.data_ptr()
    if isinstance(prop, (tuple, list)):
        a.prop = None
        a.prop_r = prop[0].data_ptr() if prop[0].numel() > 0 else None
        a.prop_c = prop[1].data_ptr() if prop[1].numel() > 0 else None
    else:
        a.prop = prop.data_ptr() if (prop is not None and prop.numel() > 0) else None
    a.positions = positions.data_ptr()
    a.batch_idx = batch_idx.data_ptr()
    a.targets = targets.data_ptr()
    a.mask = mask.data_ptr()
    a.grad_obj = grad_obj.data_ptr() if grad_obj is not None else None
    a.out_intensity = out_intensity.data_ptr() if out_intensity is not None else None
    a.out_exit = out_exit.data_ptr() if out_exit is not None else None
    a.out_waves = out_waves.data_ptr() if out_waves is not None else None
    a.n, a.S, a.P, a.B = geom.n, geom.S, geom.P, int(B)
    a.Ho, a.Wo, a.npos = geom.Ho, geom.Wo, geom.npos
    a.loss_type = _lib.LOSS_TYPES[loss_type]
    a.loss_scale = float(loss_scale)
    a.inv_mean_intensity = float(inv_mean)
    a.variant = _lib.VARIANTS[variant]
    return a


def plan_and_bind(a, device, adjoint: bool, grid=None):
    """Resolve the launch plan of ``a`` (variant, grid, workspace sizes), bind the
    device workspace and return (grid, number of probe-gradient partials)."""
    v, g, parts = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
    se, pe = ctypes.c_int64(0), ctypes.c_int64(0)
    _lib.check(_lib.lib().ptycho_batch_plan(ctypes.byref(a), int(adjoint), ctypes.byref(v), ctypes.byref(g),
                                            ctypes.byref(se), ctypes.byref(pe), ctypes.byref(parts)), "batch_plan")
    grid_v, parts_v = g.value, parts.value
    if grid is not None:  # caller-chosen grid (serial variant only)
        if v.value != _lib.VARIANTS["serial"]:
            raise ValueError("an explicit grid is only accepted with variant='serial'")
        grid_v = parts_v = int(grid)
        nn = a.n * a.n
        slots = a.P * a.S + a.P + 1 + (a.P * (a.S - 1) if a.grad_prop else 0)
        se.value, pe.value = grid_v * slots * nn, grid_v * a.P * nn
    ws = workspace(device).ensure(se.value if adjoint else 0, pe.value if adjoint else 0, grid_v)
    a.grid = grid_v
    a.scratch = ws.scratch.data_ptr() if adjoint else None
    a.probe_grad_part = ws.partials.data_ptr() if adjoint else None
    a.loss_part = ws.loss_part.data_ptr()
    a.status = ws.status.data_ptr()
    return grid_v, parts_v, ws


def _check_batch_inputs(obj_c, probe_o, prop, positions, batch_idx, targets, mask):
    dev = obj_c.device
    _req(obj_c, "obj", torch.complex64, dev)
    _req(probe_o, "probe", torch.complex64, dev)
    sep = isinstance(prop, (tuple, list))
    if sep:
        for t in prop:
            _req(t, "separable propagator factors", torch.complex64, dev)
    elif prop is not None and prop.numel() > 0:
        _req(prop, "propagators", torch.complex64, dev)
    _req(positions, "positions", torch.float32, dev)
    _req(batch_idx, "batch_indices", torch.int64, dev)
    _req(targets, "targets", torch.float32, dev)
    _req(mask, "detector_mask", torch.float32, dev)
    geom = BatchGeometry.of(obj_c, probe_o, positions.shape[0])
    if targets.shape[1:] != (geom.n, geom.n) or mask.shape != (geom.n, geom.n):
        raise ValueError("targets / mask must be (npos, n, n) / (n, n)")
    if geom.S > 1:
        if sep:
            if any(tuple(t.shape) != (geom.S - 1, geom.n) for t in prop):
                raise ValueError(f"separable propagator factors must be ({geom.S - 1}, {geom.n}) each")
        elif prop is None or tuple(prop.shape) != (geom.S - 1, geom.n, geom.n):
            raise ValueError(f"propagators must be ({geom.S - 1}, {geom.n}, {geom.n})")
    return geom


def loss_scale_of(loss_type: str, B: int, num_gpts: int, mean_intensity: float) -> float:
    # error / (B / N) / mean_I for l1/l2 (ptychography_base.py:924-931)
    return float(num_gpts) / float(B) / float(mean_intensity)


def batch_forward(obj_c, probe_o, prop, positions, batch_idx, targets, mask, num_gpts, mean_intensity,
                  loss_type="l2_amplitude", want_intensity=True, want_exit=False, want_waves=False,
                  probe_hat=None, grid=None, variant="auto", descan=None):
    """Forward model + loss of one batch with no gradients.  ``descan`` (optional
    float32 (npos, 2)): descan shifts applied to the exit waves.

    Returns dict(loss=0-d tensor, intensity=(B,n,n) detector layout or None,
    exit=(P,B,n,n) or None, waves=(S,P,B,n,n) or None).
    """
    geom = _check_batch_inputs(obj_c, probe_o, prop, positions, batch_idx, targets, mask)
    B = int(batch_idx.numel())
    dev = obj_c.device
    if probe_hat is None:
        probe_hat = fft2(probe_o)
    out_i = torch.empty((B, geom.n, geom.n), dtype=torch.float32, device=dev) if want_intensity else None
    out_e = torch.empty((geom.P, B, geom.n, geom.n), dtype=torch.complex64, device=dev) if want_exit else None
    out_w = (torch.empty((geom.S, geom.P, B, geom.n, geom.n), dtype=torch.complex64, device=dev)
             if want_waves else None)
    a = _batch_args(geom, obj_c, probe_hat, prop, positions, batch_idx, targets, mask, B, loss_type,
                    loss_scale_of(loss_type, max(B, 1), num_gpts, mean_intensity), 1.0 / mean_intensity,
                    out_intensity=out_i, out_exit=out_e, out_waves=out_w, variant=variant, descan=descan)
    grid_v, _, ws = plan_and_bind(a, dev, adjoint=False, grid=grid)
    loss = torch.empty((), dtype=torch.float32, device=dev)
    if B == 0:
        loss.zero_()
        return dict(loss=loss, intensity=out_i, exit=out_e, waves=out_w)
    _lib.check(_lib.lib().ptycho_forward_loss(ctypes.byref(a), _stream()), "forward_loss")
    _lib.check(_lib.lib().ptycho_reduce_loss(_p(ws.loss_part), grid_v, _p(loss), _stream()), "reduce_loss")
    return dict(loss=loss, intensity=out_i, exit=out_e, waves=out_w)


def batch_forward_adjoint(obj_c, probe_o, prop, positions, batch_idx, targets, mask, num_gpts, mean_intensity,
                          loss_type="l2_amplitude", probe_hat=None, grid=None, grad_obj=None,
                          grad_probe=None, variant="auto", recompute_every=None, grad_positions=None,
                          descan=None, grad_descan=None, grad_prop=None):
    """Fused forward + loss + adjoint of one batch.

    Returns (loss 0-d tensor, grad w.r.t. the constrained object (S,Ho,Wo),
    grad w.r.t. the orthogonalised probe (P,n,n)), torch gradient convention.
    ``grad_obj`` (if given) is accumulated into, not cleared.  ``grad_positions``
    (optional float32 (B, 2), zero-filled by the caller) receives dL/d(position) of
    every batch entry (the serial kernel runs then).  ``descan`` (float32 (npos, 2))
    applies descan shifts to the exit waves; ``grad_descan`` (float32 (B, 2)) receives
    dL/d(descan) of every batch entry; ``grad_prop`` (float32 (S-1, 2), zero-filled)
    accumulates the propagator sensitivities sum_k fftfreq_index(k) Im(conj(dL/dZ_s) Z_s)
    along rows and columns (the probe-tilt gradient's per-slice factors).
    """
    geom = _check_batch_inputs(obj_c, probe_o, prop, positions, batch_idx, targets, mask)
    B = int(batch_idx.numel())
    dev = obj_c.device
    if probe_hat is None:
        probe_hat = fft2(probe_o)
    if grad_obj is None:
        grad_obj = torch.zeros_like(obj_c)
    loss = torch.empty((), dtype=torch.float32, device=dev)
    if grad_probe is None:
        grad_probe = torch.empty_like(probe_o)
    if B == 0:
        loss.zero_()
        grad_probe.zero_()
        return loss, grad_obj, grad_probe
    ext = grad_positions is not None or descan is not None or grad_descan is not None or grad_prop is not None
    a = _batch_args(geom, obj_c, probe_hat, prop, positions, batch_idx, targets, mask, B, loss_type,
                    loss_scale_of(loss_type, B, num_gpts, mean_intensity), 1.0 / mean_intensity,
                    grad_obj=grad_obj, variant="serial" if ext else variant,
                    recompute_every=recompute_every, descan=descan)
    for name, t, shape in (("grad_positions", grad_positions, (B, 2)), ("grad_descan", grad_descan, (B, 2)),
                           ("grad_prop", grad_prop, (max(geom.S - 1, 0), 2))):
        if t is None:
            continue
        _req(t, name, torch.float32, dev)
        if tuple(t.shape) != shape:
            raise ValueError(f"{name} must be {shape}")
        setattr(a, name, t.data_ptr())
    grid_v, parts, ws = plan_and_bind(a, dev, adjoint=True, grid=grid)
    lib = _lib.lib()
    st = _stream()
    if PROFILE_EVENTS is not None:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
    _lib.check(lib.ptycho_forward_adjoint(ctypes.byref(a), st), "forward_adjoint")
    if PROFILE_EVENTS is not None:
        ev1.record()
        PROFILE_EVENTS.append((ev0, ev1))
    _lib.check(lib.ptycho_reduce_loss(_p(ws.loss_part), grid_v, _p(loss), st), "reduce_loss")
    nn = geom.P * geom.n * geom.n
    _lib.check(lib.ptycho_reduce_partials(_p(ws.partials), _p(grad_probe), parts, nn, st), "reduce_partials")
    inv = 1.0 / float(geom.n * geom.n)
    _lib.check(lib.ptycho_fft2(_p(grad_probe), _p(grad_probe), geom.P, geom.n, 1, inv, st), "fft2")
    return loss, grad_obj, grad_probe


def batch_analytic(obj_c, probe_o, prop, positions, batch_idx, targets, mask, num_gpts, mean_intensity,
                   loss_type="l2_amplitude", probe_hat=None):
    """Analytic (autograd=False) update directions of one batch, as the reference's
    ``Ptychography.backward(autograd=False)`` leaves them in ``_obj.grad`` and
    ``_probe.grad`` (ptychography.py:339-372, object_models.py:686-725,
    probe_models.py:774-783): Fourier-projection seed, reverse multislice,
    object update / sum over modes of max(sum_patches |psi|^2), probe update =
    minus the batch sum of the probe-plane gradient / max patch energy / the
    reference's orthonormal-FFT factor.  Returns (loss, grad_obj, grad_probe)."""
    geom = _check_batch_inputs(obj_c, probe_o, prop, positions, batch_idx, targets, mask)
    B = int(batch_idx.numel())
    dev = obj_c.device
    if probe_hat is None:
        probe_hat = fft2(probe_o)
    upd = torch.zeros_like(obj_c)
    loss = torch.zeros((), dtype=torch.float32, device=dev)
    g_probe = torch.zeros_like(probe_o)
    if B == 0:
        return loss, upd, g_probe
    an_norm = torch.zeros((geom.S, geom.P, geom.Ho, geom.Wo), dtype=torch.float32, device=dev)
    a = _batch_args(geom, obj_c, probe_hat, prop, positions, batch_idx, targets, mask, B, loss_type,
                    loss_scale_of(loss_type, B, num_gpts, mean_intensity), 1.0 / mean_intensity,
                    grad_obj=upd, variant="serial")
    a.analytic = 1
    a.an_norm = an_norm.data_ptr()
    grid_v, parts, ws = plan_and_bind(a, dev, adjoint=True)
    lib = _lib.lib()
    st = _stream()
    _lib.check(lib.ptycho_forward_adjoint(ctypes.byref(a), st), "forward_adjoint(analytic)")
    _lib.check(lib.ptycho_reduce_loss(_p(ws.loss_part), grid_v, _p(loss), st), "reduce_loss")
    nn = geom.P * geom.n * geom.n
    _lib.check(lib.ptycho_reduce_partials(_p(ws.partials), _p(g_probe), parts, nn, st), "reduce_partials")
    obj_norm = torch.empty(1, dtype=torch.float32, device=dev)
    _lib.check(lib.ptycho_patch_energy_max(_p(obj_c), _p(positions), _p(batch_idx), geom.S, geom.Ho, geom.Wo,
                                           geom.n, B, geom.npos, _p(obj_norm), st), "patch_energy_max")
    maxes = torch.empty(geom.S * geom.P, dtype=torch.float32, device=dev)
    g_obj = torch.empty_like(obj_c)
    _lib.check(lib.ptycho_analytic_obj_finalize(_p(upd), _p(an_norm), _p(maxes), geom.S, geom.P,
                                                geom.Ho * geom.Wo, _p(g_obj), st), "analytic_obj_finalize")
    hw = float(geom.n * geom.n)
    ortho = 2.0 * hw**0.5 if geom.P == 1 else 1.0 / (2.0 * hw**0.5)
    _lib.check(lib.ptycho_analytic_probe_finalize(_p(g_probe), nn, _p(obj_norm), float(ortho), st),
               "analytic_probe_finalize")
    return loss, g_obj, g_probe


class _BatchLossFn(torch.autograd.Function):
    """loss(obj_raw, probe_o, positions, descan, tilt) of one batch; gradients from the
    fused adjoint kernel."""

    @staticmethod
    def forward(ctx, obj_raw, probe_o, prop, positions, batch_idx, targets, mask, descan, tilt, cfg):
        obj_raw_c = dense(obj_raw.detach())
        probe_c = dense(probe_o.detach())
        spec = cfg.get("obj_spec") or COMPLEX_OBJECT
        ctx.spec = spec
        obj_c, work = obj_transmission(obj_raw_c, spec)
        ng = ctx.needs_input_grad
        need = ng[0] or ng[1] or ng[3] or ng[7] or ng[8]
        ctx.npos = int(positions.shape[0])
        dsc = None if descan is None else dense(descan.detach())
        dev = positions.device
        if tilt is not None:
            prop = separable_propagators_t(cfg["prop_geometry"], tilt.detach())
        B = int(batch_idx.numel())
        empty = torch.empty(0, device=dev)
        if need:
            g_pos = torch.zeros((B, 2), dtype=torch.float32, device=dev) if ng[3] else None
            g_dsc = torch.zeros((B, 2), dtype=torch.float32, device=dev) if ng[7] else None
            S = int(obj_raw.shape[0])
            g_prop = torch.zeros((max(S - 1, 0), 2), dtype=torch.float32, device=dev) if ng[8] else None
            loss, g_obj_c, g_probe = batch_forward_adjoint(
                obj_c, probe_c, prop, positions.detach(), batch_idx, targets, mask, cfg["num_gpts"],
                cfg["mean_intensity"], cfg["loss_type"], grid=cfg.get("grid"), variant=cfg.get("variant", "auto"),
                recompute_every=cfg.get("recompute_every"), grad_positions=g_pos, descan=dsc, grad_descan=g_dsc,
                grad_prop=g_prop)
            ctx.save_for_backward(obj_raw_c, work, g_obj_c, g_probe, batch_idx,
                                  g_pos if g_pos is not None else empty, g_dsc if g_dsc is not None else empty,
                                  g_prop if g_prop is not None else empty,
                                  tilt.detach() if tilt is not None else empty)
            ctx.prop_geometry = cfg.get("prop_geometry")
        else:
            loss = batch_forward(obj_c, probe_c, prop, positions.detach(), batch_idx, targets, mask, cfg["num_gpts"],
                                 cfg["mean_intensity"], cfg["loss_type"], want_intensity=False,
                                 grid=cfg.get("grid"), variant=cfg.get("variant", "auto"), descan=dsc)["loss"]
        return loss

    @staticmethod
    def _per_position(ctx, g_batch, batch_idx, gout):
        """Per batch entry -> per scan position (repeated indices add up); the kernel skips
        out-of-range indices (and reports them): route them to row 0 with a zero gradient."""
        out = torch.zeros((ctx.npos, 2), dtype=torch.float32, device=g_batch.device)
        valid = (batch_idx >= 0) & (batch_idx < ctx.npos)
        out.index_add_(0, torch.where(valid, batch_idx, torch.zeros_like(batch_idx)), g_batch * gout * valid[:, None])
        return out

    @staticmethod
    def backward(ctx, gout):
        obj_raw, work, g_obj_c, g_probe, batch_idx, g_pos, g_dsc, g_prop, tilt = ctx.saved_tensors
        gout = dense(gout.detach().to(torch.float32).reshape(1))
        ng = ctx.needs_input_grad
        g_obj = obj_transmission_vjp(obj_raw, g_obj_c, work, ctx.spec, scale=gout) if ng[0] else None
        g_pr = g_probe * gout if ng[1] else None
        g_positions = _BatchLossFn._per_position(ctx, g_pos, batch_idx, gout) if ng[3] else None
        g_descan = _BatchLossFn._per_position(ctx, g_dsc, batch_idx, gout) if ng[7] else None
        g_tilt = None
        if ng[8]:
            g_tilt = tilt_gradient(g_prop, tilt, ctx.prop_geometry) * gout
        return g_obj, g_pr, None, g_positions, None, None, None, g_descan, g_tilt, None


def batch_loss(obj_raw, probe_o, prop, positions, batch_idx, targets, mask, num_gpts, mean_intensity,
               loss_type="l2_amplitude", grid=None, variant="auto", recompute_every=None, obj_spec=None,
               descan=None, tilt=None, prop_geometry=None):
    """Differentiable consistency loss of one batch w.r.t. the raw object
    parameter (hard constraint and, for potentials, exp(i V) included), the
    orthogonalised probe, the scan positions (when they require grad), the descan
    shifts ``descan`` (float32 (npos, 2), optional) and the probe tilt ``tilt`` (float32
    (2,) mrad, optional: the propagators are then built from it, ``prop_geometry`` =
    (n, sampling, energy, slice thicknesses), and ``prop`` is ignored).  ``obj_spec``
    (default: complex object) names the object type; ``recompute_every`` (256 x 256
    windows): adjoint checkpoint interval."""
    if tilt is not None and prop_geometry is None:
        raise ValueError("a probe tilt needs prop_geometry = (n, sampling, energy, slice thicknesses)")
    cfg = dict(num_gpts=int(num_gpts), mean_intensity=float(mean_intensity), loss_type=loss_type, grid=grid,
               variant=variant, recompute_every=recompute_every, obj_spec=obj_spec, prop_geometry=prop_geometry)
    return _BatchLossFn.apply(obj_raw, probe_o, prop, positions, batch_idx, targets, mask, descan, tilt, cfg)


def separable_propagators_t(prop_geometry, tilt: torch.Tensor):
    """``separable_propagators`` with the tilt given as a device tensor (2,) [mrad], so a
    learned tilt needs no device-to-host read: Kr_s = exp(-i pi lambda dz_s kr^2 -
    2 pi i dz_s tan(theta_r / 1e3) kr), Kc likewise (probe_models.py:406-425).  The
    factors are evaluated in float32 on the tilt's device."""
    import math

    from .diffractive_imaging.complex_probe import electron_wavelength_angstrom

    n, sampling, energy, dz = prop_geometry
    dev = tilt.device
    dz = torch.as_tensor(np.asarray(dz, dtype=np.float64), device=dev).reshape(-1)
    lam = electron_wavelength_angstrom(energy)
    t = torch.tan(tilt.to(torch.float64) / 1e3)
    out = []
    for ax in range(2):
        k = torch.fft.fftfreq(int(n), float(sampling[ax]), dtype=torch.float64, device=dev)
        ph = -math.pi * lam * dz[:, None] * k[None] ** 2 - 2 * math.pi * dz[:, None] * t[ax] * k[None]
        out.append(torch.polar(torch.ones_like(ph), ph).to(torch.complex64).contiguous())
    return tuple(out)


def tilt_gradient(prop_sums: torch.Tensor, tilt: torch.Tensor, prop_geometry) -> torch.Tensor:
    """dL/d(probe tilt) (2,) from the kernel's propagator sensitivities (S-1, 2):
    K_s carries exp(-2 pi i dz_s tan(theta / 1e3) k) per axis, k = index / (n d), so
    dL/dtheta = sum_s 2 pi dz_s sec^2(theta / 1e3) / 1e3 / (n d) * prop_sums[s].  The
    reference adds the tilt ramp only for a nonzero tilt (probe_models.py:418, 421), so
    a zero tilt gets a zero gradient."""
    import math

    n, sampling, _, dz = prop_geometry
    dev = prop_sums.device
    dz = torch.as_tensor(np.asarray(dz, dtype=np.float64), device=dev).reshape(-1, 1)
    d = torch.as_tensor([float(sampling[0]), float(sampling[1])], dtype=torch.float64, device=dev)
    th = tilt.to(torch.float64)
    coef = 2 * math.pi * dz / (1e3 * int(n) * d[None]) / torch.cos(th / 1e3)[None] ** 2
    g = (coef * prop_sums.to(torch.float64)).sum(0) * (th != 0)
    return g.to(torch.float32)


def separable_propagators(n, sampling, energy, slice_thicknesses, tilt_mrad=(0.0, 0.0), device="cuda"):
    """Per-axis factors of the Fresnel propagators (probe_models.py:376-427).

    K_s[kr, kc] = exp(-i pi lambda dz_s (kr^2 + kc^2)) exp(-2 pi i dz_s tan(tr) kr)
    exp(-2 pi i dz_s tan(tc) kc) = Kr_s[kr] * Kc_s[kc].  Evaluated in float64 and
    rounded to complex64.  Returns (Kr, Kc), each (S-1, n)."""
    import math

    from .diffractive_imaging.complex_probe import electron_wavelength_angstrom

    dz = torch.as_tensor(slice_thicknesses, dtype=torch.float64).reshape(-1)
    lam = electron_wavelength_angstrom(energy)
    out = []
    for ax, tilt in ((0, tilt_mrad[0]), (1, tilt_mrad[1])):
        k = torch.fft.fftfreq(int(n), float(sampling[ax]), dtype=torch.float64)
        ph = -math.pi * lam * dz[:, None] * k[None] ** 2
        if tilt:
            ph = ph - 2 * math.pi * dz[:, None] * math.tan(float(tilt) / 1e3) * k[None]
        out.append(torch.polar(torch.ones_like(ph), ph).to(torch.complex64).to(device).contiguous())
    return tuple(out)


# ----------------------------------------------------------------------------
# optional object constraints (object_models.py:273-480) and the FOV mask
# ----------------------------------------------------------------------------

def _cwork(device) -> torch.Tensor:
    return torch.empty(int(_lib.lib().ptycho_obj_constraint_work_elems()), dtype=torch.float64, device=device)


def probe_overlap(intensity: torch.Tensor, positions: torch.Tensor, obj_shape_2d) -> torch.Tensor:
    """(Ho, Wo) float32: sum over positions of ``intensity`` (n, n) placed at each
    position's wrapped patch window (ptychography_base.py:201-216)."""
    dev = intensity.device
    _req(intensity, "intensity", torch.float32, dev)
    _req(positions, "positions", torch.float32, dev)
    Ho, Wo = (int(x) for x in obj_shape_2d)
    out = torch.empty((Ho, Wo), dtype=torch.float32, device=dev)
    _lib.check(_lib.lib().ptycho_probe_overlap(_p(intensity), int(intensity.shape[-1]), _p(positions),
                                               int(positions.shape[0]), Ho, Wo, _p(out), _stream()), "probe_overlap")
    return out


def gaussian_taps(sigma: float, device) -> torch.Tensor:
    """The normalised float32 Gaussian of object_models.py:445-451."""
    import math

    k = int(2 * math.ceil(3 * sigma) + 1)
    if k % 2 == 0:
        k += 1
    ax = np.arange(-k // 2 + 1.0, k // 2 + 1.0, dtype=np.float32)
    g = np.exp(-0.5 * (ax / np.float32(sigma)) ** 2).astype(np.float32)
    return torch.as_tensor(g / g.sum(), dtype=torch.float32, device=device)


class _FovConstrainFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, obj, mask, pure):
        o = dense(obj.detach())
        m = dense(mask.detach())
        out = torch.empty_like(o)
        work = _cwork(o.device)
        _lib.check(_lib.lib().ptycho_obj_constrain_fov(_p(o), _p(m), m.numel(), _p(out), o.numel(), int(pure),
                                                       _p(work), work.numel(), _stream()), "obj_constrain_fov")
        ctx.save_for_backward(o, m)
        ctx.pure = pure
        return out

    @staticmethod
    def backward(ctx, g):
        o, m = ctx.saved_tensors
        g = dense(g.detach().to(torch.complex64))
        out = torch.empty_like(o)
        work = _cwork(o.device)
        _lib.check(_lib.lib().ptycho_obj_constrain_fov_vjp(_p(o), _p(m), m.numel(), _p(g), _p(out), o.numel(),
                                                           int(ctx.pure), _p(work), work.numel(), _stream()),
                   "obj_constrain_fov_vjp")
        return out, None, None


class _PotentialBaseFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, v, bmask, amask, positivity, fix, factor):
        v = dense(v.detach())
        out = torch.empty_like(v)
        work = _cwork(v.device)
        hw = int(v.shape[-2] * v.shape[-1])
        _lib.check(_lib.lib().ptycho_obj_potential_base(
            _p(v), _p(bmask) if bmask is not None else None, _p(amask) if amask is not None else None, hw, _p(out),
            v.numel(), int(positivity), int(fix), float(factor), _p(work), work.numel(), _stream()),
            "obj_potential_base")
        ctx.save_for_backward(v, *(t for t in (bmask, amask) if t is not None))
        ctx.has = (bmask is not None, amask is not None)
        ctx.args = (int(positivity), int(fix), float(factor))
        return out

    @staticmethod
    def backward(ctx, g):
        saved = list(ctx.saved_tensors)
        v = saved.pop(0)
        bmask = saved.pop(0) if ctx.has[0] else None
        amask = saved.pop(0) if ctx.has[1] else None
        g = dense(g.detach().to(torch.float32))
        out = torch.empty_like(v)
        work = _cwork(v.device)
        hw = int(v.shape[-2] * v.shape[-1])
        _lib.check(_lib.lib().ptycho_obj_potential_base_vjp(
            _p(v), _p(bmask) if bmask is not None else None, _p(amask) if amask is not None else None, hw, _p(g),
            _p(out), v.numel(), *ctx.args, _p(work), work.numel(), _stream()), "obj_potential_base_vjp")
        return out, None, None, None, None, None


class _PhaseExpFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, v):
        v = dense(v.detach())
        out = torch.empty(v.shape, dtype=torch.complex64, device=v.device)
        _lib.check(_lib.lib().ptycho_phase_exp(_p(v), _p(out), v.numel(), _stream()), "phase_exp")
        ctx.save_for_backward(v)
        return out

    @staticmethod
    def backward(ctx, g):
        (v,) = ctx.saved_tensors
        g = dense(g.detach().to(torch.complex64))
        out = torch.empty_like(v)
        _lib.check(_lib.lib().ptycho_phase_exp_vjp(_p(v), _p(g), _p(out), v.numel(), _stream()), "phase_exp_vjp")
        return out


def _blur(x: torch.Tensor, taps: torch.Tensor) -> torch.Tensor:
    x = dense(x)
    out = torch.empty_like(x)
    tmp = torch.empty_like(x)
    S, Ho, Wo = (int(d) for d in x.shape)
    _lib.check(_lib.lib().ptycho_obj_blur(_p(x), _p(out), _p(tmp), S, Ho, Wo, int(x.is_complex()), _p(taps),
                                          int(taps.numel()), _stream()), "obj_blur")
    return out


class _BlurFn(torch.autograd.Function):
    """Zero-padded separable Gaussian blur: self-adjoint, so the VJP is the same blur."""

    @staticmethod
    def forward(ctx, x, taps):
        ctx.save_for_backward(taps)
        return _blur(x.detach(), taps)

    @staticmethod
    def backward(ctx, g):
        (taps,) = ctx.saved_tensors
        return _blur(g.detach(), taps), None


_ENV_CACHE: dict = {}


def butterworth_env(shape, sampling, q_lowpass, q_highpass, order, device) -> torch.Tensor:
    """The float32 Butterworth envelope (H, W) of object_models.py:495-507 (cached)."""
    key = (tuple(int(x) for x in shape), tuple(float(x) for x in sampling), q_lowpass, q_highpass, int(order),
           str(device))
    env = _ENV_CACHE.get(key)
    if env is None:
        qx = np.fft.fftfreq(key[0][0], key[1][0]).astype(np.float32)
        qy = np.fft.fftfreq(key[0][1], key[1][1]).astype(np.float32)
        qya, qxa = np.meshgrid(qy, qx, indexing="xy")
        qra = np.sqrt(qxa ** 2 + qya ** 2).astype(np.float32)
        e = np.ones_like(qra)
        if q_highpass:
            e = e * (1 - 1 / (1 + (qra / np.float32(q_highpass)) ** (2 * order)))
        if q_lowpass:
            e = e * (1 / (1 + (qra / np.float32(q_lowpass)) ** (2 * order)))
        env = torch.as_tensor(e.astype(np.float32), device=device).contiguous()
        if len(_ENV_CACHE) > 16:
            _ENV_CACHE.clear()
        _ENV_CACHE[key] = env
    return env


def _butter(x: torch.Tensor, env: torch.Tensor, vjp: bool) -> torch.Tensor:
    x = dense(x)
    S, Ho, Wo = (int(d) for d in x.shape)
    out = torch.empty_like(x)
    tmp = torch.empty((2, S, Ho, Wo), dtype=torch.complex64, device=x.device)
    means = torch.empty((2, S), dtype=torch.complex64, device=x.device)
    fn = _lib.lib().ptycho_obj_butterworth_vjp if vjp else _lib.lib().ptycho_obj_butterworth
    _lib.check(fn(_p(x), _p(out), S, Ho, Wo, int(not x.is_complex()), _p(env), _p(tmp), _p(means), _stream()),
               "obj_butterworth" + ("_vjp" if vjp else ""))
    return out


class _ButterworthFn(torch.autograd.Function):
    """The Butterworth filter of object_models.py:481-520 (per-slice mean kept, real part
    for potentials); self-adjoint up to the mean handling."""

    @staticmethod
    def forward(ctx, x, env):
        ctx.save_for_backward(env)
        return _butter(x.detach(), env, vjp=False)

    @staticmethod
    def backward(ctx, g):
        (env,) = ctx.saved_tensors
        return _butter(g.detach(), env, vjp=True), None


class _SliceMeanFn(torch.autograd.Function):
    """identical_slices: every slice replaced by the slice mean; the reference does it in
    place under no_grad, so the gradient passes straight through."""

    @staticmethod
    def forward(ctx, x):
        x = dense(x.detach())
        out = torch.empty_like(x)
        S = int(x.shape[0])
        _lib.check(_lib.lib().ptycho_obj_slice_mean(_p(x), _p(out), S, x[0].numel(), int(x.is_complex()),
                                                    _stream()), "obj_slice_mean")
        return out

    @staticmethod
    def backward(ctx, g):
        return g


def constrained_object_ext(obj_raw: torch.Tensor, obj_type: str, constraints: dict, mask=None,
                           sampling=None) -> torch.Tensor:
    """ObjectConstraints.apply_hard_constraints (object_models.py:289-339) with the optional
    constraints: the FOV mask (``apply_fov_mask``, ``mask`` (Ho, Wo)), the potential's
    baseline from the mask's background (``fix_potential_baseline``), ``gaussian_sigma``, the
    Butterworth filters (``q_lowpass`` / ``q_highpass`` with ``butterworth_order``; needs the
    object ``sampling`` [A]) and ``identical_slices``.  Differentiable; returns the complex
    object, or the real potential before exp(i V)."""
    c = constraints
    use_mask = bool(c.get("apply_fov_mask")) and mask is not None
    if obj_type in ("complex", "pure_phase"):
        if use_mask:
            out = _FovConstrainFn.apply(obj_raw, mask, obj_type == "pure_phase")
        else:
            out = object_transmission(obj_raw, ObjSpec(obj_type))
    elif obj_type == "potential":
        fix = bool(c.get("fix_potential_baseline", False))
        out = _PotentialBaseFn.apply(obj_raw, mask if fix else None, mask if use_mask else None,
                                     bool(c.get("positivity", True)), fix,
                                     float(c.get("fix_potential_baseline_factor", 1.0)))
    else:
        raise ValueError(f"unknown object type {obj_type!r}")
    if c.get("gaussian_sigma") is not None:
        out = _BlurFn.apply(out, gaussian_taps(float(c["gaussian_sigma"]), out.device))
    if c.get("q_lowpass") or c.get("q_highpass"):
        if sampling is None:
            raise ValueError("the Butterworth filters need the object sampling")
        env = butterworth_env(out.shape[-2:], sampling, c.get("q_lowpass"), c.get("q_highpass"),
                              int(c.get("butterworth_order", 4)), out.device)
        out = _ButterworthFn.apply(out, env)
    if c.get("identical_slices") and out.shape[0] > 1:
        out = _SliceMeanFn.apply(out)
    return out


def transmission_of(obj2: torch.Tensor) -> torch.Tensor:
    """What multiplies the wave: the complex object itself, exp(i V) of a potential
    (object_models.py:252-256)."""
    return obj2 if obj2.is_complex() else _PhaseExpFn.apply(obj2)


class _SoftLossFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, obj2, kind, wz, wxy, ws):
        o = dense(obj2.detach())
        S, Ho, Wo = (int(d) for d in o.shape)
        loss = torch.empty((), dtype=torch.float32, device=o.device)
        grad = torch.empty_like(o)
        work = _cwork(o.device)
        _lib.check(_lib.lib().ptycho_obj_soft_loss(_p(o), S, Ho, Wo, int(kind), float(wz), float(wxy), float(ws),
                                                   _p(work), work.numel(), _p(loss), _p(grad), _stream()),
                   "obj_soft_loss")
        ctx.save_for_backward(grad)
        return loss

    @staticmethod
    def backward(ctx, g):
        (grad,) = ctx.saved_tensors
        return grad * g.to(torch.float32), None, None, None, None


def soft_constraint_loss(obj2: torch.Tensor, obj_type: str, tv_weight_z=0.0, tv_weight_xy=0.0,
                         surface_zero_weight=0.0) -> torch.Tensor:
    """Soft constraints of the hard-constrained object (object_models.py:341-435): TV along z
    and in-plane, surface-zero terms; a differentiable scalar (zero gradient at zero-magnitude
    pixels, where the reference's autograd gives NaN)."""
    kind = {"complex": 0, "pure_phase": 1, "potential": 2}[obj_type]
    return _SoftLossFn.apply(obj2, kind, float(tv_weight_z), float(tv_weight_xy), float(surface_zero_weight))


# ----------------------------------------------------------------------------
# optimiser steps
# ----------------------------------------------------------------------------

def _real_view(t: torch.Tensor) -> torch.Tensor:
    return torch.view_as_real(t) if t.is_complex() else t


def adam_step(param, grad, exp_avg, exp_avg_sq, step: int, lr: float, betas=(0.9, 0.999), eps=1e-8,
              weight_decay=0.0, decoupled=False, lr_tensor=None, max_exp_avg_sq=None):
    """One Adam / AdamW step; with ``max_exp_avg_sq`` the AMSGrad variant."""
    p, g = _real_view(param), _real_view(grad)
    m, v = _real_view(exp_avg), _real_view(exp_avg_sq)
    vm = None if max_exp_avg_sq is None else _real_view(max_exp_avg_sq)
    for name, t in (("param", p), ("grad", g), ("exp_avg", m), ("exp_avg_sq", v), ("max_exp_avg_sq", vm)):
        if t is not None:
            _req(t.reshape(-1) if t.is_contiguous() else t, name, torch.float32)
    b1, b2 = betas
    bc1 = 1.0 - b1 ** step
    bc2s = (1.0 - b2 ** step) ** 0.5
    if vm is not None:
        _lib.check(_lib.lib().ptycho_adam_amsgrad_step(_p(p), _p(g), _p(m), _p(v), _p(vm), p.numel(), float(lr),
                                                       _p(lr_tensor), float(b1), float(b2), float(eps),
                                                       float(weight_decay), int(bool(decoupled)), float(bc1),
                                                       float(bc2s), _stream()), "adam_amsgrad_step")
        return
    _lib.check(_lib.lib().ptycho_adam_step(_p(p), _p(g), _p(m), _p(v), p.numel(), float(lr), _p(lr_tensor),
                                           float(b1), float(b2), float(eps), float(weight_decay),
                                           int(bool(decoupled)), float(bc1), float(bc2s), _stream()), "adam_step")


def sgd_step(param, grad, lr: float, weight_decay=0.0, lr_tensor=None):
    p, g = _real_view(param), _real_view(grad)
    _req(p, "param", torch.float32)
    _req(g, "grad", torch.float32)
    _lib.check(_lib.lib().ptycho_sgd_step(_p(p), _p(g), p.numel(), float(lr), _p(lr_tensor),
                                          float(weight_decay), _stream()), "sgd_step")


def sgd_momentum_step(param, grad, momentum_buffer, first: bool, lr: float, momentum: float, dampening=0.0,
                      nesterov=False, weight_decay=0.0, lr_tensor=None):
    """One torch.optim.SGD step with momentum (the buffer is seeded on the first step)."""
    p, g, b = _real_view(param), _real_view(grad), _real_view(momentum_buffer)
    for name, t in (("param", p), ("grad", g), ("momentum_buffer", b)):
        _req(t, name, torch.float32)
    _lib.check(_lib.lib().ptycho_sgd_momentum_step(_p(p), _p(g), _p(b), p.numel(), float(lr), _p(lr_tensor),
                                                   float(weight_decay), float(momentum), float(dampening),
                                                   int(bool(nesterov)), int(bool(first)), _stream()),
               "sgd_momentum_step")
