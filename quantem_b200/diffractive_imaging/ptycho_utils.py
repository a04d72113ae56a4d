"""Host-side helpers of the ptychography path (batching, probe orthogonalisation).

Behaviour follows quantem.diffractive_imaging.ptycho_utils / probe_models of the
reference (file:line cited per function).
"""
from __future__ import annotations

from math import ceil
from typing import Literal

import numpy as np
import torch


class SimpleBatcher:
    """Per-epoch shuffled position batches with an optional validation split.

    Same index arithmetic and numpy-generator call sequence as the reference's
    SimpleBatcher (ptycho_utils.py:16-117), so a seeded run visits positions in
    the same order.
    """

    def __init__(self, num: int, batch_size: int | None, shuffle: bool = True,
                 rng: np.random.Generator | int | None = None, val_ratio: float = 0.0,
                 val_mode: Literal["grid", "random"] = "grid",
                 train_indices: np.ndarray | None = None, val_indices: np.ndarray | None = None):
        self.indices = np.arange(num)
        self.batch_size = batch_size if batch_size is not None else num
        self.shuffle = shuffle
        self.rng = rng
        if train_indices is not None or val_indices is not None:
            if train_indices is None or val_indices is None:
                raise ValueError("Both train_indices and val_indices must be provided together.")
            self.train_indices = np.asarray(train_indices, dtype=int)
            self.val_indices = np.asarray(val_indices, dtype=int)
            return
        if val_ratio < 0 or val_ratio >= 1:
            val_ratio = 0.0
        n_val = int(round(len(self.indices) * val_ratio))
        if n_val > 0:
            if val_mode == "random":
                perm = self.rng.permutation(self.indices)
                self.val_indices = perm[:n_val]
                self.train_indices = np.setdiff1d(self.indices, self.val_indices, assume_unique=False)
            else:
                if val_ratio <= 0.5:
                    k = max(1, int(round(1.0 / val_ratio)))
                    invert = False
                else:
                    k = max(1, int(round(1.0 / (1.0 - val_ratio))))
                    invert = True
                grid_sel = self.indices[::k]
                if len(grid_sel) > n_val:
                    grid_sel = grid_sel[:n_val]
                if invert:
                    self.train_indices = grid_sel
                    self.val_indices = np.setdiff1d(self.indices, grid_sel, assume_unique=False)
                else:
                    self.val_indices = grid_sel
                    self.train_indices = np.setdiff1d(self.indices, self.val_indices, assume_unique=False)
        else:
            self.val_indices = np.asarray([], dtype=int)
            self.train_indices = self.indices

    @property
    def rng(self) -> np.random.Generator:
        return self._rng

    @rng.setter
    def rng(self, rng):
        if rng is None:
            rng = np.random.default_rng()
        elif isinstance(rng, (int, float)):
            rng = np.random.default_rng(rng)
        elif not isinstance(rng, np.random.Generator):
            raise TypeError(f"rng should be a np.random.Generator or a seed, got {type(rng)}")
        self._rng = rng

    def __iter__(self):
        order = self.rng.permutation(self.train_indices) if self.shuffle else self.train_indices
        for i in range(0, len(order), self.batch_size):
            yield order[i:i + self.batch_size]

    def __len__(self):
        return int(ceil(len(self.train_indices) / self.batch_size))

    def iter_val(self):
        if len(self.val_indices) == 0:
            return iter(())

        def _gen():
            for i in range(0, len(self.val_indices), self.batch_size):
                yield self.val_indices[i:i + self.batch_size]

        return _gen()

    @property
    def has_validation(self) -> bool:
        return len(self.val_indices) > 0

    def val_len(self) -> int:
        return int(ceil(len(self.val_indices) / self.batch_size)) if self.has_validation else 0


def device_batches(batcher: SimpleBatcher, device) -> list[torch.Tensor]:
    """The batches of one pass of ``batcher`` (same generator calls, same boundaries) as
    int64 index tensors on ``device``: the pass's whole order goes up in one pinned,
    asynchronous copy, so no batch waits for a pageable host copy (which would drain the
    stream before every batch).  The copy is issued here, before the caller's loop: a pinned
    copy runs on a copy engine, so a caller that streams other data up on a side stream
    issues this one first, or it queues behind that transfer."""
    batches = list(batcher)
    if not batches:
        return []
    order = torch.from_numpy(np.ascontiguousarray(np.concatenate(batches), dtype=np.int64))
    dev = torch.device(device)
    if dev.type == "cuda":
        order = order.pin_memory().to(dev, non_blocking=True)
    else:
        order = order.to(dev)
    out, start = [], 0
    for b in batches:
        out.append(order[start:start + len(b)])
        start += len(b)
    return out


class _OrthogonalizeProbes(torch.autograd.Function):
    """The orthogonalisation on the GPU: one ``ptycho_probe_orthogonalize`` launch
    forward, one ``ptycho_probe_orthogonalize_vjp`` launch backward."""

    @staticmethod
    def forward(ctx, probe):
        from .. import _lib, ops

        probe = ops.dense(probe.detach())
        P = probe.shape[0]
        nn = probe[0].numel()
        lib = _lib.lib()
        we = int(lib.ptycho_probe_ortho_work_elems(P, nn))
        work = torch.empty(we, dtype=torch.complex64, device=probe.device)
        out = torch.empty_like(probe)
        _lib.check(lib.ptycho_probe_orthogonalize(ops._p(probe), ops._p(out), P, nn, ops._p(work), we, ops._stream()),
                   "probe_orthogonalize")
        ctx.save_for_backward(probe, work)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        from .. import _lib, ops

        probe, work = ctx.saved_tensors
        P = probe.shape[0]
        nn = probe[0].numel()
        g = ops.dense(grad_out.to(torch.complex64))
        grad = torch.empty_like(probe)
        _lib.check(_lib.lib().ptycho_probe_orthogonalize_vjp(ops._p(probe), ops._p(g), ops._p(grad), P, nn,
                                                             ops._p(work), work.numel(), ops._stream()),
                   "probe_orthogonalize_vjp")
        return grad


def orthogonalize_probes(start_probe: torch.Tensor) -> torch.Tensor:
    """Mixed-state Gram-Schmidt with norm restore and intensity sort.

    probe_models.py:484-525: modified Gram-Schmidt on the running vector,
    each mode rescaled to its original norm, modes sorted by descending
    real-space intensity.  Differentiable.  CUDA complex64 stacks run on the
    orthogonalisation kernels (forward and gradient, one launch each); host
    tensors (set-up code) use the same steps as tensor ops.
    """
    if start_probe.is_cuda and start_probe.dtype == torch.complex64 and 1 <= start_probe.shape[0] <= 16:
        return _OrthogonalizeProbes.apply(start_probe)
    n_probes = start_probe.shape[0]
    original_norms = torch.sqrt(
        torch.sum(start_probe.real.square() + start_probe.imag.square(), dim=(-2, -1), keepdim=True))
    ortho = []
    for i in range(n_probes):
        probe_i = start_probe[i]
        for j in range(len(ortho)):
            probe_i = probe_i - torch.sum(ortho[j].conj() * probe_i) * ortho[j]
        norm = torch.sqrt(torch.sum(probe_i.real.square() + probe_i.imag.square())).clamp_min(1e-12)
        ortho.append(probe_i / norm)
    probes = torch.stack(ortho) * original_norms.view(-1, 1, 1)
    intensities = torch.sum(torch.abs(probes).square(), dim=(-2, -1))
    order = torch.argsort(intensities, descending=True)
    return torch.complex(probes.real[order], probes.imag[order])


_CENTER_N = (64, 96, 128, 256)


class _CenterProbe(torch.autograd.Function):
    """The centre-of-mass shift on the GPU: ``ptycho_probe_center`` forward (centres of mass,
    probe FFT, ramp, inverse FFT), ``ptycho_probe_center_vjp`` backward."""

    @staticmethod
    def forward(ctx, probe):
        from .. import _lib, ops

        probe = ops.dense(probe.detach())
        P, n = probe.shape[0], probe.shape[-1]
        lib = _lib.lib()
        we = int(lib.ptycho_probe_center_work_elems(P, n))
        work = torch.empty(we, dtype=torch.complex64, device=probe.device)
        out = torch.empty_like(probe)
        _lib.check(lib.ptycho_probe_center(ops._p(probe), ops._p(out), P, n, ops._p(work), we, ops._stream()),
                   "probe_center")
        ctx.save_for_backward(probe, work)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        from .. import _lib, ops

        probe, work = ctx.saved_tensors
        P, n = probe.shape[0], probe.shape[-1]
        g = ops.dense(grad_out.to(torch.complex64))
        grad = torch.empty_like(probe)
        _lib.check(_lib.lib().ptycho_probe_center_vjp(ops._p(probe), ops._p(g), ops._p(grad), P, n, ops._p(work),
                                                      work.numel(), ops._stream()), "probe_center_vjp")
        return grad


def center_probe(start_probe: torch.Tensor) -> torch.Tensor:
    """Probe centre-of-mass constraint (probe_models.py:467-482): every mode's |psi|^2 centre
    of mass on the fftshifted grid, minus n // 2, shifted back to the origin with a Fourier
    ramp (fourier_shift_expand, ptycho_utils.py:128-139).  Differentiable, through the centre
    of mass too.  CUDA complex64 stacks run on the probe-centring kernels; host tensors
    (set-up code) use the same steps as tensor ops."""
    P, nr, nc = start_probe.shape[-3:]
    if (start_probe.is_cuda and start_probe.dtype == torch.complex64 and 1 <= P <= 16 and nr == nc
            and nr in _CENTER_N):
        return _CenterProbe.apply(start_probe)
    inten = torch.fft.fftshift(start_probe.abs().square(), dim=(-2, -1))
    yr = torch.arange(nr, device=inten.device, dtype=inten.dtype)
    yc = torch.arange(nc, device=inten.device, dtype=inten.dtype)
    tot = inten.sum(dim=(-2, -1))
    com = torch.stack([(inten * yr[:, None]).sum(dim=(-2, -1)) / tot - nr // 2,
                       (inten * yc[None, :]).sum(dim=(-2, -1)) / tot - nc // 2], dim=-1)
    kr = torch.as_tensor(np.fft.fftfreq(nr).astype(np.float32), device=inten.device)
    kc = torch.as_tensor(np.fft.fftfreq(nc).astype(np.float32), device=inten.device)
    shift = -com
    ramp = (torch.exp(-2j * np.pi * kr[None, :, None] * shift[:, 0, None, None])
            * torch.exp(-2j * np.pi * kc[None, None, :] * shift[:, 1, None, None])).to(start_probe.dtype)
    return torch.fft.ifft2(torch.fft.fft2(start_probe) * ramp)


class _ProbeTV(torch.autograd.Function):
    """The probe TV soft loss on the GPU: one ``ptycho_probe_tv`` call computes the loss and
    its gradient together; backward scales the gradient."""

    @staticmethod
    def forward(ctx, probe, weight):
        from .. import _lib, ops

        probe = ops.dense(probe.detach())
        P, n = probe.shape[0], probe.shape[-1]
        lib = _lib.lib()
        nw = int(lib.ptycho_probe_tv_work_elems())
        work = torch.empty(nw, dtype=torch.float64, device=probe.device)
        loss = torch.empty((), dtype=torch.float32, device=probe.device)
        grad = torch.empty_like(probe)
        _lib.check(lib.ptycho_probe_tv(ops._p(probe), P, n, float(weight), ops._p(loss), ops._p(grad), ops._p(work),
                                       nw, ops._stream()), "probe_tv")
        ctx.save_for_backward(grad)
        return loss

    @staticmethod
    def backward(ctx, g):
        (grad,) = ctx.saved_tensors
        return grad * g.to(grad.real.dtype), None


def probe_tv_loss(probe: torch.Tensor, weight: float) -> torch.Tensor:
    """Probe total-variation soft loss (probe_models.py:460-466): weight x (mean |diff| along
    the last axis + mean |diff| along the second-last); CUDA complex64 stacks on the TV
    kernel, host tensors with tensor ops."""
    if not weight:
        return torch.zeros((), device=probe.device)
    P, nr, nc = probe.shape[-3:]
    if probe.is_cuda and probe.dtype == torch.complex64 and nr == nc and nr >= 2:
        return _ProbeTV.apply(probe, float(weight))
    tv = torch.zeros((), device=probe.device)
    for dim in (-1, -2):
        tv = tv + torch.mean(torch.abs(torch.diff(probe, dim=dim)))
    return weight * tv
