"""Mixed-state pixelated probe model (quantem probe_models.ProbePixelated).

Initial probe synthesis (probe_models.py:722-759 with complex_probe.py:475-507),
seeded per-mode phase ramps (846-858), mode weights (860-873), the hard constraints
(Gram-Schmidt, optional centre of mass; 452-525) on every access and the Fresnel propagators
(376-427).  The per-position Fourier shift runs inside the fused batch kernel;
``forward`` is kept for callers that want explicit shifted probes.
"""
from __future__ import annotations

import math
from copy import deepcopy

import numpy as np
import torch

from ..core import config
from ..core.optim import OptimizerMixin
from .complex_probe import POLAR_ALIASES, POLAR_SYMBOLS, electron_wavelength_angstrom, real_space_probe
from .ptycho_utils import center_probe, orthogonalize_probes, probe_tv_loss


def _standardise_aberrations(params: dict, max_order: int | None = 5) -> dict:
    """probe_models.py:171-221: polar coefficients, 'defocus' -> C10 = -defocus,
    aliases resolved, every symbol up to ``max_order`` present (zero if absent)."""
    out = {}

    def walk(p):
        for sym, val in list(p.items()):
            if isinstance(val, dict):
                walk(val)
            elif val is None:
                continue
            elif sym in POLAR_SYMBOLS:
                out[sym] = float(val)
            elif sym == "defocus":
                out["C10"] = -float(val)
            elif sym in POLAR_ALIASES:
                out[POLAR_ALIASES[sym]] = float(val)

    walk(deepcopy(params))
    if max_order is not None:
        for sym in POLAR_SYMBOLS:
            if sym.startswith(("C", "phi")) and int(sym[-2]) <= max_order and sym not in out:
                out[sym] = 0.0
    return out


class ProbePixelated(OptimizerMixin):
    DEFAULT_PROBE_PARAMS = {"energy": None, "defocus": None, "semiangle_cutoff": None, "soft_edges": True,
                            "aberration_coefs": {}}
    DEFAULT_LRS = {"probe": 1e-3}
    DEFAULT_CONSTRAINTS = {"orthogonalize_probe": True, "center_probe": False, "tv_weight": 0.0}
    _token = object()

    def __init__(self, num_probes=1, probe_params=None, probe_tilt=(0, 0), learn_probe_tilt=False, roi_shape=None,
                 dtype=torch.complex64, device="cpu", rng=None, initial_probe_weights=None,
                 vacuum_probe_intensity=None, _from_params=False, _token=None):
        if _token is not self._token:
            raise RuntimeError("Use a factory method to instantiate this class.")
        OptimizerMixin.__init__(self)
        self.num_probes = int(num_probes)
        self._device = config.validate_device(device)[0]
        self._probe_params = dict(self.DEFAULT_PROBE_PARAMS)
        self.probe_params = dict(probe_params or {})
        self._probe_tilt = torch.as_tensor(probe_tilt, dtype=torch.float32).detach().clone().reshape(2)
        self._initial_probe_tilt = self._probe_tilt.clone()
        self.learn_probe_tilt = bool(learn_probe_tilt)
        self._roi_shape = None if roi_shape is None else np.asarray(roi_shape, dtype=int)
        self.rng = rng
        self.initial_probe_weights = initial_probe_weights
        self._from_params = _from_params
        if vacuum_probe_intensity is not None:
            raise NotImplementedError("vacuum probe intensities are not part of the B200 path")
        self.vacuum_probe_intensity = None
        self._constraints = dict(self.DEFAULT_CONSTRAINTS)
        self._initial_probe = None
        self._probe = None

    @classmethod
    def from_params(cls, probe_params: dict, num_probes: int = 1, roi_shape=None, probe_tilt=(0, 0),
                    learn_probe_tilt=False, dtype=torch.complex64, device="cpu", rng=None,
                    initial_probe_weights=None, vacuum_probe_intensity=None):
        return cls(num_probes, deepcopy(probe_params), probe_tilt, learn_probe_tilt, roi_shape, dtype, device, rng,
                   initial_probe_weights, vacuum_probe_intensity, _from_params=True, _token=cls._token)

    @classmethod
    def from_array(cls, probe_array, num_probes=None, probe_params=None, probe_tilt=(0, 0), learn_probe_tilt=False,
                   dtype=torch.complex64, device="cpu", rng=None, initial_probe_weights=None):
        arr = torch.as_tensor(probe_array).to(torch.complex64)
        if arr.ndim == 3:
            if num_probes is None:
                num_probes = arr.shape[0]
            elif num_probes != arr.shape[0]:
                raise ValueError(f"num_probes {num_probes} must match probe_array shape {arr.shape[0]}")
        else:
            num_probes = 1 if num_probes is None else num_probes
            arr = torch.cat([arr[None]] * num_probes, dim=0)
        m = cls(num_probes, dict(probe_params or {}), probe_tilt, learn_probe_tilt,
                (int(arr.shape[-2]), int(arr.shape[-1])), dtype, device, rng, initial_probe_weights,
                _from_params=False, _token=cls._token)
        m._initial_probe = arr
        m._probe = arr.clone().to(m._device).requires_grad_(True)
        return m

    # ------------------------------------------------------------ properties
    @property
    def probe_params(self) -> dict:
        return self._probe_params

    @probe_params.setter
    def probe_params(self, params: dict):
        params = dict(params)
        params["aberration_coefs"] = _standardise_aberrations(params)
        self._probe_params = {**self.DEFAULT_PROBE_PARAMS, **self._probe_params, **params}

    @property
    def roi_shape(self) -> np.ndarray:
        return self._roi_shape

    @property
    def device(self):
        return self._device

    @property
    def dtype(self):
        return torch.complex64

    @property
    def rng(self):
        return self._rng

    @rng.setter
    def rng(self, rng):
        if rng is None:
            self._rng_seed = None
            rng = np.random.default_rng()
        elif isinstance(rng, (int, float)):
            self._rng_seed = int(rng)
            rng = np.random.default_rng(rng)
        else:
            self._rng_seed = None
        self._rng = rng

    @property
    def initial_probe_weights(self) -> torch.Tensor:
        return self._initial_probe_weights

    @initial_probe_weights.setter
    def initial_probe_weights(self, w):
        """probe_models.py:685-696."""
        if w is None:
            self._initial_probe_weights = torch.tensor([1 - 0.02 * (self.num_probes - 1)] + [0.02] * (self.num_probes - 1))
        else:
            if len(w) != self.num_probes:
                raise ValueError(f"initial_probe_weights must be a list of length {self.num_probes}")
            w2 = torch.as_tensor(np.asarray(w), dtype=torch.float32)
            self._initial_probe_weights = w2 / torch.sum(w2)

    @property
    def constraints(self) -> dict:
        return self._constraints

    @constraints.setter
    def constraints(self, c: dict):
        self._constraints = dict(self.DEFAULT_CONSTRAINTS)
        for k, v in (c or {}).items():
            self.add_constraint(k, v)

    def add_constraint(self, key, value):
        if key not in self.DEFAULT_CONSTRAINTS:
            raise KeyError(f"Unknown probe constraint {key!r}")
        self._constraints[key] = value

    @property
    def probe_tilt(self) -> torch.Tensor:
        """Probe tilt [mrad] (row, column) of the propagators (probe_models.py:118-131,
        418-425); a parameter of the probe optimiser with ``learn_probe_tilt``."""
        return self._probe_tilt

    @probe_tilt.setter
    def probe_tilt(self, tilt):
        t = torch.as_tensor(tilt.detach().cpu() if isinstance(tilt, torch.Tensor) else tilt,
                            dtype=torch.float32).reshape(2)
        if self.has_optimizer() and isinstance(getattr(self, "_probe_tilt", None), torch.Tensor):
            with torch.no_grad():
                self._probe_tilt.data = t.to(self._probe_tilt.device)
        else:
            self._probe_tilt = t.to(self._device)

    @property
    def params(self):
        """The tilt (when learned) and the probe modes (probe_models.py:299-304, 699-703)."""
        if self.learn_probe_tilt:
            t = self._probe_tilt
            if not (t.is_leaf and t.requires_grad and t.device == torch.device(self._device)):
                self._probe_tilt = t.detach().to(self._device).contiguous().requires_grad_(True)
            return [self._probe_tilt, self._probe]
        return [self._probe]

    @property
    def initial_probe(self):
        return self._initial_probe

    def get_optimization_parameters(self):
        return self.params

    def remove_optimizer(self):
        super().remove_optimizer()
        self._probe_tilt = self._probe_tilt.detach()

    # ------------------------------------------------------------ set-up
    def set_initial_probe(self, roi_shape, reciprocal_sampling, mean_diffraction_intensity, device=None):
        """probe_models.py:722-759."""
        if device is not None:
            self._device = config.validate_device(device)[0]
        if self._roi_shape is None:
            self._roi_shape = np.asarray(roi_shape, dtype=int)
        elif not np.array_equal(self._roi_shape, np.asarray(roi_shape)):
            raise ValueError(f"roi_shape {roi_shape} conflicts with initialized roi_shape {self._roi_shape}.")
        self.reciprocal_sampling = np.asarray(reciprocal_sampling, dtype=np.float32)
        if mean_diffraction_intensity <= 0:
            raise ValueError("mean_diffraction_intensity must be > 0")
        self.mean_diffraction_intensity = float(mean_diffraction_intensity)
        if self._from_params:
            p = self.probe_params
            for k in ("energy", "semiangle_cutoff"):
                if p.get(k) is None:
                    raise ValueError(f"Missing probe parameter '{k}' in probe_params")
            gpts = tuple(int(x) for x in self._roi_shape)
            sampling = tuple(1 / (self._roi_shape * self.reciprocal_sampling).astype(np.float64))
            probes = real_space_probe(gpts, sampling, p["energy"], p["semiangle_cutoff"],
                                      soft_edges=p.get("soft_edges", True),
                                      aberration_coefs=p["aberration_coefs"]).to(torch.complex64)
        else:
            probes = self._initial_probe.clone().cpu()
        if probes.ndim != 3:
            probes = probes[None]
        if probes.shape[0] != self.num_probes:
            probes = torch.cat([probes] * self.num_probes, dim=0)
        probes = self._apply_random_phase_shifts(probes)
        probes = self._apply_weights(probes)
        self._initial_probe = probes
        self._probe = probes.clone().to(self._device).requires_grad_(True)

    def _apply_random_phase_shifts(self, probes: torch.Tensor) -> torch.Tensor:
        """probe_models.py:846-858 (same generator call order)."""
        probes = probes.clone()
        for a0 in range(1, self.num_probes):
            sy = torch.exp(-2j * torch.pi * (self.rng.random() - 0.5) * torch.fft.fftfreq(int(self._roi_shape[0])))
            sx = torch.exp(-2j * torch.pi * (self.rng.random() - 0.5) * torch.fft.fftfreq(int(self._roi_shape[1])))
            probes[a0] = probes[a0] * sy[:, None] * sx[None]
        return probes

    def _apply_weights(self, probes: torch.Tensor) -> torch.Tensor:
        """probe_models.py:860-873."""
        probe_intensity = torch.sum(torch.abs(torch.fft.fft2(probes, norm="ortho")).square())
        probes = probes * torch.sqrt(self.mean_diffraction_intensity / probe_intensity)
        cw = torch.sum(torch.abs(probes).square(), dim=(1, 2))
        cw = cw / torch.sum(cw)
        return probes * torch.sqrt(self.initial_probe_weights / cw)[:, None, None]

    def reset(self):
        self._probe = self._initial_probe.clone().to(self._device).requires_grad_(True)
        self._probe_tilt = self._initial_probe_tilt.clone().to(self._device)
        if self._optimizer is not None:
            self.set_optimizer(self._optimizer_params)

    def to(self, device):
        dev, _ = config.validate_device(device)
        self._device = dev
        if self._probe is not None and self._probe.device != torch.device(dev):
            self._probe = self._probe.detach().to(dev).requires_grad_(True)
            self._probe_tilt = self._probe_tilt.detach().to(dev)
            if self._optimizer is not None:
                self.set_optimizer(self._optimizer_params)
        else:
            self._probe_tilt = self._probe_tilt.to(dev)
        return self

    def prop_geometry(self, sampling, slice_thicknesses):
        """(n, sampling, energy, slice thicknesses) from which the batch kernels build the
        separable propagators of a learned tilt (ops.batch_loss)."""
        return (int(self._roi_shape[0]), tuple(float(x) for x in sampling), self.probe_params["energy"],
                tuple(float(x) for x in np.atleast_1d(np.asarray(slice_thicknesses, dtype=float))))

    def reset_iter_constraint_losses(self):
        pass

    @property
    def name(self) -> str:
        return "ProbePixelated"

    @property
    def shape(self) -> np.ndarray:
        return np.array((self.num_probes, *(int(x) for x in self._roi_shape)))

    def check_probe_params(self) -> None:
        """Report missing probe parameters; a missing defocus is taken from -C10
        (probe_models.py:342-350)."""
        pp = self._probe_params
        for k in self.DEFAULT_PROBE_PARAMS:
            if pp.get(k) is None:
                c10 = (pp.get("aberration_coefs") or {}).get("C10", 0)
                if k == "defocus" and c10:
                    pp[k] = -1 * c10
                    continue
                print(f"Missing probe parameter '{k}' in probe_params")

    def apply_hard_constraints(self, probe: torch.Tensor) -> torch.Tensor:
        """The probe's hard constraints on any (P, n, n) stack (probe_models.py:452-458):
        Gram-Schmidt + sort, then the centre-of-mass shift, as enabled; differentiable."""
        if self._constraints.get("orthogonalize_probe", True):
            probe = orthogonalize_probes(probe)
        if self._constraints.get("center_probe", False):
            probe = center_probe(probe)
        return probe

    @property
    def has_soft_constraints(self) -> bool:
        return bool(self._constraints.get("tv_weight", 0))

    def apply_soft_constraints(self, probe):
        """The probe TV soft loss on the hard-constrained probe (probe_models.py:441-450,
        ptychography.py:134), zero when ``tv_weight`` is 0."""
        w = float(self._constraints.get("tv_weight", 0) or 0)
        if not w:
            return torch.zeros((), device=self._probe.device)
        return probe_tv_loss(probe, w)

    # ------------------------------------------------------------ compute
    @property
    def probe(self) -> torch.Tensor:
        """Probe modes after the hard constraints in the reference's order (probe_models.py:
        452-458): Gram-Schmidt + sort if enabled, then the centre-of-mass shift if enabled."""
        return self.apply_hard_constraints(self._probe)

    def _compute_propagator_arrays(self, sampling, num_slices, slice_thicknesses) -> torch.Tensor:
        """(S-1, H, W) complex64 propagators evaluated like probe_models.py:376-427."""
        if num_slices == 1:
            return torch.tensor([])
        kr, kc = (torch.fft.fftfreq(int(n), float(d)) for n, d in zip(self._roi_shape, sampling))
        k2 = (kr[:, None] ** 2 + kc[None] ** 2).to(torch.complex64)
        energy = self.probe_params["energy"]
        if energy is None:
            raise ValueError("probe_model energy must be set to compute propagators.")
        lam = electron_wavelength_angstrom(energy)
        dz = torch.as_tensor(np.asarray(slice_thicknesses), dtype=k2.dtype)
        props = torch.exp((-1.0j * torch.pi * lam * dz[:, None, None]) * k2)
        tr, tc = (float(x) for x in self.probe_tilt.detach())
        if tr != 0:
            props = props * torch.exp(1.0j * (-2 * math.pi * dz[:, None, None] * math.tan(tr / 1e3)) * kr[None, :, None])
        if tc != 0:
            props = props * torch.exp(1.0j * (-2 * math.pi * dz[:, None, None] * math.tan(tc / 1e3)) * kc[None, None, :])
        return props

    def separable_propagators(self, sampling, slice_thicknesses, device):
        """Per-axis factors of the same propagators for the batch kernels."""
        from .. import ops

        return ops.separable_propagators(int(self._roi_shape[0]), sampling, self.probe_params["energy"],
                                         np.asarray(slice_thicknesses, dtype=float),
                                         tuple(float(x) for x in self.probe_tilt.detach()), device=device)

    def forward(self, fract_positions: torch.Tensor) -> torch.Tensor:
        """(P, B, H, W) sub-pixel shifted probes (ptycho_utils.py:128-176)."""
        from .. import ops

        probe = self.probe.contiguous()
        nr, nc = probe.shape[-2:]
        kr = torch.fft.fftfreq(nr, device=probe.device)
        kc = torch.fft.fftfreq(nc, device=probe.device)
        r = fract_positions[:, 0][:, None, None]
        c = fract_positions[:, 1][:, None, None]
        ramp = torch.exp(-2.0j * torch.pi * kr[None, :, None] * r) * torch.exp(-2.0j * torch.pi * kc[None, None, :] * c)
        ph = ops.fft2(probe.detach())
        shifted = ph[None] * ramp[:, None].to(torch.complex64)
        out = ops.fft2(shifted.contiguous(), inverse=True, scale=1.0 / (nr * nc))
        return out.swapaxes(0, 1)

    def backward(self, *args, **kwargs):
        raise NotImplementedError("analytic probe gradients: use autograd=True")
