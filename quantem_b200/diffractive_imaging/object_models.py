"""Pixelated multislice object model (quantem object_models.ObjectPixelated).

The parameter is the raw complex object (S, Ho, Wo); ``obj`` applies the
complex hard constraint (object_models.py:289-300) with the CUDA kernels.  The
per-batch patch gather happens inside the fused batch kernel; ``forward`` is kept
for callers that want explicit (S, B, H, W) patches.
"""
from __future__ import annotations

from typing import Literal, Sequence

import numpy as np
import torch

from ..core import config
from ..core.optim import OptimizerMixin


class ObjectPixelated(OptimizerMixin):
    DEFAULT_LRS = {"object": 5e-3, "tv_weight_z": 0, "tv_weight_xy": 0}
    DEFAULT_CONSTRAINTS = {
        "positivity": True, "fix_potential_baseline": False, "fix_potential_baseline_factor": 1.0,
        "identical_slices": False, "apply_fov_mask": False, "tv_weight_z": 0, "tv_weight_xy": 0,
        "surface_zero_weight": 0, "gaussian_sigma": None, "butterworth_order": 4, "q_lowpass": None,
        "q_highpass": None,
    }
    # constraints whose non-default values need operations outside the B200 path
    _UNSUPPORTED = ("identical_slices", "apply_fov_mask", "tv_weight_z", "tv_weight_xy", "surface_zero_weight",
                    "gaussian_sigma", "q_lowpass", "q_highpass")
    _token = object()

    def __init__(self, num_slices=1, slice_thicknesses=None, obj_type="complex", initialize_mode="uniform",
                 device="cpu", rng=None, _token=None):
        if _token is not self._token:
            raise RuntimeError("Use a factory method to instantiate this class.")
        OptimizerMixin.__init__(self)
        t = str(obj_type).lower()
        if t != "complex":
            raise NotImplementedError(f"obj_type {obj_type!r}: the B200 path implements complex objects")
        self._obj_type = "complex"
        self._device = config.validate_device(device)[0]
        self._initialize_mode = initialize_mode
        self._obj = torch.ones(num_slices, 1, 1, dtype=torch.complex64)
        self._initial_obj = None
        self.slice_thicknesses = slice_thicknesses
        self._constraints = dict(self.DEFAULT_CONSTRAINTS)
        self._sampling = None
        self.rng = rng
        self._mask = None

    # ------------------------------------------------------------ factories
    @classmethod
    def from_uniform(cls, num_slices: int = 1, slice_thicknesses=None, device="cpu",
                     obj_type: Literal["complex", "pure_phase", "potential"] = "complex", rng=None):
        return cls(num_slices, slice_thicknesses, obj_type, "uniform", device, rng, _token=cls._token)

    @classmethod
    def from_random(cls, num_slices: int = 1, slice_thicknesses=None, device="cpu", obj_type="complex", rng=None):
        return cls(num_slices, slice_thicknesses, obj_type, "random", device, rng, _token=cls._token)

    @classmethod
    def from_array(cls, initial_obj, slice_thicknesses=None, device="cpu", obj_type="complex", rng=None):
        arr = torch.as_tensor(initial_obj).to(torch.complex64)
        m = cls(arr.shape[0], slice_thicknesses, obj_type, "array", device, rng, _token=cls._token)
        m._initial_obj = arr
        return m

    # ------------------------------------------------------------ properties
    @property
    def obj_type(self) -> str:
        return self._obj_type

    @property
    def dtype(self):
        return torch.complex64

    @property
    def device(self):
        return self._device

    @property
    def num_slices(self) -> int:
        return int(self._obj.shape[0])

    @property
    def shape(self):
        return tuple(self._obj.shape)

    @property
    def params(self):
        return self._obj

    @property
    def initial_obj(self):
        return self._initial_obj

    @property
    def sampling(self):
        if self._sampling is None:
            raise ValueError("ObjectModel sampling not set, call _initialize_obj() first")
        return self._sampling

    @property
    def slice_thicknesses(self) -> torch.Tensor:
        return self._slice_thicknesses

    @slice_thicknesses.setter
    def slice_thicknesses(self, val):
        """object_models.py:150-183: a scalar is repeated for the S-1 gaps."""
        if val is None:
            th = []
        elif isinstance(val, (float, int)):
            th = [val]
        else:
            th = list(np.asarray(val, dtype=float).ravel())
        if len(th) == 0:
            if self.num_slices > 1:
                raise ValueError(f"num slices = {self.num_slices}, so slice_thicknesses cannot be None")
            t = torch.tensor([])
        elif len(th) == 1:
            if float(th[0]) <= 0:
                raise ValueError("slice_thicknesses must be > 0")
            t = float(th[0]) * torch.ones(self.num_slices - 1)
        else:
            if len(th) != self.num_slices - 1:
                raise ValueError(f"slice_thicknesses must have {self.num_slices - 1} entries")
            t = torch.tensor(th)
        self._slice_thicknesses = t.to(getattr(torch, config.get("dtype_real")))

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
            raise KeyError(f"Unknown object constraint {key!r}")
        if key in self._UNSUPPORTED and value not in (None, False, 0) and value != self.DEFAULT_CONSTRAINTS[key]:
            raise NotImplementedError(f"object constraint {key}={value!r} is not part of the B200 path")
        self._constraints[key] = value

    @property
    def mask(self):
        return self._mask

    @mask.setter
    def mask(self, m):
        self._mask = None if m is None else torch.as_tensor(m)

    # ------------------------------------------------------------ state
    def _initialize_obj(self, shape, sampling=None):
        if sampling is not None:
            self._sampling = (float(sampling[0]), float(sampling[1]))
        shape = tuple(int(x) for x in shape)
        if self._obj.numel() > self.num_slices and tuple(self._obj.shape) == shape:
            return
        if self._initialize_mode == "uniform":
            arr = torch.ones(shape, dtype=torch.complex64)
        elif self._initialize_mode == "random":
            g = torch.Generator().manual_seed(int(self._rng_seed % 2**32) if self._rng_seed is not None else 0)
            ph = (torch.randn(shape, dtype=torch.float32, generator=g) - 0.5) * 1e-6
            arr = torch.exp(1.0j * ph).to(torch.complex64)
        elif self._initialize_mode == "array":
            arr = self._initial_obj
            if tuple(arr.shape) != shape:
                raise ValueError(f"initial object shape {tuple(arr.shape)} != reconstruction shape {shape}")
        else:
            raise ValueError(f"Invalid initialize mode: {self._initialize_mode}")
        self._initial_obj = arr.to(torch.complex64)
        self.reset()

    def reset(self):
        self._obj = self._initial_obj.clone().to(self._device).requires_grad_(True)
        if self._optimizer is not None:
            self.set_optimizer(self._optimizer_params)

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

    def get_optimization_parameters(self):
        return [self._obj]

    def to(self, device):
        dev, _ = config.validate_device(device)
        self._device = dev
        if self._obj.device != torch.device(dev):
            self._obj = self._obj.detach().to(dev).requires_grad_(True)
            if self._optimizer is not None:
                self.set_optimizer(self._optimizer_params)
        return self

    def reset_iter_constraint_losses(self):
        pass

    def apply_soft_constraints(self, obj, mask=None):
        return torch.zeros((), device=self._obj.device)

    # ------------------------------------------------------------ compute
    @property
    def obj(self) -> torch.Tensor:
        """Hard-constrained object (differentiable, CUDA kernels)."""
        from .. import ops

        return ops.constrained_object(self._obj)

    def forward(self, patch_indices: torch.Tensor) -> torch.Tensor:
        """(S, B, H, W) object patches at the given flat indices (object_models.py:252-265)."""
        o = self.obj.reshape(self.num_slices, -1)
        return torch.complex(o.real[:, patch_indices], o.imag[:, patch_indices])

    def backward(self, *args, **kwargs):
        raise NotImplementedError("analytic object gradients: use autograd=True")
