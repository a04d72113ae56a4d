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
    # every optional constraint of the reference is built for pixelated objects
    _UNSUPPORTED = ()
    _token = object()

    def __init__(self, num_slices=1, slice_thicknesses=None, obj_type="complex", initialize_mode="uniform",
                 device="cpu", rng=None, _token=None):
        if _token is not self._token:
            raise RuntimeError("Use a factory method to instantiate this class.")
        OptimizerMixin.__init__(self)
        self._obj_type = self._process_obj_type(obj_type)
        self._device = config.validate_device(device)[0]
        self._initialize_mode = initialize_mode
        self._obj = torch.ones(num_slices, 1, 1, dtype=self.dtype)
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
        arr = torch.as_tensor(initial_obj)
        m = cls(arr.shape[0], slice_thicknesses, obj_type, "array", device, rng, _token=cls._token)
        if m.obj_type == "potential" and arr.is_complex():
            raise TypeError("a potential object is real: pass a real initial_obj")
        m._initial_obj = arr.to(m.dtype)
        return m

    @staticmethod
    def _process_obj_type(obj_type) -> str:
        """object_models.py:123-136 (same spellings accepted)."""
        t = str(obj_type).lower()
        if t in ("potential", "potentials"):
            return "potential"
        if t in ("pure_phase", "purephase", "pure phase"):
            return "pure_phase"
        if t == "complex":
            return "complex"
        raise ValueError(f"Object type should be 'potential', 'complex', or 'pure_phase', got {obj_type}")

    # ------------------------------------------------------------ properties
    @property
    def obj_type(self) -> str:
        return self._obj_type

    @obj_type.setter
    def obj_type(self, t) -> None:
        """object_models.py:105-107 (the parameter keeps its dtype until re-initialised)."""
        self._obj_type = self._process_obj_type(t)

    @property
    def dtype(self):
        """float32 for potentials, complex64 otherwise (object_models.py:85-89)."""
        return torch.float32 if self._obj_type == "potential" else torch.complex64

    def _ext_constraints(self) -> bool:
        """Whether the optional hard constraints are active (FOV mask, Gaussian blur, identical
        slices, a potential baseline taken from the FOV mask's background)."""
        c = self._constraints
        return bool((c.get("apply_fov_mask") and self._mask is not None) or c.get("gaussian_sigma") is not None
                    or c.get("q_lowpass") or c.get("q_highpass")
                    or (c.get("identical_slices") and self.num_slices > 1)
                    or (self.obj_type == "potential" and c.get("fix_potential_baseline")))

    @property
    def has_soft_constraints(self) -> bool:
        c = self._constraints
        return bool(c.get("tv_weight_z", 0) or c.get("tv_weight_xy", 0) or c.get("surface_zero_weight", 0))

    @property
    def name(self) -> str:
        return "ObjPixelized"

    @property
    def shape_2d(self) -> tuple[int, int]:
        return tuple(self.shape[1:])

    def apply_hard_constraints(self, obj: torch.Tensor, mask=None) -> torch.Tensor:
        """The hard constraints of this model (object_models.py:289-339) on any object array of
        its type (S, Ho, Wo), differentiable, on the constraint kernels; the FOV mask applies
        only when given, as in the reference."""
        from .. import ops

        m = None
        if mask is not None:
            m = torch.as_tensor(mask.detach() if isinstance(mask, torch.Tensor) else np.asarray(mask),
                                dtype=torch.float32)
            m = (m[0] if m.ndim == 3 else m).to(obj.device).contiguous()
        c = self._constraints
        if ((c.get("apply_fov_mask") and m is not None) or c.get("gaussian_sigma") is not None
                or c.get("q_lowpass") or c.get("q_highpass") or (c.get("identical_slices") and obj.shape[0] > 1)
                or (self.obj_type == "potential" and c.get("fix_potential_baseline"))):
            return ops.constrained_object_ext(obj, self.obj_type, c, m, self._sampling)
        if self.obj_type == "complex":
            return ops.constrained_object(obj)
        if self.obj_type == "pure_phase":
            return ops.object_transmission(obj, self.transmission_spec())
        return torch.clamp(obj, min=0.0) if c.get("positivity", True) else obj

    def get_tv_loss(self, array: torch.Tensor, weights=None) -> torch.Tensor:
        """TV soft loss (object_models.py:360-411): weights (z, xy) from the constraints by
        default, a scalar for both, or a pair; the z term is dropped for one slice."""
        from .. import ops

        if weights is None:
            w = (self._constraints.get("tv_weight_z", 0), self._constraints.get("tv_weight_xy", 0))
        elif isinstance(weights, (int, float)):
            w = (weights, weights)
        else:
            if len(weights) != 2:
                raise ValueError(f"weights must be a tuple of length 2, got {weights}")
            w = tuple(weights)
        if not any(w):
            return torch.zeros((), device=array.device)
        return ops.soft_constraint_loss(array, self.obj_type, w[0], w[1], 0.0)

    def get_surface_zero_loss(self, array: torch.Tensor, weight: float = 0.0) -> torch.Tensor:
        """Surface-zero soft loss of the first and last slices (object_models.py:413-435)."""
        from .. import ops

        if weight == 0:
            return torch.zeros((), device=array.device)
        return ops.soft_constraint_loss(array, self.obj_type, 0.0, 0.0, weight)

    def gaussian_blur_2d(self, tensor: torch.Tensor, sigma: float = 1.0) -> torch.Tensor:
        """Zero-padded separable Gaussian blur along the last two axes of an (S, Ho, Wo) array
        (object_models.py:437-479), differentiable, on the blur kernel."""
        from .. import ops

        return ops._BlurFn.apply(tensor, ops.gaussian_taps(sigma, tensor.device))

    def butterworth_constraint(self, tensor: torch.Tensor, sampling) -> torch.Tensor:
        """The Butterworth low / high-pass filter of the constraints (object_models.py:481-520)
        on an (S, Ho, Wo) array, differentiable, on the line-DFT kernels."""
        from .. import ops

        c = self._constraints
        env = ops.butterworth_env(tensor.shape[-2:], sampling, c.get("q_lowpass"), c.get("q_highpass"),
                                  c.get("butterworth_order", 4), tensor.device)
        return ops._ButterworthFn.apply(tensor, env)

    def _mask_on_device(self):
        m = self._mask
        if m is None:
            return None
        if m.device != torch.device(self._obj.device) or m.dtype != torch.float32 or not m.is_contiguous():
            self._mask = m = m.to(self._obj.device, torch.float32).contiguous()
        return m

    def batch_object(self):
        """(tensor, ObjSpec) for the batch kernels: the raw object and its transmission spec,
        or, with the optional hard constraints active, the transmission itself (computed by
        the constraint kernels, differentiable) with an identity spec."""
        from .. import ops

        if self._ext_constraints():
            return self.transmission(), ops.ObjSpec("complex", hard_constraint=False)
        return self._obj, self.transmission_spec()

    def transmission_spec(self):
        """What the batch kernels need to turn the raw object into its transmission."""
        from .. import ops

        c = self._constraints
        return ops.ObjSpec(self._obj_type, positivity=bool(c.get("positivity", True)),
                           fix_baseline=bool(c.get("fix_potential_baseline", False)),
                           baseline_factor=float(c.get("fix_potential_baseline_factor", 1.0)))

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
        """The probe-overlap FOV mask (Ho, Wo) (the reference stores it expanded over the
        slices; a (S, Ho, Wo) mask is reduced to its first slice)."""
        if m is None:
            self._mask = None
            return
        t = torch.as_tensor(np.asarray(m) if not isinstance(m, torch.Tensor) else m.detach(), dtype=torch.float32)
        self._mask = (t[0] if t.ndim == 3 else t).contiguous()

    # ------------------------------------------------------------ state
    def _initialize_obj(self, shape, sampling=None):
        if sampling is not None:
            self._sampling = (float(sampling[0]), float(sampling[1]))
        shape = tuple(int(x) for x in shape)
        if self._obj.numel() > self.num_slices and tuple(self._obj.shape) == shape:
            return
        potential = self._obj_type == "potential"
        if self._initialize_mode == "uniform":  # object_models.py:660-664
            arr = torch.zeros(shape, dtype=torch.float32) if potential else torch.ones(shape, dtype=torch.complex64)
        elif self._initialize_mode == "random":
            g = torch.Generator().manual_seed(int(self._rng_seed % 2**32) if self._rng_seed is not None else 0)
            ph = (torch.randn(shape, dtype=torch.float32, generator=g) - 0.5) * 1e-6
            arr = ph if potential else torch.exp(1.0j * ph).to(torch.complex64)
        elif self._initialize_mode == "array":
            arr = self._initial_obj
            if tuple(arr.shape) != shape:
                raise ValueError(f"initial object shape {tuple(arr.shape)} != reconstruction shape {shape}")
        else:
            raise ValueError(f"Invalid initialize mode: {self._initialize_mode}")
        self._initial_obj = arr.to(self.dtype)
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
        """Soft constraints of the hard-constrained object (object_models.py:341-358): TV
        along z and in-plane and the surface-zero terms, by the constraint kernels."""
        from .. import ops

        if not self.has_soft_constraints:
            return torch.zeros((), device=self._obj.device)
        c = self._constraints
        return ops.soft_constraint_loss(obj, self.obj_type, c.get("tv_weight_z", 0), c.get("tv_weight_xy", 0),
                                        c.get("surface_zero_weight", 0))

    # ------------------------------------------------------------ compute
    @property
    def obj(self) -> torch.Tensor:
        """Hard-constrained object (object_models.py:289-339; differentiable): the complex
        or pure-phase object from the CUDA constraint kernels, or the real potential
        V - offset clamped at 0."""
        from .. import ops

        if self._ext_constraints():
            return ops.constrained_object_ext(self._obj, self._obj_type, self._constraints, self._mask_on_device(),
                                              self._sampling)
        if self._obj_type == "complex":
            return ops.constrained_object(self._obj)
        if self._obj_type == "pure_phase":
            return ops.object_transmission(self._obj, self.transmission_spec())
        spec = self.transmission_spec()
        v = self._obj
        if spec.fix_baseline:
            v = v - v.min().detach() * spec.baseline_factor
        return torch.clamp(v, min=0.0) if spec.positivity else v

    def transmission(self) -> torch.Tensor:
        """exp(i V') for potentials, the constrained object otherwise (complex64,
        differentiable, CUDA kernels): what multiplies the wave in every slice."""
        from .. import ops

        if self._ext_constraints():
            return ops.transmission_of(self.obj)
        return ops.object_transmission(self._obj, self.transmission_spec())

    def forward(self, patch_indices: torch.Tensor) -> torch.Tensor:
        """(S, B, H, W) object patches at the given flat indices (object_models.py:252-265)."""
        o = self.transmission().reshape(self.num_slices, -1)
        return torch.complex(o.real[:, patch_indices], o.imag[:, patch_indices])

    def backward(self, *args, **kwargs):
        raise NotImplementedError("analytic object gradients: use autograd=True")


class ObjectDIP(ObjectPixelated):
    """Deep-image-prior object (object_models.py:728-1226): the object is the output
    of a CNN, obj = exp(i * model(model_input (+ noise))[0]) for pure-phase objects,
    and the network weights are what the optimiser updates.

    The network is ``quantem_b200.core.ml.cnn.CNN2d`` (real-valued, BF16 tcgen05
    kernels).  With a real network (pure-phase or potential objects) its output
    (1, S, H, W) is the phase / potential of every slice and the transmission is
    exp(i output); with a complex network (``ComplexCNN2d``, complex objects, the
    reference's default) the output is the complex object itself.  As in the
    reference's ObjectDIP.forward (object_models.py:990-1008) the network output enters
    the patches without the hard constraint (for a real network exp(i phase) goes through
    the complex constraint kernel, which at unit amplitude only removes the mean phase:
    a global phase that changes neither the loss nor its gradient); ``obj`` applies the
    hard constraint of the object type.  Gradients flow from the fused adjoint into the
    CNN backward kernels by torch autograd; the pixelated-object gradient rescale
    (ptychography.py:330-332) is not applied, as in the reference."""

    # the optional constraints act on ``obj`` (and through it on the soft terms), as in the
    # reference, whose DIP forward feeds the masked network output to the patches
    _UNSUPPORTED = ()

    def __init__(self, num_slices=1, slice_thicknesses=None, input_noise_std=0.025, device="cuda",
                 obj_type="complex", rng=None, _token=None):
        t = ObjectPixelated._process_obj_type(obj_type)
        ObjectPixelated.__init__(self, num_slices, slice_thicknesses, "complex", "dip", device, rng,
                                 _token=ObjectPixelated._token)
        self._obj_type_dip = t
        self._model = None
        self._model_input = torch.tensor([])
        self._pretrain_target = torch.tensor([])
        self._pretrain_losses = []
        self._pretrain_lrs = []
        self._pretrained_weights = None
        if input_noise_std < 0:
            raise ValueError("input_noise_std must be >= 0")
        self._input_noise_std = float(input_noise_std)
        self._gen = None

    @classmethod
    def from_model(cls, model, model_input, num_slices: int = 1, slice_thicknesses=None,
                   input_noise_std: float = 0.025, device="cuda", obj_type="complex", rng=None):
        """object_models.py:768-794."""
        m = cls(num_slices, slice_thicknesses, input_noise_std, device, obj_type, rng)
        m._model = model
        if m.is_complex_model and m._obj_type_dip != "complex":
            raise ValueError("a complex network (ComplexCNN2d) describes a complex object")
        m.model_input = model_input
        m._set_pretrained_weights()
        return m

    @classmethod
    def from_pixelated(cls, model, pixelated: ObjectPixelated, input_noise_std: float = 0.025, device=None):
        """object_models.py:796-834: input and pre-training target = the pixelated object
        with a complex network; with a real network its potential (potential objects) or
        its phase (pure-phase objects, and complex objects, whose transmission then is
        exp(i output): the reference casts a complex object to the real network's dtype
        here, keeping only its real part, which this path does not reproduce)."""
        if not isinstance(pixelated, ObjectPixelated):
            raise ValueError(f"pixelated must be an ObjectPixelated, got {type(pixelated)}")
        complex_model = "complex" in str(getattr(model, "dtype", ""))
        obj = pixelated.obj.detach()
        if complex_model:
            if pixelated.obj_type != "complex":
                raise ValueError("a complex network (ComplexCNN2d) describes a complex object")
            target = obj.clone()
        elif pixelated.obj_type == "potential":
            target = obj.float().clone()
        else:
            target = torch.angle(obj).float()
        m = cls.from_model(model, target, num_slices=pixelated.num_slices,
                           slice_thicknesses=pixelated.slice_thicknesses.cpu().numpy() if
                           pixelated.slice_thicknesses.numel() else None,
                           input_noise_std=input_noise_std, device=device or pixelated.device,
                           obj_type=pixelated.obj_type, rng=pixelated._rng_seed)
        m.pretrain_target = target
        return m

    @property
    def is_complex_model(self) -> bool:
        return "complex" in str(getattr(self._model, "dtype", ""))

    def transmission_spec(self):
        """Complex network: the output is the transmission (no hard constraint, as the
        reference's DIP forward); real network: exp(i output) through the complex kernel."""
        from .. import ops

        return ops.ObjSpec("complex", hard_constraint=not self.is_complex_model)

    # ------------------------------------------------------------------ state
    @property
    def name(self) -> str:
        return "ObjectDIP"

    @property
    def obj_type(self) -> str:
        return self._obj_type_dip

    @property
    def model(self):
        return self._model

    @property
    def pretrained_weights(self):
        return self._pretrained_weights

    def _set_pretrained_weights(self):
        self._pretrained_weights = {k: v.clone() for k, v in self._model.state_dict().items()}

    @property
    def model_input(self) -> torch.Tensor:
        return self._model_input

    @model_input.setter
    def model_input(self, x):
        x = torch.as_tensor(x).detach().clone()
        x = x.to(torch.complex64) if self.is_complex_model else x.float()
        if x.shape[-3] != self.num_slices:
            raise ValueError(f"model_input.shape[-3] {x.shape[-3]} does not match num_slices {self.num_slices}")
        if x.ndim == 3:
            x = x[None]
        elif x.ndim != 4:
            raise ValueError(f"model_input must be (num_slices, h, w), got shape {tuple(x.shape)}")
        self._model_input = x.to(self._model.device).contiguous()

    @property
    def num_slices(self) -> int:
        return int(self._num_slices_dip) if hasattr(self, "_num_slices_dip") else int(self._obj.shape[0])

    @property
    def pretrain_target(self) -> torch.Tensor:
        return self._pretrain_target

    @pretrain_target.setter
    def pretrain_target(self, t):
        if t is None:
            self._pretrain_target = torch.tensor([])
            return
        t = torch.as_tensor(t)
        t = t.to(torch.complex64) if self.is_complex_model else t.float()
        if t.ndim == 4:
            t = t[0]
        if tuple(t.shape) != tuple(self.model_input.shape[-3:]):
            raise ValueError(f"pretrain target {tuple(t.shape)} != model input {tuple(self.model_input.shape[-3:])}")
        self._pretrain_target = t.to(self._model.device).contiguous()

    @property
    def pretrain_losses(self) -> np.ndarray:
        return np.array(self._pretrain_losses)

    @property
    def pretrain_lrs(self) -> np.ndarray:
        return np.array(self._pretrain_lrs)

    @property
    def shape(self):
        return tuple(int(v) for v in self._model_input.shape[1:])

    @property
    def params(self):
        return self._model.flat

    def get_optimization_parameters(self):
        return [self._model.flat]

    def _noisy_input(self, noise: bool):
        if not noise or self._input_noise_std <= 0.0:
            return self._model_input
        if self._gen is None:
            self._gen = torch.Generator(device=self._model_input.device).manual_seed(
                int(self._rng_seed) if self._rng_seed is not None else 0)
        # torch.randn of a complex dtype: real and imaginary parts each N(0, 1/2)
        return self._model_input + torch.randn(self._model_input.shape, generator=self._gen,
                                               device=self._model_input.device,
                                               dtype=self._model_input.dtype) * self._input_noise_std

    def raw_object(self, noise: bool = True, masked: bool = False) -> torch.Tensor:
        """The network's object as complex64 (S, H, W), differentiable: its output for a
        complex network, exp(i output) for a real one.  ``masked``: the output times the
        probe-overlap FOV mask first, as the reference's DIP forward does whenever the mask
        is set (object_models.py:1005-1007; Ptychography.preprocess sets it)."""
        out = self._model(self._noisy_input(noise))[0]
        if masked and self._mask is not None:
            m = self._mask
            if m.device != out.device:
                self._mask = m = m.to(out.device).contiguous()
            out = out * m
        if self.is_complex_model:
            return out.contiguous()
        return torch.polar(torch.ones_like(out), out)

    @property
    def _obj(self) -> torch.Tensor:
        """What the batch kernels take: the (noisy-input) network output, FOV-masked."""
        return self.raw_object(noise=True, masked=True)

    @_obj.setter
    def _obj(self, v):  # the base constructor stores a placeholder; the network defines the object
        self._num_slices_dip = int(v.shape[0])

    def batch_object(self):
        """The masked network output and its spec: the reference's DIP forward applies no
        hard constraint, optional or not (object_models.py:990-1008)."""
        return self._obj, self.transmission_spec()

    def transmission(self) -> torch.Tensor:
        from .. import ops

        return ops.object_transmission(self._obj, self.transmission_spec())

    @property
    def obj(self) -> torch.Tensor:
        """The network's object with the hard constraint of its type (object_models.py:975-983),
        the optional constraints included."""
        from .. import ops

        if self._ext_constraints():
            x = (self._model(self._noisy_input(False))[0] if self._obj_type_dip == "potential"
                 else self.raw_object(noise=False))
            m = self._mask
            if m is not None and m.device != x.device:
                self._mask = m = m.to(x.device).contiguous()
            return ops.constrained_object_ext(x, self._obj_type_dip, self._constraints, m, self._sampling)
        if self._obj_type_dip == "potential":
            v = self._model(self._noisy_input(False))[0]
            return torch.clamp(v, min=0.0) if self._constraints.get("positivity", True) else v
        return ops.constrained_object(self.raw_object(noise=False))

    def _initialize_obj(self, shape, sampling=None):
        if sampling is not None:
            self._sampling = (float(sampling[0]), float(sampling[1]))
        if tuple(int(s) for s in shape) != tuple(self._model_input.shape[1:]):
            raise ValueError(f"shape {tuple(shape)} does not match model_input {tuple(self._model_input.shape)}")

    def reset(self):
        """Back to the pre-trained weights (object_models.py:1032-1034)."""
        self._model.load_state_dict(self._pretrained_weights)
        if self._optimizer is not None:
            self.set_optimizer(self._optimizer_params)

    def to(self, device):
        dev, _ = config.validate_device(device)

        def norm(d):
            d = torch.device(d)
            return torch.device("cuda", torch.cuda.current_device()) if d.type == "cuda" and d.index is None else d

        if norm(dev) != norm(self._model.device):
            raise NotImplementedError("the CNN2d lives on the device it was built on")
        self._device = dev
        return self

    def forward(self, patch_indices: torch.Tensor) -> torch.Tensor:
        o = self._obj.reshape(self.num_slices, -1)
        return torch.complex(o.real[:, patch_indices], o.imag[:, patch_indices])

    # ------------------------------------------------------------------ pre-training
    def pretrain(self, model_input=None, pretrain_target=None, reset: bool = False, num_iters: int = 100,
                 optimizer_params: dict | None = None, scheduler_params: dict | None = None, loss_fn="l2",
                 apply_constraints: bool = False, show: bool = False, device=None):
        """Fit the network output to the target phase (object_models.py:1047-1154)."""
        from ..core.ml.cnn import mse_loss

        if str(loss_fn).lower() not in ("l2", "mse"):
            raise NotImplementedError("pre-training loss: l2")
        if apply_constraints:
            raise NotImplementedError("pre-training with the hard constraint applied is not part of the B200 path")
        if optimizer_params is not None:
            self.set_optimizer(optimizer_params)
        if self._optimizer is None:
            self.set_optimizer({"type": "adam", "lr": 1e-3})
        if scheduler_params is not None:
            self.set_scheduler(scheduler_params, num_iters)
        if reset:
            self._model._init_params(0)
            self._pretrain_losses, self._pretrain_lrs = [], []
        if model_input is not None:
            self.model_input = model_input
        if pretrain_target is not None:
            self.pretrain_target = pretrain_target
        if self._pretrain_target.numel() == 0:
            raise ValueError("No pretrain target set. Provide pretrain_target or set it beforehand.")
        self._model.train()
        opt = self._optimizer
        tgt = torch.view_as_real(self._pretrain_target) if self.is_complex_model else self._pretrain_target
        for _ in range(num_iters):
            out = self._model(self._noisy_input(True))[0]
            if self.is_complex_model:  # complex_l2: mean over the real and the imaginary parts
                out = torch.view_as_real(out)
            loss = mse_loss(out, tgt)
            opt.zero_grad(set_to_none=True)
            loss.backward()
            opt.step()
            if self._scheduler is not None:
                self.step_scheduler(float(loss.item()))
            self._pretrain_losses.append(float(loss.item()))
            self._pretrain_lrs.append(opt.param_groups[0]["lr"])
        self._set_pretrained_weights()
        return self
