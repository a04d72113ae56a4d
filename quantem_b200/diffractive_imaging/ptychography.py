"""Ptychography engine: drop-in for quantem.diffractive_imaging.Ptychography.

Same construction and call sequence as the reference (ptychography.py:36-58,
ptychography_base.py:135-189, ptychography.py:146-308): ``from_models`` ->
``preprocess`` -> ``reconstruct``.  Each batch runs one fused forward + loss +
adjoint CUDA launch (quantem_b200.ops) followed by the fused optimiser kernels;
the batch loss stays on the device and is read back once per iteration, or once per
call when nothing consumes it during the run (the reference reads it twice per batch).
"""
from __future__ import annotations

from typing import Literal

import numpy as np
import scipy.ndimage as ndi
import torch
from tqdm.auto import tqdm

from ..core import config
from .. import ops
from .dataset_models import PtychographyDatasetRaster
from .detector_models import DetectorPixelated
from .object_models import ObjectPixelated
from .probe_models import ProbePixelated
from .ptycho_utils import SimpleBatcher, device_batches


def adjust_padding_power2(pad, shape, power2_level):
    """Pad so that (shape + 2 pad) is divisible by 2**power2_level (ptychography_base.py:1002-1016)."""
    div = 2**power2_level
    pad = np.array(pad, dtype=np.int64)
    r0 = (shape[-2] + 2 * pad[-2]) % div
    r1 = (shape[-1] + 2 * pad[-1]) % div
    if r0:
        pad[-2] += (div - r0) // 2
    if r1:
        pad[-1] += (div - r1) // 2
    if (shape[-2] + 2 * pad[-2]) % div or (shape[-1] + 2 * pad[-1]) % div:
        raise ValueError(f"Adjustment failed to achieve divisibility by {div}")
    return pad


class Ptychography:
    """Multislice mixed-probe gradient-descent ptychography on B200."""

    _token = object()
    OPTIMIZABLE_VALS = ["object", "probe", "dataset"]
    DEFAULT_OPTIMIZER_TYPE = "adam"

    def __init__(self, dset, obj_model, probe_model, detector_model, logger=None, device="cpu", verbose=True,
                 rng=None, _token=None):
        if _token is not self._token:
            raise RuntimeError("Use Ptychography.from_models() to instantiate this class.")
        if not isinstance(dset, PtychographyDatasetRaster):
            raise TypeError(f"dset should be a PtychographyDatasetRaster, got {type(dset)}")
        if not isinstance(obj_model, ObjectPixelated):
            raise TypeError(f"obj_model must be ObjectPixelated, got {type(obj_model)}")
        if not isinstance(probe_model, ProbePixelated):
            raise TypeError(f"probe_model must be ProbePixelated, got {type(probe_model)}")
        if not isinstance(detector_model, DetectorPixelated):
            raise TypeError(f"detector_model must be DetectorPixelated, got {type(detector_model)}")
        self.verbose = verbose
        self.dset = dset
        self._device = config.validate_device(device)[0]
        self.rng = rng
        self._preprocessed = False
        self._obj_padding_force_power2_level = 3
        self._store_snapshots = False
        self._store_snapshot_every = 1
        self._iter_losses: list[float] = []
        self._iter_val_losses: list[float] = []
        self._iter_lrs: dict[str, list] = {}
        self._snapshots: list[dict] = []
        self._obj_padding_px = np.array([0, 0])
        self.batch_size = dset.num_gpts
        self._val_ratio = 0.0
        self._val_mode = "grid"
        self._probe_model = probe_model
        if dset.preprocessed:
            probe_model.set_initial_probe(self.roi_shape, self.reciprocal_sampling, dset.mean_diffraction_intensity,
                                          device=self._device)
        self._obj_model = obj_model
        self.detector_model = detector_model
        self.logger = logger
        self._propagators = torch.tensor([])
        self._prop_factors = None
        self.loss_readback: Literal["auto", "iteration"] = "auto"
        self.to(self._device)

    @classmethod
    def from_models(cls, dset, obj_model, probe_model, detector_model, logger=None, device="cpu", verbose=True,
                    rng=None):
        return cls(dset, obj_model, probe_model, detector_model, logger, device, verbose, rng, _token=cls._token)

    # ------------------------------------------------------------ basic state
    @property
    def rng(self) -> np.random.Generator:
        return self._rng

    @rng.setter
    def rng(self, rng):
        if rng is None:
            self._rng_seed = None
            rng = np.random.default_rng()
        elif isinstance(rng, (int, float)):
            self._rng_seed = int(rng)
            rng = np.random.default_rng(rng)
        elif isinstance(rng, np.random.Generator):
            self._rng_seed = None
        else:
            raise TypeError(f"rng should be a np.random.Generator or a seed, got {type(rng)}")
        self._rng = rng

    def _reset_rng(self):
        if self._rng_seed is not None:
            self.rng = self._rng_seed

    @property
    def device(self) -> str:
        return self._device

    @property
    def obj_model(self) -> ObjectPixelated:
        return self._obj_model

    @property
    def probe_model(self) -> ProbePixelated:
        return self._probe_model

    @property
    def roi_shape(self) -> np.ndarray:
        return self.dset.roi_shape

    @property
    def gpts(self) -> np.ndarray:
        return self.dset.gpts

    @property
    def reciprocal_sampling(self) -> np.ndarray:
        return self.dset.reciprocal_sampling

    @property
    def sampling(self) -> np.ndarray:
        return self.dset.obj_sampling

    @property
    def num_slices(self) -> int:
        return self.obj_model.num_slices

    @property
    def num_probes(self) -> int:
        return self.probe_model.num_probes

    @property
    def slice_thicknesses(self) -> np.ndarray:
        t = self.obj_model.slice_thicknesses
        return np.array([]) if t is None else t.cpu().numpy()

    @property
    def obj_padding_px(self) -> np.ndarray:
        return self._obj_padding_px

    @obj_padding_px.setter
    def obj_padding_px(self, pad):
        p2 = np.asarray(pad, dtype=np.int64).reshape(2)
        if self._obj_padding_force_power2_level > 0:
            p2 = adjust_padding_power2(p2, self.dset._obj_shape_full_2d((0, 0)), self._obj_padding_force_power2_level)
        self._obj_padding_px = p2
        self.obj_model._initialize_obj(shape=self.obj_shape_full, sampling=self.sampling)
        self.obj_model.to(self._device)
        self.dset._set_initial_scan_positions_px(self._obj_padding_px)
        self.dset._set_patch_indices(self._obj_padding_px)

    @property
    def obj_shape_full(self) -> np.ndarray:
        return np.concatenate([[self.num_slices], self.dset._obj_shape_full_2d(self.obj_padding_px)])

    @property
    def obj_shape_crop(self) -> np.ndarray:
        shp = np.floor(self.dset.fov / self.sampling)
        shp += shp % 2
        return np.concatenate([[self.num_slices], shp]).astype("int")

    @property
    def batch_size(self) -> int:
        return self._batch_size

    @batch_size.setter
    def batch_size(self, val):
        if val is not None:
            if int(val) <= 0:
                raise ValueError("batch_size must be > 0")
            self._batch_size = int(val)

    @property
    def val_ratio(self) -> float:
        return float(self._val_ratio)

    @val_ratio.setter
    def val_ratio(self, r):
        r = float(r)
        if r < 0.0 or r > 1.0:
            raise ValueError("val_ratio must satisfy 0 <= val_ratio <= 1")
        self._val_ratio = r

    @property
    def val_mode(self):
        return self._val_mode

    @val_mode.setter
    def val_mode(self, mode):
        if mode not in ("grid", "random"):
            raise ValueError(f"val_mode must be either 'grid' or 'random', got {mode}")
        self._val_mode = mode

    @property
    def iter_losses(self) -> np.ndarray:
        return np.array(self._iter_losses)

    @property
    def val_iter_losses(self) -> np.ndarray:
        return np.array(self._iter_val_losses)

    @property
    def num_iters(self) -> int:
        return len(self._iter_losses)

    @property
    def iter_lrs(self) -> dict:
        return {k: np.array(v) for k, v in self._iter_lrs.items()}

    @property
    def snapshots(self):
        return self._snapshots

    @property
    def propagators(self) -> torch.Tensor:
        return torch.tensor([]) if self.num_slices == 1 else self._propagators

    def to(self, device):
        dev, _ = config.validate_device(device)
        self._device = dev
        self.obj_model.to(dev)
        self.probe_model.to(dev)
        self.dset.to(dev)
        if isinstance(self._propagators, torch.Tensor):
            self._propagators = self._propagators.to(dev)
        if self._prop_factors is not None:
            self._prop_factors = tuple(t.to(dev) for t in self._prop_factors)
        return self

    def vprint(self, m, level=1):
        if self.verbose >= level:
            print(m)

    def _check_preprocessed(self):
        if not self._preprocessed:
            raise AttributeError("Preprocessing has not been completed. Please run Ptycho.preprocess()")

    # ------------------------------------------------------------ set-up
    def preprocess(self, obj_padding_px=(0, 0), val_ratio=0.0, val_mode="grid", vectorized=True, batch_size=None,
                   com_fit_function="constant", force_com_rotation=None, force_com_transpose=None,
                   padded_diffraction_intensities_shape=None, plot_rotation=True, plot_com=True,
                   plot_probe_overlap=False):
        """ptychography_base.py:135-189 (no plots)."""
        if not self.dset.preprocessed:
            self.vprint("Dataset was not preprocessed, proceeding with defaults.")
            self.dset.preprocess(com_fit_function=com_fit_function, force_com_rotation=force_com_rotation,
                                 force_com_transpose=force_com_transpose,
                                 padded_diffraction_intensities_shape=padded_diffraction_intensities_shape,
                                 obj_padding_px=obj_padding_px, device=self.device)
            self.probe_model.set_initial_probe(self.roi_shape, self.reciprocal_sampling,
                                               self.dset.mean_diffraction_intensity, device=self.device)
        self.obj_padding_px = obj_padding_px
        self.dset._set_initial_scan_positions_px(self.obj_padding_px)
        self.dset._set_patch_indices(self.obj_padding_px)
        self.compute_propagator_arrays()
        self._set_obj_fov_mask()
        self._preprocessed = True
        self.val_ratio = float(val_ratio)
        self.val_mode = val_mode
        return self

    def _get_probe_overlap(self) -> np.ndarray:
        """Sum over positions of |probe mode 0|^2 at each patch window (ptychography_base.py:
        201-216): the overlap kernel on CUDA devices, a host sum during a host set-up."""
        with torch.no_grad():
            inten = self.probe_model.probe[0].detach().abs().square().to(torch.float32).contiguous()
        pos = self.dset.scan_positions_px.detach().to(torch.float32).contiguous()
        shape = tuple(int(x) for x in self.obj_shape_full[-2:])
        if inten.device.type == "cuda":
            return ops.probe_overlap(inten, pos.to(inten.device), shape).cpu().numpy()
        n = int(inten.shape[-1])
        fr = np.fft.fftfreq(n, d=1.0 / n).astype(np.int64)
        org = np.round(pos.numpy().astype(np.float64)).astype(np.int64)
        rows = (org[:, 0][:, None] + fr[None]) % shape[0]
        cols = (org[:, 1][:, None] + fr[None]) % shape[1]
        out = np.zeros(shape, dtype=np.float32)
        a = inten.numpy()
        for b in range(org.shape[0]):
            np.add.at(out, (rows[b][:, None], cols[b][None, :]), a)
        return out

    def _set_obj_fov_mask(self, gaussian_sigma: float = 2.0):
        """The probe-overlap FOV mask (ptychography_base.py:191-199): overlap > 0.3 max,
        binary closing (5 iterations), binary dilation (min(32, min padding // 4)
        iterations), Gaussian filter; used by ``apply_fov_mask`` and by a fixed potential
        baseline."""
        overlap = self._get_probe_overlap()
        ov = overlap > overlap.max() * 0.3
        ov = ndi.binary_closing(ov, iterations=5)
        ov = ndi.binary_dilation(ov, iterations=min(32, int(np.min(self.obj_padding_px)) // 4))
        ov = ndi.gaussian_filter(ov.astype(np.float32), sigma=gaussian_sigma)
        self.obj_fov_mask = ov
        self.obj_model.mask = ov

    def compute_propagator_arrays(self):
        """Propagators like the reference (complex64, probe_models.py:376-427) plus
        their per-axis factors for the batch kernels."""
        if self.num_slices == 1:
            self._propagators = torch.tensor([])
            self._prop_factors = None
            return
        self._propagators = self.probe_model._compute_propagator_arrays(
            self.sampling, self.num_slices, self.slice_thicknesses).to(self._device)
        if torch.device(self._device).type == "cuda":
            self._prop_factors = self.probe_model.separable_propagators(self.sampling, self.slice_thicknesses,
                                                                        self._device)
        else:
            self._prop_factors = None

    # ------------------------------------------------------------ optimisers
    def _get_default_lr(self, key):
        if key == "object":
            return self.obj_model.DEFAULT_LRS.get("object", 5e-3)
        if key == "probe":
            return self.probe_model.DEFAULT_LRS.get("probe", 1e-3)
        if key == "dataset":
            return 1e-3
        raise ValueError(f"Unknown optimization key: {key}")

    @property
    def optimizer_params(self) -> dict:
        return {k: p for k, p in (("object", self.obj_model.optimizer_params),
                                  ("probe", self.probe_model.optimizer_params),
                                  ("dataset", self.dset.optimizer_params)) if p}

    @optimizer_params.setter
    def optimizer_params(self, d):
        """ptychography_opt.py:183-228."""
        if isinstance(d, (tuple, list)):
            d = {k: {} for k in d}
        for k, v in d.items():
            v = dict(v)
            v.setdefault("type", self.DEFAULT_OPTIMIZER_TYPE)
            v.setdefault("lr", self._get_default_lr(k))
            if k == "object":
                self.obj_model.optimizer_params = v
            elif k == "probe":
                self.probe_model.optimizer_params = v
            elif k == "dataset":
                self.dset.optimizer_params = v
            else:
                raise ValueError(f"key to be optimized, {k}, not in allowed keys: {self.OPTIMIZABLE_VALS}")

    @property
    def optimizers(self) -> dict:
        out = {}
        if self.obj_model.has_optimizer():
            out["object"] = self.obj_model.optimizer
        if self.probe_model.has_optimizer():
            out["probe"] = self.probe_model.optimizer
        if self.dset.has_optimizer():
            out["dataset"] = self.dset.optimizer
        return out

    def set_optimizers(self):
        models = {"object": self.obj_model, "probe": self.probe_model, "dataset": self.dset}
        for key, params in self.optimizer_params.items():
            models[key].set_optimizer(params)

    @property
    def scheduler_params(self) -> dict:
        return {"object": self.obj_model.scheduler_params, "probe": self.probe_model.scheduler_params,
                "dataset": self.dset.scheduler_params}

    @scheduler_params.setter
    def scheduler_params(self, d):
        for k in self.OPTIMIZABLE_VALS:
            d.setdefault(k, {})
        for k, v in d.items():
            if k == "object":
                self.obj_model.scheduler_params = v
            elif k == "probe":
                self.probe_model.scheduler_params = v
            elif k == "dataset":
                self.dset.scheduler_params = v
            else:
                raise ValueError(f"key to be optimized, {k}, not in allowed keys: {self.OPTIMIZABLE_VALS}")

    def set_schedulers(self, params, num_iter=None):
        for key, sp in params.items():
            if key == "object":
                self.obj_model.set_scheduler(sp, num_iter)
            elif key == "probe":
                self.probe_model.set_scheduler(sp, num_iter)
            elif key == "dataset":
                self.dset.set_scheduler(sp, num_iter)

    def step_schedulers(self, loss=None):
        self.obj_model.step_scheduler(loss)
        self.probe_model.step_scheduler(loss)
        self.dset.step_scheduler(loss)

    @property
    def constraints(self) -> dict:
        return {"object": self.obj_model.constraints, "probe": self.probe_model.constraints,
                "dataset": self.dset.constraints, "detector": {"detector_mask": None}}

    @constraints.setter
    def constraints(self, c: dict):
        handlers = {"object": self.obj_model, "probe": self.probe_model, "dataset": self.dset}
        for key, value in c.items():
            if key in handlers and isinstance(value, dict):
                for sk, sv in value.items():
                    handlers[key].add_constraint(sk, sv)
            elif key == "detector" and isinstance(value, dict):
                pass
            else:
                raise KeyError(f"Invalid constraint category '{key}'. Valid categories are: "
                               f"{list(handlers) + ['detector']}")

    def reset_recon(self):
        """ptychography_base.py:834-848 and ptychography.py:96-100."""
        self._reset_rng()
        self.obj_model.reset()
        self.probe_model.reset()
        self.dset.reset()
        self.compute_propagator_arrays()
        self.obj_model.constraints = self.obj_model.DEFAULT_CONSTRAINTS
        self._iter_losses, self._iter_val_losses, self._iter_lrs, self._snapshots = [], [], {}, []
        self.obj_model.reset_optimizer()
        self.probe_model.reset_optimizer()
        self.dset.reset_optimizer()

    # ------------------------------------------------------------ reference API surface
    @property
    def autograd(self) -> bool:
        """ptychography.py:84-90 (``reconstruct(autograd=...)`` selects the update)."""
        return getattr(self, "_autograd", True)

    @autograd.setter
    def autograd(self, autograd: bool) -> None:
        self._autograd = bool(autograd)

    @property
    def iter_recon_types(self) -> np.ndarray:
        """ptychography_base.py:403-408 (the reference records none)."""
        return np.array(getattr(self, "_iter_recon_types", []))

    @property
    def reciprocal_units(self) -> list[str]:
        return ["A^-1", "A^-1"]

    @property
    def angular_sampling(self) -> np.ndarray:
        """Detector sampling in mrad (ptychography_base.py:672-694)."""
        from .complex_probe import electron_wavelength_angstrom

        sampling = np.asarray(self.dset.detector_sampling, dtype=float)
        units = self.dset.detector_units
        if units[0] == "mrad":
            return sampling
        if units[0] == "A^-1":
            energy = self.probe_model.probe_params.get("energy")
            if energy is None:
                raise ValueError("dc units given in A^-1 but no energy defined to convert to mrad")
            return sampling * electron_wavelength_angstrom(energy) * 1e3
        if units[0] == "pixels":
            raise ValueError("dset Q units given in pixels, needs calibration")
        raise NotImplementedError(f"Unknown dset Q units: {units}")

    @property
    def angular_units(self) -> list[str]:
        return ["mrad", "mrad"]

    @property
    def store_snapshots(self) -> bool:
        return self._store_snapshots

    @store_snapshots.setter
    def store_snapshots(self, val) -> None:
        if val is not None:
            self._store_snapshots = bool(val)

    @property
    def store_snapshot_every(self) -> int:
        return self._store_snapshot_every

    @store_snapshot_every.setter
    def store_snapshot_every(self, val) -> None:
        if val is not None:
            self._store_snapshot_every = int(val)

    def get_snapshot_by_iter(self, iteration: int, closest: bool = False, cropped: bool = False) -> dict:
        """ptychography_base.py:444-493: the snapshot at ``iteration`` (or the closest one), its
        object optionally cropped to the field of view with the mean phase removed."""
        if len(self._snapshots) == 0:
            raise ValueError("No snapshots available. Use store_snapshots=True during reconstruction.")
        iteration = int(iteration)
        if closest:
            snp = min(self._snapshots, key=lambda x: abs(x["iteration"] - iteration))
        else:
            for snp in self._snapshots:
                if snp["iteration"] == iteration:
                    break
            else:
                raise ValueError(f"No snapshot found at iteration: {iteration}, "
                                 "to return the closest snapshot, set closest=True")
        if cropped:
            snp = dict(snp)
            c = self._crop_rotate_obj_fov(snp["obj"])
            if self.obj_type == "pure_phase":
                ph = np.angle(c)
                c = np.exp(1j * (ph - ph.mean()))
            if self.obj_type in ("pure_phase", "complex"):
                ph = np.angle(c)
                c = np.abs(c) * np.exp(1j * (ph - ph.mean()))
            snp["obj"] = c
        return snp

    @property
    def obj_type(self) -> str:
        return self.obj_model.obj_type

    def set_obj_type(self, t, force: bool = False) -> None:
        """ptychography_base.py:249-255: only before training unless forced."""
        new = ObjectPixelated._process_obj_type(t)
        if self.num_iters > 0 and new != self.obj_model.obj_type and not force:
            raise ValueError("Cannot change object type after training. Run with reset=True or rerun preprocess.")
        self.obj_model.obj_type = new

    def get_probe_intensities(self, probe=None) -> np.ndarray:
        """Relative intensities of the probe modes (ptychography_base.py:864-877)."""
        if probe is None:
            probe = self.probe
        probe = probe.detach().cpu().numpy() if isinstance(probe, torch.Tensor) else np.asarray(probe)
        if probe.ndim == 2:
            return np.array([1.0])
        inten = np.abs(probe) ** 2
        return inten.sum(axis=(-2, -1)) / inten.sum()

    def estimate_intensities(self, overlap_array: torch.Tensor) -> torch.Tensor:
        """sum over modes of |orthonormal fft2(exit waves)|^2, corner-centred
        (ptychography_base.py:963-968); exit waves (P, B, n, n) complex64 on the GPU, n one of the
        built window sizes."""
        return self._ortho_fft2(overlap_array.detach()).abs().square().sum(0)

    def estimate_amplitudes(self, overlap_array: torch.Tensor, corner_centered: bool = False) -> torch.Tensor:
        """sqrt of the mode sum of |orthonormal fft2(exit waves) + 1e-9|^2, fftshifted unless
        ``corner_centered`` (ptychography_base.py:949-961)."""
        far = self._ortho_fft2(overlap_array.detach())
        amps = torch.sqrt((far + 1e-9).abs().square().sum(0))
        return amps if corner_centered else torch.fft.fftshift(amps, dim=(-2, -1))

    @property
    def obj_fov_mask(self) -> np.ndarray:
        """The probe-overlap FOV mask (1, Ho, Wo) that preprocess builds (ptychography_base.py:
        346-359); the object model keeps it as (Ho, Wo)."""
        m = self.obj_model.mask
        if m is None:
            raise AttributeError("obj_fov_mask is set by preprocess()")
        return m.detach().cpu().numpy()[None]

    @obj_fov_mask.setter
    def obj_fov_mask(self, mask) -> None:
        m = np.asarray(mask.detach().cpu() if isinstance(mask, torch.Tensor) else mask, dtype=np.float32)
        if m.ndim == 2:
            m = m[None]
        if m.ndim != 3:
            raise ValueError(f"obj_fov_mask must be 2-D or 3-D, got {m.ndim} dimensions")
        self.obj_model.mask = m

    def _ortho_fft2(self, x: torch.Tensor, inverse: bool = False) -> torch.Tensor:
        """Orthonormal (i)fft2 of a (..., n, n) complex stack on the library's FFT kernels."""
        x = ops.dense(x.to(torch.complex64))
        n = int(x.shape[-1])
        return ops.fft2(x.reshape(-1, n, n), inverse=inverse, scale=1.0 / n).reshape(x.shape)

    def overlap_projection(self, obj_patches: torch.Tensor, input_probe: torch.Tensor):
        """The multislice forward of gathered patches (ptychography_base.py:934-947): the wave
        entering each slice (S, P, B, n, n) and the exit wave (P, B, n, n), propagating with
        ifft2(fft2(wave) prop_s) on the library's FFT kernels.  The reconstruction gathers the
        patches and runs this chain inside the batch kernel; this is the analysis form."""
        obj_patches = ops.dense(obj_patches.detach().to(torch.complex64))
        probe = ops.dense(input_probe.detach().to(torch.complex64))
        n = int(probe.shape[-1])
        S = int(obj_patches.shape[0])
        props = self.propagators
        waves = [probe]
        overlap = obj_patches[0] * probe
        for s in range(1, S):
            f = ops.fft2(ops.dense(overlap).reshape(-1, n, n)).reshape(overlap.shape)
            wave = ops.fft2(ops.dense(f * props[s - 1].to(f.device)).reshape(-1, n, n), inverse=True,
                            scale=1.0 / (n * n)).reshape(overlap.shape)
            waves.append(wave)
            overlap = obj_patches[s] * wave
        return torch.stack(waves, dim=0), overlap

    def fourier_projection(self, measured_amplitudes: torch.Tensor, overlap_array: torch.Tensor) -> torch.Tensor:
        """Exit waves with their far-field amplitude replaced by the measured one (detector
        layout in, ptychography.py:356-372): one mode keeps the far-field phase; several modes
        scale every mode by measured / estimated amplitude (0 where the estimate is 0)."""
        meas = torch.fft.fftshift(measured_amplitudes.to(torch.float32), dim=(-2, -1))
        far = self._ortho_fft2(overlap_array)
        if self.num_probes == 1:
            mod = meas * torch.exp(1j * torch.angle(far))
        else:
            est = self.estimate_amplitudes(overlap_array, corner_centered=True)
            est = torch.where(est == 0, torch.full_like(est, float("inf")), est)
            mod = (meas / est)[None] * far
        return self._ortho_fft2(mod, inverse=True)

    def gradient_step(self, amplitudes: torch.Tensor, overlap: torch.Tensor) -> torch.Tensor:
        """The analytic update direction of the exit waves, fourier_projection - overlap
        (ptychography.py:350-354); ``reconstruct(autograd=False)`` computes it in-kernel."""
        return self.fourier_projection(amplitudes, overlap) - overlap.to(torch.complex64)

    def error_estimate(self, pred_intensities: torch.Tensor, batch_indices, loss_type="l2_amplitude"):
        """The consistency loss of predicted (detector-layout) intensities against the batch's
        targets and those targets (ptychography_base.py:908-932): an analysis helper; the
        reconstruction computes the same loss inside the fused batch kernel."""
        dev = pred_intensities.device
        bi = torch.as_tensor(np.asarray(batch_indices, dtype=np.int64), device=self.dset.targets.device)
        targets = self.dset.targets[bi].to(dev)
        mask = self.dset.detector_mask.to(dev)
        preds = torch.sqrt(pred_intensities + 1e-9) if "amplitude" in loss_type else pred_intensities
        diff = preds * mask - targets * mask
        if "l1" in loss_type:
            error = torch.sum(torch.abs(diff)) / (diff.shape[0] / self.dset.num_gpts)
        elif "l2" in loss_type:
            error = torch.sum(torch.abs(diff) ** 2) / (diff.shape[0] / self.dset.num_gpts)
        elif loss_type == "poisson":
            error = torch.sum(preds - targets * torch.log(preds + 1e-6))
        else:
            raise ValueError(f"Unknown loss type {loss_type}, should be 'l1' or 'l2'")
        return error / self.dset.mean_diffraction_intensity, targets

    def backward(self, loss: torch.Tensor, autograd: bool = True, *args):
        """ptychography.py:317-348 for a loss from ``ops.batch_loss``: autograd, then the
        pixelated-object gradient rescale; the analytic update runs inside ``reconstruct``."""
        if not autograd:
            raise NotImplementedError("the analytic update is fused into reconstruct(autograd=False)")
        loss.backward()
        leaf = self.obj_model._obj
        if type(self.obj_model) is ObjectPixelated and leaf.grad is not None:
            leaf.grad.mul_(self.dset.upsample_factor ** 2 / 2)

    @property
    def schedulers(self) -> dict:
        out = {}
        for key, m in (("object", self.obj_model), ("probe", self.probe_model), ("dataset", self.dset)):
            if getattr(m, "scheduler", None) is not None:
                out[key] = m.scheduler
        return out

    def remove_optimizer(self, key: str) -> None:
        {"object": self.obj_model, "probe": self.probe_model, "dataset": self.dset}[key].remove_optimizer()

    def step_optimizers(self) -> None:
        for o in self.optimizers.values():
            o.step()

    def zero_grad_all(self) -> None:
        for o in self.optimizers.values():
            o.zero_grad(set_to_none=True)

    def clone(self, device="cpu"):
        """A deep copy of the reconstruction (ptychography.py:595-629), moved to ``device``."""
        import copy

        lg = self.logger
        self.logger = None  # loggers hold writers; the reference clones them separately
        try:
            cloned = copy.deepcopy(self)
        finally:
            self.logger = lg
        if lg is not None:
            cloned.logger = lg.clone() if hasattr(lg, "clone") else lg
        cloned.to(device)
        return cloned

    @classmethod
    def from_ptychography(cls, ptycho, obj_model=None, probe_model=None, logger=None):
        """ptychography.py:61-81: a reset clone of ``ptycho``, optionally with new models."""
        tmp = ptycho.logger
        ptycho.logger = None
        try:
            cloned = ptycho.clone(ptycho.device)
        finally:
            ptycho.logger = tmp
        if obj_model is not None:
            cloned._obj_model = obj_model
        if probe_model is not None:
            cloned._probe_model = probe_model
        if logger is not None:
            cloned.logger = logger
        cloned.reset_recon()
        return cloned

    # ------------------------------------------------------------ forward model API
    def _batch_tensors(self):
        dev = torch.device(self._device)
        if dev.type != "cuda":
            raise RuntimeError("the B200 ptychography path runs on CUDA devices only (use device='gpu')")
        prop = self._prop_factors if self._prop_factors is not None else self._propagators
        if self.num_slices == 1:
            n = int(self.roi_shape[0])
            prop = torch.zeros((0, n, n), dtype=torch.complex64, device=dev)
        elif self.probe_model.learn_probe_tilt:  # the propagators follow the current tilt
            prop = ops.separable_propagators_t(self._prop_geometry(), self.probe_model.probe_tilt.detach())
        return prop, self.dset.scan_positions_px.contiguous(), self.dset.targets, \
            self.dset.detector_mask.to(dev).contiguous()

    def _prop_geometry(self):
        return self.probe_model.prop_geometry(self.sampling, self.slice_thicknesses)

    def _batch_descan(self):
        d = self.dset.batch_descan()
        return None if d is None else d.detach().contiguous()

    def _device_targets(self, tg):
        """Targets on the device (a one-off copy when the dataset keeps them on the host)."""
        return tg if tg.device.type == "cuda" else tg.to(self._device, non_blocking=True)

    def forward_intensities(self, batch_indices, loss_type="l2_amplitude"):
        """Predicted detector intensities (B, H, W) and batch loss, no gradients."""
        prop, pos, tg, mask = self._batch_tensors()
        tg = self._device_targets(tg)
        bi = torch.as_tensor(np.asarray(batch_indices, dtype=np.int64), device=self._device)
        with torch.no_grad():
            obj_c = self.obj_model.transmission().detach().contiguous()
            probe_o = self.probe_model.probe.detach().contiguous()
        out = ops.batch_forward(obj_c, probe_o, prop, pos, bi, tg, mask, self.dset.num_gpts,
                                self.dset.mean_diffraction_intensity, loss_type, descan=self._batch_descan())
        return out["intensity"], out["loss"]

    def forward_operator(self, obj_patches=None, shifted_input_probes=None, descan=None, batch_indices=None):
        """(propagated probes (S,P,B,H,W), exit waves (P,B,H,W)) of a batch
        (ptychography_base.py:892-906), computed by the batch kernel."""
        if batch_indices is None:
            raise ValueError("forward_operator on the B200 path takes batch_indices (positions are gathered in-kernel)")
        prop, pos, tg, mask = self._batch_tensors()
        tg = self._device_targets(tg)
        bi = torch.as_tensor(np.asarray(batch_indices, dtype=np.int64), device=self._device)
        with torch.no_grad():
            out = ops.batch_forward(self.obj_model.transmission().detach().contiguous(),
                                    self.probe_model.probe.detach().contiguous(), prop, pos, bi, tg, mask,
                                    self.dset.num_gpts, self.dset.mean_diffraction_intensity,
                                    want_intensity=False, want_exit=True, want_waves=True,
                                    descan=self._batch_descan())
        return out["waves"], out["exit"]

    # ------------------------------------------------------------ reconstruction
    def reconstruct(self, num_iters: int = 0, reset: bool = False, optimizer_params: dict | None = None,
                    scheduler_params: dict | None = None, constraints: dict = {}, batch_size: int | None = None,
                    store_snapshots: bool | None = None, store_snapshots_every: int | None = None,
                    device: Literal["cpu", "gpu"] | None = None, autograd: bool = True,
                    loss_type: Literal["l2_amplitude", "l1_amplitude", "l2_intensity", "l1_intensity",
                                       "poisson"] = "l2_amplitude"):
        """Gradient-descent iterations (ptychography.py:146-308)."""
        self._check_preprocessed()
        if device is not None:
            self.to(device)
        self.batch_size = batch_size
        if store_snapshots_every is not None:
            self._store_snapshot_every = int(store_snapshots_every)
            if store_snapshots is None:
                store_snapshots = True
        if store_snapshots is not None:
            self._store_snapshots = bool(store_snapshots)
        if reset:
            self.reset_recon()
        self.constraints = constraints
        new_sched = reset
        if optimizer_params is not None:
            self.optimizer_params = optimizer_params
            self.set_optimizers()
            new_sched = True
        if scheduler_params is not None:
            self.scheduler_params = scheduler_params
            new_sched = True
        if new_sched:
            self.set_schedulers(self.scheduler_params, num_iter=num_iters)
        self.dset._set_targets(loss_type)
        self.compute_propagator_arrays()
        batcher = SimpleBatcher(self.dset.num_gpts, self.batch_size, rng=self.rng, val_ratio=self.val_ratio,
                                val_mode=self.val_mode)
        prop, _, tg, mask = self._batch_tensors()
        opts = [o for o in (self.obj_model.optimizer, self.probe_model.optimizer, self.dset.optimizer) if o is not None]
        dev = torch.device(self._device)
        # targets kept in host memory (dset.keep_targets_on_host): one double-buffered copy per iteration
        from ..engine import HostTargetStream  # engine imports this package's utilities

        stream = HostTargetStream(tg, dev) if tg.device.type != "cuda" and num_iters > 0 else None
        self.last_h2d_bytes_per_iter = stream.bytes_per_copy if stream is not None else 0
        nvtx = torch.cuda.nvtx  # profiler ranges (iteration, batch); no cost without a profiler
        # when nothing reads the loss during the run (no scheduler, logger, validation split,
        # snapshots or progress bar) and ``loss_readback`` is "auto", each iteration's loss stays
        # on the device and all are read once at the end, with the status word: the host queues
        # iteration after iteration without waiting.  "iteration" reads each when it ends.
        defer = (self.loss_readback == "auto" and self.logger is None and not batcher.has_validation
                 and not self._store_snapshots and not self.schedulers and not self.verbose)
        pending = []
        # progress bar with the loss when verbose (ptychography.py:206-300), on stderr
        pbar = tqdm(range(num_iters), disable=not self.verbose)
        for a0 in pbar:
            nvtx.range_push(f"reconstruct iteration {self.num_iters}")
            total = torch.zeros((), dtype=torch.float32, device=dev)
            nb = 0
            # the batch order goes up before the next targets copy takes the copy engine: that
            # copy waits for the order's upload (when the host runs iterations ahead, both would
            # otherwise become ready together and the order could queue behind the targets)
            batches = device_batches(batcher, dev)
            if stream is not None:
                tg = stream.acquire()
                if a0 + 1 < num_iters:
                    uploaded = torch.cuda.Event()
                    uploaded.record()
                    stream.prefetch_next(after=uploaded)
            consistency = torch.zeros((), dtype=torch.float32, device=dev)
            for idx in batches:
                nvtx.range_push("batch")
                for o in opts:
                    o.zero_grad(set_to_none=True)
                self.dset.apply_hard_constraints(self.obj_padding_px)
                pos = self.dset.scan_positions_px.contiguous()
                if autograd:
                    probe_o = self.probe_model.probe
                    leaf = self.obj_model._obj  # a leaf (pixelated) or a network output (DIP)
                    # the raw object and its transmission spec, or (optional / soft constraints)
                    # the hard-constrained object computed once, its transmission taken by the
                    # batch kernels with an identity spec and the object by the soft terms
                    soft_obj = None
                    if self.obj_model.has_soft_constraints and type(self.obj_model) is ObjectPixelated:
                        soft_obj = self.obj_model.obj
                        obj_raw, obj_spec = ops.transmission_of(soft_obj), ops.ObjSpec("complex", hard_constraint=False)
                    else:
                        obj_raw, obj_spec = self.obj_model.batch_object()
                    # learned descan shifts and probe tilt enter the kernels as differentiable inputs
                    descan = self.dset.batch_descan()
                    tilt = self.probe_model.probe_tilt
                    tilt = tilt if (tilt.requires_grad and self.num_slices > 1) else None
                    closs = ops.batch_loss(obj_raw, probe_o, prop, pos, idx, tg, mask,
                                           self.dset.num_gpts, self.dset.mean_diffraction_intensity, loss_type,
                                           obj_spec=obj_spec, descan=descan, tilt=tilt,
                                           prop_geometry=self._prop_geometry() if tilt is not None else None)
                    loss = closs
                    # soft constraints join the batch loss (ptychography.py:125-140, 229-231)
                    if self.obj_model.has_soft_constraints:
                        loss = loss + self.obj_model.apply_soft_constraints(
                            soft_obj if soft_obj is not None else self.obj_model.obj)
                    if self.probe_model.has_soft_constraints:
                        loss = loss + self.probe_model.apply_soft_constraints(probe_o)
                    if descan is not None and self.dset.constraints.get("descan_tv_weight", 0) > 0:
                        loss = loss + self.dset.apply_soft_constraints(descan)
                    if (obj_raw.requires_grad or self.probe_model._probe.requires_grad or pos.requires_grad
                            or (descan is not None and descan.requires_grad) or tilt is not None):
                        loss.backward()
                        if leaf.is_leaf and leaf.grad is not None:
                            # pixelated objects only (ptychography.py:330-332)
                            leaf.grad.mul_(self.dset.upsample_factor ** 2 / 2)
                else:
                    # analytic update directions (ptychography.py:339-348), no autograd graph
                    if type(self.obj_model).__name__ == "ObjectDIP":
                        raise NotImplementedError("the analytic update applies to pixelated objects (autograd=True)")
                    if self.dset.batch_descan() is not None:
                        raise NotImplementedError("learned descan shifts need autograd=True")
                    # the optional constraints act through the forward model only, as in the
                    # reference: the update directions are applied to the raw parameters, and
                    # the soft terms join the loss value but not the directions
                    with torch.no_grad():
                        probe_o = self.probe_model.probe.detach().contiguous()
                        obj_type = self.obj_model.obj_type
                        if obj_type == "complex" and not self.obj_model._ext_constraints():
                            obj_c, _ = ops.obj_constrain(self.obj_model._obj.detach().contiguous())
                        else:
                            obj_c = self.obj_model.transmission().detach().contiguous()
                        loss, g_obj, g_probe = ops.batch_analytic(
                            obj_c, probe_o, prop, pos, idx, tg, mask, self.dset.num_gpts,
                            self.dset.mean_diffraction_intensity, loss_type)
                        if obj_type == "potential":
                            # sum_patches Re(-i conj(o) conj(psi) g) (object_models.py:705-709) is
                            # Im(conj(o) sum_patches conj(psi) g): every patch covering a pixel
                            # carries that pixel's transmission o
                            g_obj = (obj_c.conj() * g_obj).imag.contiguous()
                        closs = loss
                        if self.obj_model.has_soft_constraints:
                            loss = loss + self.obj_model.apply_soft_constraints(self.obj_model.obj).detach()
                        if self.probe_model.has_soft_constraints:
                            loss = loss + self.probe_model.apply_soft_constraints(probe_o).detach()
                    self.obj_model._obj.grad = g_obj
                    self.probe_model._probe.grad = g_probe
                for o in opts:
                    o.step()
                total += loss.detach()
                consistency += closs.detach()
                nb += 1
                nvtx.range_pop()
            if stream is not None:
                stream.release()
            if defer:
                pending.append(total / max(nb, 1))
                nvtx.range_pop()
                continue
            total_loss = float((total / max(nb, 1)).item())
            # the logger receives the consistency loss alone (ptychography.py:284-292)
            consistency_loss = total_loss
            if self.logger is not None and (self.obj_model.has_soft_constraints or
                                            self.probe_model.has_soft_constraints or
                                            self.dset.constraints.get("descan_tv_weight", 0) > 0):
                consistency_loss = float((consistency / max(nb, 1)).item())
            ops.check_status(dev)  # out-of-range batch indices / non-finite intensities since the last check
            val_loss = None
            if batcher.has_validation:
                vl, vb = 0.0, 0
                for bi in batcher.iter_val():
                    _, l = self.forward_intensities(bi, loss_type)
                    vl += float(l.item())
                    vb += 1
                if vb:
                    val_loss = vl / vb
                    self._iter_val_losses.append(val_loss)
            self._record_iter(total_loss)
            self.step_schedulers(total_loss)
            if self._store_snapshots and (a0 % self._store_snapshot_every) == 0:
                self._snapshots.append(dict(iteration=self.num_iters, obj=self.obj, probe=self.probe))
            if self.logger is not None:
                self.logger.log_iter(self.obj_model, self.probe_model, self.dset, self.num_iters - 1,
                                     consistency_loss, nb, self._get_current_lrs())
            if self.verbose:
                text = f"Iter {a0 + 1}/{num_iters}, Loss: {total_loss:.3e}"
                pbar.set_description(text if val_loss is None else f"{text}, Val: {val_loss:.3e}")
            nvtx.range_pop()
        if pending:  # one read of every iteration's loss and of the status word
            losses = torch.stack(pending).cpu().tolist()
            ops.check_status(dev)
            for loss in losses:
                self._record_iter(float(loss))
        return self

    def _get_current_lrs(self):
        return {k: o.param_groups[0]["lr"] for k, o in self.optimizers.items()}

    def _record_iter(self, loss):
        self._iter_losses.append(loss)
        opts = self.optimizers
        for key in set(self._iter_lrs) | set(opts):
            if key in self._iter_lrs:
                self._iter_lrs[key].append(opts[key].param_groups[0]["lr"] if key in opts else 0.0)
            else:
                self._iter_lrs[key] = [0.0] * (self.num_iters - 1) + [opts[key].param_groups[0]["lr"]]

    # ------------------------------------------------------------ checkpoint / resume
    def state_dict(self, save_raw_data: bool = False, skip=()) -> dict:
        """The reconstruction's resumable state (quantem_b200.diffractive_imaging.checkpoint)."""
        from . import checkpoint

        return checkpoint.state_dict(self, save_raw_data=save_raw_data, skip=skip)

    def save(self, path, mode: Literal["w", "o"] = "w", store: Literal["auto", "zip", "dir"] = "auto", skip=(),
             compression_level: int | None = 4, save_raw_data: bool = False, verbose: int | bool = True):
        """Save the reconstruction (ptychography.py:376-480): object, probe, optimiser and
        scheduler states, generator state, histories and the dataset's preprocessing
        parameters and positions; the 4D-STEM array too with ``save_raw_data``.  One
        ``torch.save`` file (``store`` and ``compression_level`` are accepted for API
        compatibility; the reference's zarr store is not used).  ``mode`` "w" refuses to
        replace an existing file, "o" overwrites."""
        from pathlib import Path

        from . import checkpoint

        if self.verbose and verbose:
            print(f"Saving ptychography object to {Path(path).resolve()}")
        checkpoint.save(self, path, mode=mode, save_raw_data=save_raw_data, skip=skip)

    @classmethod
    def from_file(cls, path, dset=None, device=None, verbose=None, auto_reload_dataset: bool = True):
        """Load a reconstruction saved by ``save`` (ptychography.py:481-588).  Without
        ``dset`` the dataset is rebuilt from the stored raw data and preprocessed with the
        stored parameters; a given ``dset`` is used as is (preprocessed with the stored
        parameters if it is not yet).  Training continues exactly where it stopped."""
        from . import checkpoint

        if dset is None and not auto_reload_dataset:
            raise ValueError("this path needs a dataset: pass dset= or keep auto_reload_dataset=True")
        return checkpoint.load(cls, path, dset=dset, device=device, verbose=verbose)

    # ------------------------------------------------------------ results
    @property
    def obj(self) -> np.ndarray:
        """Constrained object with the mean phase removed (ptychography_base.py:312-318);
        the constrained real potential for potential objects."""
        with torch.no_grad():
            o = self.obj_model.obj.detach().cpu().numpy()
        if self.obj_model.obj_type == "potential":
            return o
        ph = np.angle(o)
        return np.abs(o) * np.exp(1j * (ph - ph.mean()))

    @property
    def probe(self) -> np.ndarray:
        with torch.no_grad():
            return self.probe_model.probe.detach().cpu().numpy()

    @property
    def obj_cropped(self) -> np.ndarray:
        c = self._crop_rotate_obj_fov(self.obj)
        if self.obj_model.obj_type == "potential":
            return c
        ph = np.angle(c)
        return np.abs(c) * np.exp(1j * (ph - ph.mean()))

    def _crop_rotate_obj_fov(self, array, positions_px=None, com_rotation_rad=None, transpose=None, padding=None):
        """ptychography_base.py:782-831."""
        array = np.asarray(array).copy()
        rot = self.dset.com_rotation_rad if com_rotation_rad is None else com_rotation_rad
        transpose = self.dset.com_transpose if transpose is None else transpose
        angle = rot if transpose else -1 * rot
        pos = self.dset.initial_scan_positions_px.cpu().numpy() if positions_px is None else positions_px
        origin = pos.mean(0).astype(np.float32)
        R = np.array([[np.cos(angle), -np.sin(angle)], [np.sin(angle), np.cos(angle)]], dtype=np.float32)
        pts = (pos - origin) @ R + origin + 1e-9
        min_r, min_c = np.floor(np.min(pts, axis=0)).astype("int")
        max_r, max_c = np.ceil(np.max(pts, axis=0)).astype("int")
        min_r, min_c = max(min_r, 0), max(min_c, 0)
        max_r, max_c = min(max_r, array.shape[-2]), min(max_c, array.shape[-1])
        out = ndi.rotate(array, np.rad2deg(-angle), order=1, reshape=False, axes=(-2, -1))[..., min_r:max_r,
                                                                                                min_c:max_c]
        if transpose:
            out = out.swapaxes(-2, -1)
        tgt = tuple(self.obj_shape_crop)
        sl = []
        for ax, t in zip(range(-3, 0), tgt):
            n = out.shape[ax]
            s0 = max((n - t) // 2, 0)
            sl.append(slice(s0, s0 + min(t, n)))
        return out[tuple(sl)]
