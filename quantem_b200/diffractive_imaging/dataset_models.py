"""Raster-scan ptychography dataset model (host-side set-up + per-batch positions).

Mirrors quantem.diffractive_imaging.dataset_models.PtychographyDatasetRaster of
the reference: CoM fitting (dataset_models.py:1027-1112, ptycho_utils.py:352-415),
relative rotation (1114-1370), diffraction normalisation to corner-centred target
amplitudes (1372-1480), raster scan positions (883-944), hard constraints on the
positions (597-613) and the per-batch ``forward`` (1482-1499).  Set-up runs on
the host (numpy / torch on the CPU); the batch kernels compute patch indices from
the positions on the GPU, and ``patch_indices`` is built only on request.
"""
from __future__ import annotations

from typing import Literal

import numpy as np
import torch
from scipy.optimize import curve_fit

from ..core import config
from ..core.datasets import Dataset4dstem
from ..core.optim import OptimizerMixin
from .complex_probe import electron_wavelength_angstrom


def _plane(xy, mx, my, b):
    return mx * xy[0] + my * xy[1] + b


def _parabola(xy, c0, cx1, cx2, cy1, cy2, cxy):
    return c0 + cx1 * xy[0] + cy1 * xy[1] + cx2 * xy[0] ** 2 + cy2 * xy[1] ** 2 + cxy * xy[0] * xy[1]


def fit_origin(data, mask=None, fit_function="plane"):
    """Fit of the diffraction origin over the scan (ptycho_utils.py:352-415)."""
    qr0, qc0 = data
    if fit_function == "constant":
        fr = np.mean(qr0) * np.ones_like(qr0)
        fc = np.mean(qc0) * np.ones_like(qc0)
        return fr, fc, qr0 - fr, qc0 - fc
    f = {"plane": _plane, "parabola": _parabola}.get(fit_function)
    if f is None:
        raise ValueError("fit_function must be one of 'plane', 'parabola', 'constant'")
    shape = qr0.shape
    r, c = np.indices(shape)
    rc = np.vstack((r.reshape(1, -1), c.reshape(1, -1)))
    if mask is not None:
        m1 = mask.reshape(1, -1)
        rcm = np.vstack((r.reshape(1, -1) * m1, c.reshape(1, -1) * m1))
        pr, _ = curve_fit(f, rcm, qr0[mask])
        pc, _ = curve_fit(f, rcm, qc0[mask])
    else:
        pr, _ = curve_fit(f, rc, qr0.ravel())
        pc, _ = curve_fit(f, rc, qc0.ravel())
    fr = f(rc, *pr).reshape(shape)
    fc = f(rc, *pc).reshape(shape)
    return fr, fc, qr0 - fr, qc0 - fc


def fourier_shift_real(ar: np.ndarray, rshift, cshift) -> np.ndarray:
    """Periodic sub-pixel Fourier shift of real images (ptycho_utils.py:239-300, non-bilinear).

    Works on (..., nr, nc) stacks with per-image shifts of shape (...)."""
    nr, nc = ar.shape[-2:]
    qr = np.fft.fftfreq(nr, 1)[:, None]
    qc = np.fft.fftfreq(nc, 1)[None, :]
    rs = np.asarray(rshift)[..., None, None]
    cs = np.asarray(cshift)[..., None, None]
    p = np.exp(-(2j * np.pi) * ((cs * qc) + (rs * qr)))
    return np.real(np.fft.ifft2(np.fft.fft2(ar) * p))


def bilinear_shift(ar: np.ndarray, rshift, cshift) -> np.ndarray:
    """Periodic bilinear shift of real images (ptycho_utils.py:273-284, bilinear=True): each
    image rolled by floor(shift) and blended with the roll one pixel further by the fractional
    parts, in float64.  Works on (..., nr, nc) stacks with per-image shifts of shape (...)."""
    nr, nc = ar.shape[-2:]
    a = ar.reshape(-1, nr, nc)
    rs = np.asarray(rshift, dtype=np.float64).reshape(-1)
    cs = np.asarray(cshift, dtype=np.float64).reshape(-1)
    rf, cf = np.floor(rs), np.floor(cs)
    wr, wc = (rs - rf)[:, None, None], (cs - cf)[:, None, None]
    rf, cf = rf.astype(np.int64), cf.astype(np.int64)
    b = np.arange(a.shape[0])[:, None, None]
    r0 = (np.arange(nr)[None] - rf[:, None]) % nr
    r1 = (np.arange(nr)[None] - rf[:, None] - 1) % nr
    c0 = (np.arange(nc)[None] - cf[:, None]) % nc
    c1 = (np.arange(nc)[None] - cf[:, None] - 1) % nc

    def g(ri, ci):
        return a[b, ri[:, :, None], ci[:, None, :]].astype(np.float64)

    out = g(r0, c0) * ((1 - wr) * (1 - wc)) + g(r1, c0) * (wr * (1 - wc))
    out = out + g(r0, c1) * ((1 - wr) * wc) + g(r1, c1) * (wr * wc)
    return out.reshape(ar.shape)


class PtychographyDatasetRaster(OptimizerMixin):
    """4D-STEM raster dataset: targets, scan positions and their constraints."""

    _token = object()
    DEFAULT_CONSTRAINTS = {
        "descan_tv_weight": 0.0,
        "descan_shifts_constant": False,
        "center_scan_positions": False,
        "clip_scan_positions": True,
    }

    def __init__(self, dset: Dataset4dstem, detector_mask=None, verbose=1, learn_descan=True,
                 learn_scan_positions=True, _token=None):
        if _token is not self._token:
            raise RuntimeError("Use PtychographyDatasetRaster.from_* to instantiate this class.")
        OptimizerMixin.__init__(self)
        if dset.units[-1] not in ("A^-1", "mrad"):
            raise ValueError(f"Expected diffraction units to be 'A^-1', got {dset.units[-1]}")
        self.scan_sampling = np.asarray(dset.sampling[:2], dtype=float)
        self.scan_units = list(dset.units[:2])
        self.gpts = np.asarray(dset.shape[:2], dtype=int)
        self.intensities_4d = np.asarray(dset.array).copy()
        shp = self.intensities_4d.shape
        self._array3d = self.intensities_4d.reshape(shp[0] * shp[1], shp[2], shp[3])
        self._dset = dset
        self._diffraction_padding = np.zeros(2, dtype=int)
        self.detector_sampling = np.asarray(dset.sampling[-2:], dtype=float)
        self.detector_units = list(dset.units[-2:])
        self.verbose = verbose
        self.learn_descan = bool(learn_descan)
        self.learn_scan_positions = bool(learn_scan_positions)
        self._preprocessed = False
        self._preprocessing_params = {}
        self.com_rotation_rad = 0.0
        self.com_transpose = False
        self._probe_energy = None
        self._device = "cpu"
        dt = getattr(torch, config.get("dtype_real"))
        self._scan_positions_px = torch.zeros((self.num_gpts, 2), dtype=dt)
        self._initial_scan_positions_px = torch.zeros((self.num_gpts, 2), dtype=dt)
        self._descan_shifts = torch.zeros((self.num_gpts, 2), dtype=dt)
        self._initial_descan_shifts = torch.zeros((self.num_gpts, 2), dtype=dt)
        self.detector_mask = detector_mask
        self._constraints = dict(self.DEFAULT_CONSTRAINTS)
        self._targets = None
        self._targets_on_host = False
        self._patch_indices = None
        self._last_patch_positions_px = None

    @classmethod
    def from_array(cls, array, name=None, origin=None, sampling=None, units=None, signal_units="arb. units",
                   detector_mask=None, verbose=1, learn_descan=True, learn_scan_positions=True):
        """A dataset from a 4-D array (dataset_models.py:734-780): a Dataset4dstem with the
        given metadata, then the raster dataset on it."""
        d4 = Dataset4dstem.from_array(array, name=name, origin=origin, sampling=sampling, units=units,
                                      signal_units=signal_units)
        return cls(d4, detector_mask, verbose, learn_descan, learn_scan_positions, _token=cls._token)

    @property
    def dset(self) -> Dataset4dstem:
        """The source 4D-STEM dataset (dataset_models.py:251-259)."""
        return self._dset

    @property
    def shape(self) -> np.ndarray:
        return np.array(self._dset.shape)

    @property
    def reciprocal_units(self) -> list[str]:
        return ["A^-1", "A^-1"]

    @property
    def diffraction_padding(self) -> np.ndarray:
        return self._diffraction_padding

    @diffraction_padding.setter
    def diffraction_padding(self, padding):
        pad = np.asarray(padding, dtype=int)
        if pad.shape != (2,):
            raise ValueError(f"diffraction_padding must have shape (2,), got {pad.shape}")
        self._diffraction_padding = pad

    @property
    def intensities(self) -> torch.Tensor:
        """Raw intensities (npos, qx, qy), clipped at 0 (dataset_models.py:313-327)."""
        return self._intensities

    @intensities.setter
    def intensities(self, arr):
        self._intensities = self._checked_patterns(arr, "intensities")

    @property
    def centered_intensities(self) -> torch.Tensor:
        """Intensities centred on the detector (npos, qx, qy) (dataset_models.py:295-311)."""
        return self._centered_intensities

    @centered_intensities.setter
    def centered_intensities(self, arr):
        self._centered_intensities = self._checked_patterns(arr, "centered_intensities")

    def _checked_patterns(self, arr, name):
        t = torch.as_tensor(arr.detach() if isinstance(arr, torch.Tensor) else np.asarray(arr),
                            dtype=getattr(torch, config.get("dtype_real")))
        shape = (self.num_gpts, *(int(x) for x in self.roi_shape))
        if tuple(t.shape) != shape:
            raise ValueError(f"{name} must have shape {shape}, got {tuple(t.shape)}")
        return t

    def vprint(self, m, level: int = 1, *args, **kwargs) -> None:
        """Print when verbose (dataset_models.py:509-512)."""
        if self.verbose >= level:
            print(m, *args, **kwargs)

    def patch_indices_need_update(self) -> bool:
        """Whether the rounded scan positions moved since the patch windows were last set
        (dataset_models.py:541-548).  The batch kernels form the windows from the positions
        themselves, so the answer only matters to callers of ``patch_indices``."""
        if self._last_patch_positions_px is None:
            return True
        old = torch.round(self._last_patch_positions_px.to(self.scan_positions_px.device))
        return not torch.equal(old, torch.round(self.scan_positions_px.detach()))

    def get_descan_tv_loss(self, descan_shifts: torch.Tensor, weight: float = 0.0) -> torch.Tensor:
        """weight x the mean absolute difference of consecutive descan shifts, averaged over the
        two axes (dataset_models.py:580-587)."""
        if weight == 0:
            return torch.zeros((), dtype=getattr(torch, config.get("dtype_real")), device=descan_shifts.device)
        return weight * (torch.mean(torch.abs(descan_shifts[:, 0].diff())) +
                         torch.mean(torch.abs(descan_shifts[:, 1].diff()))) / 2

    @classmethod
    def from_dataset4dstem(cls, dset: Dataset4dstem, detector_mask=None, verbose=1, learn_descan=True,
                           learn_scan_positions=True):
        return cls(dset, detector_mask, verbose, learn_descan, learn_scan_positions, _token=cls._token)

    # ------------------------------------------------------------------ props
    @property
    def num_gpts(self) -> int:
        return int(self._array3d.shape[0])

    @property
    def roi_shape(self) -> np.ndarray:
        return np.array(self._array3d.shape[-2:])

    @property
    def device(self):
        return self._device

    @property
    def preprocessed(self) -> bool:
        return self._preprocessed

    @property
    def probe_energy(self):
        return self._probe_energy

    @probe_energy.setter
    def probe_energy(self, e):
        self._probe_energy = None if e is None else float(e)

    @property
    def reciprocal_sampling(self) -> np.ndarray:
        units = self.detector_units
        s = self.detector_sampling
        if units[0] == "A^-1":
            return s
        if units[0] == "mrad":
            if self.probe_energy is None:
                raise ValueError("dset Q units given in mrad but no probe energy defined")
            return s / electron_wavelength_angstrom(self.probe_energy) / 1e3
        raise ValueError(f"Unknown dset Q units: {units}")

    @property
    def obj_sampling(self) -> np.ndarray:
        return 1 / (self.roi_shape * self.reciprocal_sampling)

    @property
    def fov(self) -> np.ndarray:
        return self.scan_sampling * (self.gpts - 1)

    @property
    def _obj_shape_crop_2d(self) -> np.ndarray:
        shp = np.floor(self.fov / self.obj_sampling)
        shp += shp % 2
        return shp.astype("int")

    @property
    def upsample_factor(self) -> float:
        return float((self._obj_shape_crop_2d / self.gpts).mean())

    @property
    def _obj_shape_rot_2d(self) -> np.ndarray:
        c = self._obj_shape_crop_2d.copy()
        a = self.com_rotation_rad
        rot = np.floor([abs(c[-1] * np.sin(a)) + abs(c[-2] * np.cos(a)),
                        abs(c[-2] * np.sin(a)) + abs(c[-1] * np.cos(a))])
        rot += rot % 2
        return rot.astype("int")

    def _obj_shape_full_2d(self, obj_padding_px) -> np.ndarray:
        return (self._obj_shape_rot_2d + 2 * np.array(obj_padding_px)).astype("int")

    @property
    def detector_mask(self) -> torch.Tensor:
        return self._detector_mask

    @detector_mask.setter
    def detector_mask(self, mask):
        dt = getattr(torch, config.get("dtype_real"))
        if mask is None:
            mask = torch.ones(*[int(x) for x in self.roi_shape], dtype=dt)
        else:
            mask = torch.as_tensor(np.asarray(mask) if not isinstance(mask, torch.Tensor) else mask, dtype=dt)
            if tuple(mask.shape) != tuple(self.roi_shape):
                raise ValueError(f"detector_mask must have shape {tuple(self.roi_shape)}")
        self._detector_mask = mask.to(self._device)

    @property
    def scan_positions_px(self) -> torch.Tensor:
        return self._scan_positions_px

    @scan_positions_px.setter
    def scan_positions_px(self, positions):
        t = torch.as_tensor(positions.detach().cpu().numpy() if isinstance(positions, torch.Tensor)
                            else np.asarray(positions), dtype=getattr(torch, config.get("dtype_real")))
        if tuple(t.shape) != (self.num_gpts, 2):
            raise ValueError(f"scan_positions_px must have shape {(self.num_gpts, 2)}")
        self._set_positions(t)

    def _set_positions(self, t: torch.Tensor):
        """New position values; kept in the same tensor while an optimiser holds it (the
        reference assigns ``.data`` of its position parameter, dataset_models.py:146-154)."""
        cur = self._scan_positions_px
        if self.has_optimizer() and isinstance(cur, torch.Tensor) and cur.shape == t.shape:
            with torch.no_grad():
                cur.data = t.detach().to(cur.device, cur.dtype).contiguous()
        else:
            self._scan_positions_px = t.detach().to(self._device).contiguous()

    @property
    def initial_scan_positions_px(self) -> torch.Tensor:
        return self._initial_scan_positions_px

    @property
    def descan_shifts(self) -> torch.Tensor:
        """Descan shifts [px] (num_positions, 2): with ``learn_descan`` and a dataset
        optimiser, the exit wave of every position is multiplied by their translation
        ramp (ptychography_base.py:903-905) and the targets are the uncentred patterns."""
        return self._descan_shifts

    @descan_shifts.setter
    def descan_shifts(self, shifts):
        t = torch.as_tensor(shifts.detach().cpu().numpy() if isinstance(shifts, torch.Tensor)
                            else np.asarray(shifts), dtype=getattr(torch, config.get("dtype_real")))
        if tuple(t.shape) != (self.num_gpts, 2):
            raise ValueError(f"descan_shifts must have shape {(self.num_gpts, 2)}")
        self._set_descan(t)

    def _set_descan(self, t: torch.Tensor):
        """New descan values, kept in the same tensor while an optimiser holds it
        (dataset_models.py:121-132 assigns ``.data``)."""
        cur = self._descan_shifts
        if self.has_optimizer() and isinstance(cur, torch.Tensor) and cur.shape == t.shape:
            with torch.no_grad():
                cur.data = t.detach().to(cur.device, cur.dtype).contiguous()
        else:
            self._descan_shifts = t.detach().to(self._device).contiguous()

    @property
    def initial_descan_shifts(self) -> torch.Tensor:
        """Descan shifts the dataset resets to (dataset_models.py:189-202)."""
        return self._initial_descan_shifts

    @initial_descan_shifts.setter
    def initial_descan_shifts(self, shifts):
        t = torch.as_tensor(shifts.detach().cpu().numpy() if isinstance(shifts, torch.Tensor)
                            else np.asarray(shifts), dtype=getattr(torch, config.get("dtype_real")))
        if tuple(t.shape) != (self.num_gpts, 2):
            raise ValueError(f"initial_descan_shifts must have shape {(self.num_gpts, 2)}")
        self._initial_descan_shifts = t.to(self._device)

    @property
    def descan_learned(self) -> bool:
        """Descan shifts enter the forward model (dataset_models.py:232, 1495): learned and
        a dataset optimiser is set."""
        return self.learn_descan and self.has_optimizer()

    def apply_descan_constraints(self, descan: torch.Tensor) -> torch.Tensor | None:
        """dataset_models.py:588-595: ``descan_shifts_constant`` replaces the shifts by zeros
        (no gradient reaches them); None stands for those zeros here."""
        if self._constraints.get("descan_shifts_constant", False):
            return None
        return descan

    def batch_descan(self) -> torch.Tensor | None:
        """The (num_positions, 2) descan shifts the batch kernels apply, or None."""
        if not self.descan_learned:
            return None
        return self.apply_descan_constraints(self._descan_shifts)

    def apply_soft_constraints(self, descan_shifts: torch.Tensor) -> torch.Tensor:
        """dataset_models.py:564-586: ``descan_tv_weight`` * the mean absolute difference of
        consecutive shifts (raster order), averaged over the two axes, when descan is
        learned; zero otherwise."""
        w = float(self._constraints.get("descan_tv_weight", 0.0))
        if w <= 0 or not self.descan_learned:
            return torch.zeros((), dtype=getattr(torch, config.get("dtype_real")), device=descan_shifts.device)
        return w * (torch.mean(torch.abs(descan_shifts[:, 0].diff())) +
                    torch.mean(torch.abs(descan_shifts[:, 1].diff()))) / 2

    @property
    def positions_px_fractional(self) -> torch.Tensor:
        return self.scan_positions_px - torch.round(self.scan_positions_px)

    @property
    def targets(self) -> torch.Tensor:
        if not self._preprocessed:
            raise ValueError("dset must be preprocessed before targets can be accessed")
        return self._targets

    @property
    def constraints(self) -> dict:
        return self._constraints

    @property
    def targets_on_host(self) -> bool:
        return self._targets_on_host

    def keep_targets_on_host(self, enable: bool = True):
        """Keep the measured targets in pinned host memory whatever device the dataset
        moves to.  ``Ptychography.reconstruct`` then copies them to the GPU once per
        iteration, double-buffered on a copy stream so that the copy for the next
        iteration overlaps the current one (for data that should not stay resident in
        device memory).  Not part of the reference API."""
        self._targets_on_host = bool(enable)
        if isinstance(self._targets, torch.Tensor):
            self._targets = self._host_or_device(self._targets)
            self._targets_kind = getattr(self, "_targets_kind", None)
        return self

    def _host_or_device(self, t: torch.Tensor) -> torch.Tensor:
        if self._targets_on_host:
            if t.device.type == "cpu" and t.is_contiguous() and (not torch.cuda.is_available() or t.is_pinned()):
                return t  # already where it belongs: no new tensor, no copy
            t = t.detach().cpu().contiguous()
            return t if not torch.cuda.is_available() or t.is_pinned() else t.pin_memory()
        return t.to(self._device).contiguous()

    def add_constraint(self, key, value):
        if key not in self.DEFAULT_CONSTRAINTS:
            raise KeyError(f"Unknown dataset constraint {key!r}")
        self._constraints[key] = value

    def get_optimization_parameters(self):
        """The descan shifts and the scan positions, each when learned, in that order
        (dataset_models.py:98-110)."""
        params = []
        if self.learn_descan:
            self._descan_shifts = self._descan_shifts.detach().contiguous().requires_grad_(True)
            params.append(self._descan_shifts)
        if self.learn_scan_positions:
            self._scan_positions_px = self._scan_positions_px.detach().contiguous().requires_grad_(True)
            params.append(self._scan_positions_px)
        if not params:
            raise RuntimeError("No parameters to optimize for dataset: learn_descan and learn_scan_positions "
                               "are both False")
        return params

    def remove_optimizer(self):
        super().remove_optimizer()
        self._scan_positions_px = self._scan_positions_px.detach()
        self._descan_shifts = self._descan_shifts.detach()

    def reset_iter_constraint_losses(self):
        pass

    def reset(self):
        self._set_positions(self._initial_scan_positions_px.clone())
        self._set_descan(self._initial_descan_shifts.clone())
        if self._optimizer is not None:
            self.set_optimizer(self._optimizer_params)

    def to(self, device):
        dev, _ = config.validate_device(device)
        self._device = dev
        for name in ("_scan_positions_px", "_initial_scan_positions_px", "_descan_shifts", "_initial_descan_shifts",
                     "_detector_mask",
                     "_targets", "_centered_amplitudes", "_amplitudes", "_centered_intensities", "_intensities"):
            v = getattr(self, name, None)
            if isinstance(v, torch.Tensor):
                setattr(self, name, self._host_or_device(v) if name == "_targets" else v.detach().to(dev))
        if self._optimizer is not None:  # the positions may be new tensors now
            self.set_optimizer(self._optimizer_params)
        return self

    # ---------------------------------------------------------- preprocessing
    def preprocess(self, com_fit_function: Literal["none", "plane", "parabola", "constant", "no_shift"] = "plane",
                   force_com_rotation: float | None = None, force_com_transpose: bool | None = None,
                   bilinear: bool = False, padded_diffraction_intensities_shape=None, obj_padding_px=(0, 0),
                   plot_rotation: bool = True, plot_com: str | bool = True, vectorized: bool = True,
                   probe_energy: float | None = None, device=None):
        """dataset_models.py:946-1025 (plots are not produced).

        ``device`` (default: the dataset's device): on a CUDA device the centre of
        mass and the intensity normalisation run in the GPU kernels
        (``ptycho_pattern_*`` + ``ptycho_fft2``) and the targets stay on the device;
        otherwise they run vectorised on the host.  Only the small CoM fit and the
        rotation search stay on the host in both cases."""
        if padded_diffraction_intensities_shape is not None:
            # the reference's own padding step forwards in_place=True to numpy.pad and raises
            # (dataset_models.py:976-983, core/datastructures/dataset.py:409-418)
            raise NotImplementedError("padded diffraction intensities are not part of the B200 path")
        self._bilinear = bool(bilinear)
        self._preprocessing_params = dict(com_fit_function=com_fit_function, force_com_rotation=force_com_rotation,
                                          force_com_transpose=force_com_transpose, bilinear=bool(bilinear),
                                          obj_padding_px=obj_padding_px)
        if probe_energy is not None:
            self.probe_energy = probe_energy
        dev = torch.device(config.validate_device(device if device is not None else self._device)[0])
        n = int(self.roi_shape[0])
        from .. import ops

        gpu = dev.type == "cuda" and self.roi_shape[0] == self.roi_shape[1] and n in ops.SUPPORTED_N
        self._preprocessed_on = "gpu" if gpu else "host"
        if gpu:
            self._inten_dev = torch.as_tensor(self.intensities_4d).to(dev, torch.float32).contiguous()
        self._set_intensities_com(self.intensities_4d, com_fit_function)
        self._set_com_relative_rotation(force_com_rotation, force_com_transpose)
        self._normalize_diffraction_intensities()
        self._inten_dev = None
        self._set_initial_scan_positions_px(obj_padding_px)
        self._set_patch_indices(obj_padding_px)
        self._set_targets("l2_amplitude")
        self._preprocessed = True

    def _set_intensities_com(self, intensities, fit_function):
        """Vectorised centre of mass (dataset_models.py:1027-1112); on the GPU when
        preprocess runs there (``ptycho_pattern_com``, FP64 sums)."""
        dt = config.get("dtype_real")
        if getattr(self, "_inten_dev", None) is not None:
            from .. import _lib, ops

            x = self._inten_dev
            nr, nc, qr, qc = x.shape
            com = torch.empty(2 * nr * nc, dtype=torch.float64, device=x.device)
            _lib.check(_lib.lib().ptycho_pattern_com(ops._p(x), None, nr * nc, qr, qc, ops._p(com), ops._stream()),
                       "pattern_com")
            com_r, com_c = com.view(2, nr, nc).cpu().numpy().astype(dt)
        else:
            kr = np.arange(intensities.shape[-2])
            kc = np.arange(intensities.shape[-1])
            krm, kcm = np.meshgrid(kr, kc, indexing="ij")
            im = intensities.astype(dt)
            com_r = np.sum(im * krm[None, None], axis=(-2, -1))
            com_c = np.sum(im * kcm[None, None], axis=(-2, -1))
            tot = np.sum(im, axis=(-2, -1))
            com_r /= tot
            com_c /= tot
        if fit_function == "none":
            fr, fc = com_r, com_c
        elif fit_function == "no_shift":
            fr = np.ones_like(com_r) * self.roi_shape[0] / 2
            fc = np.ones_like(com_c) * self.roi_shape[1] / 2
        else:
            fr, fc, _, _ = fit_origin((com_r, com_c), mask=np.isfinite(com_r), fit_function=fit_function)
        self.com_measured = np.array((com_r, com_c))
        self.com_fit = np.array((fr, fc))

    @property
    def com_normalized(self) -> np.ndarray:
        return np.nan_to_num(self.com_measured - self.com_fit) * self.reciprocal_sampling[:, None, None]

    def _set_com_relative_rotation(self, force_com_rotation=None, force_com_transpose=None,
                                   rotation_angles_deg=None):
        """Curl-minimising rotation search (dataset_models.py:1114-1370)."""

        def curl_for(angles, com, transpose):
            a = angles[:, None, None]
            cr, cc = com[0][None], com[1][None]
            if transpose:
                rr = np.cos(a) * cc - np.sin(a) * cr
                rc = np.sin(a) * cc + np.cos(a) * cr
            else:
                rr = np.cos(a) * cr - np.sin(a) * cc
                rc = np.sin(a) * cr + np.cos(a) * cc
            g1 = rr[:, 1:-1, 2:] - rr[:, 1:-1, :-2]
            g2 = rc[:, 2:, 1:-1] - rc[:, :-2, 1:-1]
            return np.mean(np.abs(g2 - g1), axis=(-2, -1))

        if rotation_angles_deg is None:
            rotation_angles_deg = np.arange(-89.0, 90.0, 1.0)
        ang = np.deg2rad(np.asarray(rotation_angles_deg))
        if force_com_rotation is not None:
            best = np.deg2rad(force_com_rotation)
            if force_com_transpose is not None:
                transpose = bool(force_com_transpose)
            else:
                c0 = curl_for(np.array([best]), self.com_normalized, False)[0]
                c1 = curl_for(np.array([best]), self.com_normalized, True)[0]
                transpose = bool(c1 < c0)
        elif force_com_transpose is not None:
            transpose = bool(force_com_transpose)
            best = ang[int(np.argmin(curl_for(ang, self.com_normalized, transpose)))]
        else:
            c0 = curl_for(ang, self.com_normalized, False)
            c1 = curl_for(ang, self.com_normalized, True)
            i0, i1 = int(np.argmin(c0)), int(np.argmin(c1))
            if c0[i0] <= c1[i1]:
                best, transpose = ang[i0], False
            else:
                best, transpose = ang[i1], True
        self.com_rotation_rad = float(best)
        self.com_transpose = bool(transpose)

    def _normalize_diffraction_intensities(self):
        """Centred target amplitudes (dataset_models.py:1372-1480), vectorised over
        positions: amplitude = sqrt(max(I,0)) Fourier-shifted by -CoM_fit,
        clipped at 0 and fftshifted."""
        if getattr(self, "_inten_dev", None) is not None:
            return self._normalize_diffraction_intensities_gpu()
        dt = config.get("dtype_real")
        di = self.intensities_4d.astype(dt)
        inten = np.maximum(di, 0)
        amp = np.maximum(np.sqrt(inten), 0)
        mean_intensity = float(np.sum(np.sum(inten, axis=(-2, -1), dtype=np.float64)))
        cr = -(self.com_fit[0] + 0.0)
        cc = -(self.com_fit[1] + 0.0)
        nr, nc = amp.shape[:2]
        centered = np.empty_like(amp)
        centered_i = np.empty_like(amp)
        chunk = max(1, 2048 // max(1, nc))
        for r0 in range(0, nr, chunk):
            if getattr(self, "_bilinear", False):
                sh = bilinear_shift(amp[r0:r0 + chunk], cr[r0:r0 + chunk], cc[r0:r0 + chunk])
            else:
                sh = fourier_shift_real(amp[r0:r0 + chunk].astype(np.float64), cr[r0:r0 + chunk], cc[r0:r0 + chunk])
            sh = np.fft.fftshift(np.maximum(sh, 0), axes=(-2, -1))
            centered[r0:r0 + chunk] = sh.astype(dt)
            centered_i[r0:r0 + chunk] = (sh**2).astype(dt)
        npos = nr * nc
        roi = tuple(int(x) for x in self.roi_shape)
        self._amplitudes = torch.as_tensor(amp.reshape(-1, *roi))
        self._centered_amplitudes = torch.as_tensor(centered.reshape(-1, *roi))
        self._intensities = torch.as_tensor(inten.reshape(-1, *roi))
        self._centered_intensities = torch.as_tensor(centered_i.reshape(-1, *roi))
        self.mean_diffraction_intensity = mean_intensity / npos
        descan = -1 * self.com_fit.reshape((2, -1)) + self.roi_shape[:, None] / 2
        self._descan_shifts = torch.as_tensor(descan.T.astype(dt))
        self._initial_descan_shifts = self._descan_shifts.clone()

    def _normalize_diffraction_intensities_gpu(self, chunk: int = 2048):
        """GPU version of the normalisation: clip / sqrt / sums (ptycho_pattern_prepare),
        forward FFT, shift ramp of -CoM_fit (ptycho_pattern_shift_ramp), inverse FFT,
        clip + fftshift (ptycho_pattern_center), in chunks of ``chunk`` patterns.
        FP32 transforms (the host path and the reference use FP64 numpy FFTs)."""
        from .. import _lib, ops

        x = self._inten_dev
        nr, nc, n, _ = x.shape
        npos = nr * nc
        dev = x.device
        lib, st = _lib.lib(), ops._stream()
        flat = x.view(npos, n, n)
        inten = torch.empty_like(flat)
        amp = torch.empty_like(flat)
        camp = torch.empty_like(flat)
        cint = torch.empty_like(flat)
        shifts = torch.as_tensor(-(np.asarray(self.com_fit, dtype=np.float64).reshape(2, -1) + 0.0), device=dev)
        work = torch.empty(2 * 592, dtype=torch.float64, device=dev)
        sums = torch.empty(2, dtype=torch.float64, device=dev)
        total = torch.zeros(2, dtype=torch.float64, device=dev)
        for c0 in range(0, npos, chunk):
            c1 = min(npos, c0 + chunk)
            m = c1 - c0
            ac = torch.empty((m, n, n), dtype=torch.complex64, device=dev)
            _lib.check(lib.ptycho_pattern_prepare(ops._p(flat[c0:c1]), m * n * n, ops._p(inten[c0:c1]),
                                                  ops._p(amp[c0:c1]), ops._p(ac), ops._p(work), work.numel(),
                                                  ops._p(sums), st), "pattern_prepare")
            total += sums
            sh = shifts[:, c0:c1].contiguous()
            if getattr(self, "_bilinear", False):
                _lib.check(lib.ptycho_pattern_bilinear(ops._p(amp[c0:c1]), ops._p(sh), m, n, ops._p(camp[c0:c1]),
                                                       ops._p(cint[c0:c1]), st), "pattern_bilinear")
                continue
            ops.fft2(ac, out=ac)
            _lib.check(lib.ptycho_pattern_shift_ramp(ops._p(ac), ops._p(sh), m, n, st), "pattern_shift_ramp")
            ops.fft2(ac, inverse=True, scale=1.0 / (n * n), out=ac)
            _lib.check(lib.ptycho_pattern_center(ops._p(ac), m, n, 1.0, ops._p(camp[c0:c1]), ops._p(cint[c0:c1]), st),
                       "pattern_center")
        tot = total.cpu().numpy()
        self._amplitudes = amp
        self._centered_amplitudes = camp
        self._intensities = inten
        self._centered_intensities = cint
        self.mean_diffraction_intensity = float(tot[0]) / npos
        self.mean_diffraction_amplitude = float(tot[1]) / npos
        dt = config.get("dtype_real")
        descan = -1 * self.com_fit.reshape((2, -1)) + self.roi_shape[:, None] / 2
        self._descan_shifts = torch.as_tensor(descan.T.astype(dt))
        self._initial_descan_shifts = self._descan_shifts.clone()

    @property
    def centered_amplitudes(self) -> torch.Tensor:
        return self._centered_amplitudes

    @property
    def amplitudes(self) -> torch.Tensor:
        return self._amplitudes

    def _set_initial_scan_positions_px(self, obj_padding_px):
        """Raster positions in object pixels (dataset_models.py:883-944)."""
        if obj_padding_px is None:
            obj_padding_px = np.array([0, 0])
        nr, nc = self.gpts
        sr, sc = self.scan_sampling
        r, c = np.meshgrid(np.arange(nr) * sr, np.arange(nc) * sc, indexing="ij")
        pos = np.stack((r.ravel(), c.ravel()), axis=-1).astype(config.get("dtype_real"))
        if self.com_rotation_rad != 0:
            # AffineTransform(angle)(x, origin) = (x - origin) @ R + origin (ptycho_utils.py:510-567)
            a = self.com_rotation_rad
            origin = np.asarray(pos.mean(0), dtype=np.float32)
            rot = np.array([[np.cos(a), -np.sin(a)], [np.sin(a), np.cos(a)]], dtype=np.float32)
            pos = ((pos - origin) @ rot + origin).astype(pos.dtype)
        sampling = self.obj_sampling
        if self.com_transpose:
            pos = np.flip(pos, axis=1)
            sampling = sampling[::-1]
        m = np.min(pos, axis=0).clip(-np.inf, 0)
        pos -= m
        pos[:, 0] /= sampling[0]
        pos[:, 1] /= sampling[1]
        pos[:, 0] += obj_padding_px[0]
        pos[:, 1] += obj_padding_px[1]
        self.scan_positions_px = pos
        self._initial_scan_positions_px = self._scan_positions_px.clone()

    def _set_patch_indices(self, obj_padding_px):
        """Remember the rounded positions the patch windows correspond to
        (dataset_models.py:514-539); the windows themselves are formed inside the
        batch kernels, and ``patch_indices`` builds them only when read."""
        self._patch_obj_shape = self._obj_shape_full_2d(obj_padding_px)
        self._last_patch_positions_px = self.scan_positions_px.clone()
        self._patch_indices = None

    @property
    def patch_indices(self) -> torch.Tensor:
        if self._patch_indices is None:
            shp = self._patch_obj_shape
            r0 = torch.round(self._last_patch_positions_px[:, 0]).to(torch.int32)
            c0 = torch.round(self._last_patch_positions_px[:, 1]).to(torch.int32)
            x = torch.fft.fftfreq(int(self.roi_shape[0]), d=1 / int(self.roi_shape[0])).to(r0.device)
            y = torch.fft.fftfreq(int(self.roi_shape[1]), d=1 / int(self.roi_shape[1])).to(r0.device)
            row = (r0[:, None, None] + x[None, :, None]) % int(shp[-2])
            col = (c0[:, None, None] + y[None, None, :]) % int(shp[-1])
            self._patch_indices = (row * int(shp[-1]) + col).to(torch.int32)
        return self._patch_indices

    def _set_targets(self, loss_type):
        """dataset_models.py:225-242: the centred patterns, or the uncentred ones while the
        descan shifts are learned (they then carry the pattern offsets)."""
        raw = self.descan_learned
        if "amplitude" in loss_type:
            t, kind = (self._amplitudes, "amplitude_raw") if raw else (self._centered_amplitudes, "amplitude")
        elif "intensity" in loss_type or loss_type == "poisson":
            t, kind = (self._intensities, "intensity_raw") if raw else (self._centered_intensities, "intensity")
        else:
            raise ValueError(f"Unknown loss type {loss_type}")
        # host-resident targets are built once per kind: a fresh pinned copy of the whole
        # stack on every reconstruct call would cost more than the iterations it feeds
        if (self._targets_on_host and isinstance(self._targets, torch.Tensor) and self._targets.device.type == "cpu"
                and getattr(self, "_targets_kind", None) == kind):
            return
        self._targets = self._host_or_device(t.clone())
        self._targets_kind = kind

    # --------------------------------------------------------- per batch
    def apply_hard_constraints(self, obj_padding_px):
        """Position clipping / centring (dataset_models.py:597-613)."""
        pos = self.scan_positions_px
        shp = torch.tensor(self._obj_shape_full_2d(obj_padding_px), device=pos.device, dtype=pos.dtype)
        if self._constraints.get("clip_scan_positions", True):
            pos = torch.minimum(torch.maximum(pos, torch.zeros_like(shp)), shp - 1)
        if self._constraints.get("center_scan_positions", False):
            pos = pos - pos.mean(dim=0, keepdim=True) + shp / 2
        self._set_positions(pos)

    def forward(self, batch_indices, obj_padding_px):
        """(patch_indices, positions_px, positions_px_fractional, descan shifts or None) of a
        batch (dataset_models.py:1482-1499)."""
        self.apply_hard_constraints(obj_padding_px)
        bi = torch.as_tensor(np.asarray(batch_indices), device=self.scan_positions_px.device)
        positions = self.scan_positions_px[bi]
        frac = positions - torch.round(positions)
        if not torch.equal(torch.round(self._last_patch_positions_px.to(positions.device)),
                           torch.round(self.scan_positions_px)):
            self._set_patch_indices(obj_padding_px)
        descan = self.batch_descan()
        return self.patch_indices.to(positions.device)[bi], positions, frac, (None if descan is None else descan[bi])
