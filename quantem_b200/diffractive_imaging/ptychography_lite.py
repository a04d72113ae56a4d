"""PtychoLite: the reference's high-level wrapper (ptychography_lite.py:27-217)
routed to the fused B200 path.

``from_dataset`` builds the pixelated object / probe / detector models from
simple flags, preprocesses the dataset (on the GPU when ``device`` is a GPU) and
returns a ready ``Ptychography``; ``reconstruct`` sets AdamW optimisers and
optional schedulers from flat arguments and runs the fused iterations.
``PtychoLiteDIP`` turns a PtychoLite into a deep-image-prior reconstruction on the
CNN kernels.  The tensorboard logger is not part of the B200 path (``log_dir``
must be None).
"""
from __future__ import annotations

from typing import Any, Literal, Sequence

import numpy as np
import torch

from ..core.datasets import Dataset4dstem
from .dataset_models import PtychographyDatasetRaster
from .detector_models import DetectorPixelated
from .object_models import ObjectPixelated
from .probe_models import ProbePixelated
from .ptychography import Ptychography


class PtychoLite(Ptychography):
    """High-level convenience wrapper around Ptychography (ptychography_lite.py:18-25)."""

    @classmethod
    def from_dataset(cls, dset: Dataset4dstem | PtychographyDatasetRaster, *, num_slices: int = 1,
                     slice_thicknesses: float | Sequence | None = None,
                     obj_type: Literal["complex", "pure_phase", "potential"] = "complex", num_probes: int = 1,
                     energy: float | None = None, defocus: float | None = None,
                     semiangle_cutoff: float | None = None, polar_parameters: dict | None = None,
                     middle_focus: bool = False, vacuum_probe_intensity=None,
                     initial_probe_weights: list[float] | np.ndarray | None = None,
                     obj_padding_px: tuple[int, int] = (0, 0), log_dir=None, log_prefix: str = "",
                     log_images_every: int = 10, log_probe_images: bool = False,
                     device: Literal["cpu", "gpu"] = "cpu", verbose: int | bool = True, rng=None):
        """ptychography_lite.py:27-160: dataset model, uniform object, probe from
        parameters, pixelated detector, ``from_models`` and ``preprocess``."""
        if log_dir is not None:
            raise NotImplementedError("the tensorboard logger is not part of the B200 path (log_dir=None)")
        if isinstance(dset, PtychographyDatasetRaster):
            dset_model = dset
        elif isinstance(dset, Dataset4dstem):
            dset_model = PtychographyDatasetRaster.from_dataset4dstem(dset)
        else:
            raise TypeError(f"dset must be Dataset4dstem or PtychographyDatasetRaster, got {type(dset)}")
        if not dset_model.preprocessed:
            dset_model.preprocess(com_fit_function="constant", device=device)

        obj_model = ObjectPixelated.from_uniform(num_slices=num_slices, slice_thicknesses=slice_thicknesses,
                                                 obj_type=obj_type, device="cpu", rng=rng)
        probe_params: dict[str, Any] = {"energy": energy, "defocus": defocus, "semiangle_cutoff": semiangle_cutoff}
        if polar_parameters is not None:
            probe_params.update(polar_parameters)
        if middle_focus and num_slices > 1:  # focus at mid-thickness (ptychography_lite.py:117-123)
            half = float(obj_model.slice_thicknesses.sum()) / 2
            if probe_params.get("C10") is not None:
                probe_params["C10"] -= half
            if probe_params.get("defocus") is not None:
                probe_params["defocus"] += half
        probe_model = ProbePixelated.from_params(probe_params=probe_params, num_probes=num_probes, device="cpu",
                                                 rng=rng, initial_probe_weights=initial_probe_weights,
                                                 vacuum_probe_intensity=vacuum_probe_intensity)
        ptycho = cls.from_models(dset=dset_model, obj_model=obj_model, probe_model=probe_model,
                                 detector_model=DetectorPixelated(), device=device, verbose=verbose, rng=rng)
        ptycho.preprocess(obj_padding_px=obj_padding_px)
        return ptycho

    def reconstruct(self, num_iters: int = 0, reset: bool = False, lr_obj: float = 5e-3, learn_probe: bool = True,
                    lr_probe: float = 1e-3, batch_size: int | None = None,
                    scheduler_type: Literal["exp", "cyclic", "plateau", "none"] = "none",
                    scheduler_factor: float = 0.5, new_optimizers: bool = False, constraints: dict = {},
                    store_iterations_every: int | None = None, device: Literal["cpu", "gpu"] | None = None,
                    verbose: int | bool = True):
        """ptychography_lite.py:162-217: AdamW on the object (and the probe when
        ``learn_probe``), optional schedulers, then Ptychography.reconstruct."""
        return _lite_reconstruct(self, num_iters, reset, lr_obj, learn_probe, lr_probe, batch_size, scheduler_type,
                                 scheduler_factor, new_optimizers, constraints, store_iterations_every, device,
                                 verbose)


def _lite_reconstruct(pt, num_iters, reset, lr_obj, learn_probe, lr_probe, batch_size, scheduler_type,
                      scheduler_factor, new_optimizers, constraints, store_iterations_every, device, verbose):
    """Flat-argument reconstruct shared by PtychoLite and PtychoLiteDIP: new AdamW
    optimisers (and schedulers) on the first call, after a reset or on request."""
    pt.verbose = verbose
    if new_optimizers or reset or pt.num_iters == 0:
        opt_params = {"object": {"type": "adamw", "lr": lr_obj}}
        scheduler_params = {"object": {"type": scheduler_type, "factor": scheduler_factor}}
        if learn_probe:
            opt_params["probe"] = {"type": "adamw", "lr": lr_probe}
            scheduler_params["probe"] = {"type": scheduler_type, "factor": scheduler_factor}
    else:
        opt_params = None
        scheduler_params = None
    return Ptychography.reconstruct(pt, num_iters=num_iters, reset=reset, optimizer_params=opt_params,
                                    scheduler_params=scheduler_params, constraints=constraints,
                                    batch_size=batch_size, store_snapshots_every=store_iterations_every,
                                    device=device)


class PtychoLiteDIP(Ptychography):
    """Deep-image-prior variant of PtychoLite (ptychography_lite.py:255-427) on the B200
    path: the object becomes an ``ObjectDIP`` on the BF16 tcgen05 kernels -- a complex
    network (``ComplexCNN2d``) for complex objects, a real ``CNN2d`` otherwise, as the
    reference chooses -- optionally pre-trained on the PtychoLite object, and the
    network weights are optimised through the fused forward / adjoint kernels.

    The probe stays the PtychoLite's pixelated probe (the reference's probe DIP is not
    built here, so ``pretrain_probe`` has nothing to pre-train)."""

    @classmethod
    def from_ptycholite(cls, ptycholite: PtychoLite, pretrain_iters: int | None = None, pretrain_lr: float = 1e-3,
                        pretrain_probe: bool = True, pretrain_object: bool = True, cnn_num_layers: int = 3,
                        log_dir=None, log_prefix: str = "", log_images_every: int = 10,
                        log_probe_images: bool = False, device: Literal["cpu", "gpu", "cuda"] = "gpu",
                        verbose: int | bool = True):
        """ptychography_lite.py:263-370: CNN2d object model from the pixelated object,
        optional pre-training (AdamW, plateau scheduler), ``from_models`` with the same
        dataset / probe / detector and ``preprocess`` with the same padding."""
        from ..core.ml.cnn import CNN2d, ComplexCNN2d
        from .object_models import ObjectDIP

        if log_dir is not None:
            raise NotImplementedError("the tensorboard logger is not part of the B200 path (log_dir=None)")
        if str(device).lower() == "cpu":
            raise ValueError("PtychoLiteDIP runs its CNN on the GPU kernels: device must be 'gpu' or 'cuda'")
        S = ptycholite.obj_model.num_slices
        dev = torch.device("cuda", torch.cuda.current_device())
        kind = ComplexCNN2d if ptycholite.obj_model.obj_type == "complex" else CNN2d
        net = kind(in_channels=S, out_channels=S, num_layers=cnn_num_layers, device=dev)
        obj_model = ObjectDIP.from_pixelated(net, ptycholite.obj_model)
        if pretrain_iters is not None and pretrain_object:
            obj_model.pretrain(reset=True, num_iters=pretrain_iters,
                               optimizer_params={"type": "adamw", "lr": pretrain_lr},
                               scheduler_params={"type": "plateau", "factor": 0.5}, apply_constraints=False)
        ptycho = cls.from_models(dset=ptycholite.dset, obj_model=obj_model, probe_model=ptycholite.probe_model,
                                 detector_model=ptycholite.detector_model, logger=ptycholite.logger,
                                 device=device, verbose=ptycholite.verbose if verbose is True else verbose,
                                 rng=ptycholite.rng)
        pad = ptycholite.obj_padding_px
        ptycho.preprocess(obj_padding_px=(int(pad[0]), int(pad[1])))
        return ptycho

    def reconstruct(self, num_iters: int = 0, reset: bool = False, lr_obj: float = 5e-4, learn_probe: bool = True,
                    lr_probe: float = 5e-4, batch_size: int | None = None,
                    scheduler_type: Literal["exp", "cyclic", "plateau", "none"] = "none",
                    scheduler_factor: float = 0.5, new_optimizers: bool = False, constraints: dict = {},
                    store_iterations_every: int | None = None, device: Literal["cpu", "gpu"] | None = None,
                    verbose: int | bool = True):
        """ptychography_lite.py:372-427: AdamW on the network weights (and the probe
        when ``learn_probe``), optional schedulers, then Ptychography.reconstruct."""
        return _lite_reconstruct(self, num_iters, reset, lr_obj, learn_probe, lr_probe, batch_size, scheduler_type,
                                 scheduler_factor, new_optimizers, constraints, store_iterations_every, device,
                                 verbose)
