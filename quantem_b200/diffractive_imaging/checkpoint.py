"""Checkpoint / resume of a reconstruction (``Ptychography.save`` / ``from_file``).

The reference serialises the whole object graph through its AutoSerialize zarr
store (ptychography.py:376-588, core/io/serialize.py).  zarr is not part of this
path's dependencies, so a checkpoint here is one ``torch.save`` file holding an
explicit state: the model classes and their construction arguments, the raw object
and probe parameters and their initial values, the optimiser and scheduler states
(Adam moments and step counts included), the reconstruction's numpy generator state,
the loss / learning-rate histories and the dataset's preprocessing parameters and
scan positions.  With ``save_raw_data=True`` the 4D-STEM array is stored too and
``from_file`` rebuilds and preprocesses the dataset from it (the reference reloads it
from the dataset's file path); otherwise a preprocessed dataset is passed to
``from_file``.

Resuming continues exactly where the saved run stopped: the next ``reconstruct`` call
draws the same batch order and takes the same optimiser steps as an uninterrupted run.
"""
from __future__ import annotations

import os

import numpy as np
import torch

FORMAT = "quantem_b200.Ptychography"
VERSION = 1


def _cpu(t):
    return None if t is None else t.detach().cpu().clone()


def _opt_state(model):
    out = {"optimizer_params": dict(model.optimizer_params), "scheduler_params": dict(model.scheduler_params),
           "optimizer": None, "scheduler": None}
    if model.optimizer is not None:
        sd = model.optimizer.state_dict()
        out["optimizer"] = {"state": {k: {n: (_cpu(v) if isinstance(v, torch.Tensor) else v) for n, v in st.items()}
                                      for k, st in sd["state"].items()},
                            "param_groups": sd["param_groups"]}
    if model.scheduler is not None:
        out["scheduler"] = model.scheduler.state_dict()
    return out


def _restore_opt_state(model, st, num_iter=None):
    if st["optimizer_params"]:
        model.set_optimizer(st["optimizer_params"])
        if st["optimizer"] is not None:
            model.optimizer.load_state_dict(st["optimizer"])
    if st["scheduler_params"] and model.optimizer is not None:
        model.set_scheduler(st["scheduler_params"], num_iter)
        if st["scheduler"] is not None and model.scheduler is not None:
            model.scheduler.load_state_dict(st["scheduler"])
    elif st["scheduler_params"]:
        model.scheduler_params = st["scheduler_params"]


def _object_state(obj):
    from .object_models import ObjectDIP

    dip = isinstance(obj, ObjectDIP)
    state = {"class": type(obj).__name__, "obj_type": obj.obj_type, "initialize_mode": obj._initialize_mode,
             "num_slices": obj.num_slices, "slice_thicknesses": obj.slice_thicknesses.tolist(),
             "rng_seed": obj._rng_seed, "constraints": dict(obj.constraints),
             "obj": None if dip else _cpu(obj._obj), "initial_obj": None if dip else _cpu(obj._initial_obj),
             "sampling": obj._sampling, "mask": _cpu(obj.mask) if isinstance(obj.mask, torch.Tensor) else None}
    if dip:
        # the network (class, construction arguments, weights and batch-norm statistics), its
        # input, pre-training target and weights, and the input-noise generator's state
        m = obj.model
        state["dip"] = {"model_class": type(m).__name__, "model_config": m.config(),
                        "model_state": {k: _cpu(v) for k, v in m.state_dict().items()},
                        "model_input": _cpu(obj._model_input), "pretrain_target": _cpu(obj._pretrain_target),
                        "pretrained_weights": None if obj._pretrained_weights is None else
                        {k: _cpu(v) for k, v in obj._pretrained_weights.items()},
                        "pretrain_losses": list(obj._pretrain_losses), "pretrain_lrs": list(obj._pretrain_lrs),
                        "input_noise_std": obj._input_noise_std,
                        "noise_generator": None if obj._gen is None else obj._gen.get_state()}
    state.update(_opt_state(obj))
    return state


def _build_dip(os_, device):
    """The DIP object model of a checkpoint, its network rebuilt on ``device`` (CUDA)."""
    from ..core import config
    from ..core.ml.cnn import CNN2d, ComplexCNN2d
    from .object_models import ObjectDIP

    d = os_["dip"]
    dev = torch.device(config.validate_device(device if device is not None else "gpu")[0])
    if dev.type != "cuda":
        raise ValueError("a DIP object model is restored onto a CUDA device (its network runs there)")
    mcls = ComplexCNN2d if d["model_class"] == "ComplexCNN2d" else CNN2d
    model = mcls(**d["model_config"], device=dev)
    model.load_state_dict(d["model_state"])  # host tensors: the networks place them themselves
    th = os_["slice_thicknesses"]
    obj = ObjectDIP.from_model(model, d["model_input"].to(dev), num_slices=os_["num_slices"],
                               slice_thicknesses=np.asarray(th) if th else None,
                               input_noise_std=d["input_noise_std"], device=dev, obj_type=os_["obj_type"],
                               rng=os_["rng_seed"])
    if d["pretrained_weights"] is not None:
        obj._pretrained_weights = dict(d["pretrained_weights"])
    if d["pretrain_target"] is not None and d["pretrain_target"].numel():
        obj.pretrain_target = d["pretrain_target"].to(dev)
    obj._pretrain_losses = list(d["pretrain_losses"])
    obj._pretrain_lrs = list(d["pretrain_lrs"])
    if d["noise_generator"] is not None:
        obj._gen = torch.Generator(device=dev)
        obj._gen.set_state(d["noise_generator"])
    return obj, dev


def _probe_state(probe):
    return {"class": type(probe).__name__, "num_probes": probe.num_probes, "probe_params": dict(probe.probe_params),
            "probe_tilt": probe.probe_tilt.detach().cpu().tolist(),
            "initial_probe_tilt": probe._initial_probe_tilt.tolist(),
            "learn_probe_tilt": probe.learn_probe_tilt, "from_params": probe._from_params,
            "roi_shape": None if probe.roi_shape is None else [int(x) for x in probe.roi_shape],
            "initial_probe_weights": _cpu(probe.initial_probe_weights), "rng_seed": probe._rng_seed,
            "constraints": dict(probe.constraints), "probe": _cpu(probe._probe),
            "initial_probe": _cpu(probe._initial_probe), **_opt_state(probe)}


def _dataset_state(dset, save_raw_data):
    state = {"preprocessing_params": dict(dset._preprocessing_params), "constraints": dict(dset.constraints),
             "scan_positions_px": _cpu(dset.scan_positions_px),
             "initial_scan_positions_px": _cpu(dset.initial_scan_positions_px),
             "descan_shifts": _cpu(dset.descan_shifts), "initial_descan_shifts": _cpu(dset.initial_descan_shifts),
             "probe_energy": dset.probe_energy, "targets_on_host": dset.targets_on_host,
             "learn_descan": dset.learn_descan, "learn_scan_positions": dset.learn_scan_positions,
             "raw": None, **{"optim": _opt_state(dset)}}
    if save_raw_data:
        mask = dset.detector_mask
        state["raw"] = {"array": np.asarray(dset.intensities_4d),
                        "sampling": np.concatenate([dset.scan_sampling, dset.detector_sampling]).tolist(),
                        "units": list(dset.scan_units) + list(dset.detector_units),
                        "detector_mask": None if mask is None else np.asarray(torch.as_tensor(mask).cpu())}
    return state


def state_dict(pt, save_raw_data=False, skip=()) -> dict:
    """Everything needed to resume ``pt`` (see the module docstring)."""
    skip = {skip} if isinstance(skip, str) else set(skip)
    rng_state = pt.rng.bit_generator.state
    return {
        "format": FORMAT, "version": VERSION,
        "ptychography": {
            "rng_state": rng_state, "rng_bit_generator": type(pt.rng.bit_generator).__name__,
            "rng_seed": pt._rng_seed, "obj_padding_px": [int(x) for x in pt.obj_padding_px],
            "power2_level": pt._obj_padding_force_power2_level, "batch_size": pt.batch_size,
            "val_ratio": pt.val_ratio, "val_mode": pt.val_mode, "store_snapshots": pt._store_snapshots,
            "store_snapshot_every": pt._store_snapshot_every, "iter_losses": list(pt._iter_losses),
            "iter_val_losses": list(pt._iter_val_losses),
            "iter_lrs": {k: list(v) for k, v in pt._iter_lrs.items()},
            "snapshots": [] if "snapshots" in skip else list(pt._snapshots),
            "device": pt.device, "verbose": pt.verbose,
        },
        "object": _object_state(pt.obj_model),
        "probe": _probe_state(pt.probe_model),
        "dataset": _dataset_state(pt.dset, save_raw_data),
    }


def save(pt, path, mode="w", save_raw_data=False, skip=()):
    if mode not in ("w", "o"):
        raise ValueError(f"mode must be 'w' (write) or 'o' (overwrite), got {mode!r}")
    path = os.fspath(path)
    if mode == "w" and os.path.exists(path):
        raise FileExistsError(f"{path} exists; use mode='o' to overwrite")
    torch.save(state_dict(pt, save_raw_data, skip), path)


def _build_dataset(ds_state, verbose):
    from ..core.datasets import Dataset4dstem
    from .dataset_models import PtychographyDatasetRaster

    raw = ds_state["raw"]
    if raw is None:
        raise ValueError("the checkpoint holds no raw data (saved with save_raw_data=False): pass the "
                         "preprocessed dataset as from_file(path, dset=...)")
    d4 = Dataset4dstem.from_array(raw["array"], sampling=raw["sampling"], units=raw["units"])
    pd = PtychographyDatasetRaster.from_dataset4dstem(d4, detector_mask=raw["detector_mask"],
                                                      verbose=verbose if verbose is not None else 0,
                                                      learn_descan=ds_state["learn_descan"],
                                                      learn_scan_positions=ds_state["learn_scan_positions"])
    params = dict(ds_state["preprocessing_params"])
    pd.preprocess(probe_energy=ds_state["probe_energy"], plot_rotation=False, plot_com=False, **params)
    return pd


def from_state(cls, state, dset=None, device=None, verbose=None):
    from .detector_models import DetectorPixelated
    from .object_models import ObjectPixelated
    from .probe_models import ProbePixelated

    if state.get("format") != FORMAT:
        raise ValueError(f"not a {FORMAT} checkpoint")
    if int(state.get("version", 0)) > VERSION:
        raise ValueError(f"checkpoint version {state['version']} is newer than this library ({VERSION})")
    ps, os_, pr, ds = state["ptychography"], state["object"], state["probe"], state["dataset"]
    if dset is None:
        dset = _build_dataset(ds, verbose)
    elif not dset.preprocessed:
        dset.preprocess(probe_energy=ds["probe_energy"], plot_rotation=False, plot_com=False,
                        **ds["preprocessing_params"])
    dip = os_["class"] == "ObjectDIP"
    if os_["class"] not in ("ObjectPixelated", "ObjectDIP"):
        raise NotImplementedError(f"object model {os_['class']} cannot be restored from a checkpoint")
    build_dev = "cpu"
    if dip:  # the network lives on its device from the start
        obj, build_dev = _build_dip(os_, device)
    else:
        th = os_["slice_thicknesses"]
        obj = ObjectPixelated(os_["num_slices"], th if th else None, os_["obj_type"], os_["initialize_mode"],
                              "cpu", os_["rng_seed"], _token=ObjectPixelated._token)
    probe = ProbePixelated(pr["num_probes"], pr["probe_params"], tuple(pr["probe_tilt"]),
                           bool(pr.get("learn_probe_tilt", False)), pr["roi_shape"],
                           torch.complex64, "cpu", pr["rng_seed"], pr["initial_probe_weights"], None,
                           _from_params=pr["from_params"], _token=ProbePixelated._token)
    if pr["initial_probe"] is not None:
        probe._initial_probe = pr["initial_probe"].clone()
        probe._from_params = False  # the initial probe is restored as saved, no regeneration
    pt = cls.from_models(dset, obj, probe, DetectorPixelated(), device=build_dev,
                         verbose=ps["verbose"] if verbose is None else verbose)
    probe._from_params = pr["from_params"]
    pt._obj_padding_force_power2_level = ps["power2_level"]
    pt.obj_padding_px = ps["obj_padding_px"]
    # raw parameters and initial values exactly as saved
    if not dip:
        obj._initial_obj = os_["initial_obj"].clone()
        obj._obj = os_["obj"].clone().requires_grad_(True)
    obj.constraints = os_["constraints"]
    if os_["mask"] is not None:
        obj.mask = os_["mask"]
    probe._initial_probe = pr["initial_probe"].clone()
    probe._probe = pr["probe"].clone().requires_grad_(True)
    if "initial_probe_tilt" in pr:
        probe._initial_probe_tilt = torch.tensor(pr["initial_probe_tilt"], dtype=torch.float32)
    probe.constraints = pr["constraints"]
    dset._constraints = dict(ds["constraints"])
    dset._initial_scan_positions_px = ds["initial_scan_positions_px"].clone()
    dset.scan_positions_px = ds["scan_positions_px"].clone()
    if "descan_shifts" in ds:
        dset.descan_shifts = ds["descan_shifts"].clone()
        dset.initial_descan_shifts = ds["initial_descan_shifts"].clone()
    dset._set_patch_indices(pt.obj_padding_px)
    if ds["targets_on_host"]:
        dset.keep_targets_on_host(True)
    pt.batch_size = ps["batch_size"]
    pt.val_ratio = ps["val_ratio"]
    pt.val_mode = ps["val_mode"]
    pt._store_snapshots = ps["store_snapshots"]
    pt._store_snapshot_every = ps["store_snapshot_every"]
    pt._iter_losses = list(ps["iter_losses"])
    pt._iter_val_losses = list(ps["iter_val_losses"])
    pt._iter_lrs = {k: list(v) for k, v in ps["iter_lrs"].items()}
    pt._snapshots = list(ps["snapshots"])
    pt._preprocessed = True
    # device first: moving a model re-creates its optimiser, so states are loaded after the move
    pt.to(device if device is not None else build_dev)
    pt.compute_propagator_arrays()
    _restore_opt_state(obj, os_)
    _restore_opt_state(probe, pr)
    if ds.get("optim"):  # learned scan positions (dataset optimiser)
        _restore_opt_state(dset, ds["optim"])
    gen = getattr(np.random, ps["rng_bit_generator"])()
    gen.state = ps["rng_state"]
    pt._rng = np.random.Generator(gen)
    pt._rng_seed = ps["rng_seed"]
    return pt


def load(cls, path, dset=None, device=None, verbose=None):
    state = torch.load(os.fspath(path), map_location="cpu", weights_only=False)
    return from_state(cls, state, dset=dset, device=device, verbose=verbose)
