"""PtychoLite (ptychography_lite.py:27-217) on the fused path: from_dataset builds
the same models and preprocessing as the explicit Ptychography construction, and
reconstruct with its flat AdamW arguments follows the same loss trajectory."""
import numpy as np
import pytest

from tests.conftest import load_golden

pytestmark = pytest.mark.gpu


def test_ptycholite_equals_explicit_construction(cuda_device):
    from quantem_b200.diffractive_imaging import (Dataset4dstem, DetectorPixelated, ObjectPixelated,
                                                  ProbePixelated, PtychoLite, Ptychography,
                                                  PtychographyDatasetRaster)

    z = load_golden("mixed64")
    H, nscan = int(z["H"]), int(z["nscan"])
    px, step = float(z["px"]), float(z["step_px"])
    rs = 1.0 / (H * px)
    S, P, seed, pad = int(z["S"]), int(z["P"]), int(z["seed"]), int(z["pad"])
    w = z["weights"] if z["weights"].size else None

    def d4():
        return Dataset4dstem.from_array(z["data"].reshape(nscan, nscan, H, H), sampling=(step * px, step * px, rs, rs),
                                        units=("A", "A", "A^-1", "A^-1"))

    lite = PtychoLite.from_dataset(d4(), num_slices=S, slice_thicknesses=float(z["dz"]), num_probes=P,
                                   energy=float(z["energy"]), defocus=200.0, semiangle_cutoff=20.0,
                                   initial_probe_weights=w, obj_padding_px=(pad, pad), device="gpu", verbose=0,
                                   rng=seed)
    assert lite.dset._preprocessed_on == "gpu"
    lite.reconstruct(num_iters=4, lr_obj=5e-3, lr_probe=1e-3, batch_size=16, verbose=0)

    pd = PtychographyDatasetRaster.from_dataset4dstem(d4())
    pd.preprocess(com_fit_function="constant", device="gpu")
    obj = ObjectPixelated.from_uniform(num_slices=S, slice_thicknesses=float(z["dz"]), obj_type="complex", rng=seed)
    probe = ProbePixelated.from_params(probe_params={"energy": float(z["energy"]), "defocus": 200.0,
                                                     "semiangle_cutoff": 20.0},
                                       num_probes=P, rng=seed, initial_probe_weights=w)
    pt = Ptychography.from_models(dset=pd, obj_model=obj, probe_model=probe, detector_model=DetectorPixelated(),
                                  device="gpu", verbose=0, rng=seed)
    pt.preprocess(obj_padding_px=(pad, pad))
    pt.reconstruct(num_iters=4, optimizer_params={"object": {"type": "adamw", "lr": 5e-3},
                                                  "probe": {"type": "adamw", "lr": 1e-3}},
                   scheduler_params={"object": {"type": "none"}, "probe": {"type": "none"}}, batch_size=16)
    a, b = np.asarray(lite.iter_losses), np.asarray(pt.iter_losses)
    assert a.shape == (4,) and np.all(np.isfinite(a))
    np.testing.assert_allclose(a, b, rtol=1e-6)
    assert a[-1] < a[0]


def test_ptycholite_dip_from_ptycholite(cuda_device):
    """PtychoLiteDIP.from_ptycholite (ptychography_lite.py:263-370): the object becomes
    a pre-trained ObjectDIP on the PtychoLite's dataset, probe and padding, and its
    flat-argument reconstruct optimises the network weights through the fused path."""
    from quantem_b200.diffractive_imaging import Dataset4dstem, ObjectDIP, PtychoLite, PtychoLiteDIP

    z = load_golden("mixed64")
    H, nscan = int(z["H"]), int(z["nscan"])
    px, step = float(z["px"]), float(z["step_px"])
    rs = 1.0 / (H * px)
    S, P, seed, pad = int(z["S"]), int(z["P"]), int(z["seed"]), int(z["pad"])
    w = z["weights"] if z["weights"].size else None
    d4 = Dataset4dstem.from_array(z["data"].reshape(nscan, nscan, H, H), sampling=(step * px, step * px, rs, rs),
                                  units=("A", "A", "A^-1", "A^-1"))
    lite = PtychoLite.from_dataset(d4, num_slices=S, slice_thicknesses=float(z["dz"]), num_probes=P,
                                   energy=float(z["energy"]), defocus=200.0, semiangle_cutoff=20.0,
                                   initial_probe_weights=w, obj_padding_px=(pad, pad), device="gpu", verbose=0,
                                   rng=seed)
    lite.reconstruct(num_iters=3, lr_obj=5e-3, lr_probe=1e-3, batch_size=16, verbose=0)

    dip = PtychoLiteDIP.from_ptycholite(lite, pretrain_iters=40, pretrain_lr=3e-3, device="gpu", verbose=0)
    assert isinstance(dip.obj_model, ObjectDIP)
    # a complex PtychoLite object gets a complex network, as in the reference
    from quantem_b200.core.ml.cnn import ComplexCNN2d

    assert isinstance(dip.obj_model.model, ComplexCNN2d) and dip.obj_model.obj_type == "complex"
    assert dip.probe_model is lite.probe_model and dip.dset is lite.dset
    assert tuple(dip.obj_model.obj.shape) == tuple(lite.obj_model.obj.shape)
    pl = dip.obj_model.pretrain_losses
    assert pl.shape == (40,) and pl[-1] < pl[0]
    w0 = dip.obj_model.model.flat.detach().clone()
    dip.reconstruct(num_iters=3, lr_obj=5e-4, lr_probe=5e-4, batch_size=16, verbose=0)
    losses = np.asarray(dip.iter_losses)
    assert losses.shape == (3,) and np.all(np.isfinite(losses))
    assert float((dip.obj_model.model.flat.detach() - w0).abs().max()) > 0
    with pytest.raises(ValueError):
        PtychoLiteDIP.from_ptycholite(lite, device="cpu")
