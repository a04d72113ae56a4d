"""Pure-phase and potential objects (object_models.py:87, 123-136, 289-339, 252-256) on
the CUDA path: the transmission kernels and their VJP against the FP64 oracle, and the
batch loss / gradients / reconstruct trajectory against the reference's own run
(fixtures purephase64, potential64)."""
import numpy as np
import pytest
import torch

from oracle import ptycho_oracle as O
from tests.conftest import load_golden, rel

pytestmark = pytest.mark.gpu

TOL_I = 1e-5
TOL_G = 1e-4


def _t(x, dev, dtype=None):
    return torch.as_tensor(np.ascontiguousarray(x), device=dev, dtype=dtype)


@pytest.mark.parametrize("obj_type,positivity,fix", [("complex", True, False), ("pure_phase", True, False),
                                                      ("potential", True, False), ("potential", False, False),
                                                      ("potential", True, True)])
def test_transmission_and_vjp_match_fp64_oracle(cuda_device, obj_type, positivity, fix):
    from quantem_b200 import ops

    rng = np.random.default_rng(3)
    shape = (3, 70, 90)
    if obj_type == "potential":
        obj = (0.05 + 0.3 * rng.standard_normal(shape)).astype(np.float32)
    else:
        obj = ((1 - 0.4 * rng.random(shape)) * np.exp(1j * 0.7 * rng.standard_normal(shape))).astype(np.complex64)
        obj.flat[:5] *= 2.0  # amplitudes above 1: clamped (complex) or dropped (pure phase)
    g = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    spec = ops.ObjSpec(obj_type, positivity=positivity, fix_baseline=fix, baseline_factor=0.8)
    o64 = obj.astype(np.float64 if obj_type == "potential" else np.complex128)
    kw = dict(positivity=positivity, fix_baseline=fix, baseline_factor=0.8)
    t_ref = O.object_transmission(o64, obj_type, **kw)
    g_ref = O.object_transmission_vjp(o64, g.astype(np.complex128), obj_type, **kw)
    t, work = ops.obj_transmission(_t(obj, cuda_device), spec)
    gr = ops.obj_transmission_vjp(_t(obj, cuda_device), _t(g, cuda_device), work, spec,
                                  scale=torch.tensor(0.5, device=cuda_device))
    assert rel(t.cpu().numpy(), t_ref) < 1e-6
    assert gr.dtype == (torch.float32 if obj_type == "potential" else torch.complex64)
    assert rel(gr.cpu().numpy(), 0.5 * g_ref) < 1e-5


def _spec_of(z):
    from quantem_b200 import ops

    return ops.ObjSpec(str(z["obj_type"]))


@pytest.mark.parametrize("case", ["purephase64", "potential64"])
def test_batch_gradients_match_reference_object_types(cuda_device, case):
    from quantem_b200 import ops
    from quantem_b200.diffractive_imaging.ptycho_utils import orthogonalize_probes

    z = load_golden(case)
    dev = cuda_device
    H = int(z["H"])
    obj = _t(z["obj_perturbed"], dev).requires_grad_(True)
    probe = _t(z["probe_init"], dev).requires_grad_(True)
    loss = ops.batch_loss(obj, orthogonalize_probes(probe), _t(z["propagators"], dev),
                          _t(z["positions"], dev, torch.float32), _t(z["batch_indices"].astype(np.int64), dev),
                          _t(z["targets"], dev, torch.float32), torch.ones((H, H), device=dev),
                          int(z["positions"].shape[0]), float(z["mean_intensity"]), obj_spec=_spec_of(z))
    loss.backward()
    assert abs(loss.item() - float(z["batch_loss"])) / float(z["batch_loss"]) < TOL_I
    g_obj = obj.grad.cpu().numpy() * float(z["upsample_factor"]) ** 2 / 2
    assert rel(g_obj, z["grad_obj"]) < TOL_G
    assert rel(probe.grad.cpu().numpy(), z["grad_probe"]) < TOL_G


@pytest.mark.parametrize("case", ["purephase64", "potential64"])
def test_reconstruct_matches_reference_object_types(cuda_device, case):
    """Ptychography.reconstruct from the drop-in API with obj_type pure_phase / potential:
    the reference's loss trajectory, and the parameters within 3x the reference's own
    float32 drift from the FP64 oracle (floor 1e-5)."""
    from quantem_b200.diffractive_imaging import (Dataset4dstem, DetectorPixelated, ObjectPixelated,
                                                  ProbePixelated, Ptychography, PtychographyDatasetRaster)

    z = load_golden(case)
    dev = cuda_device
    H, nscan = int(z["H"]), int(z["nscan"])
    px, step = float(z["px"]), float(z["step_px"])
    rs = 1.0 / (H * px)
    d4 = Dataset4dstem.from_array(z["data"].reshape(nscan, nscan, H, H), sampling=(step * px, step * px, rs, rs),
                                  units=("A", "A", "A^-1", "A^-1"))
    pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
    pd.preprocess(com_fit_function="constant", force_com_rotation=0, force_com_transpose=False,
                  probe_energy=float(z["energy"]), device="gpu")
    obj = ObjectPixelated.from_uniform(num_slices=int(z["S"]), slice_thicknesses=float(z["dz"]),
                                       obj_type=str(z["obj_type"]))
    probe = ProbePixelated.from_params(probe_params={"energy": float(z["energy"]), "defocus": 200.0,
                                                     "semiangle_cutoff": 20.0},
                                       num_probes=int(z["P"]), rng=int(z["seed"]) + 1,
                                       initial_probe_weights=list(z["weights"]))
    pt = Ptychography.from_models(dset=pd, obj_model=obj, probe_model=probe, detector_model=DetectorPixelated(),
                                  device="gpu", verbose=0, rng=int(z["seed"]) + 2)
    pt.preprocess(obj_padding_px=(int(z["pad"]), int(z["pad"])))
    assert obj.dtype == (torch.float32 if str(z["obj_type"]) == "potential" else torch.complex64)
    pt.dset.scan_positions_px = torch.as_tensor(z["positions"])
    pt.obj_model._obj = torch.as_tensor(z["obj_perturbed"]).to(dev).requires_grad_(True)
    pt.probe_model._probe = torch.as_tensor(z["probe_init"]).to(dev).requires_grad_(True)
    pt.rng = int(z["recon_rng_seed"])
    pt.reconstruct(num_iters=int(z["iters"]), batch_size=int(z["batch"]),
                   optimizer_params={"object": {"type": "adam"}, "probe": {"type": "adam"}},
                   constraints={"probe": {"orthogonalize_probe": True}}, device="gpu")
    np.testing.assert_allclose(pt.iter_losses, z["recon_losses"], rtol=1e-4)
    fp = (lambda x: x.astype(np.float64)) if str(z["obj_type"]) == "potential" else (lambda x: x.astype(np.complex128))
    obj64, probe64, _ = O.reconstruct(fp(z["obj_perturbed"]), z["probe_init"].astype(np.complex128),
                                      z["positions"].astype(np.float64), z["propagators"].astype(np.complex128),
                                      z["targets"].astype(np.float64), np.ones((H, H)), float(z["mean_intensity"]),
                                      float(z["upsample_factor"]), int(z["iters"]), int(z["batch"]),
                                      np.random.default_rng(int(z["recon_rng_seed"])), obj_type=str(z["obj_type"]))
    # Adam's first steps move every parameter component by about lr * sign(gradient).  A
    # pure-phase object's gradient has no radial part, so the real (imaginary) component of
    # the gradient at pixels whose phase is near 0 (pi/2) is a small difference that float32
    # rounding flips in sign: any float32 path drifts further from FP64 there (floor 3e-5).
    floor = 3e-5 if str(z["obj_type"]) == "pure_phase" else 1e-5
    for mine, ref, truth in ((pt.obj_model._obj, z["recon_obj"], obj64), (pt.probe_model._probe, z["recon_probe"],
                                                                          probe64)):
        assert rel(mine.detach().cpu().numpy(), truth) < max(3 * rel(ref, truth), floor)
    if str(z["obj_type"]) == "potential":
        v = pt.obj  # the constrained potential: real, non-negative
        assert np.isrealobj(v) and v.min() >= 0.0


def _dropin_objtype(z, dev):
    from quantem_b200.diffractive_imaging import (Dataset4dstem, DetectorPixelated, ObjectPixelated,
                                                  ProbePixelated, Ptychography, PtychographyDatasetRaster)

    H, nscan = int(z["H"]), int(z["nscan"])
    px, step = float(z["px"]), float(z["step_px"])
    rs = 1.0 / (H * px)
    d4 = Dataset4dstem.from_array(z["data"].reshape(nscan, nscan, H, H), sampling=(step * px, step * px, rs, rs),
                                  units=("A", "A", "A^-1", "A^-1"))
    pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
    pd.preprocess(com_fit_function="constant", force_com_rotation=0, force_com_transpose=False,
                  probe_energy=float(z["energy"]), device="gpu")
    obj = ObjectPixelated.from_uniform(num_slices=int(z["S"]), slice_thicknesses=float(z["dz"]),
                                       obj_type=str(z["obj_type"]))
    probe = ProbePixelated.from_params(probe_params={"energy": float(z["energy"]), "defocus": 200.0,
                                                     "semiangle_cutoff": 20.0},
                                       num_probes=int(z["P"]), rng=int(z["seed"]) + 1,
                                       initial_probe_weights=list(z["weights"]))
    pt = Ptychography.from_models(dset=pd, obj_model=obj, probe_model=probe, detector_model=DetectorPixelated(),
                                  device="gpu", verbose=0, rng=int(z["seed"]) + 2)
    pt.preprocess(obj_padding_px=(int(z["pad"]), int(z["pad"])))
    pt.dset.scan_positions_px = torch.as_tensor(z["positions"])
    pt.obj_model._obj = torch.as_tensor(z["obj_perturbed"]).to(dev).requires_grad_(True)
    pt.probe_model._probe = torch.as_tensor(z["probe_init"]).to(dev).requires_grad_(True)
    return pt


@pytest.mark.parametrize("case", ["purephase64", "potential64"])
def test_analytic_update_of_object_types_through_reconstruct(cuda_device, case):
    """reconstruct(autograd=False) with pure-phase and potential objects: one full-batch pass
    with zero-step SGD leaves the analytic update directions in .grad; they equal the FP64
    oracle's (pinned to the reference's own analytic gradients of these object types)."""
    z = load_golden(case)
    pt = _dropin_objtype(z, cuda_device)
    obj_type = str(z["obj_type"])
    pt.reconstruct(num_iters=1, batch_size=pt.dset.num_gpts, autograd=False,
                   optimizer_params={"object": {"type": "sgd", "lr": 0.0}, "probe": {"type": "sgd", "lr": 0.0}},
                   constraints={"probe": {"orthogonalize_probe": True}}, device="gpu")
    raw = z["obj_perturbed"].astype(np.float64 if obj_type == "potential" else np.complex128)
    g_obj, g_probe, _ = O.analytic_gradients(raw, z["probe_init"].astype(np.complex128),
                                             z["positions"].astype(np.float64), z["propagators"].astype(np.complex128),
                                             z["targets"].astype(np.float64), orthogonalize=True, obj_type=obj_type)
    got = pt.obj_model._obj.grad
    assert got.dtype == (torch.float32 if obj_type == "potential" else torch.complex64)
    assert rel(got.cpu().numpy(), g_obj) < 1e-4
    assert rel(pt.probe_model._probe.grad.cpu().numpy(), g_probe) < 1e-4
