"""Learned descan shifts and probe tilt on the CUDA path.

Descan (ptychography_base.py:903-905, dataset_models.py:225-242, 1482-1499): the exit
wave of each position times the translation ramp of its descan shift, the targets the
uncentred patterns; the fused adjoint returns dL/d(descan) of every batch entry.
Probe tilt (probe_models.py:376-427): a per-axis phase ramp of every propagator; the
fused adjoint returns the per-slice sensitivities sum_k k Im(conj(dL/dZ) Z), from which
ops.tilt_gradient forms dL/d(tilt).  Checked against the FP64 oracle (pinned to finite
differences and to the reference's autograd) and against the reference's own
reconstruction with a dataset optimiser and learn_probe_tilt (fixture descantilt64)."""
import numpy as np
import pytest
import torch

from oracle import ptycho_oracle as O
from tests.conftest import load_golden, rel

pytestmark = pytest.mark.gpu


def _t(x, dev, dtype=None):
    return torch.as_tensor(np.ascontiguousarray(x), device=dev, dtype=dtype)


@pytest.mark.parametrize("n,S,P", [(64, 2, 2), (96, 3, 1), (128, 8, 4)])
def test_descan_and_propagator_gradients_match_fp64_oracle(cuda_device, n, S, P):
    from quantem_b200 import ops

    rng = np.random.default_rng(60 + n)
    Ho, B = n + 96, 5
    obj = np.exp(1j * 0.3 * rng.standard_normal((S, Ho, Ho))) * (1 - 0.2 * rng.random((S, Ho, Ho)))
    probe = rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))
    probe *= np.exp(-((np.fft.fftfreq(n) * n)[:, None] ** 2 + (np.fft.fftfreq(n) * n)[None] ** 2) / (n * 2.0))
    props = O.propagators((n, n), (0.2, 0.2), 300e3, [20.0] * (S - 1), tilt_mrad=(1.0, -2.0))
    pos = rng.uniform(0, Ho, size=(B, 2)).astype(np.float32).astype(np.float64)
    descan = rng.uniform(-0.8, 0.8, size=(B, 2)).astype(np.float32).astype(np.float64)
    tg = np.abs(rng.standard_normal((B, n, n))) * 3
    obj_c = O.constrain_object(obj)
    loss_o, g_obj_o, g_probe_o, st = O.batch_loss_and_grads(obj_c, probe, pos, props, tg, np.ones((n, n)), 50,
                                                            20.0, descan=descan)
    dev = cuda_device
    gd = torch.zeros((B, 2), device=dev)
    gp = torch.zeros((S - 1, 2), device=dev)
    args = (_t(obj_c.astype(np.complex64), dev), _t(probe.astype(np.complex64), dev),
            _t(props.astype(np.complex64), dev), _t(pos, dev, torch.float32), torch.arange(B, device=dev),
            _t(tg, dev, torch.float32), torch.ones((n, n), device=dev), 50, 20.0)
    dsc = _t(descan, dev, torch.float32)
    loss, g_obj, g_probe = ops.batch_forward_adjoint(*args, descan=dsc, grad_descan=gd, grad_prop=gp)
    assert abs(loss.item() - loss_o) / loss_o < 1e-5
    assert rel(g_obj.cpu().numpy(), g_obj_o) < 1e-4
    assert rel(g_probe.cpu().numpy(), g_probe_o) < 1e-4
    assert rel(gd.cpu().numpy(), O.descan_gradients(st)) < 1e-4
    assert rel(gp.cpu().numpy(), st.prop_sums) < 1e-4
    # the forward-only kernel applies the same descan ramp
    out = ops.batch_forward(*args, descan=dsc)
    assert rel(out["intensity"].cpu().numpy(), np.fft.fftshift(st.intensity, axes=(-2, -1))) < 1e-5
    assert abs(out["loss"].item() - loss_o) / loss_o < 1e-5


def test_descan_and_tilt_gradients_match_reference(cuda_device):
    """ops.batch_loss with the descan shifts and the tilt as differentiable inputs, at the
    reference fixture's batch: loss, object / probe / descan / tilt gradients."""
    from quantem_b200 import ops
    from quantem_b200.diffractive_imaging.ptycho_utils import orthogonalize_probes

    z = load_golden("descantilt64")
    dev = cuda_device
    H, S = int(z["H"]), int(z["S"])
    geom = (H, tuple(float(x) for x in z["sampling"]), float(z["energy"]), [float(z["dz"])] * (S - 1))
    obj = _t(z["obj_perturbed"], dev).requires_grad_(True)
    probe = _t(z["probe_init"], dev).requires_grad_(True)
    descan = _t(z["descan"], dev, torch.float32).requires_grad_(True)
    tilt = _t(z["tilt"], dev, torch.float32).requires_grad_(True)
    loss = ops.batch_loss(obj, orthogonalize_probes(probe), None, _t(z["positions"], dev, torch.float32),
                          _t(z["batch_indices"].astype(np.int64), dev), _t(z["targets"], dev, torch.float32),
                          torch.ones((H, H), device=dev), int(z["positions"].shape[0]), float(z["mean_intensity"]),
                          descan=descan, tilt=tilt, prop_geometry=geom)
    loss.backward()
    assert abs(loss.item() - float(z["batch_loss"])) / float(z["batch_loss"]) < 1e-5
    up = float(z["upsample_factor"]) ** 2 / 2
    assert rel(obj.grad.cpu().numpy() * up, z["grad_obj"]) < 1e-4
    assert rel(probe.grad.cpu().numpy(), z["grad_probe"]) < 1e-4
    g = descan.grad.cpu().numpy()
    assert rel(g, z["grad_descan"]) < 1e-4
    assert np.abs(g[len(z["batch_indices"]):]).max() == 0.0
    assert rel(tilt.grad.cpu().numpy(), z["grad_tilt"]) < 1e-3  # the reference's float32 propagator phases


def test_zero_tilt_gets_no_gradient(cuda_device):
    """The reference multiplies the tilt ramp in only for a nonzero tilt, so autograd gives
    a zero tilt no gradient (probe_models.py:418-425)."""
    from quantem_b200 import ops
    from quantem_b200.diffractive_imaging.ptycho_utils import orthogonalize_probes

    z = load_golden("descantilt64")
    dev = cuda_device
    H, S = int(z["H"]), int(z["S"])
    geom = (H, tuple(float(x) for x in z["sampling"]), float(z["energy"]), [float(z["dz"])] * (S - 1))
    tilt = torch.tensor([0.0, 1.5], device=dev).requires_grad_(True)
    loss = ops.batch_loss(_t(z["obj_perturbed"], dev), orthogonalize_probes(_t(z["probe_init"], dev)), None,
                          _t(z["positions"], dev, torch.float32), _t(z["batch_indices"].astype(np.int64), dev),
                          _t(z["centered_targets"], dev, torch.float32), torch.ones((H, H), device=dev),
                          int(z["positions"].shape[0]), float(z["mean_intensity"]), tilt=tilt, prop_geometry=geom)
    loss.backward()
    g = tilt.grad.cpu().numpy()
    assert g[0] == 0.0 and g[1] != 0.0


def _dropin(z, dev, **dset_kw):
    from quantem_b200.diffractive_imaging import (Dataset4dstem, DetectorPixelated, ObjectPixelated,
                                                  ProbePixelated, Ptychography, PtychographyDatasetRaster)

    H, nscan = int(z["H"]), int(z["nscan"])
    px, step = float(z["px"]), float(z["step_px"])
    rs = 1.0 / (H * px)
    d4 = Dataset4dstem.from_array(z["data"].reshape(nscan, nscan, H, H), sampling=(step * px, step * px, rs, rs),
                                  units=("A", "A", "A^-1", "A^-1"))
    pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0, **dset_kw)
    pd.preprocess(com_fit_function="constant", force_com_rotation=0, force_com_transpose=False,
                  probe_energy=float(z["energy"]), device="gpu")
    obj = ObjectPixelated.from_uniform(num_slices=int(z["S"]), slice_thicknesses=float(z["dz"]))
    probe = ProbePixelated.from_params(probe_params={"energy": float(z["energy"]), "defocus": 200.0,
                                                     "semiangle_cutoff": 20.0},
                                       num_probes=int(z["P"]), rng=int(z["seed"]) + 1,
                                       initial_probe_weights=list(z["weights"]), probe_tilt=tuple(z["tilt"]),
                                       learn_probe_tilt=True)
    pt = Ptychography.from_models(dset=pd, obj_model=obj, probe_model=probe, detector_model=DetectorPixelated(),
                                  device="gpu", verbose=0, rng=int(z["seed"]) + 2)
    pt.preprocess(obj_padding_px=(int(z["pad"]), int(z["pad"])))
    return pt, pd


def test_reconstruct_learns_descan_and_tilt_like_reference(cuda_device):
    """Ptychography.reconstruct with a dataset optimiser over the descan shifts (Adam, lr
    1e-2 px) and learn_probe_tilt (in the probe's Adam) from the reference run's start:
    set-up (uncentred targets), loss trajectory, descan / tilt updates and the object
    against the FP64 oracle within 3x the reference's own float32 drift from it."""
    z = load_golden("descantilt64")
    dev = cuda_device
    H, S = int(z["H"]), int(z["S"])
    pt, pd = _dropin(z, dev, learn_descan=True, learn_scan_positions=False)
    pd.descan_shifts = torch.as_tensor(z["descan"])
    pt.obj_model._obj = torch.as_tensor(z["obj_perturbed"]).to(dev).requires_grad_(True)
    pt.probe_model._probe = torch.as_tensor(z["probe_init"]).to(dev).requires_grad_(True)
    pt.rng = int(z["recon_rng_seed"])
    opt = {"object": {"type": "adam"}, "probe": {"type": "adam"}, "dataset": {"type": "adam", "lr": 1e-2}}
    pt.reconstruct(num_iters=int(z["iters"]), batch_size=int(z["batch"]), optimizer_params=opt,
                   constraints={"probe": {"orthogonalize_probe": True}}, device="gpu")
    assert rel(pd.targets.detach().cpu().numpy(), z["targets"]) < 1e-6  # the uncentred amplitudes
    np.testing.assert_allclose(pt.iter_losses, z["recon_losses"], rtol=1e-4)
    geom = ((H, H), tuple(z["sampling"]), float(z["energy"]), [float(z["dz"])] * (S - 1))
    obj64, _, _, learned = O.reconstruct(
        z["obj_perturbed"].astype(np.complex128), z["probe_init"].astype(np.complex128),
        z["positions"].astype(np.float64), O.propagators(*geom, tilt_mrad=tuple(z["tilt"])),
        z["targets"].astype(np.float64), np.ones((H, H)), float(z["mean_intensity"]), float(z["upsample_factor"]),
        int(z["iters"]), int(z["batch"]), np.random.default_rng(int(z["recon_rng_seed"])), descan=z["descan"],
        lr_descan=1e-2, tilt=z["tilt"], prop_geometry=geom)
    moved = pd.descan_shifts.detach().cpu().numpy() - z["descan"]
    moved64 = learned["descan"] - z["descan"]
    assert rel(moved, moved64) < max(3 * rel(z["recon_descan"] - z["descan"], moved64), 1e-3)
    dt = pt.probe_model.probe_tilt.detach().cpu().numpy() - z["tilt"]
    dt64 = learned["tilt"] - z["tilt"]
    assert rel(dt, dt64) < max(3 * rel(z["recon_tilt"] - z["tilt"], dt64), 1e-3)
    assert rel(pt.obj_model._obj.detach().cpu().numpy(), obj64) < max(3 * rel(z["recon_obj"], obj64), 1e-5)
    # the forward paths follow the learned descan and tilt
    inten, _ = pt.forward_intensities(np.arange(4))
    assert torch.isfinite(inten).all()


def test_reconstruct_with_reference_default_dataset_flags(cuda_device):
    """A dataset made with the reference's defaults (learn_descan and learn_scan_positions
    both True) and a dataset optimiser learns descan shifts and positions together; the
    descan_shifts_constant constraint freezes the shifts (zero shifts, no gradient)."""
    z = load_golden("descantilt64")
    dev = cuda_device
    pt, pd = _dropin(z, dev)
    d0 = pd.descan_shifts.detach().clone()
    p0 = pd.scan_positions_px.detach().clone()
    opt = {"object": {"type": "adam"}, "probe": {"type": "adam"}, "dataset": {"type": "adam", "lr": 1e-2}}
    pt.reconstruct(num_iters=2, batch_size=10, optimizer_params=opt, device="gpu")
    assert np.isfinite(pt.iter_losses).all()
    assert (pd.descan_shifts.detach() - d0.to(dev)).abs().max().item() > 1e-3
    assert (pd.scan_positions_px.detach() - p0.to(dev)).abs().max().item() > 1e-3
    pt2, pd2 = _dropin(z, dev)
    pt2.reconstruct(num_iters=1, batch_size=10, optimizer_params=opt, device="gpu",
                    constraints={"dataset": {"descan_shifts_constant": True}})
    assert torch.equal(pd2.descan_shifts.detach().cpu(), pd2.initial_descan_shifts.detach().cpu())


def test_extension_arguments_are_rejected_where_not_built(cuda_device):
    from quantem_b200 import ops

    dev = cuda_device
    n, S, P, B = 256, 2, 1, 2
    obj = torch.ones((S, 512, 512), dtype=torch.complex64, device=dev)
    probe = torch.ones((P, n, n), dtype=torch.complex64, device=dev)
    props = torch.ones((S - 1, n, n), dtype=torch.complex64, device=dev)
    pos = torch.full((B, 2), 200.0, device=dev)
    tg = torch.ones((B, n, n), device=dev)
    with pytest.raises(RuntimeError, match="256"):
        ops.batch_forward(obj, probe, props, pos, torch.arange(B, device=dev), tg, torch.ones((n, n), device=dev),
                          B, 1.0, descan=torch.zeros((B, 2), device=dev))
