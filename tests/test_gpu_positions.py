"""Learned scan positions on the CUDA path (dataset_models.py:30-120, 1482-1499): the
positions enter only through the fractional probe shift, and the fused adjoint returns
dL/d(position) of every batch entry.  Checked against the FP64 oracle (which is pinned to
finite differences and to the reference's autograd) and against the reference's own
reconstruction with a dataset optimiser (fixture positions64, learn_descan=False)."""
import numpy as np
import pytest
import torch

from oracle import ptycho_oracle as O
from tests.conftest import load_golden, rel

pytestmark = pytest.mark.gpu


def _t(x, dev, dtype=None):
    return torch.as_tensor(np.ascontiguousarray(x), device=dev, dtype=dtype)


@pytest.mark.parametrize("n,S,P", [(64, 2, 2), (96, 3, 1), (128, 8, 4)])
def test_position_gradients_match_fp64_oracle(cuda_device, n, S, P):
    from quantem_b200 import ops

    rng = np.random.default_rng(40 + n)
    Ho, B = n + 96, 5
    obj = np.exp(1j * 0.3 * rng.standard_normal((S, Ho, Ho))) * (1 - 0.2 * rng.random((S, Ho, Ho)))
    probe = rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))
    probe *= np.exp(-((np.fft.fftfreq(n) * n)[:, None] ** 2 + (np.fft.fftfreq(n) * n)[None] ** 2) / (n * 2.0))
    props = O.propagators((n, n), (0.2, 0.2), 300e3, [20.0] * (S - 1))
    pos = rng.uniform(0, Ho, size=(B, 2)).astype(np.float32).astype(np.float64)
    tg = np.abs(rng.standard_normal((B, n, n))) * 3
    obj_c = O.constrain_object(obj)
    loss_o, _, _, st = O.batch_loss_and_grads(obj_c, probe, pos, props, tg, np.ones((n, n)), 50, 20.0)
    g_ref = O.position_gradients(probe, st, st.g_probe_plane)
    dev = cuda_device
    gpos = torch.zeros((B, 2), device=dev)
    loss, _, _ = ops.batch_forward_adjoint(
        _t(obj_c.astype(np.complex64), dev), _t(probe.astype(np.complex64), dev),
        _t(props.astype(np.complex64), dev) if S > 1 else torch.zeros((0, n, n), dtype=torch.complex64, device=dev),
        _t(pos, dev, torch.float32), torch.arange(B, device=dev), _t(tg, dev, torch.float32),
        torch.ones((n, n), device=dev), 50, 20.0, grad_positions=gpos)
    assert abs(loss.item() - loss_o) / loss_o < 1e-5
    assert rel(gpos.cpu().numpy(), g_ref) < 1e-4


def test_position_gradients_match_reference(cuda_device):
    from quantem_b200 import ops
    from quantem_b200.diffractive_imaging.ptycho_utils import orthogonalize_probes

    z = load_golden("positions64")
    dev = cuda_device
    H = int(z["H"])
    positions = _t(z["positions"], dev, torch.float32).requires_grad_(True)
    loss = ops.batch_loss(_t(z["obj_perturbed"], dev), orthogonalize_probes(_t(z["probe_init"], dev)),
                          _t(z["propagators"], dev), positions, _t(z["batch_indices"].astype(np.int64), dev),
                          _t(z["targets"], dev, torch.float32), torch.ones((H, H), device=dev),
                          int(z["positions"].shape[0]), float(z["mean_intensity"]))
    loss.backward()
    assert abs(loss.item() - float(z["batch_loss"])) / float(z["batch_loss"]) < 1e-5
    g = positions.grad.cpu().numpy()
    assert rel(g, z["grad_positions"]) < 1e-4
    assert np.abs(g[len(z["batch_indices"]):]).max() == 0.0


def test_reconstruct_learns_positions_like_reference(cuda_device):
    """Ptychography.reconstruct with a dataset optimiser (Adam, lr 1e-2 px) from the
    reference run's start: loss trajectory, the position updates and the object against
    the FP64 oracle within 3x the reference's own float32 drift from it."""
    from quantem_b200.diffractive_imaging import (Dataset4dstem, DetectorPixelated, ObjectPixelated,
                                                  ProbePixelated, Ptychography, PtychographyDatasetRaster)

    z = load_golden("positions64")
    dev = cuda_device
    H, nscan = int(z["H"]), int(z["nscan"])
    px, step = float(z["px"]), float(z["step_px"])
    rs = 1.0 / (H * px)
    d4 = Dataset4dstem.from_array(z["data"].reshape(nscan, nscan, H, H), sampling=(step * px, step * px, rs, rs),
                                  units=("A", "A", "A^-1", "A^-1"))
    pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0, learn_descan=False)
    pd.preprocess(com_fit_function="constant", force_com_rotation=0, force_com_transpose=False,
                  probe_energy=float(z["energy"]), device="gpu")
    obj = ObjectPixelated.from_uniform(num_slices=int(z["S"]), slice_thicknesses=float(z["dz"]))
    probe = ProbePixelated.from_params(probe_params={"energy": float(z["energy"]), "defocus": 200.0,
                                                     "semiangle_cutoff": 20.0},
                                       num_probes=int(z["P"]), rng=int(z["seed"]) + 1,
                                       initial_probe_weights=list(z["weights"]))
    pt = Ptychography.from_models(dset=pd, obj_model=obj, probe_model=probe, detector_model=DetectorPixelated(),
                                  device="gpu", verbose=0, rng=int(z["seed"]) + 2)
    pt.preprocess(obj_padding_px=(int(z["pad"]), int(z["pad"])))
    pd.scan_positions_px = torch.as_tensor(z["positions"])
    pt.obj_model._obj = torch.as_tensor(z["obj_perturbed"]).to(dev).requires_grad_(True)
    pt.probe_model._probe = torch.as_tensor(z["probe_init"]).to(dev).requires_grad_(True)
    pt.rng = int(z["recon_rng_seed"])
    pt.reconstruct(num_iters=int(z["iters"]), batch_size=int(z["batch"]),
                   optimizer_params={"object": {"type": "adam"}, "probe": {"type": "adam"},
                                     "dataset": {"type": "adam", "lr": 1e-2}},
                   constraints={"probe": {"orthogonalize_probe": True}}, device="gpu")
    np.testing.assert_allclose(pt.iter_losses, z["recon_losses"], rtol=1e-4)
    obj64, probe64, _, pos64 = O.reconstruct(
        z["obj_perturbed"].astype(np.complex128), z["probe_init"].astype(np.complex128),
        z["positions"].astype(np.float64), z["propagators"].astype(np.complex128), z["targets"].astype(np.float64),
        np.ones((H, H)), float(z["mean_intensity"]), float(z["upsample_factor"]), int(z["iters"]), int(z["batch"]),
        np.random.default_rng(int(z["recon_rng_seed"])), lr_positions=1e-2)
    moved = pd.scan_positions_px.detach().cpu().numpy() - z["positions"]
    moved64 = pos64 - z["positions"]
    assert rel(moved, moved64) < max(3 * rel(z["recon_positions"] - z["positions"], moved64), 1e-3)
    assert rel(pt.obj_model._obj.detach().cpu().numpy(), obj64) < max(3 * rel(z["recon_obj"], obj64), 1e-5)
    # the reference's defaults learn the descan shifts and the positions together
    pd2 = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
    pd2.set_optimizer({"type": "adam", "lr": 1e-3})
    assert [tuple(p.shape) for p in pd2.optimizer.param_groups[0]["params"]] == [(nscan * nscan, 2)] * 2
    assert pd2.optimizer.param_groups[0]["params"][0] is pd2.descan_shifts
