"""The headline geometry against the reference's own run (fixture c2small, made by
tests/golden/make_golden.py): 8 slices of 20 A, 4 probe modes at 128^2 with weights
0.7/0.15/0.1/0.05, a 512^2 object, +-0.5 px jitter, two windows wrapping both object
edges.  Tolerances: intensities 1e-5 relative L2, gradients 1e-4 relative L2 (FP32
kernels against the reference's float32 autograd and the FP64 oracle)."""
import numpy as np
import pytest
import torch

from oracle import ptycho_oracle as O
from tests.conftest import rel
from tests.golden.c2small import load_c2small, sampled
from tests.test_oracle_fd import fd_directional, random_directions

pytestmark = pytest.mark.gpu

TOL_I = 1e-5
TOL_G = 1e-4


def _t(x, dev, dtype=None):
    return torch.as_tensor(np.ascontiguousarray(x), device=dev, dtype=dtype)


@pytest.fixture(scope="module")
def z():
    return load_c2small()


def _inputs(z, dev):
    H = int(z["H"])
    return dict(prop=_t(z["propagators"], dev), positions=_t(z["positions"], dev, torch.float32),
                targets=_t(z["targets"], dev, torch.float32), mask=torch.ones((H, H), device=dev),
                batch_idx=_t(z["batch_indices"].astype(np.int64), dev))


@pytest.mark.parametrize("variant", ["serial", "cluster"])
def test_c2small_forward_matches_reference(cuda_device, z, variant):
    from quantem_b200 import ops

    inp = _inputs(z, cuda_device)
    obj_c, _ = ops.obj_constrain(_t(z["obj_perturbed"], cuda_device))
    out = ops.batch_forward(obj_c, _t(z["probe_ortho"], cuda_device), inp["prop"], inp["positions"],
                            inp["batch_idx"], inp["targets"], inp["mask"], int(z["positions"].shape[0]),
                            float(z["mean_intensity"]), variant=variant)
    assert rel(out["intensity"].cpu().numpy(), z["batch_intensities"]) < TOL_I
    assert abs(out["loss"].item() - float(z["batch_loss"])) / float(z["batch_loss"]) < TOL_I


def _cuda_raw_gradients(z, dev, obj_raw, probe_raw, variant="auto"):
    """Loss and gradients w.r.t. the raw object and probe through the drop-in chain:
    hard constraint, probe orthogonalisation, fused forward + adjoint, and the
    reference's object-gradient rescale upsample_factor^2 / 2."""
    from quantem_b200 import ops
    from quantem_b200.diffractive_imaging.ptycho_utils import orthogonalize_probes

    inp = _inputs(z, dev)
    obj = _t(obj_raw.astype(np.complex64), dev).requires_grad_(True)
    probe = _t(probe_raw.astype(np.complex64), dev).requires_grad_(True)
    loss = ops.batch_loss(obj, orthogonalize_probes(probe), inp["prop"], inp["positions"], inp["batch_idx"],
                          inp["targets"], inp["mask"], int(z["positions"].shape[0]), float(z["mean_intensity"]),
                          variant=variant)
    loss.backward()
    g_obj = obj.grad.cpu().numpy().astype(np.complex128) * float(z["upsample_factor"]) ** 2 / 2
    return loss.item(), g_obj, probe.grad.cpu().numpy().astype(np.complex128)


@pytest.mark.parametrize("variant", ["serial", "cluster"])
def test_c2small_gradients_match_reference(cuda_device, z, variant):
    loss, g_obj, g_probe = _cuda_raw_gradients(z, cuda_device, z["obj_perturbed"], z["probe_init"], variant)
    assert abs(loss - float(z["batch_loss"])) / float(z["batch_loss"]) < TOL_I
    assert rel(sampled(g_obj, z["grad_idx"]), z["grad_obj_sampled"]) < TOL_G
    assert rel(g_probe, z["grad_probe"]) < TOL_G


@pytest.mark.parametrize("which", ["obj", "probe", "both"])
def test_c2small_gradients_match_fp64_finite_differences(cuda_device, z, which):
    """<CUDA gradient, d> against the FP64 central difference of the oracle's loss along
    random complex directions d (object amplitude scaled by 0.999, away from the |o| = 1
    clamp).  Bar: 1e-4 of |<g, d>| plus 1e-6 of |g| |d| (FP32 gradient rounding over
    ~10^6 components)."""
    obj_raw = z["obj_perturbed"].astype(np.complex128) * 0.999
    probe_raw = z["probe_init"].astype(np.complex128)
    _, g_obj, g_probe = _cuda_raw_gradients(z, cuda_device, obj_raw, probe_raw)
    g_obj = g_obj * 2.0 / float(z["upsample_factor"]) ** 2  # plain dL/d(obj) for the difference quotient
    rng = np.random.default_rng(7 + len(which))
    for _ in range(2):
        d_obj, d_probe = random_directions(rng, obj_raw, probe_raw, which)
        adj = float(np.sum(g_obj.real * d_obj.real + g_obj.imag * d_obj.imag)
                    + np.sum(g_probe.real * d_probe.real + g_probe.imag * d_probe.imag))
        fd = fd_directional(z, obj_raw, probe_raw, d_obj, d_probe, 1e-6)
        scale = np.sqrt(np.vdot(g_obj, g_obj).real + np.vdot(g_probe, g_probe).real) * np.sqrt(
            np.vdot(d_obj, d_obj).real + np.vdot(d_probe, d_probe).real)
        assert abs(adj - fd) <= 1e-4 * abs(fd) + 1e-6 * scale, (adj, fd)


def test_c2small_reconstruct_matches_reference(cuda_device, z):
    """Ptychography.reconstruct at the headline geometry (3 Adam iterations, batches of 5
    and 4 positions) from the reference run's start: the loss trajectory, and the object
    (sampled pixels) and probe against the FP64 oracle within 3x the reference's own
    float32 drift from it (floor 1e-5)."""
    from tests.test_host_setup import build_from_golden

    pt = build_from_golden(z, device="gpu")
    dev = cuda_device
    pt.dset.scan_positions_px = torch.as_tensor(z["positions"])
    pt.obj_model._obj = torch.as_tensor(z["obj_perturbed"]).to(dev).requires_grad_(True)
    pt.probe_model._probe = torch.as_tensor(z["probe_init"]).to(dev).requires_grad_(True)
    pt.rng = int(z["recon_rng_seed"])
    pt.reconstruct(num_iters=int(z["iters"]), batch_size=int(z["batch"]),
                   optimizer_params={"object": {"type": "adam"}, "probe": {"type": "adam"}},
                   constraints={"probe": {"orthogonalize_probe": True}}, device="gpu")
    np.testing.assert_allclose(pt.iter_losses, z["recon_losses"], rtol=1e-4)
    H = int(z["H"])
    obj64, probe64, _ = O.reconstruct(z["obj_perturbed"].astype(np.complex128), z["probe_init"].astype(np.complex128),
                                      z["positions"].astype(np.float64), z["propagators"].astype(np.complex128),
                                      z["targets"].astype(np.float64), np.ones((H, H)), float(z["mean_intensity"]),
                                      float(z["upsample_factor"]), int(z["iters"]), int(z["batch"]),
                                      np.random.default_rng(int(z["recon_rng_seed"])))
    idx = z["recon_idx"]
    mine_obj = sampled(pt.obj_model._obj.detach().cpu().numpy(), idx)
    truth_obj = sampled(obj64, idx)
    assert rel(mine_obj, truth_obj) < max(3 * rel(z["recon_obj_sampled"], truth_obj), 1e-5)
    mine_probe = pt.probe_model._probe.detach().cpu().numpy()
    assert rel(mine_probe, probe64) < max(3 * rel(z["recon_probe"], probe64), 1e-5)
