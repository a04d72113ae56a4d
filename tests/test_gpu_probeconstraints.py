"""The optional probe constraints on the GPU (probe_models.py:430-482): the centre-of-mass
shift and its gradient, the TV soft loss and its gradient, against the FP64 oracle, and the
drop-in reconstruction with them against the reference's own run (fixtures
probecons_*64, made by tests/golden/make_golden.py).  Tolerances: the constrained probe 1e-5
relative L2 (float32 FFTs), gradients 1e-4."""
import numpy as np
import pytest
import torch

from oracle import ptycho_oracle as O
from tests.conftest import load_golden, rel
from tests.test_oracle_golden import PROBECONS_CASES

pytestmark = pytest.mark.gpu


def _probe(rng, P, n):
    y, x = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    base = np.exp(-(((y - 7.3) % n) ** 2 + ((x - n + 5.6) % n) ** 2) / (0.02 * n * n))  # off-centre blob
    return np.stack([base * np.exp(1j * 0.2 * (k + 1) * x) * (1.0 - 0.2 * k)
                     + 0.03 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) for k in range(P)])


@pytest.mark.parametrize("n", [64, 96, 128, 256])
@pytest.mark.parametrize("P", [1, 3])
def test_center_probe_kernels_match_fp64_oracle(cuda_device, n, P):
    from quantem_b200.diffractive_imaging.ptycho_utils import center_probe

    rng = np.random.default_rng(7 * n + P)
    p = _probe(rng, P, n)
    g = rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))
    ref, cache = O.center_probe(p)
    ref_g = O.center_probe_vjp(cache, g)
    x = torch.as_tensor(p.astype(np.complex64), device=cuda_device).requires_grad_(True)
    out = center_probe(x)
    assert rel(out.detach().cpu().numpy(), ref) < 1e-5
    out.backward(torch.as_tensor(g.astype(np.complex64), device=cuda_device))
    assert rel(x.grad.cpu().numpy(), ref_g) < 1e-4


@pytest.mark.parametrize("n", [64, 128])
@pytest.mark.parametrize("P", [1, 4])
def test_probe_tv_kernel_matches_fp64_oracle(cuda_device, n, P):
    from quantem_b200.diffractive_imaging.ptycho_utils import probe_tv_loss

    rng = np.random.default_rng(11 * n + P)
    p = _probe(rng, P, n)
    p[:, :3, :3] = 0.0  # equal neighbours: zero differences take a zero gradient
    loss_o, g_o = O.probe_tv_loss(p, 0.3)
    x = torch.as_tensor(p.astype(np.complex64), device=cuda_device).requires_grad_(True)
    loss = probe_tv_loss(x, 0.3)
    assert abs(loss.item() - loss_o) <= 1e-5 * abs(loss_o)
    (2.5 * loss).backward()
    assert rel(x.grad.cpu().numpy(), 2.5 * g_o) < 1e-5


def test_probe_constraint_kernels_are_deterministic(cuda_device):
    from quantem_b200.diffractive_imaging.ptycho_utils import center_probe, probe_tv_loss

    rng = np.random.default_rng(3)
    p = torch.as_tensor(_probe(rng, 4, 128).astype(np.complex64), device=cuda_device)
    a = [center_probe(p) for _ in range(2)]
    b = [probe_tv_loss(p, 0.1) for _ in range(2)]
    assert torch.equal(a[0], a[1]) and torch.equal(b[0], b[1])


def _dropin(z, dev):
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
    obj = ObjectPixelated.from_uniform(num_slices=int(z["S"]), slice_thicknesses=float(z["dz"]), obj_type="complex")
    probe = ProbePixelated.from_params(probe_params={"energy": float(z["energy"]), "defocus": 200.0,
                                                     "semiangle_cutoff": 20.0},
                                       num_probes=int(z["P"]), rng=132, initial_probe_weights=list(z["weights"]))
    pt = Ptychography.from_models(dset=pd, obj_model=obj, probe_model=probe, detector_model=DetectorPixelated(),
                                  device="gpu", verbose=0, rng=133)
    pt.preprocess(obj_padding_px=(int(z["pad"]), int(z["pad"])))
    pt.probe_model._probe = torch.as_tensor(z["probe_init"]).to(dev).requires_grad_(True)
    pt.obj_model._obj = torch.as_tensor(z["obj_perturbed"]).to(dev).requires_grad_(True)
    return pt


@pytest.mark.parametrize("case", sorted(PROBECONS_CASES))
def test_constrained_probe_and_batch_gradients_match_reference(cuda_device, case):
    from quantem_b200 import ops

    cons = PROBECONS_CASES[case]
    z = load_golden(f"probecons_{case}64")
    dev = cuda_device
    pt = _dropin(z, dev)
    pt.constraints = {"probe": dict(cons)}
    pm = pt.probe_model
    probe_c = pm.probe
    assert rel(probe_c.detach().cpu().numpy(), z["probe_constrained"]) < 2e-5
    soft = pm.apply_soft_constraints(probe_c)
    assert abs(soft.item() - float(z["probe_soft_loss"])) <= 1e-5 * max(float(z["probe_soft_loss"]), 1e-3)
    H = int(z["H"])
    obj_in, spec = pt.obj_model.batch_object()
    loss = ops.batch_loss(obj_in, probe_c, ops.dense(pt.propagators.to(dev)),
                          torch.as_tensor(z["positions"], device=dev),
                          torch.as_tensor(z["batch_indices"].astype(np.int64), device=dev),
                          torch.as_tensor(z["targets"], device=dev), torch.ones((H, H), device=dev),
                          int(z["positions"].shape[0]), float(z["mean_intensity"]), obj_spec=spec)
    total = loss + soft
    total.backward()
    assert abs(total.item() - float(z["batch_total_loss"])) / float(z["batch_total_loss"]) < 1e-5
    up = float(z["upsample_factor"]) ** 2 / 2
    assert rel(pt.obj_model._obj.grad.cpu().numpy() * up, z["grad_obj"]) < 2e-4
    assert rel(pm._probe.grad.cpu().numpy(), z["grad_probe"]) < 2e-4


@pytest.mark.parametrize("case", sorted(PROBECONS_CASES))
def test_reconstruct_with_probe_constraints_like_reference(cuda_device, case):
    """Two Adam iterations through Ptychography.reconstruct with the probe constraints: loss
    trajectory against the reference's, object and probe against the FP64 oracle within 3x
    the reference's own float32 drift from it."""
    cons = PROBECONS_CASES[case]
    z = load_golden(f"probecons_{case}64")
    dev = cuda_device
    pt = _dropin(z, dev)
    pt.rng = int(z["recon_rng_seed"])
    pt.reconstruct(num_iters=int(z["iters"]), batch_size=int(z["batch"]),
                   optimizer_params={"object": {"type": "adam"}, "probe": {"type": "adam"}},
                   constraints={"probe": dict(cons)}, device="gpu")
    np.testing.assert_allclose(pt.iter_losses, z["recon_losses"], rtol=1e-4)
    H = int(z["H"])
    obj64, probe64, _ = O.reconstruct(
        z["obj_perturbed"].astype(np.complex128), z["probe_init"].astype(np.complex128),
        z["positions"].astype(np.float64), z["propagators"].astype(np.complex128), z["targets"].astype(np.float64),
        np.ones((H, H)), float(z["mean_intensity"]), float(z["upsample_factor"]), int(z["iters"]), int(z["batch"]),
        np.random.default_rng(int(z["recon_rng_seed"])), probe_constraints=cons)
    for mine, ref, truth in ((pt.obj_model._obj, z["recon_obj"], obj64), (pt.probe_model._probe, z["recon_probe"],
                                                                           probe64)):
        assert rel(mine.detach().cpu().numpy(), truth) < max(3 * rel(ref, truth), 1e-5)
