"""The drop-in API end to end on the GPU: ``Ptychography.reconstruct`` from the
same state as the reference run recorded in the golden fixtures."""
import numpy as np
import pytest
import torch

from oracle import ptycho_oracle as O
from tests.conftest import load_golden, rel
from tests.test_host_setup import build_from_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["single64", "mixed64"])
def test_reconstruct_matches_reference(cuda_device, case):
    z = load_golden(case)
    pt = build_from_golden(z, device="gpu")
    dev = cuda_device
    pt.dset.scan_positions_px = torch.as_tensor(z["positions"])
    pt.obj_model._obj = torch.as_tensor(z["obj_perturbed"]).to(dev).requires_grad_(True)
    pt.probe_model._probe = torch.as_tensor(z["probe_init"]).to(dev).requires_grad_(True)
    pt.rng = int(z["recon_rng_seed"])
    pt.reconstruct(num_iters=int(z["iters"]), batch_size=int(z["batch"]),
                   optimizer_params={"object": {"type": "adam"}, "probe": {"type": "adam"}},
                   constraints={"probe": {"orthogonalize_probe": bool(z["orthogonalize"])}}, device="gpu")
    np.testing.assert_allclose(pt.iter_losses, z["recon_losses"], rtol=1e-4)
    # Adam's first steps are ~lr * sign(g): float32 rounding of near-zero gradient
    # components flips some of them, so any float32 run drifts from the float64
    # trajectory.  Bound: 3x the reference's own measured drift from the FP64
    # oracle on the same case (floor 1e-5).
    H = int(z["H"])
    props = z["propagators"].astype(np.complex128) if int(z["S"]) > 1 else np.zeros((0, H, H))
    obj64, probe64, _ = O.reconstruct(z["obj_perturbed"].astype(np.complex128), z["probe_init"].astype(np.complex128),
                                      z["positions"].astype(np.float64), props, z["targets"].astype(np.float64),
                                      np.ones((H, H)), float(z["mean_intensity"]), float(z["upsample_factor"]),
                                      int(z["iters"]), int(z["batch"]), np.random.default_rng(int(z["recon_rng_seed"])))
    for mine, ref, truth in ((pt.obj_model._obj, z["recon_obj"], obj64), (pt.probe_model._probe, z["recon_probe"], probe64)):
        bound = max(3 * rel(ref, truth), 1e-5)
        assert rel(mine.detach().cpu().numpy(), truth) < bound


def test_reference_gradient_test_case_on_gpu(cuda_device):
    """The reference's own gradient-test inputs through the CUDA path (see
    tests/test_oracle_golden.py for why the gradient bar is set by float32
    conditioning here)."""
    from quantem_b200 import ops
    from quantem_b200.diffractive_imaging import Dataset4dstem, PtychographyDatasetRaster
    from tests.golden.whitenoise import whitenoise_inputs

    inp = whitenoise_inputs()
    z = load_golden("whitenoise64")
    N = inp["N"]
    d4 = Dataset4dstem.from_array(inp["data4d"], sampling=inp["sampling4d"], units=("A", "A", "A^-1", "A^-1"))
    pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
    pd.preprocess(com_fit_function="constant", force_com_rotation=0, force_com_transpose=False,
                  probe_energy=inp["energy"])
    dev = cuda_device
    probe = torch.as_tensor(z["probe_used_p1_ad"]).to(dev)
    obj = torch.ones((1, N, N), dtype=torch.complex64, device=dev)
    loss, g_obj, _ = ops.batch_forward_adjoint(
        ops.obj_constrain(obj)[0], probe, torch.zeros((0, N, N), dtype=torch.complex64, device=dev),
        pd.scan_positions_px.to(dev), torch.arange(pd.num_gpts, device=dev), pd.targets.to(dev),
        torch.ones((N, N), device=dev), pd.num_gpts, pd.mean_diffraction_intensity)
    assert abs(loss.item() - z["loss_p1_ad"][0]) / z["loss_p1_ad"][0] < 1e-5
    _, g_ref, _, _ = O.batch_loss_and_grads(np.ones((1, N, N), np.complex128),
                                            z["probe_used_p1_ad"].astype(np.complex128),
                                            pd.scan_positions_px.numpy().astype(np.float64), np.zeros((0, N, N)),
                                            pd.targets.numpy().astype(np.float64), np.ones((N, N)), pd.num_gpts,
                                            pd.mean_diffraction_intensity)
    assert rel(g_obj.cpu().numpy(), g_ref) < 2e-2


@pytest.mark.parametrize("case", ["single64", "mixed64"])
def test_reconstruct_analytic_matches_oracle(cuda_device, case):
    """reconstruct(autograd=False): one SGD iteration over seeded batches against
    the FP64 oracle applying the reference's analytic update directions."""
    z = load_golden(case)
    pt = build_from_golden(z, device="gpu")
    dev = cuda_device
    pt.dset.scan_positions_px = torch.as_tensor(z["positions"])
    pt.obj_model._obj = torch.as_tensor(z["obj_perturbed"]).to(dev).requires_grad_(True)
    pt.probe_model._probe = torch.as_tensor(z["probe_init"]).to(dev).requires_grad_(True)
    pt.rng = 7
    lr = 0.1
    pt.reconstruct(num_iters=1, batch_size=int(z["batch"]), autograd=False,
                   optimizer_params={"object": {"type": "sgd", "lr": lr}, "probe": {"type": "sgd", "lr": lr}},
                   constraints={"probe": {"orthogonalize_probe": bool(z["orthogonalize"])}}, device="gpu")
    H = int(z["H"])
    props = z["propagators"].astype(np.complex128) if int(z["S"]) > 1 else np.zeros((0, H, H))
    obj = z["obj_perturbed"].astype(np.complex128)
    probe = z["probe_init"].astype(np.complex128)
    pos = z["positions"].astype(np.float64)
    tg = z["targets"].astype(np.float64)
    for bi in O.batch_order(np.random.default_rng(7), pos.shape[0], int(z["batch"])):
        g_obj, g_probe, _ = O.analytic_gradients(obj, probe, pos[bi], props, tg[bi],
                                                 orthogonalize=bool(z["orthogonalize"]))
        obj = obj - lr * g_obj
        probe = probe - lr * g_probe
    assert rel(pt.obj_model._obj.detach().cpu().numpy(), obj) < 1e-5
    assert rel(pt.probe_model._probe.detach().cpu().numpy(), probe) < 1e-5


def test_graphed_iteration_matches_eager(cuda_device):
    """engine.GraphedIteration (the full-batch iteration captured in a CUDA graph, device-side
    Adam step counts) follows the eager batch_step + torch-style Adam trajectory."""
    from quantem_b200 import engine

    rng = np.random.default_rng(9)
    S, P, n, Ho, npos = 2, 2, 64, 128, 24
    dev = cuda_device
    obj0 = torch.tensor(np.exp(1j * 0.1 * rng.standard_normal((S, Ho, Ho))), dtype=torch.complex64, device=dev)
    probe0 = torch.tensor((rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))) * 0.3,
                          dtype=torch.complex64, device=dev)
    props = torch.tensor(O.propagators((n, n), (0.2, 0.2), 300e3, [20.0] * (S - 1)), dtype=torch.complex64,
                         device=dev)
    pos = torch.tensor(rng.uniform(32, 96, (npos, 2)), dtype=torch.float32, device=dev)
    tg = torch.tensor(np.abs(rng.standard_normal((npos, n, n))) * 2, dtype=torch.float32, device=dev)
    mask = torch.ones((n, n), device=dev)

    def problem():
        return engine.ProblemTensors(obj=obj0.clone().requires_grad_(True), probe=probe0.clone().requires_grad_(True),
                                     prop=props, positions=pos, targets=tg, mask=mask, mean_intensity=4.0,
                                     upsample_factor=2.0)

    pe = problem()
    opts = [engine.make_optimizer([pe.obj], {"type": "adam", "lr": 5e-3}),
            engine.make_optimizer([pe.probe], {"type": "adam", "lr": 1e-3})]
    idx = torch.arange(npos, device=dev)
    le, ge = [], None
    for k in range(4):
        le.append(float(engine.batch_step(pe, idx, opts)))
        if k == 0:
            ge = (pe.obj.grad.detach().cpu().numpy(), pe.probe.grad.detach().cpu().numpy())
    pg = problem()
    it = engine.GraphedIteration(pg, batch_idx=idx).capture(warmup=0)
    lg, gg = [], None
    for k in range(4):
        lg.append(float(it.replay()))
        if k == 0:
            gg = (pg.obj.grad.detach().cpu().numpy(), pg.probe.grad.detach().cpu().numpy())
    # the first step's gradients to the gradient tolerance, the loss trajectory to 1e-5 (the
    # parameters themselves are not compared: Adam's first steps move every pixel by about
    # lr whatever the size of its gradient, so weakly lit pixels follow rounding noise)
    assert rel(gg[0], ge[0]) < 1e-4 and rel(gg[1], ge[1]) < 1e-4
    np.testing.assert_allclose(lg, le, rtol=1e-5)


def test_host_resident_targets_match_device_targets(cuda_device):
    """dset.keep_targets_on_host: the targets stay in pinned host memory and reconstruct
    copies them to the GPU every iteration; the trajectory equals the device-resident one
    (up to the order of the float atomics), and the pinned copy is built once, not per call."""
    z = load_golden("mixed64")
    runs = []
    for host in (False, True):
        pt = build_from_golden(z, device="gpu")
        pt.dset.scan_positions_px = torch.as_tensor(z["positions"])
        pt.obj_model._obj = torch.as_tensor(z["obj_perturbed"]).to(cuda_device).requires_grad_(True)
        pt.probe_model._probe = torch.as_tensor(z["probe_init"]).to(cuda_device).requires_grad_(True)
        pt.rng = int(z["recon_rng_seed"])
        if host:
            pt.dset.keep_targets_on_host(True)
        pt.reconstruct(num_iters=2, batch_size=int(z["batch"]),
                       optimizer_params={"object": {"type": "adam"}, "probe": {"type": "adam"}}, device="gpu")
        if host:
            tg = pt.dset.targets
            assert tg.device.type == "cpu" and tg.is_pinned()
            assert pt.last_h2d_bytes_per_iter == tg.numel() * 4
        pt.reconstruct(num_iters=2, batch_size=int(z["batch"]), device="gpu")
        if host:
            assert pt.dset.targets is tg  # kept across reconstruct calls
        runs.append((np.asarray(pt.iter_losses), pt.obj_model._obj.detach().cpu().numpy()))
    np.testing.assert_allclose(runs[1][0], runs[0][0], rtol=1e-6)
    assert rel(runs[1][1], runs[0][1]) < 1e-5


def test_deferred_loss_readback_matches_per_iteration_readback(cuda_device):
    """loss_readback='auto' (every iteration's loss read once at the end of the call, nothing
    consuming it in between) gives the same losses and parameters as reading each iteration."""
    z = load_golden("mixed64")
    out = {}
    for mode in ("iteration", "auto"):
        pt = build_from_golden(z, device="gpu")
        pt.dset.scan_positions_px = torch.as_tensor(z["positions"])
        pt.obj_model._obj = torch.as_tensor(z["obj_perturbed"]).to(cuda_device).requires_grad_(True)
        pt.probe_model._probe = torch.as_tensor(z["probe_init"]).to(cuda_device).requires_grad_(True)
        pt.rng = int(z["recon_rng_seed"])
        pt.loss_readback = mode
        pt.reconstruct(num_iters=4, batch_size=int(z["batch"]),
                       optimizer_params={"object": {"type": "adam"}, "probe": {"type": "adam"}}, device="gpu")
        out[mode] = pt
    a, b = out["iteration"], out["auto"]
    assert len(b.iter_losses) == 4
    np.testing.assert_allclose(b.iter_losses, a.iter_losses, rtol=1e-6)
    assert rel(b.obj_model._obj.detach().cpu().numpy(), a.obj_model._obj.detach().cpu().numpy()) < 1e-5
