"""GPU parity of the sm_100a kernels against the FP64 oracle and the golden
fixtures produced by the reference.  Tolerances: forward intensities 1e-5
relative L2, gradients 1e-4 relative L2 (FP32 kernels vs FP64 / reference)."""
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


@pytest.mark.parametrize("n", [64, 128])
@pytest.mark.parametrize("inverse", [False, True])
def test_fft2_matches_numpy(cuda_device, n, inverse):
    from quantem_b200 import ops

    rng = np.random.default_rng(n + inverse)
    x = (rng.standard_normal((5, n, n)) + 1j * rng.standard_normal((5, n, n))).astype(np.complex64)
    got = ops.fft2(_t(x, cuda_device), inverse=inverse, scale=0.5).cpu().numpy()
    ref = (np.fft.ifft2(x.astype(np.complex128)) * n * n if inverse else np.fft.fft2(x.astype(np.complex128))) * 0.5
    assert rel(got, ref) < 2e-6


def test_obj_constrain_and_vjp(cuda_device):
    from quantem_b200 import ops

    rng = np.random.default_rng(3)
    shp = (3, 40, 56)
    obj = ((0.5 + rng.random(shp)) * np.exp(1j * rng.normal(size=shp))).astype(np.complex64)
    obj[0, 0, 0] = 0.0
    g = (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)).astype(np.complex64)
    o = _t(obj, cuda_device)
    out, work = ops.obj_constrain(o)
    ref = O.constrain_object(obj.astype(np.complex128))
    assert rel(out.cpu().numpy(), ref) < 1e-6
    gr = ops.obj_constrain_vjp(o, _t(g, cuda_device), work).cpu().numpy()
    gref = O.constrain_object_vjp(obj.astype(np.complex128), g.astype(np.complex128))
    assert rel(gr, gref) < 1e-5


def _golden_inputs(z, dev):
    S, P = int(z["S"]), int(z["P"])
    props = z["propagators"] if S > 1 else np.zeros((0, int(z["H"]), int(z["H"])), np.complex64)
    return dict(
        prop=_t(props, dev),
        positions=_t(z["positions"], dev, torch.float32),
        targets=_t(z["targets"], dev, torch.float32),
        mask=torch.ones((int(z["H"]),) * 2, device=dev, dtype=torch.float32),
        batch_idx=_t(z["batch_indices"].astype(np.int64), dev),
    )


@pytest.mark.parametrize("variant", ["serial", "cluster"])
@pytest.mark.parametrize("case", ["single64", "mixed64", "mixed128"])
def test_batch_forward_matches_reference(cuda_device, case, variant):
    from quantem_b200 import ops

    z = load_golden(case)
    dev = cuda_device
    inp = _golden_inputs(z, dev)
    obj_c, _ = ops.obj_constrain(_t(z["obj_perturbed"], dev))
    probe_o = _t(z["probe_ortho"], dev)
    out = ops.batch_forward(obj_c, probe_o, inp["prop"], inp["positions"], inp["batch_idx"], inp["targets"],
                            inp["mask"], int(z["positions"].shape[0]), float(z["mean_intensity"]), variant=variant)
    assert rel(out["intensity"].cpu().numpy(), z["batch_intensities"]) < TOL_I
    assert abs(out["loss"].item() - float(z["batch_loss"])) / float(z["batch_loss"]) < TOL_I


@pytest.mark.parametrize("variant", ["serial", "cluster"])
@pytest.mark.parametrize("case", ["single64", "mixed64", "mixed128"])
def test_batch_gradients_match_reference(cuda_device, case, variant):
    from quantem_b200 import ops
    from quantem_b200.diffractive_imaging.ptycho_utils import orthogonalize_probes

    z = load_golden(case)
    dev = cuda_device
    inp = _golden_inputs(z, dev)
    obj = _t(z["obj_perturbed"], dev).requires_grad_(True)
    probe = _t(z["probe_init"], dev).requires_grad_(True)
    probe_o = orthogonalize_probes(probe) if int(z["orthogonalize"]) else probe
    loss = ops.batch_loss(obj, probe_o, inp["prop"], inp["positions"], inp["batch_idx"], inp["targets"],
                          inp["mask"], int(z["positions"].shape[0]), float(z["mean_intensity"]), variant=variant)
    loss.backward()
    g_obj = obj.grad.cpu().numpy() * float(z["upsample_factor"]) ** 2 / 2
    assert abs(loss.item() - float(z["batch_loss"])) / float(z["batch_loss"]) < TOL_I
    assert rel(g_obj, z["grad_obj"]) < TOL_G
    assert rel(probe.grad.cpu().numpy(), z["grad_probe"]) < TOL_G


def _c2_like(rng, S=8, P=4, n=128, Ho=512, B=6):
    obj = (np.exp(1j * 0.3 * rng.standard_normal((S, Ho, Ho))) * (1 - 0.2 * rng.random((S, Ho, Ho))))
    probe = rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))
    probe *= np.exp(-((np.fft.fftfreq(n) * n)[:, None] ** 2 + (np.fft.fftfreq(n) * n)[None] ** 2) / 200.0)
    props = O.propagators((n, n), (0.2, 0.2), 300e3, [20.0] * (S - 1))
    positions = rng.uniform(0, Ho, size=(B, 2)).astype(np.float32).astype(np.float64)
    targets = np.abs(rng.standard_normal((B, n, n))) * 3
    return obj, probe, props, positions, targets


@pytest.mark.parametrize("variant", ["serial", "cluster"])
def test_c2_geometry_matches_fp64_oracle(cuda_device, variant):
    """512^2 x 8 slices, 4 modes at 128^2 (the multislice mixed-probe configuration)."""
    from quantem_b200 import ops

    rng = np.random.default_rng(7)
    obj, probe, props, positions, targets = _c2_like(rng)
    dev = cuda_device
    B = positions.shape[0]
    mean_i = 50.0
    npos = 4096
    obj_c = O.constrain_object(obj)
    loss_o, g_obj_o, g_probe_o, st = O.batch_loss_and_grads(obj_c, probe, positions, props, targets,
                                                            np.ones((128, 128)), npos, mean_i)
    I_o = O.detector_intensities(st)
    pos_full = np.zeros((npos, 2)); pos_full[:B] = positions
    tg_full = np.zeros((npos, 128, 128)); tg_full[:B] = targets
    args = (_t(obj_c.astype(np.complex64), dev), _t(probe.astype(np.complex64), dev),
            _t(props.astype(np.complex64), dev), _t(pos_full, dev, torch.float32),
            torch.arange(B, device=dev, dtype=torch.int64), _t(tg_full, dev, torch.float32),
            torch.ones((128, 128), device=dev), npos, mean_i)
    out = ops.batch_forward(*args, variant=variant)
    assert rel(out["intensity"].cpu().numpy(), I_o) < TOL_I
    loss, g_obj, g_probe = ops.batch_forward_adjoint(*args, variant=variant)
    assert abs(loss.item() - loss_o) / loss_o < TOL_I
    assert rel(g_obj.cpu().numpy(), g_obj_o) < TOL_G
    assert rel(g_probe.cpu().numpy(), g_probe_o) < TOL_G


@pytest.mark.parametrize("variant", ["serial", "cluster"])
def test_c2_geometry_separable_propagators(cuda_device, variant):
    """Same geometry with the propagators passed as per-axis factors (shared-memory path)."""
    from quantem_b200 import ops

    rng = np.random.default_rng(8)
    obj, probe, props, positions, targets = _c2_like(rng)
    dev = cuda_device
    B, npos, mean_i = positions.shape[0], 4096, 50.0
    kr, kc = ops.separable_propagators(128, (0.2, 0.2), 300e3, [20.0] * 7, device=dev)
    full = (kr[:, :, None] * kc[:, None, :]).cpu().numpy()
    assert rel(full, props) < 1e-6
    obj_c = O.constrain_object(obj)
    loss_o, g_obj_o, g_probe_o, st = O.batch_loss_and_grads(obj_c, probe, positions, props, targets,
                                                            np.ones((128, 128)), npos, mean_i)
    pos_full = np.zeros((npos, 2)); pos_full[:B] = positions
    tg_full = np.zeros((npos, 128, 128)); tg_full[:B] = targets
    args = (_t(obj_c.astype(np.complex64), dev), _t(probe.astype(np.complex64), dev), (kr, kc),
            _t(pos_full, dev, torch.float32), torch.arange(B, device=dev, dtype=torch.int64),
            _t(tg_full, dev, torch.float32), torch.ones((128, 128), device=dev), npos, mean_i)
    out = ops.batch_forward(*args, variant=variant)
    assert rel(out["intensity"].cpu().numpy(), O.detector_intensities(st)) < TOL_I
    loss, g_obj, g_probe = ops.batch_forward_adjoint(*args, variant=variant)
    assert abs(loss.item() - loss_o) / loss_o < TOL_I
    assert rel(g_obj.cpu().numpy(), g_obj_o) < TOL_G
    assert rel(g_probe.cpu().numpy(), g_probe_o) < TOL_G


def test_adam_matches_torch(cuda_device):
    from quantem_b200 import ops

    torch.manual_seed(0)
    p = torch.randn(1000, dtype=torch.complex64, device=cuda_device)
    p_ref = p.clone().requires_grad_(True)
    opt = torch.optim.Adam([p_ref], lr=5e-3)
    m = torch.zeros_like(p); v = torch.zeros_like(p)
    for step in range(1, 4):
        g = torch.randn_like(p)
        p_ref.grad = g.clone()
        opt.step()
        ops.adam_step(p, g, m, v, step, 5e-3)
    assert rel(p.cpu().numpy(), p_ref.detach().cpu().numpy()) < 1e-6


@pytest.mark.parametrize("case", ["single64", "mixed64", "mixed128"])
def test_analytic_update_matches_reference(cuda_device, case):
    """autograd=False update directions (ptychography.py:339-372) against the
    reference's own analytic gradients recorded at the same state."""
    from quantem_b200 import ops
    from quantem_b200.diffractive_imaging.ptycho_utils import orthogonalize_probes

    z = load_golden(case)
    dev = cuda_device
    inp = _golden_inputs(z, dev)
    obj_c, _ = ops.obj_constrain(_t(z["obj_perturbed"], dev))
    probe = _t(z["probe_init"], dev)
    probe_o = orthogonalize_probes(probe) if int(z["orthogonalize"]) else probe
    loss, g_obj, g_probe = ops.batch_analytic(obj_c, probe_o.contiguous(), inp["prop"], inp["positions"],
                                              inp["batch_idx"], inp["targets"], inp["mask"],
                                              int(z["positions"].shape[0]), float(z["mean_intensity"]))
    assert abs(loss.item() - float(z["batch_loss"])) / float(z["batch_loss"]) < TOL_I
    assert rel(g_obj.cpu().numpy(), z["grad_obj_an"]) < TOL_G
    assert rel(g_probe.cpu().numpy(), z["grad_probe_an"]) < TOL_G


@pytest.mark.parametrize("n", [64, 96])
@pytest.mark.parametrize("loss_type", O.LOSS_TYPES)
def test_loss_types_match_fp64_oracle(cuda_device, n, loss_type):
    """Every consistency loss of the reference (ptychography_base.py:908-932) through the
    fused forward + adjoint kernel, with a partial detector mask: loss, object and probe
    gradients against the FP64 oracle, whose losses are pinned to the reference's own
    error_estimate (tests/golden/loss_types.npz)."""
    from quantem_b200 import ops

    rng = np.random.default_rng(23)
    S, P, Ho, B, npos, mean_i = 2, 2, 160, 6, 300, 20.0
    obj = np.exp(1j * 0.3 * rng.standard_normal((S, Ho, Ho))) * (1 - 0.2 * rng.random((S, Ho, Ho)))
    probe = rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))
    probe *= np.exp(-((np.fft.fftfreq(n) * n)[:, None] ** 2 + (np.fft.fftfreq(n) * n)[None] ** 2) / 150.0)
    props = O.propagators((n, n), (0.2, 0.2), 300e3, [20.0] * (S - 1))
    positions = rng.uniform(0, Ho, size=(B, 2)).astype(np.float32).astype(np.float64)
    targets = np.abs(rng.standard_normal((B, n, n))) * (2.0 if "amplitude" in loss_type else 6.0)
    mask = (rng.random((n, n)) > 0.15).astype(np.float64)
    obj_c = O.constrain_object(obj)
    loss_o, g_obj_o, g_probe_o, _ = O.batch_loss_and_grads(obj_c, probe, positions, props, targets, mask, npos,
                                                           mean_i, loss_type)
    dev = cuda_device
    args = (_t(obj_c.astype(np.complex64), dev), _t(probe.astype(np.complex64), dev),
            _t(props.astype(np.complex64), dev), _t(positions, dev, torch.float32),
            torch.arange(B, device=dev, dtype=torch.int64), _t(targets, dev, torch.float32),
            _t(mask, dev, torch.float32), npos, mean_i)
    loss, g_obj, g_probe = ops.batch_forward_adjoint(*args, loss_type=loss_type)
    assert abs(loss.item() - loss_o) / abs(loss_o) < TOL_I
    assert rel(g_obj.cpu().numpy(), g_obj_o) < TOL_G
    assert rel(g_probe.cpu().numpy(), g_probe_o) < TOL_G


def test_status_word_reports_invalid_indices_and_nonfinite(cuda_device):
    """The batch kernels skip positions whose index is outside [0, npos) and count them,
    and count non-finite predicted intensities; ops.check_status surfaces both."""
    import warnings

    from quantem_b200 import ops

    rng = np.random.default_rng(5)
    S, P, n, Ho, B, npos = 2, 1, 64, 96, 3, 3
    obj = np.exp(1j * 0.2 * rng.standard_normal((S, Ho, Ho)))
    probe = (rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))) * 0.5
    props = O.propagators((n, n), (0.2, 0.2), 300e3, [20.0] * (S - 1))
    pos = rng.uniform(0, Ho, (npos, 2))
    tg = np.abs(rng.standard_normal((npos, n, n)))
    dev = cuda_device
    args = dict(prop=_t(props.astype(np.complex64), dev), positions=_t(pos, dev, torch.float32),
                targets=_t(tg, dev, torch.float32), mask=torch.ones((n, n), device=dev), num_gpts=npos,
                mean_intensity=2.0)
    obj_t, probe_t = _t(O.constrain_object(obj).astype(np.complex64), dev), _t(probe.astype(np.complex64), dev)
    ops.read_status(dev)  # start clean
    ops.batch_forward_adjoint(obj_t, probe_t, batch_idx=torch.tensor([0, 5, 1], device=dev), **args)
    st = ops.read_status(dev, reset=False)
    assert st["invalid_indices"] == 1 and st["nonfinite"] == 0
    with pytest.raises(RuntimeError, match="outside"):
        ops.check_status(dev)
    assert ops.read_status(dev)["raw"] == 0  # cleared by the check
    bad = obj_t.clone()
    bad[0, 0:Ho, 0:Ho] = float("nan")
    ops.batch_forward_adjoint(bad, probe_t, batch_idx=torch.arange(B, device=dev), **args)
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        st = ops.check_status(dev)
    assert st["nonfinite"] > 0 and st["invalid_indices"] == 0
    assert any("not finite" in str(x.message) for x in w)


def test_status_word_saturates_without_reporting_bad_indices(cuda_device):
    """A NaN object over more than 2^20 predicted pixels (80 positions x 128^2) fills the
    non-finite field of the status word to its maximum; the count must not carry into
    the invalid-index field, so check_status warns and does not raise."""
    import warnings

    from quantem_b200 import ops

    rng = np.random.default_rng(9)
    S, P, n, Ho, B = 1, 1, 128, 256, 80
    dev = cuda_device
    obj = torch.full((S, Ho, Ho), float("nan"), dtype=torch.complex64, device=dev)
    probe = _t(((rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))) * 0.5).astype(np.complex64),
               dev)
    pos = _t(rng.uniform(0, Ho, (B, 2)), dev, torch.float32)
    tg = _t(np.abs(rng.standard_normal((B, n, n))), dev, torch.float32)
    ops.read_status(dev)  # start clean
    ops.batch_forward_adjoint(obj, probe, torch.empty((0, n, n), dtype=torch.complex64, device=dev), pos,
                              torch.arange(B, device=dev), tg, torch.ones((n, n), device=dev), B, 2.0)
    st = ops.read_status(dev, reset=False)
    assert B * n * n > ops.STATUS_NONFINITE_MASK
    assert st["nonfinite"] == ops.STATUS_NONFINITE_MASK and st["invalid_indices"] == 0
    with warnings.catch_warnings(record=True):
        warnings.simplefilter("always")
        ops.check_status(dev)  # warns, does not raise
    assert ops.read_status(dev)["raw"] == 0


@pytest.mark.parametrize("n", [128, 256])
@pytest.mark.parametrize("B", [1, 2])
def test_small_batches_at_the_object_edge(cuda_device, n, B):
    """Batches smaller than the grid (one or two positions) whose windows wrap around the
    object's edges (periodic patch indices, dataset_models.py:514-535): loss and
    gradients against the FP64 oracle."""
    from quantem_b200 import ops

    rng = np.random.default_rng(31 + n + B)
    S, P, Ho = 2, 2, n + 64
    obj = np.exp(1j * 0.3 * rng.standard_normal((S, Ho, Ho))) * (1 - 0.2 * rng.random((S, Ho, Ho)))
    probe = rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))
    probe *= np.exp(-((np.fft.fftfreq(n) * n)[:, None] ** 2 + (np.fft.fftfreq(n) * n)[None] ** 2) / (n * 2.0))
    props = O.propagators((n, n), (0.2, 0.2), 300e3, [20.0] * (S - 1))
    edge = np.array([[1.3, Ho - 2.6], [Ho - 0.4, 3.7]])[:B].astype(np.float32).astype(np.float64)  # both edges
    targets = np.abs(rng.standard_normal((B, n, n))) * 2
    obj_c = O.constrain_object(obj)
    npos, mean_i = 50, 10.0
    loss_o, g_obj_o, g_probe_o, _ = O.batch_loss_and_grads(obj_c, probe, edge, props, targets, np.ones((n, n)),
                                                           npos, mean_i)
    dev = cuda_device
    loss, g_obj, g_probe = ops.batch_forward_adjoint(
        _t(obj_c.astype(np.complex64), dev), _t(probe.astype(np.complex64), dev), _t(props.astype(np.complex64), dev),
        _t(edge, dev, torch.float32), torch.arange(B, device=dev, dtype=torch.int64), _t(targets, dev, torch.float32),
        torch.ones((n, n), device=dev), npos, mean_i)
    assert abs(loss.item() - loss_o) / abs(loss_o) < TOL_I
    assert rel(g_obj.cpu().numpy(), g_obj_o) < TOL_G
    assert rel(g_probe.cpu().numpy(), g_probe_o) < TOL_G


@pytest.mark.parametrize("n", [64, 96, 128, 256])
def test_rectangular_object(cuda_device, n):
    """Objects with Ho != Wo (row and column wrap maps, row pitch Wo): forward intensities,
    loss and gradients against the FP64 oracle for every built window size."""
    from quantem_b200 import ops

    rng = np.random.default_rng(7 + n)
    S, P, B, npos, mean_i = 2, 2, 4, 40, 10.0
    Ho, Wo = n + 40, n + 104
    obj = np.exp(1j * 0.3 * rng.standard_normal((S, Ho, Wo))) * (1 - 0.2 * rng.random((S, Ho, Wo)))
    probe = rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))
    probe *= np.exp(-((np.fft.fftfreq(n) * n)[:, None] ** 2 + (np.fft.fftfreq(n) * n)[None] ** 2) / (n * 2.0))
    props = O.propagators((n, n), (0.2, 0.2), 300e3, [20.0] * (S - 1))
    pos = np.stack([rng.uniform(0, Ho, B), rng.uniform(0, Wo, B)], -1).astype(np.float32).astype(np.float64)
    targets = np.abs(rng.standard_normal((B, n, n))) * 2
    obj_c = O.constrain_object(obj)
    loss_o, g_obj_o, g_probe_o, st = O.batch_loss_and_grads(obj_c, probe, pos, props, targets, np.ones((n, n)),
                                                            npos, mean_i)
    dev = cuda_device
    args = (_t(obj_c.astype(np.complex64), dev), _t(probe.astype(np.complex64), dev),
            _t(props.astype(np.complex64), dev), _t(pos, dev, torch.float32),
            torch.arange(B, device=dev, dtype=torch.int64), _t(targets, dev, torch.float32),
            torch.ones((n, n), device=dev), npos, mean_i)
    out = ops.batch_forward(*args)
    assert rel(out["intensity"].cpu().numpy(), O.detector_intensities(st)) < TOL_I
    loss, g_obj, g_probe = ops.batch_forward_adjoint(*args)
    assert abs(loss.item() - loss_o) / abs(loss_o) < TOL_I
    assert rel(g_obj.cpu().numpy(), g_obj_o) < TOL_G
    assert rel(g_probe.cpu().numpy(), g_probe_o) < TOL_G


@pytest.mark.parametrize("P,n", [(1, 64), (2, 96), (4, 128), (6, 256)])
def test_probe_orthogonalization_kernels_match_fp64_oracle(cuda_device, P, n):
    """ptycho_probe_orthogonalize / _vjp (probe_models.py:484-525) against the FP64 oracle's
    Gram-Schmidt and its reverse mode, through orthogonalize_probes and torch autograd."""
    from quantem_b200.diffractive_imaging.ptycho_utils import orthogonalize_probes

    rng = np.random.default_rng(P * 1000 + n)
    probe = (rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))) * rng.uniform(0.2, 2.0, (P, 1, 1))
    probe = probe.astype(np.complex64).astype(np.complex128)
    gs = (rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n)))
    out_o, order_o, cache = O.gram_schmidt(probe)
    g_o = O.gram_schmidt_vjp(cache, gs)
    pt = torch.tensor(probe, dtype=torch.complex64, device=cuda_device, requires_grad=True)
    out = orthogonalize_probes(pt)
    assert rel(out.detach().cpu().numpy(), out_o) < TOL_I
    # a real loss whose gradient w.r.t. the output is gs (torch convention)
    loss = torch.sum(torch.real(torch.conj(torch.tensor(gs, dtype=torch.complex64, device=cuda_device)) * out))
    loss.backward()
    assert rel(pt.grad.cpu().numpy(), g_o) < TOL_G


@pytest.mark.parametrize("kind,kw", [
    ("adam", {"amsgrad": True}), ("adamw", {"amsgrad": True, "weight_decay": 0.05}),
    ("sgd", {"momentum": 0.9}), ("sgd", {"momentum": 0.8, "dampening": 0.3, "weight_decay": 0.01}),
    ("sgd", {"momentum": 0.9, "nesterov": True})])
def test_fused_optimiser_options_match_torch(cuda_device, kind, kw):
    """AMSGrad and SGD momentum / dampening / Nesterov of the fused optimisers against
    torch.optim on complex parameters (optimizer_mixin.py:117-123)."""
    from quantem_b200 import engine

    torch.manual_seed(1)
    p = torch.randn(3000, dtype=torch.complex64, device=cuda_device).requires_grad_(True)
    p_ref = p.detach().clone().requires_grad_(True)
    lr = 5e-3 if kind != "sgd" else 0.05
    ref_cls = {"adam": torch.optim.Adam, "adamw": torch.optim.AdamW, "sgd": torch.optim.SGD}[kind]
    opt_ref = ref_cls([p_ref], lr=lr, **kw)
    opt = engine.make_optimizer([p], {"type": kind, "lr": lr, **kw})
    for _ in range(5):
        g = torch.randn_like(p)
        p.grad, p_ref.grad = g.clone(), g.clone()
        opt.step()
        opt_ref.step()
    assert rel(p.detach().cpu().numpy(), p_ref.detach().cpu().numpy()) < 1e-6
