"""Deep-image-prior object (ObjectDIP, object_models.py:728-1226) on the CNN and
batch kernels: the phase -> exp -> fused-loss chain against the FP64 oracle, network
pre-training to a target phase, and a DIP reconstruction through Ptychography."""
import numpy as np
import pytest
import torch

from oracle import ptycho_oracle as O
from tests.conftest import load_golden, rel
from tests.test_host_setup import build_from_golden

pytestmark = pytest.mark.gpu


def test_phase_chain_matches_fp64_oracle(cuda_device):
    """dL/dphi for obj = exp(i phi) through the fused adjoint + constraint VJP equals
    Re(conj(g_raw) i z) of the oracle (torch complex-gradient convention)."""
    from quantem_b200 import ops

    rng = np.random.default_rng(31)
    S, P, n, Ho, B = 2, 2, 64, 96, 6
    phi = 0.4 * rng.standard_normal((S, Ho, Ho))
    z = np.exp(1j * phi)
    probe = rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))
    probe *= np.exp(-((np.fft.fftfreq(n) * n)[:, None] ** 2 + (np.fft.fftfreq(n) * n)[None] ** 2) / 100.0)
    props = O.propagators((n, n), (0.2, 0.2), 300e3, [20.0] * (S - 1))
    pos = rng.uniform(0, Ho, size=(B, 2)).astype(np.float32).astype(np.float64)
    tg = np.abs(rng.standard_normal((B, n, n))) * 3
    obj_c = O.constrain_object(z)
    loss_o, g_c, _, _ = O.batch_loss_and_grads(obj_c, probe, pos, props, tg, np.ones((n, n)), 400, 30.0)
    g_raw = O.constrain_object_vjp(z, g_c)
    dphi_o = np.real(np.conj(g_raw) * 1j * z)
    dev = cuda_device
    phi_t = torch.tensor(phi, dtype=torch.float32, device=dev, requires_grad=True)
    zt = torch.polar(torch.ones_like(phi_t), phi_t)
    loss = ops.batch_loss(zt, torch.as_tensor(probe.astype(np.complex64), device=dev),
                          torch.as_tensor(props.astype(np.complex64), device=dev),
                          torch.as_tensor(pos, dtype=torch.float32, device=dev),
                          torch.arange(B, device=dev, dtype=torch.int64),
                          torch.as_tensor(tg, dtype=torch.float32, device=dev), torch.ones((n, n), device=dev),
                          400, 30.0)
    loss.backward()
    assert abs(loss.item() - loss_o) / loss_o < 1e-5
    assert rel(phi_t.grad.cpu().numpy(), dphi_o) < 1e-4


def test_dip_pretrain_and_reconstruct(cuda_device):
    from quantem_b200.core.ml.cnn import CNN2d
    from quantem_b200.diffractive_imaging import ObjectDIP, Ptychography

    z = load_golden("mixed64")
    base = build_from_golden(z, device="cuda")
    base.reconstruct(num_iters=2, optimizer_params={"object": {"type": "adam", "lr": 5e-3},
                                                    "probe": {"type": "adam", "lr": 1e-3}}, batch_size=8)
    S = base.obj_model.num_slices
    net = CNN2d(S, S, start_filters=8, num_layers=3, device=cuda_device, seed=2)
    dip = ObjectDIP.from_pixelated(net, base.obj_model, input_noise_std=0.0)
    with torch.no_grad():  # a visible target: the pixelated phase plus a smooth pattern
        yy = torch.linspace(-1, 1, dip.shape[1], device=cuda_device)
        dip.pretrain_target = dip.pretrain_target + 0.2 * torch.cos(3 * yy)[None, :, None]
    dip.pretrain(num_iters=60, optimizer_params={"type": "adam", "lr": 3e-3})
    pl = dip.pretrain_losses
    assert pl[-1] < 0.2 * pl[0]
    assert tuple(dip.obj.shape) == tuple(base.obj_model.shape) and dip.obj.dtype == torch.complex64

    pt = Ptychography.from_models(dset=base.dset, obj_model=dip, probe_model=base.probe_model,
                                  detector_model=base.detector_model, device="gpu", verbose=0, rng=3)
    pt.preprocess(obj_padding_px=base.obj_padding_px)
    # the network was pre-trained on the unmasked object: without the FOV mask (which the
    # preprocess sets and the batch path applies, tested below) the first iterations descend
    dip.mask = None
    w0 = net.flat.detach().clone()
    pt.reconstruct(num_iters=3, optimizer_params={"object": {"type": "adam", "lr": 1e-3}}, batch_size=8)
    losses = np.asarray(pt.iter_losses)
    assert losses.shape == (3,) and np.all(np.isfinite(losses))
    assert losses[-1] < losses[0]
    assert float((net.flat.detach() - w0).abs().max()) > 0  # the network weights are what moved


def test_complex_dip_chain_matches_fp64_oracle(cuda_device):
    """A complex network's output is the transmission itself (no hard constraint in the
    reference's DIP forward): dL/d(output) through the fused adjoint equals the oracle's
    batch gradient at that object."""
    from quantem_b200 import ops

    rng = np.random.default_rng(33)
    S, P, n, Ho, B = 2, 2, 64, 96, 6
    z = (1.1 - 0.4 * rng.random((S, Ho, Ho))) * np.exp(1j * 0.4 * rng.standard_normal((S, Ho, Ho)))
    probe = rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))
    probe *= np.exp(-((np.fft.fftfreq(n) * n)[:, None] ** 2 + (np.fft.fftfreq(n) * n)[None] ** 2) / 100.0)
    props = O.propagators((n, n), (0.2, 0.2), 300e3, [20.0] * (S - 1))
    pos = rng.uniform(0, Ho, size=(B, 2)).astype(np.float32).astype(np.float64)
    tg = np.abs(rng.standard_normal((B, n, n))) * 3
    loss_o, g_o, _, _ = O.batch_loss_and_grads(z, probe, pos, props, tg, np.ones((n, n)), 400, 30.0)
    dev = cuda_device
    zt = torch.tensor(z.astype(np.complex64), device=dev, requires_grad=True)
    loss = ops.batch_loss(zt, torch.as_tensor(probe.astype(np.complex64), device=dev),
                          torch.as_tensor(props.astype(np.complex64), device=dev),
                          torch.as_tensor(pos, dtype=torch.float32, device=dev),
                          torch.arange(B, device=dev, dtype=torch.int64),
                          torch.as_tensor(tg, dtype=torch.float32, device=dev), torch.ones((n, n), device=dev),
                          400, 30.0, obj_spec=ops.ObjSpec("complex", hard_constraint=False))
    loss.backward()
    assert abs(loss.item() - loss_o) / loss_o < 1e-5
    assert rel(zt.grad.cpu().numpy(), g_o) < 1e-4


def test_complex_dip_pretrain_and_reconstruct(cuda_device):
    """PtychoLiteDIP-style use with the reference's default complex object: a complex
    network (ComplexCNN2d) pre-trained on the pixelated complex object, then optimised
    through Ptychography.reconstruct."""
    from quantem_b200.core.ml.cnn import ComplexCNN2d
    from quantem_b200.diffractive_imaging import ObjectDIP, Ptychography

    z = load_golden("mixed64")
    base = build_from_golden(z, device="cuda")
    base.reconstruct(num_iters=2, optimizer_params={"object": {"type": "adam", "lr": 5e-3},
                                                    "probe": {"type": "adam", "lr": 1e-3}}, batch_size=8)
    S = base.obj_model.num_slices
    net = ComplexCNN2d(S, S, start_filters=8, num_layers=3, device=cuda_device, seed=4)
    dip = ObjectDIP.from_pixelated(net, base.obj_model, input_noise_std=0.0)
    assert dip.obj_type == "complex" and dip.model_input.dtype == torch.complex64
    dip.pretrain(num_iters=60, optimizer_params={"type": "adam", "lr": 3e-3})
    pl = dip.pretrain_losses
    assert pl[-1] < 0.2 * pl[0]
    assert tuple(dip.obj.shape) == tuple(base.obj_model.shape) and dip.obj.dtype == torch.complex64
    pt = Ptychography.from_models(dset=base.dset, obj_model=dip, probe_model=base.probe_model,
                                  detector_model=base.detector_model, device="gpu", verbose=0, rng=3)
    pt.preprocess(obj_padding_px=base.obj_padding_px)
    # the network was pre-trained on the unmasked object: without the FOV mask (which the
    # preprocess sets and the batch path applies, tested below) the first iterations descend
    dip.mask = None
    w0 = net.flat.detach().clone()
    pt.reconstruct(num_iters=3, optimizer_params={"object": {"type": "adam", "lr": 1e-3}}, batch_size=8)
    losses = np.asarray(pt.iter_losses)
    assert losses.shape == (3,) and np.all(np.isfinite(losses))
    assert losses[-1] < losses[0]
    assert float((net.flat.detach() - w0).abs().max()) > 0


def test_dip_batch_object_carries_the_fov_mask(cuda_device):
    """The reference's DIP forward multiplies the network output by the probe-overlap FOV
    mask whenever Ptychography.preprocess has set it (object_models.py:1005-1007); the
    object the batch kernels take does the same, while ``obj`` stays unmasked."""
    from quantem_b200.core.ml.cnn import CNN2d
    from quantem_b200.diffractive_imaging import ObjectDIP, Ptychography

    z = load_golden("mixed64")
    base = build_from_golden(z, device="cuda")
    S = base.obj_model.num_slices
    net = CNN2d(S, S, start_filters=8, num_layers=3, device=cuda_device, seed=2)
    dip = ObjectDIP.from_pixelated(net, base.obj_model, input_noise_std=0.0)
    pt = Ptychography.from_models(dset=base.dset, obj_model=dip, probe_model=base.probe_model,
                                  detector_model=base.detector_model, device="gpu", verbose=0, rng=3)
    pt.preprocess(obj_padding_px=base.obj_padding_px)
    m = dip.mask
    assert m is not None and float(m.min()) < 0.5 and float(m.max()) > 0.5
    with torch.no_grad():
        out = net(dip._noisy_input(False))[0]
        want = torch.polar(torch.ones_like(out), out * m.to(out.device))
        assert torch.allclose(dip._obj, want, atol=1e-6)
        assert not torch.allclose(dip._obj, torch.polar(torch.ones_like(out), out), atol=1e-3)


def test_dip_optional_constraints_act_on_obj_and_soft_terms(cuda_device):
    """On a DIP object the optional hard constraints shape ``obj`` (and the soft terms that
    read it) while the batch path keeps the masked network output, as the reference's DIP
    does (object_models.py:975-1008); checked against the FP64 oracle's constraint chain."""
    from quantem_b200.core.ml.cnn import CNN2d
    from quantem_b200.diffractive_imaging import ObjectDIP, Ptychography

    z = load_golden("mixed64")
    base = build_from_golden(z, device="cuda")
    S = base.obj_model.num_slices
    net = CNN2d(S, S, start_filters=8, num_layers=3, device=cuda_device, seed=5)
    dip = ObjectDIP.from_pixelated(net, base.obj_model, input_noise_std=0.0)
    pt = Ptychography.from_models(dset=base.dset, obj_model=dip, probe_model=base.probe_model,
                                  detector_model=base.detector_model, device="gpu", verbose=0, rng=3)
    pt.preprocess(obj_padding_px=base.obj_padding_px)
    cons = {"gaussian_sigma": 1.2, "apply_fov_mask": True, "tv_weight_xy": 0.05}
    pt.constraints = {"object": dict(cons)}
    with torch.no_grad():
        raw = dip.raw_object(noise=False).cpu().numpy().astype(np.complex128)
        assert dip.obj_type == "complex"  # a real network on a complex object: exp(i output)
        ext = O._ext_args(cons, dip.mask.cpu().numpy().astype(np.float64))
        want = O.constrain_object_ext(raw, "complex", **ext)
        assert rel(dip.obj.cpu().numpy(), want) < 2e-5
        out = net(dip._noisy_input(False))[0]
        assert torch.allclose(dip.batch_object()[0], torch.polar(torch.ones_like(out), out * dip.mask), atol=1e-6)
    w0 = net.flat.detach().clone()
    pt.reconstruct(num_iters=2, optimizer_params={"object": {"type": "adam", "lr": 1e-3}}, batch_size=8)
    assert np.all(np.isfinite(pt.iter_losses))
    assert float((net.flat.detach() - w0).abs().max()) > 0
