"""The reference's analysis members of ``Ptychography`` on the GPU: far-field intensity
and amplitude estimates from exit waves (ptychography_base.py:949-968), the consistency
error of predicted intensities (ptychography_base.py:908-932) and ``backward``
(ptychography.py:317-348), against torch FP32 restatements and the fused batch kernel."""
import numpy as np
import pytest
import torch

from tests.conftest import load_golden, rel
from tests.test_host_setup import build_from_golden

pytestmark = pytest.mark.gpu


def _problem(dev, case="mixed64"):
    z = load_golden(case)
    pt = build_from_golden(z, device="gpu")
    pt.dset.scan_positions_px = torch.as_tensor(z["positions"])
    pt.obj_model._obj = torch.as_tensor(z["obj_perturbed"]).to(dev).requires_grad_(True)
    pt.probe_model._probe = torch.as_tensor(z["probe_init"]).to(dev).requires_grad_(True)
    return z, pt


@pytest.mark.parametrize("case", ["single64", "mixed64"])
def test_estimates_and_error_match_the_batch_kernel(cuda_device, case):
    z, pt = _problem(cuda_device, case)
    batch = np.arange(0, pt.dset.num_gpts, 3)
    _, exits = pt.forward_operator(batch_indices=batch)
    ex = exits.detach()
    ref = torch.fft.fft2(ex, norm="ortho")
    inten = pt.estimate_intensities(ex)
    assert rel(inten.cpu().numpy(), ref.abs().square().sum(0).cpu().numpy()) < 1e-5
    amps = pt.estimate_amplitudes(ex)
    ref_amps = torch.fft.fftshift(torch.sqrt((ref + 1e-9).abs().square().sum(0)), dim=(-2, -1))
    assert rel(amps.cpu().numpy(), ref_amps.cpu().numpy()) < 1e-5
    assert rel(pt.estimate_amplitudes(ex, corner_centered=True).cpu().numpy(),
               torch.fft.ifftshift(ref_amps, dim=(-2, -1)).cpu().numpy()) < 1e-5
    # the fused kernel's predicted intensities are in the detector layout (the reference's
    # DetectorPixelated fftshifts the corner-centred estimate), and its batch loss is the
    # error estimate of those intensities
    pred, loss = pt.forward_intensities(batch)
    det = torch.fft.fftshift(inten, dim=(-2, -1))
    assert rel(pred.cpu().numpy(), det.cpu().numpy()) < 1e-5
    err, targets = pt.error_estimate(det, batch)
    assert targets.shape == det.shape
    assert abs(float(err) - float(loss)) <= 1e-4 * abs(float(loss))
    for lt in ("l1_amplitude", "l2_intensity", "l1_intensity", "poisson"):
        err_lt, _ = pt.error_estimate(pred, batch, loss_type=lt)
        _, loss_lt = pt.forward_intensities(batch, loss_type=lt)
        assert abs(float(err_lt) - float(loss_lt)) <= 1e-4 * abs(float(loss_lt))


def test_backward_rescales_the_pixelated_object_gradient(cuda_device):
    from quantem_b200 import ops

    z, pt = _problem(cuda_device)
    prop, pos, tg, mask = pt._batch_tensors()
    bi = torch.arange(0, pt.dset.num_gpts, 2, device=cuda_device)
    obj, probe = pt.obj_model._obj, pt.probe_model._probe

    def loss():
        return ops.batch_loss(obj, probe, prop, pos, bi, tg, mask, pt.dset.num_gpts,
                              pt.dset.mean_diffraction_intensity, "l2_amplitude")

    loss().backward()
    g_obj, g_probe = obj.grad.clone(), probe.grad.clone()
    obj.grad = probe.grad = None
    pt.backward(loss())
    # the object gradient is a scatter-add whose float32 atomics land in any order
    assert rel(obj.grad.cpu().numpy(), (g_obj * (pt.dset.upsample_factor ** 2 / 2)).cpu().numpy()) < 1e-5
    assert rel(probe.grad.cpu().numpy(), g_probe.cpu().numpy()) < 1e-5
    with pytest.raises(NotImplementedError):
        pt.backward(loss(), autograd=False)


@pytest.mark.parametrize("case", ["single64", "mixed64"])
def test_overlap_projection_and_fourier_projection(cuda_device, case):
    """overlap_projection on gathered patches against the batch kernel's own waves and exit
    waves; fourier_projection / gradient_step against a torch FP32 restatement of
    ptychography.py:350-372, and a zero step where the measured amplitudes are the estimate."""
    z, pt = _problem(cuda_device, case)
    batch = np.arange(0, pt.dset.num_gpts, 4)
    waves, exits = pt.forward_operator(batch_indices=batch)
    n = int(z["H"])
    obj_t = pt.obj_model.transmission().detach()
    pos = pt.dset.scan_positions_px.detach().to(cuda_device)[torch.as_tensor(batch, device=cuda_device)]
    origin = torch.round(pos).to(torch.int64)
    fr = torch.as_tensor(np.fft.fftfreq(n, d=1.0 / n).astype(np.int64), device=cuda_device)
    rows = (origin[:, 0, None] + fr[None]) % obj_t.shape[-2]
    cols = (origin[:, 1, None] + fr[None]) % obj_t.shape[-1]
    patches = obj_t[:, rows[:, :, None], cols[:, None, :]]  # (S, B, n, n)
    got_w, got_e = pt.overlap_projection(patches, waves[0])
    assert rel(got_w.cpu().numpy(), waves.cpu().numpy()) < 1e-5
    assert rel(got_e.cpu().numpy(), exits.cpu().numpy()) < 1e-5
    amps = pt.dset.targets[torch.as_tensor(batch, device=pt.dset.targets.device)].to(cuda_device)
    proj = pt.fourier_projection(amps, exits)
    meas = torch.fft.fftshift(amps, dim=(-2, -1))
    far = torch.fft.fft2(exits, norm="ortho")
    if exits.shape[0] == 1:
        ref = torch.fft.ifft2(meas * torch.exp(1j * torch.angle(far)), norm="ortho")
    else:
        est = torch.sqrt((far + 1e-9).abs().square().sum(0))
        est[est == 0] = torch.inf
        ref = torch.fft.ifft2((meas / est)[None] * far, norm="ortho")
    assert rel(proj.cpu().numpy(), ref.cpu().numpy()) < 1e-5
    assert rel(pt.gradient_step(amps, exits).cpu().numpy(), (ref - exits).cpu().numpy()) < 1e-4
    step = pt.gradient_step(pt.estimate_amplitudes(exits), exits)
    assert float(step.abs().square().sum().sqrt()) < 1e-4 * float(exits.abs().square().sum().sqrt())


@pytest.mark.parametrize("case", ["complex", "potential"])
def test_object_model_helpers_match_the_constraint_path(cuda_device, case):
    """ObjectPixelated.apply_hard_constraints on an arbitrary array equals the model's own
    constrained object; the TV / surface / blur / Butterworth helpers equal the oracle."""
    from oracle import ptycho_oracle as O
    from tests.test_gpu_objconstraints import _dropin
    from tests.test_oracle_golden import OBJCONS_CASES

    obj_type, cons = OBJCONS_CASES[case]
    z = load_golden(f"objcons_{case}64")
    pt = _dropin(z, cuda_device, obj_type)
    pt.constraints = {"object": dict(cons)}
    om = pt.obj_model
    mask = om.mask
    got = om.apply_hard_constraints(om._obj, mask)
    assert torch.equal(got.detach(), om.obj.detach())
    x = got.detach()
    xs = x.cpu().numpy().astype(np.complex128 if obj_type != "potential" else np.float64)
    tv = om.get_tv_loss(x, (0.02, 0.05))
    tv_o, _ = O.soft_constraint_loss(xs, obj_type, 0.02, 0.05, 0.0)
    assert abs(tv.item() - tv_o) <= 1e-5 * abs(tv_o)
    sz = om.get_surface_zero_loss(x, 0.01)
    sz_o, _ = O.soft_constraint_loss(xs, obj_type, 0.0, 0.0, 0.01)
    assert abs(sz.item() - sz_o) <= 1e-5 * max(abs(sz_o), 1e-6)
    bl = om.gaussian_blur_2d(x, 1.3)
    assert rel(bl.cpu().numpy(), O.blur(xs, O.gaussian_taps(1.3))) < 1e-5
    om.add_constraint("q_lowpass", 1.4)
    bw = om.butterworth_constraint(x, om._sampling)
    env = O.butterworth_env(x.shape[-2:], om._sampling, 1.4, om.constraints.get("q_highpass"),
                            om.constraints.get("butterworth_order", 4))
    assert rel(bw.cpu().numpy(), O.butterworth(xs, env)) < 1e-5
