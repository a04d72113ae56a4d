"""Resume on the GPU: 2 iterations, save, load, 2 more iterations equal 4 uninterrupted
iterations.  The object gradient is accumulated with float atomics, whose order varies
from run to run, so two uninterrupted runs may already differ in the last bits; the
resumed run must sit within that run-to-run spread (and match exactly when the
uninterrupted runs do)."""
import numpy as np
import pytest
import torch

from tests.conftest import load_golden, rel
from tests.test_host_setup import build_from_golden

pytestmark = pytest.mark.gpu

OPT = {"object": {"type": "adam"}, "probe": {"type": "adam"}}


def _fresh(z):
    pt = build_from_golden(z, device="gpu")
    dev = torch.device("cuda", 0)
    pt.dset.scan_positions_px = torch.as_tensor(z["positions"])
    pt.obj_model._obj = torch.as_tensor(z["obj_perturbed"]).to(dev).requires_grad_(True)
    pt.probe_model._probe = torch.as_tensor(z["probe_init"]).to(dev).requires_grad_(True)
    pt.rng = int(z["recon_rng_seed"])
    return pt


def _state(pt):
    return (pt.obj_model._obj.detach().cpu().numpy(), pt.probe_model._probe.detach().cpu().numpy(),
            np.asarray(pt.iter_losses))


@pytest.mark.parametrize("raw", [True, False])
def test_resume_equals_uninterrupted(cuda_device, tmp_path, raw):
    from quantem_b200.diffractive_imaging import Ptychography

    z = load_golden("mixed64")
    bs = 7  # 25 positions: 4 batches per iteration, the last one short
    runs = []
    for _ in range(2):
        pt = _fresh(z)
        pt.reconstruct(num_iters=4, batch_size=bs, optimizer_params=OPT, device="gpu")
        runs.append(_state(pt))
    pt = _fresh(z)
    pt.reconstruct(num_iters=2, batch_size=bs, optimizer_params=OPT, device="gpu")
    path = tmp_path / "mid.pt"
    pt.save(path, save_raw_data=raw, verbose=False)
    q = Ptychography.from_file(path, dset=None if raw else _fresh(z).dset, device="gpu")
    del pt
    assert q.num_iters == 2
    q.reconstruct(num_iters=2, device="gpu")
    obj, probe, losses = _state(q)
    (obj_a, probe_a, losses_a), (obj_b, probe_b, losses_b) = runs
    assert losses.shape == (4,)
    spread = max(rel(obj_b, obj_a), rel(probe_b, probe_a))
    if spread == 0.0:
        np.testing.assert_array_equal(losses, losses_a)
    np.testing.assert_allclose(losses, losses_a, rtol=1e-6)
    assert rel(obj, obj_a) <= 3 * spread + 1e-6
    assert rel(probe, probe_a) <= 3 * spread + 1e-6


@pytest.mark.parametrize("complex_net", [False, True])
def test_dip_resume_equals_uninterrupted(cuda_device, tmp_path, complex_net):
    """A DIP reconstruction (real or complex network, input noise on) saved after 2 iterations
    comes back exactly (network weights and batch-norm statistics, Adam moments and step, the
    input-noise generator), and 2 more iterations from the loaded copy equal 2 more from the
    saved one.  The BF16 GEMMs reduce split-K partials with float atomics, so two continuations
    of the same state differ by the run-to-run spread, measured on two uninterrupted runs."""
    from quantem_b200.core.ml.cnn import CNN2d, ComplexCNN2d
    from quantem_b200.diffractive_imaging import ObjectDIP, Ptychography

    z = load_golden("mixed64")
    opt = {"object": {"type": "adam", "lr": 1e-3}, "probe": {"type": "adam"}}

    def fresh():
        base = _fresh(z)
        S = base.obj_model.num_slices
        net = (ComplexCNN2d if complex_net else CNN2d)(S, S, start_filters=8, num_layers=3, device=cuda_device,
                                                       seed=7)
        dip = ObjectDIP.from_pixelated(net, base.obj_model, input_noise_std=0.01)
        pt = Ptychography.from_models(dset=base.dset, obj_model=dip, probe_model=base.probe_model,
                                      detector_model=base.detector_model, device="gpu", verbose=0,
                                      rng=int(z["recon_rng_seed"]))
        pt.preprocess(obj_padding_px=base.obj_padding_px)
        return pt

    def flat(sd):
        return np.concatenate([v.detach().cpu().numpy().ravel().view(np.float32) if v.is_complex()
                               else v.detach().cpu().numpy().ravel().astype(np.float32)
                               for k, v in sorted(sd.items()) if v.is_floating_point() or v.is_complex()])

    def adam(pt):
        st = pt.obj_model.optimizer.state_dict()["state"]
        return {k: {n: (v.cpu() if isinstance(v, torch.Tensor) else v) for n, v in s.items()} for k, s in st.items()}

    runs = []
    for _ in range(2):
        pt = fresh()
        pt.reconstruct(num_iters=4, batch_size=9, optimizer_params=opt, device="gpu")
        runs.append((flat(pt.obj_model.model.state_dict()), np.asarray(pt.iter_losses)))
    spread = rel(runs[1][0], runs[0][0])
    pt = fresh()
    pt.reconstruct(num_iters=2, batch_size=9, optimizer_params=opt, device="gpu")
    path = tmp_path / "dip.pt"
    pt.save(path, save_raw_data=True, verbose=False)
    q = Ptychography.from_file(path, device="gpu")
    assert type(q.obj_model).__name__ == "ObjectDIP" and q.num_iters == 2
    np.testing.assert_array_equal(flat(q.obj_model.model.state_dict()), flat(pt.obj_model.model.state_dict()))
    a, b = adam(q), adam(pt)
    assert a.keys() == b.keys()
    for k in a:
        assert a[k]["step"] == b[k]["step"]
        for n in ("exp_avg", "exp_avg_sq"):
            assert torch.equal(a[k][n], b[k][n])
    assert torch.equal(q.obj_model._gen.get_state(), pt.obj_model._gen.get_state())
    q.reconstruct(num_iters=2, device="gpu")
    pt.reconstruct(num_iters=2, device="gpu")
    assert len(q.iter_losses) == 4
    np.testing.assert_allclose(q.iter_losses, pt.iter_losses, rtol=max(1e-5, 10 * spread))
    assert rel(flat(q.obj_model.model.state_dict()), flat(pt.obj_model.model.state_dict())) <= 3 * spread + 1e-5
