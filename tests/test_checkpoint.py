"""Checkpoint / resume (Ptychography.save / from_file, ptychography.py:376-588) on the
host: every tensor and counter of the resumable state comes back bit for bit."""
import numpy as np
import pytest
import torch

from tests.conftest import load_golden
from tests.test_host_setup import build_from_golden


def _populate(pt, rng):
    """A mid-run state without a GPU: perturbed parameters, Adam moments and step
    counts, a scheduler, advanced generator, loss / learning-rate histories."""
    with torch.no_grad():
        pt.obj_model._obj.mul_(torch.exp(0.1j * torch.as_tensor(rng.standard_normal(pt.obj_model.shape))))
        pt.probe_model._probe.mul_(1.1)
    pt.optimizer_params = {"object": {"type": "adam", "lr": 5e-3}, "probe": {"type": "adam", "lr": 1e-3}}
    pt.set_optimizers()
    pt.scheduler_params = {"object": {"type": "exp", "gamma": 0.97}}
    pt.set_schedulers(pt.scheduler_params, num_iter=10)
    for model in (pt.obj_model, pt.probe_model):
        p = model.get_optimization_parameters()[0]
        model.optimizer.state[p] = {"step": 7, "exp_avg": torch.randn_like(p), "exp_avg_sq": torch.rand_like(p.real)
                                    .to(p.dtype)}
    for _ in range(3):
        pt.obj_model.scheduler.step()
    pt.rng.permutation(50)
    pt._iter_losses = [3.0, 2.5, 2.25]
    pt._iter_lrs = {"object": [5e-3, 4.8e-3, 4.7e-3], "probe": [1e-3] * 3}
    pt.dset.scan_positions_px = pt.dset.scan_positions_px + 0.25


def _equal(a, b):
    return torch.equal(torch.as_tensor(a), torch.as_tensor(b))


@pytest.mark.parametrize("raw", [True, False])
def test_checkpoint_round_trip_is_exact(tmp_path, raw):
    from quantem_b200.diffractive_imaging import Ptychography

    z = load_golden("mixed64")
    pt = build_from_golden(z)
    _populate(pt, np.random.default_rng(0))
    path = tmp_path / "recon.pt"
    pt.save(path, save_raw_data=raw, verbose=False)
    with pytest.raises(FileExistsError):
        pt.save(path, verbose=False)
    pt.save(path, mode="o", save_raw_data=raw, verbose=False)
    if raw:
        q = Ptychography.from_file(path)
    else:
        with pytest.raises(ValueError, match="raw data"):
            Ptychography.from_file(path)
        q = Ptychography.from_file(path, dset=build_from_golden(z).dset)
    assert _equal(q.obj_model._obj.detach(), pt.obj_model._obj.detach())
    assert _equal(q.obj_model.initial_obj, pt.obj_model.initial_obj)
    assert _equal(q.probe_model._probe.detach(), pt.probe_model._probe.detach())
    assert _equal(q.probe_model.initial_probe, pt.probe_model.initial_probe)
    assert _equal(q.dset.scan_positions_px, pt.dset.scan_positions_px)
    assert _equal(q.dset.targets, pt.dset.targets)
    np.testing.assert_array_equal(q.obj_padding_px, pt.obj_padding_px)
    assert q.iter_losses.tolist() == pt.iter_losses.tolist() and q.num_iters == pt.num_iters
    assert {k: v.tolist() for k, v in q.iter_lrs.items()} == {k: v.tolist() for k, v in pt.iter_lrs.items()}
    for a, b in ((q.obj_model, pt.obj_model), (q.probe_model, pt.probe_model)):
        pa, pb = a.get_optimization_parameters()[0], b.get_optimization_parameters()[0]
        sa, sb = a.optimizer.state[pa], b.optimizer.state[pb]
        assert sa["step"] == sb["step"] == 7
        assert _equal(sa["exp_avg"], sb["exp_avg"]) and _equal(sa["exp_avg_sq"], sb["exp_avg_sq"])
        assert a.optimizer.param_groups[0]["lr"] == b.optimizer.param_groups[0]["lr"]
    assert q.obj_model.scheduler.last_epoch == pt.obj_model.scheduler.last_epoch == 3
    # the generator continues with the same draws
    assert q.rng.permutation(100).tolist() == pt.rng.permutation(100).tolist()
    assert _equal(q.propagators, pt.propagators)


def test_checkpoint_rejects_foreign_files(tmp_path):
    from quantem_b200.diffractive_imaging import Ptychography

    path = tmp_path / "other.pt"
    torch.save({"format": "something else"}, path)
    with pytest.raises(ValueError, match="checkpoint"):
        Ptychography.from_file(path)
