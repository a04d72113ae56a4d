"""Several datasets of uneven scan size, slices and modes in one persistent launch,
the CUDA-graph captured iteration and the launch autotuner."""
import numpy as np
import pytest
import torch

from tests.conftest import rel

pytestmark = pytest.mark.gpu


def _problems(dev, specs, n=64):
    from quantem_b200 import multi, synthetic

    out = []
    for k, spec in enumerate(specs):
        scan, S, P = spec[:3]
        n = spec[3] if len(spec) > 3 else n
        cfg = synthetic.SyntheticConfig(n=n, slices=S, modes=P, mode_weights=(0.7, 0.2, 0.1, 0.05)[:P],
                                        scan=(scan, scan), step_px=4.0, pad_px=n // 2, seed=40 + k)
        ds = synthetic.make_dataset(cfg, dev)
        obj = (torch.ones(ds["obj_shape"], dtype=torch.complex64, device=dev)
               * torch.exp(1j * 0.05 * torch.randn(ds["obj_shape"], device=dev, generator=torch.Generator(dev).manual_seed(k)))
               ).contiguous().requires_grad_(True)
        probe = (ds["probes"] * ds["mean_intensity"] ** 0.5 * 1.1).contiguous().requires_grad_(True)
        out.append(multi.Problem(obj, probe, ds["propagators"], ds["positions"], ds["amplitudes"].contiguous(),
                                 torch.ones((n, n), device=dev), ds["mean_intensity"], cfg.step_px))
    return out


SPECS = [(5, 1, 1), (7, 3, 2), (9, 2, 3), (6, 4, 1)]


def test_multi_launch_matches_single_launches(cuda_device):
    from quantem_b200 import multi, ops

    probs = _problems(cuda_device, SPECS)
    grids = multi.default_grids(probs, total=13)
    obj_cs = [ops.obj_constrain(p.obj.detach().contiguous())[0] for p in probs]
    probe_os = [p.probe.detach().contiguous() for p in probs]
    res = multi.multi_forward_adjoint(probs, obj_cs, probe_os, grids)
    for p, oc, po, (loss, gobj, gp) in zip(probs, obj_cs, probe_os, res):
        l1, g1, gp1 = ops.batch_forward_adjoint(oc, po, p.prop, p.positions, p.batch_idx, p.targets, p.mask,
                                                p.num_gpts, p.mean_intensity)
        assert abs(loss.item() - l1.item()) / abs(l1.item()) < 1e-6
        assert rel(gobj.cpu().numpy(), g1.cpu().numpy()) < 1e-5
        assert rel(gp.cpu().numpy(), gp1.cpu().numpy()) < 1e-5


def test_graphed_iteration_matches_eager(cuda_device):
    from quantem_b200 import multi

    a = _problems(cuda_device, SPECS)
    b = _problems(cuda_device, SPECS)
    grids = multi.default_grids(a, total=13)
    ea = multi.MultiIteration(a, grids)
    for _ in range(3):
        la = ea.run_eager()
    gb = multi.MultiIteration(b, grids).capture(warmup=2)  # two eager warm-up iterations
    lb = gb.replay()
    torch.cuda.synchronize()
    assert rel(lb.cpu().numpy(), la.cpu().numpy()) < 1e-5
    for pa, pb in zip(a, b):
        assert rel(pb.obj.detach().cpu().numpy(), pa.obj.detach().cpu().numpy()) < 1e-5
        assert rel(pb.probe.detach().cpu().numpy(), pa.probe.detach().cpu().numpy()) < 1e-5
    st = gb.check_status()  # clean data: no skipped positions, finite intensities
    assert len(st) == len(b) and all(x["raw"] == 0 for x in st)


def test_autotune_returns_valid_partition(cuda_device):
    from quantem_b200 import multi

    probs = _problems(cuda_device, SPECS)
    g = multi.autotune_grids(probs, total=16)
    assert len(g) == len(probs)
    assert all(1 <= x <= int(p.batch_idx.numel()) for x, p in zip(g, probs))


def test_mixed_windows_96_and_128(cuda_device):
    """The uneven-workload pattern with 96 x 96 and 128 x 128 windows: one persistent
    launch per window size inside one call, results equal to single launches, and
    a graphed iteration equal to the eager one."""
    from quantem_b200 import multi, ops

    specs = [(5, 1, 1, 96), (6, 3, 2, 128), (7, 2, 1, 96), (5, 2, 2, 128)]
    probs = _problems(cuda_device, specs)
    grids = multi.default_grids(probs, total=11)
    obj_cs = [ops.obj_constrain(p.obj.detach().contiguous())[0] for p in probs]
    probe_os = [p.probe.detach().contiguous() for p in probs]
    res = multi.multi_forward_adjoint(probs, obj_cs, probe_os, grids)
    for p, oc, po, (loss, gobj, gp) in zip(probs, obj_cs, probe_os, res):
        l1, g1, gp1 = ops.batch_forward_adjoint(oc, po, p.prop, p.positions, p.batch_idx, p.targets, p.mask,
                                                p.num_gpts, p.mean_intensity)
        assert abs(loss.item() - l1.item()) / abs(l1.item()) < 1e-6
        assert rel(gobj.cpu().numpy(), g1.cpu().numpy()) < 1e-5
        assert rel(gp.cpu().numpy(), gp1.cpu().numpy()) < 1e-5
    a, b = _problems(cuda_device, specs), _problems(cuda_device, specs)
    ea = multi.MultiIteration(a, grids)
    for _ in range(3):
        la = ea.run_eager()
    lb = multi.MultiIteration(b, grids).capture(warmup=2).replay()
    torch.cuda.synchronize()
    assert rel(lb.cpu().numpy(), la.cpu().numpy()) < 1e-5
