"""The learned initialiser: a CNN2d trained on the GPU with the tcgen05 BF16 kernels
on pairs simulated by the method's own forward kernel, compared with the plain
(flat-object) start it replaces, and the plain forward model as its judge."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _setup(dev, seed=0):
    from quantem_b200 import ops, synthetic
    from quantem_b200.diffractive_imaging.learned_init import LearnedInitConfig, LearnedInitializer
    from quantem_b200.diffractive_imaging.ptycho_utils import orthogonalize_probes

    scfg = synthetic.SyntheticConfig(n=64, slices=2, modes=2, mode_weights=(0.8, 0.2), step_px=4, scan=(32, 32),
                                     pad_px=35, seed=5)
    probes = orthogonalize_probes(synthetic.make_probe_modes(scfg, dev))
    props = ops.separable_propagators(64, (scfg.pixel, scfg.pixel), scfg.energy, [scfg.slice_thickness], device=dev)
    # smooth atoms (sigma 3 px) make the phase learnable from 16 x 16-binned patterns within
    # a few thousand objects; the sharp sigma 1.5 px atoms of the benchmark need ~20k
    cfg = LearnedInitConfig(n=64, bin=4, scan_crop=16, step_px=4, start_filters=32, num_layers=3, lr=2e-3,
                            sigma_px=3.0)
    return scfg, LearnedInitializer(probes, props, cfg, dev, seed=seed)


def test_trained_network_beats_flat_start(cuda_device):
    """Held-out objects from the training distribution: the flat start has phase
    NRMSE 1 by definition (zero phase); the trained network's prediction must be
    clearly better."""
    _, li = _setup(cuda_device)
    before = li.evaluate(16)
    li.train(3200, total_objects=3200, log_every=20)
    after = li.evaluate(32)
    losses = [l for _, l in li.history]
    assert losses[-1] < 0.5 * losses[0]
    assert after < 0.7, (before, after)


def test_plain_model_judges_the_learned_start(cuda_device):
    """initial_object keeps the learned start when the forward model fits the data
    better with it, and falls back to the flat object when it does not."""
    from quantem_b200 import synthetic

    scfg, li = _setup(cuda_device, seed=1)
    li.train(3200, total_objects=3200)
    ds = synthetic.make_dataset(scfg, cuda_device)
    S, Ho, Wo = ds["obj_shape"]
    probe = ds["probes"] * (ds["mean_intensity"] / ds["probes"].abs().square().sum()) ** 0.5
    judge = dict(probe=probe.contiguous(), prop=ds["propagators"], positions=ds["positions"],
                 targets=ds["amplitudes"].contiguous(), mask=torch.ones((64, 64), device=cuda_device),
                 mean_intensity=ds["mean_intensity"],
                 batch=torch.arange(ds["positions"].shape[0], device=cuda_device))
    obj = li.initial_object(ds["amplitudes"], (32, 32), (S, Ho, Wo), (scfg.pad_px, scfg.pad_px), judge=judge)
    assert obj.shape == (S, Ho, Wo) and obj.dtype == torch.complex64
    losses = li.judge_losses
    assert len(losses) == len(li.JUDGE_SCALES)
    assert li.judge_scale == li.JUDGE_SCALES[int(np.argmin(losses))]
    assert li.used_learned == (li.judge_scale > 0)
    # a network with scrambled weights predicts garbage: the plain model rejects it or
    # shrinks it towards the flat start
    with torch.no_grad():
        li.net.flat.data.mul_(-3.0)
    obj2 = li.initial_object(ds["amplitudes"], (32, 32), (S, Ho, Wo), (scfg.pad_px, scfg.pad_px), judge=judge)
    assert li.judge_scale < 1.0
    if not li.used_learned:
        assert torch.equal(obj2, torch.ones_like(obj2))


def test_learned_start_shortens_the_time_to_the_plain_methods_best_at_c4_scale(cuda_device):
    """The learned-initialiser benchmark geometry (128^2 probe, 8 slices of 20 A, 4 modes,
    64x64 scan, 1e5 counts) on a held-out Gaussian-atom object from the dense, strong end
    of the training range (peak 0.4 rad, 0.008 atoms / px^2 / slice): a network trained on
    6000 simulated objects, judged by the plain forward model, then the plain iterations
    (known probe, Adam 5e-3 x 0.97 per iteration, batch 256) from the flat and from the
    learned start.  Target: 1.05 x the best projected-phase NRMSE the flat start reaches in
    12 iterations (at this dose the plain method plateaus within a few iterations).  The
    learned start (inference and judging included) must reach it in at most 0.85 of the
    flat start's wall time (measured 0.75 with 4000 training objects, 0.68 with 20000)."""
    import time

    from quantem_b200 import engine, ops, synthetic
    from quantem_b200.diffractive_imaging.learned_init import LearnedInitConfig, LearnedInitializer
    from quantem_b200.diffractive_imaging.ptycho_utils import SimpleBatcher, orthogonalize_probes

    dev = cuda_device
    scfg = synthetic.SyntheticConfig(seed=0, peak_phase=0.4, atom_density=0.008)
    probes = orthogonalize_probes(synthetic.make_probe_modes(scfg, dev))
    props = ops.separable_propagators(scfg.n, (scfg.pixel, scfg.pixel), scfg.energy,
                                      [scfg.slice_thickness] * (scfg.slices - 1), device=dev)
    li = LearnedInitializer(probes, props, LearnedInitConfig(lr=2e-3), dev, seed=0)
    li.train(6000, total_objects=6000)
    ds = synthetic.make_dataset(scfg, dev)
    S, Ho, Wo = ds["obj_shape"]
    probe = (ds["probes"] * (ds["mean_intensity"] / ds["probes"].abs().square().sum()) ** 0.5).contiguous()

    def proj(o):
        p = o[0]
        for k in range(1, o.shape[0]):
            p = p * o[k]
        return torch.angle(p)

    lo, hi = scfg.pad_px, scfg.pad_px + int((scfg.scan[0] - 1) * scfg.step_px)
    truth = proj(ds["obj"])[lo:hi, lo:hi].double()
    assert float(ds["obj"].angle().sum(0).abs().max()) < 3.0  # the projected phase does not wrap

    def nrmse(o):
        a = proj(ops.constrained_object(o))[lo:hi, lo:hi].double()
        d = (a - a.mean()) - (truth - truth.mean())
        return float(d.norm() / (truth - truth.mean()).norm())

    curves = {}
    for arm in ("plain", "learned"):
        torch.cuda.synchronize()
        t0 = time.time()
        if arm == "learned":
            judge = dict(probe=probe, prop=ds["propagators"], positions=ds["positions"],
                         targets=ds["amplitudes"].contiguous(), mask=torch.ones((scfg.n, scfg.n), device=dev),
                         mean_intensity=ds["mean_intensity"], batch=torch.arange(0, 4096, 4, device=dev))
            o0 = li.initial_object(ds["amplitudes"], scfg.scan, (S, Ho, Wo), (scfg.pad_px, scfg.pad_px), judge=judge)
        else:
            o0 = torch.ones((S, Ho, Wo), dtype=torch.complex64, device=dev)
        torch.cuda.synchronize()
        elapsed = time.time() - t0
        obj = o0.clone().requires_grad_(True)
        pt = engine.ProblemTensors(obj=obj, probe=probe.clone().requires_grad_(True), prop=ds["propagators"],
                                   positions=ds["positions"], targets=ds["amplitudes"].contiguous(),
                                   mask=torch.ones((scfg.n, scfg.n), device=dev),
                                   mean_intensity=ds["mean_intensity"], upsample_factor=scfg.step_px)
        opt = engine.make_optimizer([obj], {"type": "adam", "lr": 5e-3})
        sched = torch.optim.lr_scheduler.ExponentialLR(opt, 0.97)
        bt = SimpleBatcher(pt.num_gpts, 256, rng=0)
        curve = [(elapsed, nrmse(obj.detach()))]
        for _ in range(12):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            engine.run_iteration(pt, bt, [opt])
            e1.record()
            sched.step()
            torch.cuda.synchronize()
            elapsed += e0.elapsed_time(e1) / 1e3
            curve.append((elapsed, nrmse(obj.detach())))
        curves[arm] = curve
    assert li.used_learned, li.judge_losses
    assert curves["learned"][0][1] < 0.85, curves["learned"][0]
    target = 1.05 * min(v for _, v in curves["plain"])
    t_plain = next(t for t, v in curves["plain"] if v <= target)
    t_learned = next((t for t, v in curves["learned"] if v <= target), None)
    assert t_learned is not None and t_learned <= 0.85 * t_plain, (target, curves)
