"""Benchmark of the multislice mixed-probe ptychography iteration on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one full gradient iteration over every scan position):
object 512 x 512 x 8 slices (20 A), 4 probe modes at 128 x 128 (weights
0.7/0.15/0.1/0.05), 64 x 64 raster with 6 px step and +-0.5 px jitter, 1e5
counts/pattern Poisson data, l2_amplitude loss, Adam on object and probe, batch
= all 4096 positions (the reference's default batch size).  Data are seeded
synthetic inputs simulated with this package's forward kernels.

``--impl ours`` times the CUDA path: ``value`` is the device-resident iteration
replayed from a CUDA graph; ``e2e`` is ``Ptychography.reconstruct`` of the drop-in
API on a dataset built from host arrays whose targets stay in pinned host memory
and are copied to the GPU every iteration.  ``--impl reference`` times the
reference's own ``Ptychography.reconstruct(device="cpu")`` (package under
``baseline/_ref``) on the host cores on a bounded sample of the same geometry (an
8 x 8 sub-scan, 64 positions, batch 64); ``--impl reference --torch-gpu`` times the
reference's own PyTorch iteration on the GPU (also reported in the default line as
``reference_torch_gpu``).
With ``--gpus N`` (torchrun), every rank reconstructs its own dataset: N
independent replicas, no collective.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "scan positions/s per iteration"
WORKLOAD = "multislice mixed-probe: 512x512x8 object, 4 modes at 128x128, 64x64 scan, batch 4096"
FLOPS_PER_POS = 167.8e6     # 4*P*S FFTs * 5*HW*log2(HW) + 40*P*S*HW (c2)
BYTES_PER_POS = 3.06 * 2**20  # streaming lower bound per position (c2)


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        try:
            with open(self.path) as fh:
                for line in fh:
                    f = [x.strip() for x in line.split(",")]
                    if len(f) < 9:
                        continue
                    try:
                        sm.append(float(f[1]))
                        smax = float(f[2])
                    except ValueError:
                        continue
                    for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                        "sw_power_cap"), f[5:9]):
                        if v.lower().startswith("active"):
                            reasons.add(name)
        except Exception:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(values, dist, device="cpu"):
    """Element-wise maximum of per-rank timings (identity on one rank)."""
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def _dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def _init_dist(world, backend):
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
        return dist
    return None


def build_problem(seed, device, batch_size, cfg=None):
    import torch

    from quantem_b200 import engine, synthetic
    from quantem_b200.diffractive_imaging.ptycho_utils import SimpleBatcher

    cfg = cfg or synthetic.SyntheticConfig(seed=seed)
    ds = synthetic.make_dataset(cfg, device)
    S, Ho, Wo = ds["obj_shape"]
    obj = torch.ones((S, Ho, Wo), dtype=torch.complex64, device=device).requires_grad_(True)
    probe = (ds["probes"][:1].repeat(cfg.modes, 1, 1) * torch.linspace(1.0, 0.3, cfg.modes, device=device)[:, None, None]
             ).to(torch.complex64)
    k = torch.fft.fftfreq(cfg.n, device=device)
    for m in range(1, cfg.modes):  # decorrelate the initial modes
        probe[m] *= torch.exp(-2j * torch.pi * (0.3 * m) * k[:, None]).to(torch.complex64)
    # Parseval: sum over modes of |probe|^2 equals the mean pattern intensity
    # (the reference's _apply_weights normalisation, probe_models.py:860-873)
    probe = probe * torch.sqrt(ds["mean_intensity"] / probe.abs().square().sum())
    probe = probe.contiguous().requires_grad_(True)
    pt = engine.ProblemTensors(
        obj=obj, probe=probe, prop=ds["propagators"], positions=ds["positions"],
        targets=ds["amplitudes"].contiguous(), mask=torch.ones((cfg.n, cfg.n), device=device),
        mean_intensity=ds["mean_intensity"], upsample_factor=cfg.step_px)
    opts = [engine.make_optimizer([obj], {"type": "adam", "lr": 5e-3}),
            engine.make_optimizer([probe], {"type": "adam", "lr": 1e-3})]
    batcher = SimpleBatcher(pt.num_gpts, batch_size, rng=seed)
    return cfg, ds, pt, opts, batcher


def build_dropin(cfg, device, seed):
    """The drop-in API set up the way a user of the reference would: a host
    ``Dataset4dstem`` of the simulated patterns, ``PtychographyDatasetRaster.preprocess``
    (on the GPU), ``ObjectPixelated.from_uniform``, ``ProbePixelated.from_params`` with
    the configuration's mode weights, ``Ptychography.from_models(...).preprocess(...)``,
    jittered positions.  The targets stay in pinned host memory
    (``keep_targets_on_host``), so every ``reconstruct`` iteration copies them to the
    GPU."""
    import torch

    from quantem_b200 import synthetic
    from quantem_b200.diffractive_imaging import (Dataset4dstem, DetectorPixelated, ObjectPixelated,
                                                  ProbePixelated, Ptychography, PtychographyDatasetRaster)

    ds = synthetic.make_dataset(cfg, device)
    nr, nc = cfg.scan
    data = ds["intensities"].cpu().numpy().reshape(nr, nc, cfg.n, cfg.n)
    positions = ds["positions"]
    del ds
    rs = 1.0 / (cfg.n * cfg.pixel)
    d4 = Dataset4dstem.from_array(data, sampling=(cfg.step_px * cfg.pixel, cfg.step_px * cfg.pixel, rs, rs),
                                  units=("A", "A", "A^-1", "A^-1"))
    pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
    pd.preprocess(com_fit_function="no_shift", force_com_rotation=0, force_com_transpose=False,
                  plot_rotation=False, plot_com=False, probe_energy=cfg.energy, device="gpu")
    obj = ObjectPixelated.from_uniform(num_slices=cfg.slices, slice_thicknesses=cfg.slice_thickness,
                                       obj_type="complex")
    probe = ProbePixelated.from_params(probe_params={"energy": cfg.energy, "defocus": cfg.defocus,
                                                     "semiangle_cutoff": cfg.semiangle},
                                       num_probes=cfg.modes, rng=seed + 1, initial_probe_weights=list(cfg.mode_weights))
    pt = Ptychography.from_models(dset=pd, obj_model=obj, probe_model=probe, detector_model=DetectorPixelated(),
                                  device="gpu", verbose=0, rng=seed + 2)
    pt.preprocess(obj_padding_px=(cfg.pad_px, cfg.pad_px))
    pd.scan_positions_px = positions.float().to(pd.scan_positions_px.device).contiguous()  # simulated positions
    pd.keep_targets_on_host(True)
    return pt


def fp32_peak_tflops(device):
    """FP32 FMA throughput of this GPU (own microbenchmark kernel), TFLOP/s."""
    import ctypes

    import torch

    from quantem_b200 import _lib

    lib = _lib.lib()
    if not hasattr(lib, "ptycho_fp32_fma_probe"):
        return None
    fn = lib.ptycho_fp32_fma_probe
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    out = torch.empty(148 * 4 * 1024, dtype=torch.float32, device=device)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    iters = 4096
    blocks = 148 * 4
    for _ in range(3):
        _lib.check(fn(ctypes.c_void_p(out.data_ptr()), iters, blocks, st), "fma probe")
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(5):
        fn(ctypes.c_void_p(out.data_ptr()), iters, blocks, st)
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e) / 5
    flops = blocks * 512 * iters * 16 * 2  # 16 independent FMA chains per thread
    return flops / (ms * 1e-3) / 1e12


def run_ours(args):
    import torch

    from quantem_b200 import engine, ops

    rank, world, local = _dist_env()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    dist = _init_dist(world, "nccl")
    cfg, ds, pt, opts, batcher = build_problem(1234 + rank, device, args.batch_size)
    npos = pt.num_gpts

    # warm-up
    for _ in range(args.warmup):
        engine.run_iteration(pt, batcher, opts)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()

    # ---- device-resident timed region ----
    fused_events = []
    ops.PROFILE_EVENTS = fused_events
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        losses = []
        for _ in range(args.steps):
            losses.append(engine.run_iteration(pt, batcher, opts))
        t1.record()
        torch.cuda.synchronize()
    ops.PROFILE_EVENTS = None
    ms_eager = t0.elapsed_time(t1) / args.steps
    fused_ms = [a.elapsed_time(b) for a, b in fused_events]
    # ours per batch: probe orthogonalisation and its gradient, object constraint (2) and its
    # VJP (2), probe FFT, fused batch kernel, loss and partial reductions, probe-gradient FFT,
    # two Adam steps
    launches_per_batch = 13
    nbatches = len(batcher) * args.steps

    # ---- the same full-batch iteration captured in a CUDA graph and replayed ----
    ms_graph = None
    if len(batcher) == 1:
        git = engine.GraphedIteration(pt).capture(warmup=args.warmup)
        with ClockSampler(local) as clk_g:
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
            g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            g0.record()
            for _ in range(args.steps):
                gl = git.replay()
            g1.record()
            torch.cuda.synchronize()
        ms_graph = g0.elapsed_time(g1) / args.steps
        losses.append(gl.clone())
        del git
    ms = ms_graph if ms_graph is not None else ms_eager

    # ---- end to end through the drop-in API: Ptychography.reconstruct on a dataset whose
    # targets stay in pinned host memory and are copied to the GPU every iteration; the
    # loss and the status word are read back every iteration ----
    drop = build_dropin(cfg, device, 1234 + rank)
    opt = {"object": {"type": "adam", "lr": 5e-3}, "probe": {"type": "adam", "lr": 1e-3}}
    drop.reconstruct(num_iters=args.warmup, batch_size=args.batch_size, optimizer_params=opt, device="gpu")
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    drop.loss_readback = "iteration"  # every step's loss (and the status word) read when the step ends
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    drop.reconstruct(num_iters=args.steps, batch_size=args.batch_size, device="gpu")
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    h2d = drop.last_h2d_bytes_per_iter + drop.dset.num_gpts * 8  # targets + batch indices
    e2e_final_loss = float(drop.iter_losses[-1])
    # the same call with the default readback: the losses of all steps read once at its end
    drop.loss_readback = "auto"
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    drop.reconstruct(num_iters=args.steps, batch_size=args.batch_size, device="gpu")
    f1.record()
    torch.cuda.synchronize()
    e2e_deferred_ms = f0.elapsed_time(f1) / args.steps
    del drop
    torch.cuda.empty_cache()

    ms, ms_eager, e2e_ms, e2e_deferred_ms = max_over_ranks([ms, ms_eager, e2e_ms, e2e_deferred_ms], dist, device)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    value = npos * world / (ms * 1e-3)
    e2e = npos * world / (e2e_ms * 1e-3)
    hbm_peak, peak_kind = _peaks()
    fused_avg_ms = statistics.mean(fused_ms) if fused_ms else None
    pos_per_launch = args.batch_size if args.batch_size else npos
    # The binding roof of this FFT path is the FP32 CUDA-core pipe (no GEMM: tensor cores do
    # not apply); its peak is measured in the same run by the library's FMA probe kernel
    # (MEASURED_PEAKS.json carries HBM and BF16 figures only).  The HBM roof is reported
    # beside it.
    roofline = roofline_hbm = None
    fp32 = fp32_peak_tflops(device)
    if fused_avg_ms:
        achieved = BYTES_PER_POS * pos_per_launch / (fused_avg_ms * 1e-3) / 1e9
        roofline_hbm = {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                        "frac": round(achieved / hbm_peak, 4), "traffic": _ncu_traffic(),
                        "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                        else "fallback 6650 GB/s", "bytes_per_position": BYTES_PER_POS}
    if fused_avg_ms and fp32:
        ach = FLOPS_PER_POS * pos_per_launch / (fused_avg_ms * 1e-3) / 1e12
        roofline = {"bound": "fp32", "achieved": round(ach, 2), "peak": round(fp32, 2), "unit": "TFLOP/s",
                    "frac": round(ach / fp32, 4), "traffic": _ncu_traffic(),
                    "peak_source": "measured in this run (ptycho_fp32_fma_probe: 148 x 4 CTAs of FMA chains)",
                    "flops_per_position": FLOPS_PER_POS, "positions_per_launch": pos_per_launch,
                    "kernel": "fused_batch_kernel<128,adjoint>", "kernel_ms": round(fused_avg_ms, 4)}
    cpu = reference_cpu_subprocess(local, steps=2, warmup=1)
    try:  # the oracle as the checker: FP32 CUDA path against an FP64 run on a bounded sample
        accuracy = accuracy_vs_fp64(pt)
    except Exception as exc:
        accuracy = {"unavailable": f"{type(exc).__name__}: {exc}"[:300]}
    torch_ref = torch_eager_reference(pt, args.batch_size) if not args.skip_torch_reference else None
    ref_gpu = None
    if not args.skip_torch_reference:
        ref_gpu = reference_torch_gpu_subprocess(local, args.batch_size, steps=10, warmup=3)
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "positions/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "iteration": "CUDA-graph replay of the full-batch iteration" if ms_graph is not None else "eager",
        "value_eager": round(npos * world / (ms_eager * 1e-3), 1),
        "scaling": "weak", "vs_baseline": None, "dtype": "c64/f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "global_batch": pos_per_launch * world, "positions": npos,
                   "object": [cfg.slices, 512, 512], "probe": [cfg.modes, cfg.n, cfg.n],
                   "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (targets 256 MiB/step)"},
        "e2e": {"value": round(e2e, 1), "unit": "positions/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": 8,
                "path": "quantem_b200.diffractive_imaging.Ptychography.reconstruct(num_iters=steps, device='gpu') "
                        "on a host Dataset4dstem preprocessed through the drop-in API; targets in pinned host "
                        "memory copied to the GPU every iteration (double-buffered on a copy stream), loss and "
                        "status word read back every iteration (loss_readback='iteration')",
                "final_loss": e2e_final_loss,
                "deferred_readback": {"value": round(npos * world / (e2e_deferred_ms * 1e-3), 1),
                                      "unit": "positions/s",
                                      "what": "the same call with the default loss_readback='auto': no scheduler, "
                                              "logger or validation reads the loss during the run, so every "
                                              "step's loss and the status word are read once at its end"}},
        "gpu_launches": launches_per_batch * nbatches,
        "roofline": roofline, "roofline_hbm": roofline_hbm,
        "cpu_baseline": cpu,
        "accuracy_vs_fp64": accuracy,
        "torch_eager_reference_gpu": torch_ref,
        "reference_torch_gpu": ref_gpu,
        "clocks": clk_g.summary() if ms_graph is not None else clk.summary(),
        "clocks_eager": clk.summary(),
        "final_loss": float(losses[-1].item()),
    }
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def _ncu_traffic():
    """DRAM bytes per launch of the fused kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "fused_batch_kernel_traffic.json")
    try:
        with open(path) as fh:
            return json.load(fh)["dram_bytes_per_launch_full_batch"]
    except Exception:
        return None


def torch_eager_reference(pt, batch_size, steps=3, warmup=2):
    """Positions/s of the reference's PyTorch op sequence run eagerly on this GPU.

    A restatement (not the reference's code) of what quantem's
    Ptychography.reconstruct does per batch on device="gpu": probe
    Gram-Schmidt, fourier_shift_expand (fft2 * ramp -> ifft2, ptycho_utils.py:128-176),
    hard-constrained object and real/imag patch gather with int32 flat patch
    indices (object_models.py:252-339, dataset_models.py:514-535), multislice with
    torch.fft (ptychography_base.py:934-989), detector fft2(ortho)/|.|^2/mode
    sum/fftshift (detector_models.py:22-30), l2_amplitude loss (908-932), autograd
    backward, obj-grad rescale and torch.optim.Adam (optimizer_mixin.py:117-123).
    Batches that do not fit in memory are split; the number of positions per
    batch used is reported."""
    import torch

    from quantem_b200.diffractive_imaging.ptycho_utils import orthogonalize_probes

    dev = pt.obj.device
    obj = pt.obj.detach().clone().requires_grad_(True)
    probe = pt.probe.detach().clone().requires_grad_(True)
    P, n, _ = probe.shape
    S, Ho, Wo = obj.shape
    kr, kc = pt.prop
    prop = (kr[:, :, None] * kc[:, None, :]).contiguous()
    opt_o = torch.optim.Adam([obj], lr=5e-3)
    opt_p = torch.optim.Adam([probe], lr=1e-3)
    pos_all = pt.positions
    f = torch.fft.fftfreq(n, d=1 / n, device=dev)
    kf = torch.fft.fftfreq(n, d=1.0, device=dev).to(torch.float32)
    npos = pos_all.shape[0]

    def one_batch(bi):
        pos = pos_all[bi]
        frac = pos - torch.round(pos)
        r0 = torch.round(pos[:, 0]).to(torch.int32)
        c0 = torch.round(pos[:, 1]).to(torch.int32)
        rows = (r0[:, None, None] + f[None, :, None]) % Ho
        cols = (c0[:, None, None] + f[None, None, :]) % Wo
        pidx = (rows * Wo + cols).to(torch.int32).long()
        pr = orthogonalize_probes(probe)
        ramp = (torch.exp(-2j * torch.pi * kf[None, :, None] * frac[:, 0][:, None, None])
                * torch.exp(-2j * torch.pi * kf[None, None, :] * frac[:, 1][:, None, None]))
        shifted = torch.fft.ifft2(torch.fft.fft2(pr) * ramp[:, None]).swapaxes(0, 1)
        amp = torch.clamp(torch.abs(obj), 0.0, 1.0)
        phase = obj.angle() - obj.angle().mean()
        oc = (amp * torch.exp(1.0j * phase)).reshape(S, -1)
        patches = torch.complex(oc.real[:, pidx], oc.imag[:, pidx])
        ov = patches[0] * shifted
        for s in range(1, S):
            ov = patches[s] * torch.fft.ifft2(torch.fft.fft2(ov) * prop[s - 1])
        inten = torch.fft.fftshift(torch.sum(torch.abs(torch.fft.fft2(ov, norm="ortho")) ** 2, dim=0), dim=(-2, -1))
        tg = pt.targets[bi]
        diff = torch.sqrt(inten + 1e-9) * pt.mask - tg * pt.mask
        loss = torch.sum(torch.abs(diff) ** 2) / (diff.shape[0] / npos) / pt.mean_intensity
        return loss

    def iteration(bs):
        order = torch.randperm(npos, device=dev)
        for i in range(0, npos, bs):
            bi = order[i:i + bs]
            opt_o.zero_grad()
            opt_p.zero_grad()
            loss = one_batch(bi)
            loss.backward()
            obj.grad.mul_(pt.upsample_factor ** 2 / 2)
            opt_o.step()
            opt_p.step()

    bs = batch_size
    while True:
        try:
            iteration(bs)
            torch.cuda.synchronize()
            break
        except torch.OutOfMemoryError:
            torch.cuda.empty_cache()
            bs //= 2
            if bs < 1:
                return None
    for _ in range(warmup - 1):
        iteration(bs)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        iteration(bs)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    del opt_o, opt_p, obj, probe
    torch.cuda.empty_cache()
    return {"value": round(npos / (ms * 1e-3), 1), "unit": "positions/s", "batch_size": bs,
            "ms_per_step": round(ms, 2),
            "what": "PyTorch-eager restatement of the reference's per-batch op sequence (torch.fft/cuFFT, "
                    "autograd, torch.optim.Adam) on this GPU"}


def cpu_baseline_sample(args, positions=8):
    """Time the oracle port (the reference algorithm restated in numpy/scipy,
    complex64, scipy.fft with every host core) on a bounded sample of the
    workload: one batch of `positions` positions, forward + loss + adjoint."""
    from oracle import ptycho_oracle as O

    ncores = os.cpu_count() or 1
    O.set_workers(ncores)
    rng = np.random.default_rng(0)
    S, P, n, Ho = 8, 4, 128, 512
    obj = np.exp(1j * 0.1 * rng.standard_normal((S, Ho, Ho))).astype(np.complex64)
    probe = (rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))).astype(np.complex64)
    props = O.propagators((n, n), (0.2, 0.2), 300e3, [20.0] * (S - 1), cdtype=np.complex64)
    pos = rng.uniform(70, 440, size=(positions, 2)).astype(np.float32)
    tg = np.abs(rng.standard_normal((positions, n, n))).astype(np.float32)
    mask = np.ones((n, n), np.float32)
    reps = 0
    t0 = time.perf_counter()
    while True:
        O.full_gradients(obj, probe, pos, props, tg, mask, 4096, 1e5, 6.0)
        reps += 1
        el = time.perf_counter() - t0
        if el > args.cpu_seconds or reps >= 50:
            break
    rate = reps * positions / el
    return {"value": round(rate, 2), "unit": "positions/s", "cores": ncores, "kind": "port",
            "sample": f"{reps} x {positions}-position batches of the same geometry, forward+loss+adjoint "
                      f"(optimizer step excluded), complex64, scipy.fft workers={ncores}"}


def accuracy_vs_fp64(pt, nsub=16, iters=3):
    """Accuracy of the FP32 CUDA path against an FP64 run of the oracle (the checker)
    on a bounded sample of the workload: `nsub` positions spread over the scan.

    * forward intensities at the bench's current object and probe: relative L2;
    * `iters` full iterations (forward, loss, adjoint, object-gradient rescale, Adam
      on object lr 5e-3 and probe lr 1e-3, probe orthogonalisation) on those positions
      from the flat object: relative L2 of the first object gradient and phase NRMSE
      of the constrained object (mean phase removed) against the FP64 run.  Adam
      moves every pixel by about lr on its first steps whatever the size of its
      gradient, so pixels the sample barely reaches carry most of the phase error."""
    import torch

    from oracle import ptycho_oracle as O
    from quantem_b200 import engine, ops
    from quantem_b200.diffractive_imaging.ptycho_utils import orthogonalize_probes

    dev = pt.obj.device
    idx = (torch.arange(nsub, device=dev) * (pt.num_gpts // nsub)).to(torch.int64)
    kr, kc = pt.prop
    props64 = (kr.cpu().numpy().astype(np.complex128)[:, :, None] * kc.cpu().numpy().astype(np.complex128)[:, None, :])
    pos = pt.positions[idx].double().cpu().numpy()
    tg = pt.targets[idx].double().cpu().numpy()
    mask = pt.mask.double().cpu().numpy()
    mean_i, up = float(pt.mean_intensity), float(pt.upsample_factor)
    # forward intensities at the current state
    with torch.no_grad():
        obj_c, _ = ops.obj_constrain(pt.obj.detach())
        probe_o = orthogonalize_probes(pt.probe.detach())
        out = ops.batch_forward(obj_c, probe_o, pt.prop, pt.positions, idx, pt.targets, pt.mask, pt.num_gpts,
                                pt.mean_intensity)
    st = O.forward(obj_c.cpu().numpy().astype(np.complex128), probe_o.cpu().numpy().astype(np.complex128), pos,
                   props64)
    i64 = O.detector_intensities(st)
    i32 = out["intensity"].double().cpu().numpy()
    inten_rel = float(np.linalg.norm(i32 - i64) / np.linalg.norm(i64))
    # a few iterations from the flat object, FP32 CUDA vs FP64 oracle
    S, Ho, Wo = pt.obj.shape
    probe0 = pt.probe.detach().clone()
    sub = engine.ProblemTensors(
        obj=torch.ones((S, Ho, Wo), dtype=torch.complex64, device=dev).requires_grad_(True),
        probe=probe0.clone().requires_grad_(True), prop=pt.prop, positions=pt.positions[idx].contiguous(),
        targets=pt.targets[idx].contiguous(), mask=pt.mask, mean_intensity=pt.mean_intensity, upsample_factor=up)
    opts = [engine.make_optimizer([sub.obj], {"type": "adam", "lr": 5e-3}),
            engine.make_optimizer([sub.probe], {"type": "adam", "lr": 1e-3})]
    all_idx = torch.arange(nsub, device=dev, dtype=torch.int64)
    o64 = np.ones((S, Ho, Wo), np.complex128)
    p64 = probe0.cpu().numpy().astype(np.complex128)
    adam = {}

    def adam_step(key, x, g, lr, t):  # torch.optim.Adam on the real and imaginary parts
        m, v = adam.get(key, (np.zeros_like(x), np.zeros_like(x)))
        m = 0.9 * m + 0.1 * g
        v = 0.999 * v + 0.001 * (g.real ** 2 + 1j * g.imag ** 2)
        adam[key] = (m, v)
        den = lambda a: np.sqrt(a) / np.sqrt(1 - 0.999 ** t) + 1e-8  # noqa: E731
        return x - lr / (1 - 0.9 ** t) * (m.real / den(v.real) + 1j * m.imag / den(v.imag))

    grad_rel = None
    for t in range(1, iters + 1):
        engine.batch_step(sub, all_idx, opts)
        if t == 1:
            g32 = sub.obj.grad.detach().cpu().numpy().astype(np.complex128)
        _, g_o, g_p, _ = O.full_gradients(o64, p64, pos, props64, tg, mask, nsub, mean_i, up)
        if t == 1:
            grad_rel = float(np.linalg.norm(g32 - g_o) / np.linalg.norm(g_o))
        o64 = adam_step("o", o64, g_o, 5e-3, t)
        p64 = adam_step("p", p64, g_p, 1e-3, t)
    ph64 = np.angle(O.constrain_object(o64))
    ph32 = np.angle(O.constrain_object(sub.obj.detach().cpu().numpy().astype(np.complex128)))
    d64 = ph64 - ph64.mean()
    nrmse = float(np.linalg.norm((ph32 - ph32.mean()) - d64) / np.linalg.norm(d64))
    return {"forward_intensity_rel_l2": inten_rel, "first_object_gradient_rel_l2": grad_rel,
            "phase_nrmse_after_iters": nrmse, "iters": iters,
            "sample": f"{nsub} positions spread over the scan; FP64 oracle (numpy/scipy) vs FP32 CUDA"}


def c1_config():
    """Single-slice, single-mode configuration: 256^2 object with 200 Gaussian atoms
    (sigma 1.5 px, peak 0.3 rad), 64^2 probe (300 kV, 20 mrad, 200 A defocus, 0.2 A
    pixels), 16 x 16 raster with 4 px step, 1e5 counts per pattern."""
    from quantem_b200 import synthetic

    return synthetic.SyntheticConfig(n=64, slices=1, modes=1, mode_weights=(1.0,), scan=(16, 16), step_px=4.0,
                                     jitter_px=0.0, pad_px=98, peak_phase=0.3, atom_density=200 / 256 ** 2,
                                     sigma_px=1.5, counts=1e5, seed=0)


def run_c1(args):
    """The single-slice, single-mode configuration (256 positions, 20 iterations of the
    amplitude loss, Adam, full batch): the fused path on the GPU against the reference's
    own PyTorch iteration on the GPU and on the host cores (package under baseline/_ref)."""
    import torch

    from quantem_b200 import engine

    dev = torch.device("cuda", 0)
    iters = 20
    cfg = c1_config()
    _, _, pt, opts, batcher = build_problem(0, dev, None, cfg=cfg)
    for _ in range(args.warmup):
        engine.run_iteration(pt, batcher, opts)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(iters):
        loss = engine.run_iteration(pt, batcher, opts)
    e1.record()
    torch.cuda.synchronize()
    ms_eager = e0.elapsed_time(e1) / iters
    eager_loss = float(loss)
    # the same full-batch iteration captured in a CUDA graph and replayed (the iteration is
    # launch-bound at this size: 256 positions of 64 x 64 on one slice)
    git = engine.GraphedIteration(pt).capture(warmup=args.warmup)
    torch.cuda.synchronize()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record()
    for _ in range(iters):
        gl = git.replay()
    g1.record()
    torch.cuda.synchronize()
    ms = g0.elapsed_time(g1) / iters
    npos = pt.num_gpts
    ours = {"positions_per_s": round(npos / (ms * 1e-3), 1), "ms_per_iteration": round(ms, 4),
            "final_loss": float(gl), "graphed": True,
            "eager": {"positions_per_s": round(npos / (ms_eager * 1e-3), 1), "ms_per_iteration": round(ms_eager, 4),
                      "final_loss": eager_loss}}
    del git
    ref = {name: reference_torch_gpu_subprocess(0, npos, steps=iters, warmup=args.warmup,
                                                 extra=["--workload", "c1", "--ref-device", name])
           for name in ("gpu", "cpu")}
    print(json.dumps({"metric": METRIC, "value": ours["positions_per_s"], "unit": "positions/s",
                      "higher_is_better": True, "data": "synthetic", "dtype": "c64/f32",
                      "config": {"workload": "single slice, single mode: 256x256 object, 64x64 probe, 16x16 scan, "
                                             "4 px step, 1e5 counts, 20 iterations, batch 256, Adam",
                                 "iterations": iters},
                      "ours": ours, "reference_torch_gpu": ref.get("gpu"), "reference_torch_cpu": ref.get("cpu"),
                      "cpu_threads": os.cpu_count()}))


def run_kernel_only(args):
    """Launch only the fused forward+adjoint batch kernel on `--positions`
    positions of the same geometry (small cases for ncu captures)."""
    import torch

    from quantem_b200 import ops, synthetic

    device = torch.device("cuda", 0)
    cfg = synthetic.SyntheticConfig(seed=7, scan=(32, 32))  # 1024 positions: small device footprint
    ds = synthetic.make_dataset(cfg, device)
    S, Ho, Wo = ds["obj_shape"]
    obj_c, _ = ops.obj_constrain(ds["obj"])
    probes = ds["probes"] * (ds["mean_intensity"] ** 0.5)
    idx = torch.arange(args.positions, device=device, dtype=torch.int64)
    mask = torch.ones((cfg.n, cfg.n), device=device)
    times = []
    for i in range(args.warmup + args.steps):
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        ops.batch_forward_adjoint(obj_c, probes, ds["propagators"], ds["positions"], idx, ds["amplitudes"], mask,
                                  ds["positions"].shape[0], ds["mean_intensity"], variant=args.variant)
        s1.record()
        torch.cuda.synchronize()
        if i >= args.warmup:
            times.append(s0.elapsed_time(s1))
    print(json.dumps({"mode": "kernel-only", "variant": args.variant, "positions": args.positions, "ms_per_batch": statistics.mean(times),
                      "positions_per_s": args.positions / (statistics.mean(times) * 1e-3)}))


def run_c3(args):
    """Uneven multi-dataset workload: six independent datasets (scans 24^2 ... 64^2,
    slice counts 1..8, one probe mode, 96 x 96 and 128 x 128 windows) in one
    persistent launch per window size per iteration, the iteration captured in a
    CUDA graph, CTA partition from the autotuner.  Compared with the same iteration run eagerly and with one launch
    per dataset."""
    import torch

    from quantem_b200 import engine, multi, synthetic
    from quantem_b200.diffractive_imaging.ptycho_utils import SimpleBatcher

    dev = torch.device("cuda", 0)
    # (scan, slices, probe window): 96 x 96 and 128 x 128 windows alternate
    specs = [(24, 1, 96), (32, 2, 128), (40, 3, 96), (48, 5, 128), (56, 6, 96), (64, 8, 128)]

    def make():
        probs = []
        for k, (scan, S, n) in enumerate(specs):
            cfg = synthetic.SyntheticConfig(n=n, slices=S, modes=1, mode_weights=(1.0,), scan=(scan, scan),
                                            step_px=4.0, pad_px=n // 2, seed=100 + k)
            ds = synthetic.make_dataset(cfg, dev)
            obj = torch.ones(ds["obj_shape"], dtype=torch.complex64, device=dev).requires_grad_(True)
            probe = (ds["probes"] * ds["mean_intensity"] ** 0.5).contiguous().requires_grad_(True)
            probs.append(multi.Problem(obj, probe, ds["propagators"], ds["positions"], ds["amplitudes"].contiguous(),
                                       torch.ones((n, n), device=dev), ds["mean_intensity"], cfg.step_px))
        return probs

    probs = make()
    npos = sum(p.num_gpts for p in probs)
    grids = multi.autotune_grids(probs)
    it = multi.MultiIteration(probs, grids).capture(warmup=args.warmup)

    def timed(fn, k):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(k):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    ms_graph = timed(it.replay, args.steps)
    eager = multi.MultiIteration(make(), grids)
    for _ in range(args.warmup):
        eager.run_eager()
    ms_eager = timed(eager.run_eager, args.steps)
    # one launch per dataset (the reference loops over datasets), same optimiser
    singles = []
    for p in make():
        pt = engine.ProblemTensors(obj=p.obj, probe=p.probe, prop=p.prop, positions=p.positions, targets=p.targets,
                                   mask=p.mask, mean_intensity=p.mean_intensity, upsample_factor=p.upsample_factor)
        opts = [engine.make_optimizer([p.obj], {"type": "adam", "lr": 5e-3}),
                engine.make_optimizer([p.probe], {"type": "adam", "lr": 1e-3})]
        singles.append((pt, opts, SimpleBatcher(pt.num_gpts, pt.num_gpts, rng=0)))

    def loop():
        for pt, opts, bt in singles:
            engine.run_iteration(pt, bt, opts)

    for _ in range(args.warmup):
        loop()
    ms_loop = timed(loop, args.steps)
    print(json.dumps({"workload": "c3: 6 datasets, scans 24^2-64^2, 1-8 slices, 1 mode, 96x96 and 128x128 "
                                  "windows (one persistent launch per window size, one CUDA graph)",
                      "positions": npos, "grids": grids, "unit": "positions/s",
                      "graphed_persistent": round(npos / (ms_graph * 1e-3), 1),
                      "eager_persistent": round(npos / (ms_eager * 1e-3), 1),
                      "one_launch_per_dataset": round(npos / (ms_loop * 1e-3), 1),
                      "ms_per_iteration": {"graphed": round(ms_graph, 3), "eager": round(ms_eager, 3),
                                           "per_dataset": round(ms_loop, 3)}}))


def _bf16_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


# held-out test objects of the learned-initialiser benchmark (peak phase per atom [rad], atoms / px^2
# / slice): the multislice problem's own object and two denser, stronger draws from the training range
C4_OBJECTS = {"c2": (0.1, 0.003), "mid": (0.25, 0.006), "strong": (0.4, 0.008)}


def run_c4(args):
    """Learned initialiser: train the CNN2d (5 levels, 32 base filters, BF16 tcgen05
    kernels) on objects simulated by the forward kernel, then compare the time to a
    phase NRMSE target of the plain reconstruction from a flat start and from the
    learned start, on the 512x512x8 / 4-mode / 128^2 / 64x64-scan problem at the
    configured dose (1e5 counts) and noiseless, for the held-out objects of
    ``C4_OBJECTS``.  Probe known and fixed in both arms, Adam lr 5e-3 decaying 0.97 per
    iteration, batch 256.  Targets: NRMSE 1e-2 and 1.05 x the best NRMSE the flat start
    reaches in the run (the plain method's own plateau)."""
    import torch

    from quantem_b200 import engine, ops, synthetic
    from quantem_b200.core.ml import kernels as kk
    from quantem_b200.diffractive_imaging.learned_init import LearnedInitConfig, LearnedInitializer
    from quantem_b200.diffractive_imaging.ptycho_utils import SimpleBatcher, orthogonalize_probes

    dev = torch.device("cuda", 0)
    scfg = synthetic.SyntheticConfig(seed=0)
    probes = orthogonalize_probes(synthetic.make_probe_modes(scfg, dev))
    props = ops.separable_propagators(scfg.n, (scfg.pixel, scfg.pixel), scfg.energy,
                                      [scfg.slice_thickness] * (scfg.slices - 1), device=dev)
    cfg = LearnedInitConfig(lr=2e-3)
    li = LearnedInitializer(probes, props, cfg, dev, seed=0)
    nobj = args.c4_objects
    torch.cuda.synchronize()
    t0 = time.time()
    li.train(nobj, total_objects=nobj)
    torch.cuda.synchronize()
    train_s = time.time() - t0
    held_out = li.evaluate(32)

    # dominant CNN kernel: the first-layer convolution GEMM (im2col rows x 9*1024) of a training step
    M, K, N = cfg.batch_objects * cfg.scan_crop ** 2, 9 * li.C, cfg.start_filters
    A = torch.randn(M, K, device=dev).to(torch.bfloat16)
    B = torch.randn(N, K, device=dev).to(torch.bfloat16)
    C = torch.empty(M, N, device=dev)
    for _ in range(3):
        kk.gemm(A, B, C)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    reps = 20
    for _ in range(reps):
        kk.gemm(A, B, C)
    e1.record()
    torch.cuda.synchronize()
    gemm_s = e0.elapsed_time(e1) / 1e3 / reps
    gemm_bytes = 2 * M * K + 2 * N * K + 4 * M * N
    hbm, hbm_src = _peaks()
    bf16, bf16_src = _bf16_peak()
    del A, B, C

    proj_phase, nrmse = _proj_phase, _nrmse
    # the reference's own reconstruction of the same data (fresh process, GPU): its best phase
    # NRMSE is the target both arms are timed to
    ref = {}
    for dose, counts in (() if args.skip_torch_reference else (("1e5", 1e5), ("noiseless", 1e12))):
        try:
            env = dict(os.environ)
            cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--torch-gpu", "--workload",
                   "c4", "--c4-iters", str(args.c4_iters), "--c4-counts", str(counts)]
            o = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=1800)
            ref[dose] = json.loads(o.stdout.strip().splitlines()[-1])["reference_torch_gpu"]
        except Exception as exc:
            ref[dose] = {"unavailable": f"{type(exc).__name__}: {exc}"[:300]}
    base_thresholds = [0.5, 0.3, 0.1, 0.05, 0.02, 0.01]
    results = {}
    for oname, (peak, density) in C4_OBJECTS.items():
        results[oname] = {}
        for dose in ("1e5", "noiseless"):
            thresholds = list(base_thresholds)
            if oname == "c2" and "best_nrmse" in ref.get(dose, {}):
                thresholds.append(round(ref[dose]["best_nrmse"] * 1.05, 5))
            dcfg = synthetic.SyntheticConfig(seed=0, counts=1e5 if dose == "1e5" else 1e12, peak_phase=peak,
                                             atom_density=density)
            ds = synthetic.make_dataset(dcfg, dev)
            truth = proj_phase(ds["obj"])
            true_sum = ds["obj"].angle().sum(0)  # unwrapped projected phase
            lo, hi = dcfg.pad_px, dcfg.pad_px + int((dcfg.scan[0] - 1) * dcfg.step_px)
            crop = (slice(lo, hi), slice(lo, hi))
            S, Ho, Wo = ds["obj_shape"]
            probe = (ds["probes"] * (ds["mean_intensity"] / ds["probes"].abs().square().sum()) ** 0.5).contiguous()
            arms = {}
            for arm in ("plain", "learned"):
                torch.cuda.synchronize()
                t0 = time.time()
                if arm == "learned":
                    judge = dict(probe=probe, prop=ds["propagators"], positions=ds["positions"],
                                 targets=ds["amplitudes"].contiguous(), mask=torch.ones((dcfg.n, dcfg.n), device=dev),
                                 mean_intensity=ds["mean_intensity"],
                                 batch=torch.arange(0, ds["positions"].shape[0], 4, device=dev))
                    o0 = li.initial_object(ds["amplitudes"], dcfg.scan, (S, Ho, Wo), (dcfg.pad_px, dcfg.pad_px),
                                           judge=judge)
                else:
                    o0 = torch.ones((S, Ho, Wo), dtype=torch.complex64, device=dev)
                torch.cuda.synchronize()
                elapsed = time.time() - t0
                obj = o0.clone().requires_grad_(True)
                pt = engine.ProblemTensors(obj=obj, probe=probe.clone().requires_grad_(True), prop=ds["propagators"],
                                           positions=ds["positions"], targets=ds["amplitudes"].contiguous(),
                                           mask=torch.ones((dcfg.n, dcfg.n), device=dev),
                                           mean_intensity=ds["mean_intensity"], upsample_factor=dcfg.step_px)
                opt = engine.make_optimizer([obj], {"type": "adam", "lr": 5e-3})
                sched = torch.optim.lr_scheduler.ExponentialLR(opt, 0.97)
                bt = SimpleBatcher(pt.num_gpts, 256, rng=0)
                with torch.no_grad():
                    err = lambda: round(nrmse(proj_phase(ops.constrained_object(obj.detach()))[crop],  # noqa: E731
                                              truth[crop]), 5)
                    curve = [(0, round(elapsed, 4), err())]
                for it in range(1, args.c4_iters + 1):
                    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    s0.record()
                    engine.run_iteration(pt, bt, [opt])
                    s1.record()
                    sched.step()
                    torch.cuda.synchronize()
                    elapsed += s0.elapsed_time(s1) / 1e3
                    with torch.no_grad():
                        curve.append((it, round(elapsed, 4), err()))
                if arm == "plain":
                    thresholds.append(round(1.05 * min(c[2] for c in curve), 5))
                reach = {}
                for th in thresholds:
                    hit = next((c for c in curve if c[2] <= th), None)
                    reach[str(th)] = None if hit is None else hit[1]
                arms[arm] = dict(time_to_nrmse_s=reach, start_nrmse=curve[0][2], best_nrmse=min(c[2] for c in curve),
                                 final_nrmse=curve[-1][2], curve=curve[:: max(1, len(curve) // 12)],
                                 used_learned_start=(getattr(li, "used_learned", None) if arm == "learned" else None),
                                 judge_scale=(getattr(li, "judge_scale", None) if arm == "learned" else None))
            key = str(thresholds[-1])  # 1.05 x the flat start's best
            tp, tl = arms["plain"]["time_to_nrmse_s"][key], arms["learned"]["time_to_nrmse_s"][key]
            arms["to_plain_best"] = {"target_nrmse": float(key), "plain_s": tp, "learned_s": tl,
                                     "ratio": round(tl / tp, 4) if (tp and tl) else None}
            arms["max_abs_projected_phase"] = round(float(true_sum.abs().max()), 3)
            results[oname][dose] = arms
    tp = results["c2"]["noiseless"]["plain"]["time_to_nrmse_s"]["0.01"]
    tl = results["c2"]["noiseless"]["learned"]["time_to_nrmse_s"]["0.01"]
    # at the benchmark dose: both arms timed to within 5 % of the best NRMSE the reference reaches
    vs_ref = None
    if "best_nrmse" in ref.get("1e5", {}):
        key = str(round(ref["1e5"]["best_nrmse"] * 1.05, 5))
        rp = results["c2"]["1e5"]["plain"]["time_to_nrmse_s"].get(key)
        rl = results["c2"]["1e5"]["learned"]["time_to_nrmse_s"].get(key)
        vs_ref = {"target_nrmse": float(key), "plain_s": rp, "learned_s": rl,
                  "ratio": round(rl / rp, 4) if (rp and rl) else None}
    # NRMSE 1e-2 is out of reach in these runs for both arms and for the reference itself (its
    # best: ~0.69 at 1e5 counts, ~0.016 noiseless after 120 iterations), so the headline is the
    # median over the held-out objects and doses of the learned / plain time to 1.05 x the
    # flat start's best NRMSE (inference and judging included)
    ratios = [results[o][d]["to_plain_best"]["ratio"] for o in results for d in results[o]]
    ratios = sorted(r for r in ratios if r is not None)
    med = (ratios[len(ratios) // 2] if len(ratios) % 2 else 0.5 * (ratios[len(ratios) // 2 - 1] +
                                                                    ratios[len(ratios) // 2])) if ratios else None
    reached = {arm: any(results[o][d][arm]["time_to_nrmse_s"]["0.01"] is not None for o in results
                        for d in results[o]) for arm in ("plain", "learned")}
    reached["reference"] = any(ref[d].get("best_nrmse", 1.0) <= 0.01 for d in ref)
    print(json.dumps({
        "metric": "time to phase NRMSE<=1e-2, learned vs plain",
        "value": (round(med, 4) if med is not None else None), "unit": "ratio (learned time / plain time)",
        "value_definition": "median over held-out objects x doses of the learned / plain wall time to 1.05 x the "
                            "flat start's best phase NRMSE",
        "ratio_to_nrmse_1e-2_c2_noiseless": (round(tl / tp, 4) if (tp and tl) else None),
        "nrmse_1e-2_reached": reached,
        "higher_is_better": False, "data": "synthetic",
        "reference_reconstruction": ref,
        "time_to_reference_best_1e5": vs_ref,
        "config": {"workload": "c4: CNN2d 5 levels x 32 filters on 32x32-binned patterns of a 64x64 scan -> "
                               "projected phase; refinement 512x512x8, 4 modes at 128x128",
                   "objects": {k: {"peak_phase": v[0], "atom_density": v[1]} for k, v in C4_OBJECTS.items()},
                   "training_objects": nobj, "refine_iterations": args.c4_iters, "probe": "known, fixed"},
        "cnn": {"train_s": round(train_s, 2), "objects_per_s": round(nobj / train_s, 1),
                "held_out_phase_nrmse": round(held_out, 4),
                "first_layer_gemm": {"M": M, "N": N, "K": K, "ms": round(gemm_s * 1e3, 4),
                                     "tflops": round(2 * M * N * K / gemm_s / 1e12, 2),
                                     "gbs": round(gemm_bytes / gemm_s / 1e9, 1),
                                     "roofline": {"bound": "hbm", "achieved": round(gemm_bytes / gemm_s / 1e9, 1),
                                                  "peak": hbm, "unit": "GB/s",
                                                  "frac": round(gemm_bytes / gemm_s / 1e9 / hbm, 4),
                                                  "peak_source": hbm_src},
                                     "tensor_frac_of_bf16_peak": round(2 * M * N * K / gemm_s / 1e12 / bf16, 4),
                                     "bf16_peak_source": bf16_src}},
        "results": results,
    }))


def run_c5_kernel(args):
    """One 256^2 cluster forward+adjoint launch over --positions positions (profiling case):
    the 1024x1024x16 / 6-mode / 128x128-scan problem, a seeded random subset of the
    positions (as a shuffled batch of the reconstruction), --recompute-every."""
    import torch

    from quantem_b200 import ops, synthetic

    dev = torch.device("cuda", 0)
    cfg = synthetic.SyntheticConfig(n=256, slices=16, modes=6, mode_weights=(0.5, 0.2, 0.1, 0.08, 0.07, 0.05),
                                    scan=(128, 128), step_px=6.0, pad_px=131, counts=1e6, seed=0)
    ds = synthetic.make_dataset(cfg, dev)
    npos = ds["positions"].shape[0]
    probe_o = (ds["probes"] * (ds["mean_intensity"] / ds["probes"].abs().square().sum()) ** 0.5).contiguous()
    obj_c, _ = ops.obj_constrain(torch.ones(ds["obj_shape"], dtype=torch.complex64, device=dev))
    g = torch.Generator().manual_seed(0)
    idx = torch.randperm(npos, generator=g)[:args.positions].to(dev)
    run = lambda: ops.batch_forward_adjoint(obj_c, probe_o, ds["propagators"], ds["positions"], idx,  # noqa: E731
                                            ds["amplitudes"].contiguous(), torch.ones((256, 256), device=dev),
                                            npos, ds["mean_intensity"], recompute_every=args.recompute_every)
    for _ in range(args.warmup):
        run()
    ops.PROFILE_EVENTS = []
    for _ in range(args.steps):
        run()
    torch.cuda.synchronize()
    ms = statistics.median(a.elapsed_time(b) for a, b in ops.PROFILE_EVENTS)
    ops.PROFILE_EVENTS = None
    flops = 4 * 6 * 16 * 5 * 256 ** 2 * 16 + 40 * 6 * 16 * 256 ** 2
    print(json.dumps({"workload": "c5 kernel: 256^2, 16 slices, 6 modes, forward+adjoint",
                      "positions": args.positions, "recompute_every": args.recompute_every,
                      "ms_per_launch": round(ms, 3), "positions_per_s": round(args.positions / (ms * 1e-3), 1),
                      "fp32_tflops": round(flops * args.positions / (ms * 1e-3) / 1e12, 2)}))


def run_c4_gemm(args):
    """The first-layer convolution GEMM of a c4 training step alone (profiling case)."""
    import torch

    from quantem_b200.core.ml import kernels as kk

    dev = torch.device("cuda", 0)
    M, K, N = 16 * 32 * 32, 9 * 1024, 32
    A = torch.randn(M, K, device=dev).to(torch.bfloat16)
    B = torch.randn(N, K, device=dev).to(torch.bfloat16)
    C = torch.empty(M, N, device=dev)
    for _ in range(args.warmup):
        kk.gemm(A, B, C)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        kk.gemm(A, B, C)
    e1.record()
    torch.cuda.synchronize()
    s_ = e0.elapsed_time(e1) / 1e3 / args.steps
    byt = 2 * M * K + 2 * N * K + 4 * M * N
    print(json.dumps({"workload": "c4 first-layer conv GEMM", "M": M, "N": N, "K": K, "ms": round(s_ * 1e3, 4),
                      "gbs": round(byt / s_ / 1e9, 1), "tflops": round(2 * M * N * K / s_ / 1e12, 2)}))


def c5_config(scan=(128, 128)):
    """Large multislice: 1024 x 1024 x 16 object, 6 modes at 256^2, 6 px raster step with
    +-0.5 px jitter, 1e6 counts; the padding keeps the object at 1024^2 for any scan."""
    from quantem_b200 import synthetic

    pad = (1024 - (scan[0] - 1) * 6) // 2
    return synthetic.SyntheticConfig(n=256, slices=16, modes=6, mode_weights=(0.5, 0.2, 0.1, 0.08, 0.07, 0.05),
                                     scan=scan, step_px=6.0, pad_px=pad, counts=1e6, seed=0)


def run_c5(args):
    """Large multislice: 1024x1024x16 object, 6 modes at 256x256 on 4-CTA clusters, 128x128 scan
    (16384 positions, 6 px step, jitter), 1e6 counts, full-batch Adam iterations.  The
    adjoint keeps every wave (recompute_every=0) or recomputes from a checkpoint every
    4 slices; both are timed."""
    import torch

    from quantem_b200 import engine, ops, synthetic
    from quantem_b200.diffractive_imaging.ptycho_utils import SimpleBatcher

    dev = torch.device("cuda", 0)
    cfg = c5_config()
    t0 = time.time()
    ds = synthetic.make_dataset(cfg, dev)
    torch.cuda.synchronize()
    sim_s = time.time() - t0
    S, Ho, Wo = ds["obj_shape"]
    npos = ds["positions"].shape[0]
    hbm, hbm_src = _peaks()
    fp32 = fp32_peak_tflops(dev)
    flops_pos = 4 * cfg.modes * S * 5 * cfg.n ** 2 * math.log2(cfg.n ** 2) + 40 * cfg.modes * S * cfg.n ** 2
    out = {}
    for ck in (4, 0):
        obj = torch.ones((S, Ho, Wo), dtype=torch.complex64, device=dev).requires_grad_(True)
        probe = (ds["probes"] * (ds["mean_intensity"] / ds["probes"].abs().square().sum()) ** 0.5
                 ).contiguous().requires_grad_(True)
        pt = engine.ProblemTensors(obj=obj, probe=probe, prop=ds["propagators"], positions=ds["positions"],
                                   targets=ds["amplitudes"].contiguous(), mask=torch.ones((cfg.n, cfg.n), device=dev),
                                   mean_intensity=ds["mean_intensity"], upsample_factor=cfg.step_px,
                                   recompute_every=ck)
        opts = [engine.make_optimizer([obj], {"type": "adam", "lr": 5e-3}),
                engine.make_optimizer([probe], {"type": "adam", "lr": 1e-3})]
        bt = SimpleBatcher(npos, npos, rng=0)
        for _ in range(args.warmup):
            engine.run_iteration(pt, bt, opts)
        ops.PROFILE_EVENTS = []
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            engine.run_iteration(pt, bt, opts)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        kms = sum(a.elapsed_time(b) for a, b in ops.PROFILE_EVENTS) / max(len(ops.PROFILE_EVENTS), 1)
        ops.PROFILE_EVENTS = None
        ws = ops.workspace(dev)
        out[f"recompute_every_{ck}"] = {
            "positions_per_s": round(npos / (ms * 1e-3), 1), "ms_per_iteration": round(ms, 2),
            "kernel_ms": round(kms, 2),
            "kernel_fp32_tflops": round(flops_pos * npos / (kms * 1e-3) / 1e12, 2),
            "scratch_gb": round(ws.scratch.numel() * 8 / 1e9, 3)}
        del pt, opts, obj, probe
        torch.cuda.empty_cache()
    del ds
    torch.cuda.empty_cache()
    # the reference's own iteration at this geometry, in a fresh process, on a 32 x 32 sub-scan
    # (1024 positions; same object, probe and slices), the batch halved from 1024 until it fits
    ref = None if args.skip_torch_reference else reference_torch_gpu_subprocess(
        0, 1024, steps=2, warmup=1, extra=["--workload", "c5"])
    print(json.dumps({
        "metric": METRIC, "value": out["recompute_every_4"]["positions_per_s"], "unit": "positions/s",
        "reference_torch_gpu": ref,
        "higher_is_better": True, "data": "synthetic",
        "config": {"workload": "c5: 1024x1024x16 object, 6 modes at 256x256 (4-CTA cluster FFT), 128x128 scan, "
                               "16384 positions, full batch, Adam", "simulate_s": round(sim_s, 2)},
        "algorithmic_gflop_per_position": round(flops_pos / 1e9, 3),
        "fp32_peak_tflops": (round(fp32, 2) if fp32 else None), "results": out}))


def run_preprocess(args):
    """PtychographyDatasetRaster.preprocess (CoM, plane fit, rotation, intensity
    normalisation) on the 64x64-scan, 128x128-pattern dataset: host path vs GPU kernels."""
    import numpy as np
    import torch

    from quantem_b200 import synthetic
    from quantem_b200.diffractive_imaging import Dataset4dstem, PtychographyDatasetRaster

    dev = torch.device("cuda", 0)
    cfg = synthetic.SyntheticConfig(seed=0)
    ds = synthetic.make_dataset(cfg, dev)
    # raw 4D data: the simulated counts back in detector (centred) layout order, scan 64 x 64
    raw = torch.fft.fftshift(ds["intensities"], dim=(-2, -1)).view(64, 64, 128, 128).cpu().numpy()
    res = {}
    for where in ("cpu", "cuda"):
        times = []
        for _ in range(2 if where == "cpu" else 4):
            d4 = Dataset4dstem.from_array(raw, sampling=(1.2, 1.2, 1 / 25.6, 1 / 25.6),
                                          units=("A", "A", "A^-1", "A^-1"))
            pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
            torch.cuda.synchronize()
            t0 = time.time()
            pd.preprocess(com_fit_function="plane", force_com_rotation=0, force_com_transpose=False,
                          plot_rotation=False, plot_com=False, probe_energy=300e3, device=where)
            torch.cuda.synchronize()
            times.append(time.time() - t0)
        res[where] = dict(seconds=round(min(times), 4), on=pd._preprocessed_on,
                          mean_intensity=pd.mean_diffraction_intensity)
    print(json.dumps({"workload": "dataset preprocess: 64x64 scan, 128x128 patterns (CoM, plane fit, "
                                  "rotation search, Fourier-shift centring)",
                      "host_s": res["cpu"]["seconds"], "gpu_s": res["cuda"]["seconds"],
                      "speedup": round(res["cpu"]["seconds"] / res["cuda"]["seconds"], 1),
                      "mean_intensity_rel_diff": abs(res["cpu"]["mean_intensity"] - res["cuda"]["mean_intensity"])
                      / res["cpu"]["mean_intensity"]}))


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def reference_cpu_config():
    """The bounded CPU sample of the headline geometry: an 8 x 8 sub-scan (64 positions,
    6 px step, +-0.5 px jitter) with the padding that keeps the object at 512 x 512 x 8;
    4 modes at 128^2, 1e5 counts."""
    from quantem_b200 import synthetic

    return synthetic.SyntheticConfig(seed=0, scan=(8, 8), pad_px=235)


def reference_cpu_sample(steps, warmup):
    """The reference's own ``Ptychography.reconstruct(device="cpu")`` (autograd, Adam,
    probe orthogonalisation; package under baseline/_ref) on every host core, over the
    bounded sample of ``reference_cpu_config`` with batch 64 (one batch per iteration).
    Falls back to the oracle port (kind "port") when the reference package is absent."""
    import torch

    ncores = os.cpu_count() or 1
    torch.set_num_threads(ncores)
    cfg = reference_cpu_config()
    npos = cfg.scan[0] * cfg.scan[1]
    if torch.cuda.is_available():  # the sample's data are simulated with this package's CUDA kernels
        try:
            res = reference_torch_gpu(cfg, "cpu", steps, warmup, npos)
        except Exception as exc:  # a reported baseline: report why, never fail the bench
            res = {"unavailable": f"{type(exc).__name__}: {exc}"[:300]}
    else:
        res = {"unavailable": "no CUDA device to simulate the sample's data"}
    if "unavailable" not in res:
        return {"value": res["value"], "unit": "positions/s", "cores": torch.get_num_threads(), "kind": "reference",
                "cpu_model": _cpu_model(), "ms_per_step": res["ms_per_step"],
                "sample": f"quantem Ptychography.reconstruct(device='cpu') from baseline/_ref, {steps} timed "
                          f"iterations after {warmup} warm-up: {npos} positions (8x8 sub-scan) of the 512x512x8 "
                          "object / 4 modes at 128^2 geometry, batch 64, autograd + Adam + probe "
                          "orthogonalisation, complex64, torch threads = host cores"}
    port = cpu_baseline_sample(argparse.Namespace(cpu_seconds=15.0))
    port["reference_unavailable"] = res["unavailable"]
    return port


def reference_cpu_subprocess(local_device: int, steps: int, warmup: int):
    """``reference_cpu_sample`` in a fresh process (its own torch threads and allocator)."""
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "LOCAL_WORLD_SIZE", "MASTER_ADDR", "MASTER_PORT",
                        "GROUP_RANK", "ROLE_RANK", "TORCHELASTIC_RUN_ID")}
    visible = os.environ.get("CUDA_VISIBLE_DEVICES")
    env["CUDA_VISIBLE_DEVICES"] = visible.split(",")[local_device] if visible else str(local_device)
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--cpu-sample",
           "--steps", str(steps), "--warmup", str(warmup)]
    try:
        out = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=900)
        line = json.loads(out.stdout.strip().splitlines()[-1])
    except Exception as exc:  # a reported baseline: never fail the bench over it
        return {"unavailable": f"{type(exc).__name__}: {exc}"[:300]}
    return line.get("cpu_baseline", line)


def run_reference(args):
    """``--impl reference``: the reference's own CPU iteration (see reference_cpu_sample),
    rank 0 only; the other ranks exit without work."""
    rank, world, _ = _dist_env()
    if rank != 0:
        return
    cpu = reference_cpu_sample(args.steps, args.warmup)
    line = {"metric": METRIC, "value": cpu["value"], "unit": "positions/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64/f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "parallelism": "host cores",
                       "sample": "64 positions (8x8 sub-scan) per step, batch 64"},
            "cpu_baseline": cpu, "e2e": {"value": cpu["value"], "unit": "positions/s",
                                          "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if "ms_per_step" in cpu:
        line["ms_per_step"] = cpu["ms_per_step"]
    print(json.dumps(line))


def _reference_setup(cfg, dev, ref_dir=None, probe_known=False):
    """The reference's own set-up for a dataset simulated for ``cfg``: ``Dataset4dstem``,
    ``PtychographyDatasetRaster.preprocess``, ``ObjectPixelated.from_uniform``,
    ``ProbePixelated.from_params`` with the mode weights, ``Ptychography.from_models(...)
    .preprocess(...)`` and the jittered positions.  ``probe_known`` replaces the initial probe
    by the simulation's probe modes.  Returns (ptycho, dataset, simulated data) or a dict
    with ``unavailable``."""
    import numpy as np
    import torch

    from baseline.reference_import import import_reference
    from quantem_b200 import synthetic

    ref_dir = ref_dir or os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isdir(os.path.join(ref_dir, "quantem")):
        return {"unavailable": f"reference package not installed under {os.path.relpath(ref_dir, ROOT)} "
                               "(baseline/install_reference.sh)"}
    import_reference(ref_dir)
    from quantem.core.datastructures.dataset4dstem import Dataset4dstem
    from quantem.diffractive_imaging.dataset_models import PtychographyDatasetRaster
    from quantem.diffractive_imaging.detector_models import DetectorPixelated
    from quantem.diffractive_imaging.object_models import ObjectPixelated
    from quantem.diffractive_imaging.probe_models import ProbePixelated
    from quantem.diffractive_imaging.ptychography import Ptychography

    # the data are simulated with this package's forward kernels (on the GPU) in every case
    sim_dev = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else dev
    ds = synthetic.make_dataset(cfg, sim_dev)
    nr, nc = cfg.scan
    data = ds["intensities"].cpu().numpy().reshape(nr, nc, cfg.n, cfg.n)
    rs = 1.0 / (cfg.n * cfg.pixel)
    d4 = Dataset4dstem.from_array(data, sampling=(cfg.step_px * cfg.pixel, cfg.step_px * cfg.pixel, rs, rs),
                                  units=("A", "A", "A^-1", "A^-1"))
    pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
    # the simulated patterns are centred exactly: "no_shift" keeps them as simulated (a fitted
    # centre of mass would shift every pattern by its sub-pixel mean offset, a descan error the
    # reconstruction then fits with a phase ramp)
    pd.preprocess(com_fit_function="no_shift", force_com_rotation=0, force_com_transpose=False,
                  plot_rotation=False, plot_com=False, probe_energy=cfg.energy)
    obj_model = ObjectPixelated.from_uniform(num_slices=cfg.slices, slice_thicknesses=cfg.slice_thickness,
                                             obj_type="complex")
    probe_model = ProbePixelated.from_params(
        probe_params={"energy": cfg.energy, "defocus": cfg.defocus, "semiangle_cutoff": cfg.semiangle},
        num_probes=cfg.modes, rng=cfg.seed + 1, initial_probe_weights=list(cfg.mode_weights))
    pt = Ptychography.from_models(dset=pd, obj_model=obj_model, probe_model=probe_model,
                                  detector_model=DetectorPixelated(), device="cpu", verbose=0, rng=cfg.seed + 2)
    pt.preprocess(obj_padding_px=(cfg.pad_px, cfg.pad_px))
    # the positions the data were simulated at (raster + the simulation's jitter)
    pd.scan_positions_px = ds["positions"].float().cpu().contiguous()
    if probe_known:
        # the simulation's mode shapes at the reference's own intensity scale (its targets are
        # normalised by its preprocessing, and its initial probe is scaled to match them)
        ref_scale = float(probe_model._probe.detach().abs().square().sum())
        known = (ds["probes"] * (ref_scale / float(ds["probes"].abs().square().sum())) ** 0.5).cpu()
        with torch.no_grad():
            probe_model._probe.data = known.to(probe_model._probe.dtype).clone()
            probe_model._initial_probe = known.clone()
    return pt, pd, ds


def reference_torch_gpu(cfg, device, steps, warmup, batch_size, ref_dir=None, verbose=False):
    """Positions/s of the reference's own PyTorch iteration on `device`.

    Runs quantem's ``Ptychography.reconstruct`` (ptychography.py:146-308) unmodified:
    autograd, probe orthogonalisation, Adam on object (lr 5e-3) and probe (lr 1e-3),
    on a dataset simulated for `cfg` and set up by ``_reference_setup`` (the reference's
    own classes, imported from ``ref_dir``, default ``baseline/_ref``, with the import
    shim in ``baseline/reference_import.py``).  The batch starts at `batch_size` and is
    halved while the GPU runs out of memory; the batch used is reported.  Timed:
    ``reconstruct(num_iters=steps)`` as one call between CUDA events (one end-of-call
    ``gc.collect`` / ``empty_cache`` per `steps` iterations)."""
    import torch

    dev = torch.device(device)
    t0 = time.perf_counter()
    got = _reference_setup(cfg, dev, ref_dir)
    if isinstance(got, dict):
        return got
    pt, pd, _ = got
    setup_s = time.perf_counter() - t0
    dev_arg = "gpu" if dev.type == "cuda" else "cpu"
    opt = {"object": {"type": "adam", "lr": 5e-3}, "probe": {"type": "adam", "lr": 1e-3}}
    sync = torch.cuda.synchronize if dev.type == "cuda" else (lambda: None)

    bs = batch_size
    while True:  # the whole warm-up and timed run at one batch; halved while the GPU runs out of memory
        try:
            pt.reconstruct(num_iters=1, reset=True, optimizer_params=opt, batch_size=bs, device=dev_arg)
            if warmup > 1:
                pt.reconstruct(num_iters=warmup - 1, batch_size=bs)
            sync()
            if dev.type == "cuda":
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                pt.reconstruct(num_iters=steps, batch_size=bs)
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / steps
            else:
                t1 = time.perf_counter()
                pt.reconstruct(num_iters=steps, batch_size=bs)
                ms = (time.perf_counter() - t1) * 1e3 / steps
            break
        except torch.OutOfMemoryError:
            if dev.type == "cuda":
                torch.cuda.empty_cache()
            bs //= 2
            if bs < 1:
                return {"unavailable": "out of memory at batch 1"}
    npos = pd.num_gpts
    losses = [float(x) for x in pt.iter_losses]
    if verbose:
        print(f"reference setup {setup_s:.1f} s, batch {bs}, {ms:.1f} ms/iteration", file=sys.stderr)
    return {"value": round(npos / (ms * 1e-3), 1), "unit": "positions/s", "batch_size": bs,
            "ms_per_step": round(ms, 2), "positions": npos, "setup_s": round(setup_s, 1),
            "final_loss": losses[-1] if losses else None,
            "what": "quantem Ptychography.reconstruct (reference PyTorch path, autograd, Adam) on this device"}


def _proj_phase(o):
    import torch

    p = o[0]
    for k in range(1, o.shape[0]):
        p = p * o[k]
    return torch.angle(p)


def _nrmse(a, t):
    a, t = a.double(), t.double()
    d = (a - a.mean()) - (t - t.mean())
    return float(d.norm() / (t - t.mean()).norm())


def reference_c4_curve(counts, iters, batch=256):
    """The reference's own ``Ptychography.reconstruct`` on the learned-initialiser
    benchmark data (512x512x8 object, 4 modes at 128^2, 64x64 scan, ``counts`` per pattern)
    on the GPU, with the same schedule as this package's arms: probe known and fixed (no
    probe optimiser), Adam on the object at lr 5e-3 decaying 0.97 per iteration
    (scheduler "exp"), batch 256, flat start.  Returns the phase-NRMSE curve of the
    projected transmission over the scanned field (mean removed), its best value and the
    CUDA-event time per iteration."""
    import torch

    from quantem_b200 import synthetic

    dev = torch.device("cuda", 0)
    dcfg = synthetic.SyntheticConfig(seed=0, counts=counts)
    got = _reference_setup(dcfg, dev, probe_known=True)
    if isinstance(got, dict):
        return got
    pt, pd, ds = got
    truth = _proj_phase(ds["obj"]).cpu()
    lo, hi = dcfg.pad_px, dcfg.pad_px + int((dcfg.scan[0] - 1) * dcfg.step_px)
    crop = (slice(lo, hi), slice(lo, hi))
    opt = {"object": {"type": "adam", "lr": 5e-3}}
    sched = {"object": {"type": "exp", "gamma": 0.97}}
    curve = [(0, 0.0, round(_nrmse(_proj_phase(pt.obj_model.obj.detach().cpu())[crop], truth[crop]), 5))]
    elapsed = 0.0
    for it in range(1, iters + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        if it == 1:  # no reset: it would put the raster positions back in place of the simulated ones
            pt.reconstruct(num_iters=1, optimizer_params=opt, scheduler_params=sched, batch_size=batch,
                           device="gpu")
        else:
            pt.reconstruct(num_iters=1, batch_size=batch, device="gpu")
        e1.record()
        torch.cuda.synchronize()
        elapsed += e0.elapsed_time(e1) / 1e3
        with torch.no_grad():
            ph = _proj_phase(pt.obj_model.obj.detach().cpu())
        curve.append((it, round(elapsed, 4), round(_nrmse(ph[crop], truth[crop]), 5)))
    best = min(c[2] for c in curve)
    return {"best_nrmse": best, "best_at_iteration": next(c[0] for c in curve if c[2] == best),
            "final_nrmse": curve[-1][2], "s_per_iteration": round(elapsed / iters, 4),
            "curve": curve[:: max(1, len(curve) // 16)] + [curve[-1]],
            "what": "quantem Ptychography.reconstruct on the GPU, probe known and fixed, Adam 5e-3 x 0.97^it, "
                    "batch 256, flat start"}


def reference_torch_gpu_subprocess(local_device: int, batch_size: int, steps: int = 3, warmup: int = 3,
                                   extra=()):
    """``reference_torch_gpu`` in a fresh process on the same GPU (its own allocator and host
    threads, nothing of this process's state), via ``bench.py --impl reference --torch-gpu``."""
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "LOCAL_WORLD_SIZE", "MASTER_ADDR", "MASTER_PORT",
                        "GROUP_RANK", "ROLE_RANK", "TORCHELASTIC_RUN_ID")}
    visible = os.environ.get("CUDA_VISIBLE_DEVICES")
    if visible:
        env["CUDA_VISIBLE_DEVICES"] = visible.split(",")[local_device]
    else:
        env["CUDA_VISIBLE_DEVICES"] = str(local_device)
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--torch-gpu", "--steps", str(steps),
           "--warmup", str(warmup), "--batch-size", str(batch_size), *extra]
    out = None
    try:
        out = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=1800)
        line = json.loads(out.stdout.strip().splitlines()[-1])
    except Exception as exc:  # the reference is a baseline here: report, never fail the bench
        err = out.stderr.strip().splitlines()[-1] if out is not None and out.stderr.strip() else ""
        return {"unavailable": f"{type(exc).__name__}: {exc}; {err}"[:400]}
    if "unavailable" in line:
        return {"unavailable": line["unavailable"]}
    return line.get("reference_torch_gpu", line)


def run_reference_torch_gpu(args):
    rank, world, _ = _dist_env()
    if rank != 0:
        return
    import torch

    from quantem_b200 import synthetic

    if args.workload == "c4":
        res = reference_c4_curve(float(args.c4_counts), args.c4_iters)
        print(json.dumps({"impl": "reference", "workload": "c4", "counts": args.c4_counts,
                          "reference_torch_gpu": res}))
        return
    c1 = args.workload == "c1"
    c5 = args.workload == "c5"
    cfg = c1_config() if c1 else (c5_config(scan=(32, 32)) if c5 else synthetic.SyntheticConfig(seed=0))
    device = "cuda:0" if args.ref_device == "gpu" else "cpu"
    if device == "cpu":
        torch.set_num_threads(os.cpu_count() or 1)
    res = reference_torch_gpu(cfg, device, args.steps, args.warmup,
                              cfg.scan[0] * cfg.scan[1] if c1 else args.batch_size)
    line = {"metric": METRIC, "unit": "positions/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64/f32",
            "data": "synthetic", "impl": "reference", "device": args.ref_device,
            "config": {"workload": "c1" if c1 else ("c5 geometry, 32x32 sub-scan" if c5 else WORKLOAD),
                       "parallelism": "replicas1"}}
    if "unavailable" in res:
        line["unavailable"] = res["unavailable"]
    else:
        line.update(value=res["value"], ms_per_step=res["ms_per_step"], reference_torch_gpu=res)
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch-size", type=int, default=4096)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--kernel-only", action="store_true", help="time only the fused batch kernel")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5", "preprocess"],
                    help="c2: the headline multislice mixed-probe iteration; c3: uneven multi-dataset launch; "
                         "c4: learned initialiser vs flat start; c5: 256x256 windows on thread-block clusters")
    ap.add_argument("--c4-objects", type=int, default=20000, help="training objects for --workload c4")
    ap.add_argument("--recompute-every", type=int, default=0, help="adjoint checkpoint interval (--workload c5)")
    ap.add_argument("--c4-iters", type=int, default=120, help="refinement iterations per arm for --workload c4")
    ap.add_argument("--c4-counts", type=float, default=1e5, help="dose of the reference's c4 curve (--impl reference)")
    ap.add_argument("--torch-gpu", action="store_true",
                    help="with --impl reference: time the reference's own PyTorch iteration on the GPU "
                         "(package under baseline/_ref) instead of the CPU oracle port")
    ap.add_argument("--ref-device", default="gpu", choices=["gpu", "cpu"],
                    help="with --impl reference --torch-gpu: the device the reference's iteration runs on")
    ap.add_argument("--skip-torch-reference", action="store_true",
                    help="do not time the PyTorch-eager restatement of the reference path nor the "
                         "reference's own PyTorch iteration on the GPU")
    ap.add_argument("--positions", type=int, default=296, help="positions per launch with --kernel-only")
    ap.add_argument("--cpu-sample", action="store_true",
                    help="with --impl reference: the bounded reference CPU sample for the cpu_baseline key "
                         "(keeps the given --warmup)")
    ap.add_argument("--variant", default="auto", choices=["auto", "serial", "cluster"],
                    help="mapping of probe modes onto CTAs (--kernel-only)")
    args = ap.parse_args()
    if args.warmup < 3 and not args.cpu_sample:
        args.warmup = 3
    if args.impl == "reference" and args.torch_gpu:
        run_reference_torch_gpu(args)
    elif args.workload == "c1":
        run_c1(args)
    elif args.workload == "c3":
        run_c3(args)
    elif args.workload == "c4":
        run_c4_gemm(args) if args.kernel_only else run_c4(args)
    elif args.workload == "c5":
        run_c5_kernel(args) if args.kernel_only else run_c5(args)
    elif args.workload == "preprocess":
        run_preprocess(args)
    elif args.kernel_only:
        run_kernel_only(args)
    elif args.impl == "reference":
        run_reference_torch_gpu(args) if args.torch_gpu else run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
