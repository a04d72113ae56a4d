"""Generate golden fixtures by running the reference quantem package itself.

Run in a container where the reference source tree is mounted:

    python tests/golden/make_golden.py <reference checkout>/src

For each seeded case this records the reference's own set-up products
(targets, mean intensity, scan positions, object shape, initial probe,
propagators), the predicted intensities / loss / autograd gradients of one
batch, and the object, probe and losses after a few ``reconstruct`` iterations.
The fixtures pin the CPU oracle (``oracle/ptycho_oracle.py``), the host-side
set-up of ``quantem_b200.diffractive_imaging`` and the CUDA path.

Inputs are synthetic: Gaussian-atom phase objects, probes from the reference's
``real_space_probe`` and Poisson-noised intensities simulated with the oracle's
forward model.  The reference's own gradient test (tests/diffractive_imaging/
test_ptychography.py:31-146) is restated as case ``whitenoise64`` with the same
recipe (white-noise phase, analytic soft-aperture probe, 1 px raster).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ptycho_oracle as O  # noqa: E402
from baseline.reference_import import import_reference  # noqa: E402
from tests.golden.c2small import perturbed_object  # noqa: E402


def _c64(x):
    return np.asarray(x).astype(np.complex64)


def _f32(x):
    return np.asarray(x).astype(np.float32)


def simulate_data(true_obj, probes, positions_px, props, counts, rng):
    """Poisson diffraction data in detector (centred) layout, shape (N, H, W)."""
    st = O.forward(true_obj, probes, positions_px, props)
    inten = O.detector_intensities(st)
    inten = inten / inten.sum(axis=(-2, -1), keepdims=True).mean() * counts
    return rng.poisson(inten).astype(np.float32)


def run_case(name, *, H, S, P, nscan, step_px, pad, dz, counts, jitter, batch, iters,
             weights=None, seed=0, opt=None, orthogonalize=True, keep_data=True, obj_type="complex"):
    import torch
    from quantem.core.datastructures.dataset4dstem import Dataset4dstem
    from quantem.diffractive_imaging.complex_probe import real_space_probe
    from quantem.diffractive_imaging.dataset_models import PtychographyDatasetRaster
    from quantem.diffractive_imaging.detector_models import DetectorPixelated
    from quantem.diffractive_imaging.object_models import ObjectPixelated
    from quantem.diffractive_imaging.probe_models import ProbePixelated
    from quantem.diffractive_imaging.ptychography import Ptychography

    rng = np.random.default_rng(seed)
    px = 0.2  # real-space pixel [A]
    rs = 1.0 / (H * px)
    energy = 300e3
    # --- synthetic truth (oracle forward model, FP64) ---
    probe1 = real_space_probe(gpts=(H, H), sampling=(px, px), energy=energy, semiangle_cutoff=20.0,
                              aberration_coefs={"C10": -200.0}).numpy().astype(np.complex128)
    probes = np.stack([probe1] + [np.roll(probe1, k + 1, axis=1) * 0.3 for k in range(P - 1)])
    ext = (nscan - 1) * step_px
    obj_hw = int(ext + 2 * pad)
    obj_hw += (-obj_hw) % 8
    phase = np.stack([O.gaussian_atom_phase((obj_hw, obj_hw), max(4, obj_hw * obj_hw // 400), 1.5,
                                            0.3 if S == 1 else 0.1, rng) for _ in range(S)])
    true_obj = np.exp(1j * phase)
    grid = np.stack(np.meshgrid(np.arange(nscan), np.arange(nscan), indexing="ij"), -1).reshape(-1, 2)
    pos_true = grid * step_px + pad
    if jitter:
        pos_true = pos_true + rng.uniform(-0.5, 0.5, size=pos_true.shape)
    props_true = O.propagators((H, H), (px, px), energy, [dz] * (S - 1))
    data = simulate_data(true_obj, probes, pos_true, props_true, counts, rng)

    d4 = Dataset4dstem.from_array(data.reshape(nscan, nscan, H, H),
                                  sampling=(step_px * px, step_px * px, rs, rs),
                                  units=("A", "A", "A^-1", "A^-1"))
    pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
    pd.preprocess(com_fit_function="constant", force_com_rotation=0, force_com_transpose=False,
                  plot_rotation=False, plot_com=False, probe_energy=energy)
    obj_model = ObjectPixelated.from_uniform(num_slices=S, slice_thicknesses=dz, obj_type=obj_type)
    probe_model = ProbePixelated.from_params(
        probe_params={"energy": energy, "defocus": 200.0, "semiangle_cutoff": 20.0},
        num_probes=P, rng=seed + 1, initial_probe_weights=weights)
    pt = Ptychography.from_models(dset=pd, obj_model=obj_model, probe_model=probe_model,
                                  detector_model=DetectorPixelated(), device="cpu", verbose=0,
                                  rng=seed + 2)
    pt.preprocess(obj_padding_px=(pad, pad))
    if jitter:
        jit = rng.uniform(-0.5, 0.5, size=(pd.num_gpts, 2)).astype(np.float32)
        pd.scan_positions_px = pd.scan_positions_px.detach() + torch.tensor(jit)

    out = dict(
        H=H, S=S, P=P, nscan=nscan, step_px=step_px, pad=pad, dz=dz, px=px, energy=energy,
        jitter=int(jitter), batch=batch, iters=iters, seed=seed, counts=counts, obj_type=obj_type,
        weights=np.asarray(weights if weights is not None else [], dtype=np.float64),
        orthogonalize=int(orthogonalize),
        data=data if keep_data else np.zeros(0, np.float32),
        targets=_f32(pd.targets.numpy()),
        mean_intensity=np.float64(pd.mean_diffraction_intensity),
        positions=_f32(pd.scan_positions_px.detach().numpy()),
        initial_positions=_f32(pd.initial_scan_positions_px.numpy()),
        obj_shape=np.asarray(pt.obj_shape_full),
        obj_padding_px=np.asarray(pt.obj_padding_px),
        upsample_factor=np.float64(pd.upsample_factor),
        probe_init=_c64(probe_model._probe.detach().numpy()),
        propagators=_c64(pt._propagators.numpy()) if S > 1 else np.zeros((0, H, H), np.complex64),
        sampling=np.asarray(pt.sampling, dtype=np.float64),
    )

    # --- one batch at a perturbed object: intensities, loss, gradients ---
    constraints = {"probe": {"orthogonalize_probe": bool(orthogonalize)}}
    pt.constraints = constraints
    with torch.no_grad():
        shp = tuple(obj_model._obj.shape)
        if obj_type == "potential":
            # a real potential with negative values, so that the positivity clamp acts
            obj_model._obj.data = torch.tensor(0.05 + 0.1 * rng.standard_normal(shp), dtype=torch.float32)
        else:
            amp = 1.0 - 0.3 * rng.random(shp)
            ph = 0.4 * rng.standard_normal(shp)
            obj_model._obj.data = torch.tensor(amp * np.exp(1j * ph), dtype=torch.complex64)
    out["obj_perturbed"] = obj_model._obj.detach().numpy().copy()
    bi = np.arange(min(batch, pd.num_gpts))
    obj_model._obj.grad = None
    probe_model._probe.grad = None
    pt.dset._set_targets("l2_amplitude")
    pt.compute_propagator_arrays()
    patch_indices, _pos, frac, descan = pt.dset.forward(bi, pt.obj_padding_px)
    sp = probe_model.forward(frac)
    op = obj_model.forward(patch_indices)
    prop, ov = pt.forward_operator(op, sp, descan)
    inten = pt.detector_model.forward(ov)
    loss, tg = pt.error_estimate(inten, bi)
    pt.backward(loss, True, op, prop, ov, patch_indices, tg)
    out.update(
        batch_indices=bi,
        batch_intensities=_f32(inten.detach().numpy()),
        batch_loss=np.float64(loss.item()),
        grad_obj=obj_model._obj.grad.numpy().copy(),
        grad_probe=_c64(probe_model._probe.grad.numpy()),
        probe_ortho=_c64(probe_model.probe.detach().numpy()),
    )

    # --- analytic (autograd=False) update directions at the same state (complex objects) ---
    with torch.no_grad():
        obj_model._obj.grad = None
        probe_model._probe.grad = None
        patch_indices, _pos, frac, descan = pt.dset.forward(bi, pt.obj_padding_px)
        sp = probe_model.forward(frac)
        op = obj_model.forward(patch_indices)
        prop, ov = pt.forward_operator(op, sp, descan)
        inten = pt.detector_model.forward(ov)
        loss_an, tg = pt.error_estimate(inten, bi)
        pt.backward(loss_an, False, op, prop, ov, patch_indices, tg)
    out.update(grad_obj_an=obj_model._obj.grad.numpy().copy(),
               grad_probe_an=_c64(probe_model._probe.grad.numpy()))

    # --- a few reconstruct iterations from the same state ---
    with torch.no_grad():
        obj_model._obj.grad = None
        probe_model._probe.grad = None
    opt = opt or {"object": {"type": "adam"}, "probe": {"type": "adam"}}
    pt.rng = seed + 3
    pt.reconstruct(num_iters=iters, batch_size=batch, optimizer_params=opt,
                   constraints=constraints, device="cpu")
    out.update(
        recon_obj=obj_model._obj.detach().numpy().copy(),
        recon_probe=_c64(probe_model._probe.detach().numpy()),
        recon_losses=np.asarray(pt._iter_losses, dtype=np.float64),
        recon_rng_seed=np.int64(seed + 3),
    )
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: obj {tuple(pt.obj_shape_full)} N={pd.num_gpts} losses={out['recon_losses']}")


def c2small_case(name="c2small", nscan=3, batch=5, iters=3, seed=41):
    """The headline geometry at a small scan: 8 slices of 20 A, 4 probe modes at 128^2 with
    mode weights 0.7/0.15/0.1/0.05, a 512^2 object, +-0.5 px jitter, and two windows that
    wrap around both object edges (positions 1 and 3 moved next to opposite corners).
    Object-sized arrays are stored on sampled pixels only (flat row-major indices of one
    slice, the same for every slice): the batch's autograd object gradient on every
    pixel a window touches plus 4096 random untouched ones (``grad_idx``; off the windows
    only the constraint's mean-phase term acts), and the object after ``iters`` Adam
    iterations on 8192 touched plus 4096 untouched pixels (``recon_idx``)."""
    import torch
    from quantem.core.datastructures.dataset4dstem import Dataset4dstem
    from quantem.diffractive_imaging.complex_probe import real_space_probe
    from quantem.diffractive_imaging.dataset_models import PtychographyDatasetRaster
    from quantem.diffractive_imaging.detector_models import DetectorPixelated
    from quantem.diffractive_imaging.object_models import ObjectPixelated
    from quantem.diffractive_imaging.probe_models import ProbePixelated
    from quantem.diffractive_imaging.ptychography import Ptychography

    H, S, P, step_px, dz, counts = 128, 8, 4, 6, 20.0, 1e5
    weights = [0.7, 0.15, 0.1, 0.05]
    rng = np.random.default_rng(seed)
    px, energy = 0.2, 300e3
    rs = 1.0 / (H * px)
    ext = (nscan - 1) * step_px
    pad = (512 - ext) // 2
    obj_hw = ext + 2 * pad
    assert obj_hw == 512
    probe1 = real_space_probe(gpts=(H, H), sampling=(px, px), energy=energy, semiangle_cutoff=20.0,
                              aberration_coefs={"C10": -200.0}).numpy().astype(np.complex128)
    probes = np.stack([probe1 * np.sqrt(w) * np.exp(2j * np.pi * k * np.arange(H)[None, :] / H)
                       for k, w in enumerate(weights)])
    phase = np.stack([O.gaussian_atom_phase((obj_hw, obj_hw), obj_hw * obj_hw // 400, 1.5, 0.1, rng)
                      for _ in range(S)])
    true_obj = np.exp(1j * phase)
    grid = np.stack(np.meshgrid(np.arange(nscan), np.arange(nscan), indexing="ij"), -1).reshape(-1, 2)
    pos_true = grid * step_px + pad + rng.uniform(-0.5, 0.5, size=(nscan * nscan, 2))
    props_true = O.propagators((H, H), (px, px), energy, [dz] * (S - 1))
    data = simulate_data(true_obj, probes, pos_true, props_true, counts, rng)

    d4 = Dataset4dstem.from_array(data.reshape(nscan, nscan, H, H), sampling=(step_px * px, step_px * px, rs, rs),
                                  units=("A", "A", "A^-1", "A^-1"))
    pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
    pd.preprocess(com_fit_function="constant", force_com_rotation=0, force_com_transpose=False,
                  plot_rotation=False, plot_com=False, probe_energy=energy)
    obj_model = ObjectPixelated.from_uniform(num_slices=S, slice_thicknesses=dz, obj_type="complex")
    probe_model = ProbePixelated.from_params(
        probe_params={"energy": energy, "defocus": 200.0, "semiangle_cutoff": 20.0},
        num_probes=P, rng=seed + 1, initial_probe_weights=weights)
    pt = Ptychography.from_models(dset=pd, obj_model=obj_model, probe_model=probe_model,
                                  detector_model=DetectorPixelated(), device="cpu", verbose=0, rng=seed + 2)
    pt.preprocess(obj_padding_px=(pad, pad))
    assert tuple(pt.obj_shape_full) == (S, 512, 512), pt.obj_shape_full
    jit = rng.uniform(-0.5, 0.5, size=(pd.num_gpts, 2)).astype(np.float32)
    pos = pd.scan_positions_px.detach().numpy() + jit
    pos[1] = (3.4, 509.2)    # window wraps the top and right edges
    pos[3] = (508.6, 4.1)    # window wraps the bottom and left edges
    pd.scan_positions_px = torch.tensor(pos.astype(np.float32))

    out = dict(
        H=H, S=S, P=P, nscan=nscan, step_px=step_px, pad=pad, dz=dz, px=px, energy=energy, jitter=1,
        batch=batch, iters=iters, seed=seed, counts=counts, weights=np.asarray(weights, dtype=np.float64),
        orthogonalize=1, data=data,
        targets=_f32(pd.targets.numpy()),
        mean_intensity=np.float64(pd.mean_diffraction_intensity),
        positions=_f32(pd.scan_positions_px.detach().numpy()),
        initial_positions=_f32(pd.initial_scan_positions_px.numpy()),
        obj_shape=np.asarray(pt.obj_shape_full),
        obj_padding_px=np.asarray(pt.obj_padding_px),
        upsample_factor=np.float64(pd.upsample_factor),
        probe_init=_c64(probe_model._probe.detach().numpy()),
        propagators=_c64(pt._propagators.numpy()),
        sampling=np.asarray(pt.sampling, dtype=np.float64),
    )
    # windows of every position, one slice (the gradient vanishes elsewhere)
    origins, _ = O.split_positions(out["positions"].astype(np.float64))
    rows, cols = O.patch_rows_cols(origins, (H, H), (512, 512))
    touched = np.unique((rows[:, :, None] * 512 + cols[:, None, :]).ravel()).astype(np.int32)
    untouched = np.setdiff1d(np.arange(512 * 512, dtype=np.int32), touched)
    srng = np.random.default_rng(seed + 4)
    grad_idx = np.sort(np.concatenate([touched, srng.choice(untouched, 4096, replace=False)])).astype(np.int32)
    recon_idx = np.sort(np.concatenate([srng.choice(touched, 8192, replace=False),
                                        srng.choice(untouched, 4096, replace=False)])).astype(np.int32)
    out.update(touched_count=np.int64(touched.size), grad_idx=grad_idx, recon_idx=recon_idx)

    constraints = {"probe": {"orthogonalize_probe": True}}
    pt.constraints = constraints
    perturb_seed = seed + 100
    obj0 = perturbed_object((S, 512, 512), perturb_seed)
    with torch.no_grad():
        obj_model._obj.data = torch.tensor(obj0)
    out["perturb_seed"] = np.int64(perturb_seed)
    out["obj_perturbed_abs_sum"] = np.float64(np.abs(obj0.astype(np.complex128)).sum())
    bi = np.arange(batch)
    obj_model._obj.grad = None
    probe_model._probe.grad = None
    pt.dset._set_targets("l2_amplitude")
    pt.compute_propagator_arrays()
    patch_indices, _pos, frac, descan = pt.dset.forward(bi, pt.obj_padding_px)
    sp = probe_model.forward(frac)
    op = obj_model.forward(patch_indices)
    prop, ov = pt.forward_operator(op, sp, descan)
    inten = pt.detector_model.forward(ov)
    loss, tg = pt.error_estimate(inten, bi)
    pt.backward(loss, True, op, prop, ov, patch_indices, tg)
    g_obj = obj_model._obj.grad.numpy().reshape(S, -1)
    out.update(
        batch_indices=bi,
        batch_intensities=_f32(inten.detach().numpy()),
        batch_loss=np.float64(loss.item()),
        grad_obj_sampled=_c64(g_obj[:, grad_idx]),
        grad_probe=_c64(probe_model._probe.grad.numpy()),
        probe_ortho=_c64(probe_model.probe.detach().numpy()),
    )
    with torch.no_grad():
        obj_model._obj.grad = None
        probe_model._probe.grad = None
    pt.rng = seed + 3
    pt.reconstruct(num_iters=iters, batch_size=batch, optimizer_params={"object": {"type": "adam"},
                                                                         "probe": {"type": "adam"}},
                   constraints=constraints, device="cpu")
    rec = obj_model._obj.detach().numpy().reshape(S, -1)
    out.update(
        recon_obj_sampled=_c64(rec[:, recon_idx]),
        recon_probe=_c64(probe_model._probe.detach().numpy()),
        recon_losses=np.asarray(pt._iter_losses, dtype=np.float64),
        recon_rng_seed=np.int64(seed + 3),
    )
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: N={pd.num_gpts} touched={touched.size} losses={out['recon_losses']}")


def positions_case(name="positions64", seed=71):
    """Learned scan positions (dataset_models.py:30-120, 1482-1499): the reference's scan
    positions are a parameter whose gradient comes through the fractional probe shift.
    Records the autograd position gradient of one batch (positions perturbed off the
    raster so the gradient is not small) and 3 Adam iterations with a dataset optimiser
    (lr 1e-2 px; descan not learned: learn_descan=False)."""
    import torch
    from quantem.core.datastructures.dataset4dstem import Dataset4dstem
    from quantem.diffractive_imaging.complex_probe import real_space_probe
    from quantem.diffractive_imaging.dataset_models import PtychographyDatasetRaster
    from quantem.diffractive_imaging.detector_models import DetectorPixelated
    from quantem.diffractive_imaging.object_models import ObjectPixelated
    from quantem.diffractive_imaging.probe_models import ProbePixelated
    from quantem.diffractive_imaging.ptychography import Ptychography

    H, S, P, nscan, step_px, pad, dz, counts, batch, iters = 64, 2, 2, 5, 6, 32, 20.0, 1e5, 10, 3
    weights = [0.8, 0.2]
    rng = np.random.default_rng(seed)
    px, energy = 0.2, 300e3
    rs = 1.0 / (H * px)
    probe1 = real_space_probe(gpts=(H, H), sampling=(px, px), energy=energy, semiangle_cutoff=20.0,
                              aberration_coefs={"C10": -200.0}).numpy().astype(np.complex128)
    probes = np.stack([probe1 * np.sqrt(w) * np.exp(2j * np.pi * k * np.arange(H)[None, :] / H)
                       for k, w in enumerate(weights)])
    ext = (nscan - 1) * step_px
    obj_hw = int(ext + 2 * pad)
    obj_hw += (-obj_hw) % 8
    phase = np.stack([O.gaussian_atom_phase((obj_hw, obj_hw), obj_hw * obj_hw // 400, 1.5, 0.1, rng)
                      for _ in range(S)])
    grid = np.stack(np.meshgrid(np.arange(nscan), np.arange(nscan), indexing="ij"), -1).reshape(-1, 2)
    pos_true = grid * step_px + pad + rng.uniform(-0.5, 0.5, size=(nscan * nscan, 2))
    props_true = O.propagators((H, H), (px, px), energy, [dz] * (S - 1))
    data = simulate_data(np.exp(1j * phase), probes, pos_true, props_true, counts, rng)
    d4 = Dataset4dstem.from_array(data.reshape(nscan, nscan, H, H), sampling=(step_px * px, step_px * px, rs, rs),
                                  units=("A", "A", "A^-1", "A^-1"))
    pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0, learn_descan=False)
    pd.preprocess(com_fit_function="constant", force_com_rotation=0, force_com_transpose=False,
                  plot_rotation=False, plot_com=False, probe_energy=energy)
    obj_model = ObjectPixelated.from_uniform(num_slices=S, slice_thicknesses=dz, obj_type="complex")
    probe_model = ProbePixelated.from_params(
        probe_params={"energy": energy, "defocus": 200.0, "semiangle_cutoff": 20.0},
        num_probes=P, rng=seed + 1, initial_probe_weights=weights)
    pt = Ptychography.from_models(dset=pd, obj_model=obj_model, probe_model=probe_model,
                                  detector_model=DetectorPixelated(), device="cpu", verbose=0, rng=seed + 2)
    pt.preprocess(obj_padding_px=(pad, pad))
    # start off the true positions: the raster plus a +-0.7 px error (fractional parts away from 0.5)
    start = pd.scan_positions_px.detach().numpy() + rng.uniform(-0.7, 0.7, size=(pd.num_gpts, 2))
    fr = start - np.round(start)
    start = np.where(np.abs(np.abs(fr) - 0.5) < 0.02, start + 0.05, start).astype(np.float32)
    pd.scan_positions_px = torch.tensor(start)
    out = dict(H=H, S=S, P=P, nscan=nscan, step_px=step_px, pad=pad, dz=dz, px=px, energy=energy, jitter=1,
               batch=batch, iters=iters, seed=seed, counts=counts, weights=np.asarray(weights, dtype=np.float64),
               orthogonalize=1, data=data, targets=_f32(pd.targets.numpy()),
               mean_intensity=np.float64(pd.mean_diffraction_intensity),
               positions=_f32(pd.scan_positions_px.detach().numpy()),
               initial_positions=_f32(pd.initial_scan_positions_px.numpy()),
               positions_true=pos_true.astype(np.float32), obj_shape=np.asarray(pt.obj_shape_full),
               obj_padding_px=np.asarray(pt.obj_padding_px), upsample_factor=np.float64(pd.upsample_factor),
               probe_init=_c64(probe_model._probe.detach().numpy()), propagators=_c64(pt._propagators.numpy()),
               sampling=np.asarray(pt.sampling, dtype=np.float64))
    constraints = {"probe": {"orthogonalize_probe": True}}
    pt.constraints = constraints
    with torch.no_grad():
        shp = tuple(obj_model._obj.shape)
        amp = 1.0 - 0.3 * rng.random(shp)
        ph = 0.4 * rng.standard_normal(shp)
        obj_model._obj.data = torch.tensor(amp * np.exp(1j * ph), dtype=torch.complex64)
    out["obj_perturbed"] = obj_model._obj.detach().numpy().copy()
    bi = np.arange(batch)
    obj_model._obj.grad = None
    probe_model._probe.grad = None
    pd._scan_positions_px.grad = None
    pt.dset._set_targets("l2_amplitude")
    pt.compute_propagator_arrays()
    patch_indices, _pos, frac, descan = pt.dset.forward(bi, pt.obj_padding_px)
    sp = probe_model.forward(frac)
    op = obj_model.forward(patch_indices)
    prop, ov = pt.forward_operator(op, sp, descan)
    inten = pt.detector_model.forward(ov)
    loss, tg = pt.error_estimate(inten, bi)
    pt.backward(loss, True, op, prop, ov, patch_indices, tg)
    out.update(batch_indices=bi, batch_loss=np.float64(loss.item()),
               batch_intensities=_f32(inten.detach().numpy()),
               grad_positions=pd._scan_positions_px.grad.numpy().astype(np.float64).copy(),
               grad_obj=obj_model._obj.grad.numpy().copy(), grad_probe=_c64(probe_model._probe.grad.numpy()))
    with torch.no_grad():
        obj_model._obj.grad = None
        probe_model._probe.grad = None
        pd._scan_positions_px.grad = None
    pt.rng = seed + 3
    pt.reconstruct(num_iters=iters, batch_size=batch,
                   optimizer_params={"object": {"type": "adam"}, "probe": {"type": "adam"},
                                     "dataset": {"type": "adam", "lr": 1e-2}},
                   constraints=constraints, device="cpu")
    out.update(recon_obj=obj_model._obj.detach().numpy().copy(), recon_probe=_c64(probe_model._probe.detach().numpy()),
               recon_positions=pd.scan_positions_px.detach().numpy().astype(np.float32).copy(),
               recon_losses=np.asarray(pt._iter_losses, dtype=np.float64), recon_rng_seed=np.int64(seed + 3))
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: losses={out['recon_losses']} |grad_pos|={np.abs(out['grad_positions']).max():.3g} "
          f"moved={np.abs(out['recon_positions'] - out['positions']).max():.3g}")


def descan_tilt_case(name="descantilt64", seed=83):
    """Learned descan shifts (dataset_models.py:30-120, 225-242, 1482-1499;
    ptychography_base.py:892-906) and a learned probe tilt (probe_models.py:56-131,
    295-304, 376-427).  Data simulated with per-position descan shifts of up to 0.6 px
    and a (1.0, -1.5) mrad tilt; the reference starts from zero descan and a
    (0.5, -0.5) mrad tilt (a zero tilt would get no gradient: the reference adds the
    ramp only for a nonzero tilt).  Records one batch's autograd gradients, the descan
    and tilt ones included, with the dataset optimiser set (so the targets are the
    uncentred amplitudes), and 3 Adam iterations of object, probe (+ tilt) and dataset
    (descan; scan positions not learned)."""
    import torch
    from quantem.core.datastructures.dataset4dstem import Dataset4dstem
    from quantem.diffractive_imaging.complex_probe import real_space_probe
    from quantem.diffractive_imaging.dataset_models import PtychographyDatasetRaster
    from quantem.diffractive_imaging.detector_models import DetectorPixelated
    from quantem.diffractive_imaging.object_models import ObjectPixelated
    from quantem.diffractive_imaging.probe_models import ProbePixelated
    from quantem.diffractive_imaging.ptychography import Ptychography

    H, S, P, nscan, step_px, pad, dz, counts, batch, iters = 64, 3, 2, 5, 6, 32, 20.0, 1e5, 10, 3
    weights = [0.8, 0.2]
    tilt_true, tilt_start = (1.0, -1.5), (0.5, -0.5)
    rng = np.random.default_rng(seed)
    px, energy = 0.2, 300e3
    rs = 1.0 / (H * px)
    probe1 = real_space_probe(gpts=(H, H), sampling=(px, px), energy=energy, semiangle_cutoff=20.0,
                              aberration_coefs={"C10": -200.0}).numpy().astype(np.complex128)
    probes = np.stack([probe1 * np.sqrt(w) * np.exp(2j * np.pi * k * np.arange(H)[None, :] / H)
                       for k, w in enumerate(weights)])
    ext = (nscan - 1) * step_px
    obj_hw = int(ext + 2 * pad)
    obj_hw += (-obj_hw) % 8
    phase = np.stack([O.gaussian_atom_phase((obj_hw, obj_hw), obj_hw * obj_hw // 400, 1.5, 0.1, rng)
                      for _ in range(S)])
    grid = np.stack(np.meshgrid(np.arange(nscan), np.arange(nscan), indexing="ij"), -1).reshape(-1, 2)
    pos = (grid * step_px + pad).astype(np.float64)
    descan_true = rng.uniform(-0.6, 0.6, size=(nscan * nscan, 2))
    props_true = O.propagators((H, H), (px, px), energy, [dz] * (S - 1), tilt_mrad=tilt_true)
    st = O.forward(np.exp(1j * phase), probes, pos, props_true, descan=descan_true)
    inten = O.detector_intensities(st)
    inten = inten / inten.sum(axis=(-2, -1), keepdims=True).mean() * counts
    data = rng.poisson(inten).astype(np.float32)
    d4 = Dataset4dstem.from_array(data.reshape(nscan, nscan, H, H), sampling=(step_px * px, step_px * px, rs, rs),
                                  units=("A", "A", "A^-1", "A^-1"))
    pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0, learn_descan=True, learn_scan_positions=False)
    pd.preprocess(com_fit_function="constant", force_com_rotation=0, force_com_transpose=False,
                  plot_rotation=False, plot_com=False, probe_energy=energy)
    obj_model = ObjectPixelated.from_uniform(num_slices=S, slice_thicknesses=dz, obj_type="complex")
    probe_model = ProbePixelated.from_params(
        probe_params={"energy": energy, "defocus": 200.0, "semiangle_cutoff": 20.0},
        num_probes=P, rng=seed + 1, initial_probe_weights=weights, probe_tilt=tilt_start, learn_probe_tilt=True)
    pt = Ptychography.from_models(dset=pd, obj_model=obj_model, probe_model=probe_model,
                                  detector_model=DetectorPixelated(), device="cpu", verbose=0, rng=seed + 2)
    pt.preprocess(obj_padding_px=(pad, pad))
    # start the descan shifts off zero so the batch gradient is not the trivial one
    with torch.no_grad():
        pd.descan_shifts = torch.tensor(rng.uniform(-0.3, 0.3, size=(pd.num_gpts, 2)), dtype=torch.float32)
    opt = {"object": {"type": "adam"}, "probe": {"type": "adam"}, "dataset": {"type": "adam", "lr": 1e-2}}
    constraints = {"probe": {"orthogonalize_probe": True}}
    pt.constraints = constraints
    pt.optimizer_params = {k: dict(v) for k, v in opt.items()}
    pt.set_optimizers()
    pt.dset._set_targets("l2_amplitude")  # the uncentred amplitudes: descan is learned
    out = dict(H=H, S=S, P=P, nscan=nscan, step_px=step_px, pad=pad, dz=dz, px=px, energy=energy, jitter=0,
               batch=batch, iters=iters, seed=seed, counts=counts, weights=np.asarray(weights, dtype=np.float64),
               orthogonalize=1, data=data, targets=_f32(pd.targets.numpy()),
               centered_targets=_f32(pd.centered_amplitudes.numpy()),
               mean_intensity=np.float64(pd.mean_diffraction_intensity),
               positions=_f32(pd.scan_positions_px.detach().numpy()),
               descan=_f32(pd.descan_shifts.detach().numpy()), descan_true=descan_true.astype(np.float32),
               tilt=np.asarray(tilt_start, dtype=np.float64), tilt_true=np.asarray(tilt_true, dtype=np.float64),
               obj_shape=np.asarray(pt.obj_shape_full), obj_padding_px=np.asarray(pt.obj_padding_px),
               upsample_factor=np.float64(pd.upsample_factor),
               probe_init=_c64(probe_model._probe.detach().numpy()),
               sampling=np.asarray(pt.sampling, dtype=np.float64))
    pt.compute_propagator_arrays()
    out["propagators"] = _c64(pt._propagators.detach().numpy())
    with torch.no_grad():
        shp = tuple(obj_model._obj.shape)
        amp = 1.0 - 0.3 * rng.random(shp)
        ph = 0.4 * rng.standard_normal(shp)
        obj_model._obj.data = torch.tensor(amp * np.exp(1j * ph), dtype=torch.complex64)
    out["obj_perturbed"] = obj_model._obj.detach().numpy().copy()
    bi = np.arange(batch)
    for prm in (obj_model._obj, probe_model._probe, probe_model._probe_tilt, pd._descan_shifts):
        prm.grad = None
    patch_indices, _pos, frac, descan = pt.dset.forward(bi, pt.obj_padding_px)
    assert descan is not None
    sp = probe_model.forward(frac)
    op = obj_model.forward(patch_indices)
    prop, ov = pt.forward_operator(op, sp, descan)
    inten = pt.detector_model.forward(ov)
    loss, tg = pt.error_estimate(inten, bi)
    pt.backward(loss, True, op, prop, ov, patch_indices, tg)
    out.update(batch_indices=bi, batch_loss=np.float64(loss.item()),
               batch_intensities=_f32(inten.detach().numpy()),
               grad_descan=pd._descan_shifts.grad.numpy().astype(np.float64).copy(),
               grad_tilt=probe_model._probe_tilt.grad.numpy().astype(np.float64).copy(),
               grad_obj=obj_model._obj.grad.numpy().copy(), grad_probe=_c64(probe_model._probe.grad.numpy()))
    for prm in (obj_model._obj, probe_model._probe, probe_model._probe_tilt, pd._descan_shifts):
        prm.grad = None
    pt.rng = seed + 3
    pt.reconstruct(num_iters=iters, batch_size=batch, optimizer_params={k: dict(v) for k, v in opt.items()},
                   constraints=constraints, device="cpu")
    out.update(recon_obj=obj_model._obj.detach().numpy().copy(), recon_probe=_c64(probe_model._probe.detach().numpy()),
               recon_descan=pd.descan_shifts.detach().numpy().astype(np.float32).copy(),
               recon_tilt=probe_model.probe_tilt.detach().numpy().astype(np.float64).copy(),
               recon_positions=pd.scan_positions_px.detach().numpy().astype(np.float32).copy(),
               recon_losses=np.asarray(pt._iter_losses, dtype=np.float64), recon_rng_seed=np.int64(seed + 3))
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: losses={out['recon_losses']} grad_tilt={out['grad_tilt']} "
          f"|grad_descan|={np.abs(out['grad_descan']).max():.3g} tilt {out['tilt']} -> {out['recon_tilt']} "
          f"descan moved={np.abs(out['recon_descan'] - out['descan']).max():.3g}")


def objconstraints_cases(seed=91):
    """Optional object constraints (object_models.py:273-480) with the probe-overlap FOV
    mask the reference builds in preprocess (ptychography_base.py:191-216); the cases are
    listed below.  Each records the FOV mask, the hard-constrained
    object, the soft-constraint loss, one batch's loss (consistency + soft) and autograd
    gradients, and 2 Adam iterations of object and probe."""
    import torch
    from quantem.core.datastructures.dataset4dstem import Dataset4dstem
    from quantem.diffractive_imaging.complex_probe import real_space_probe
    from quantem.diffractive_imaging.dataset_models import PtychographyDatasetRaster
    from quantem.diffractive_imaging.detector_models import DetectorPixelated
    from quantem.diffractive_imaging.object_models import ObjectPixelated
    from quantem.diffractive_imaging.probe_models import ProbePixelated
    from quantem.diffractive_imaging.ptychography import Ptychography

    H, S, P, nscan, step_px, pad, dz, counts, batch, iters = 64, 3, 2, 5, 6, 32, 20.0, 1e5, 10, 2
    weights = [0.8, 0.2]
    px, energy = 0.2, 300e3
    rs = 1.0 / (H * px)
    # (name, object type, constraints).  The FOV mask is exactly 0 far from the scan, where the
    # reference's autograd gives the phase of a zero pixel a NaN gradient, so the phase soft
    # terms are recorded without the mask on complex objects.
    cases = [
        ("complex", "complex", {"gaussian_sigma": 1.0, "tv_weight_xy": 0.05, "tv_weight_z": 0.02,
                                "surface_zero_weight": 0.01}),
        ("complexfov", "complex", {"apply_fov_mask": True, "gaussian_sigma": 1.0}),
        ("potential", "potential", {"fix_potential_baseline": True, "apply_fov_mask": True,
                                    "identical_slices": True, "tv_weight_xy": 0.05}),
        ("pure_phase", "pure_phase", {"gaussian_sigma": 0.7, "identical_slices": True, "tv_weight_xy": 0.04}),
        ("butter_complex", "complex", {"q_lowpass": 1.5, "q_highpass": 0.05, "butterworth_order": 3}),
        ("butter_potential", "potential", {"q_lowpass": 1.2, "gaussian_sigma": 0.8}),
    ]
    for k, (name, obj_type, cons) in enumerate(cases):
        rng = np.random.default_rng(seed + k)
        probe1 = real_space_probe(gpts=(H, H), sampling=(px, px), energy=energy, semiangle_cutoff=20.0,
                                  aberration_coefs={"C10": -200.0}).numpy().astype(np.complex128)
        probes = np.stack([probe1 * np.sqrt(w) * np.exp(2j * np.pi * j * np.arange(H)[None, :] / H)
                           for j, w in enumerate(weights)])
        obj_hw = int((nscan - 1) * step_px + 2 * pad)
        obj_hw += (-obj_hw) % 8
        phase = np.stack([O.gaussian_atom_phase((obj_hw, obj_hw), obj_hw * obj_hw // 400, 1.5, 0.1, rng)
                          for _ in range(S)])
        grid = np.stack(np.meshgrid(np.arange(nscan), np.arange(nscan), indexing="ij"), -1).reshape(-1, 2)
        pos = grid * step_px + pad + rng.uniform(-0.5, 0.5, size=(nscan * nscan, 2))
        props_true = O.propagators((H, H), (px, px), energy, [dz] * (S - 1))
        data = simulate_data(np.exp(1j * phase), probes, pos, props_true, counts, rng)
        d4 = Dataset4dstem.from_array(data.reshape(nscan, nscan, H, H), sampling=(step_px * px, step_px * px, rs, rs),
                                      units=("A", "A", "A^-1", "A^-1"))
        pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
        pd.preprocess(com_fit_function="constant", force_com_rotation=0, force_com_transpose=False,
                      plot_rotation=False, plot_com=False, probe_energy=energy)
        obj_model = ObjectPixelated.from_uniform(num_slices=S, slice_thicknesses=dz, obj_type=obj_type)
        probe_model = ProbePixelated.from_params(
            probe_params={"energy": energy, "defocus": 200.0, "semiangle_cutoff": 20.0},
            num_probes=P, rng=seed + 1, initial_probe_weights=weights)
        pt = Ptychography.from_models(dset=pd, obj_model=obj_model, probe_model=probe_model,
                                      detector_model=DetectorPixelated(), device="cpu", verbose=0, rng=seed + 2)
        pt.preprocess(obj_padding_px=(pad, pad))
        constraints = {"object": dict(cons), "probe": {"orthogonalize_probe": True}}
        pt.constraints = constraints
        with torch.no_grad():
            shp = tuple(obj_model._obj.shape)
            if obj_type == "potential":
                obj_model._obj.data = torch.tensor(0.05 + 0.1 * rng.standard_normal(shp), dtype=torch.float32)
            else:
                amp = 1.0 - 0.3 * rng.random(shp)
                ph = 0.4 * rng.standard_normal(shp)
                obj_model._obj.data = torch.tensor(amp * np.exp(1j * ph), dtype=torch.complex64)
        out = dict(H=H, S=S, P=P, nscan=nscan, step_px=step_px, pad=pad, dz=dz, px=px, energy=energy, batch=batch,
                   iters=iters, seed=seed + k, counts=counts, weights=np.asarray(weights, dtype=np.float64),
                   obj_type=obj_type, constraints=np.asarray(repr(cons)), data=data,
                   targets=_f32(pd.targets.numpy()), mean_intensity=np.float64(pd.mean_diffraction_intensity),
                   positions=_f32(pd.scan_positions_px.detach().numpy()), obj_shape=np.asarray(pt.obj_shape_full),
                   obj_padding_px=np.asarray(pt.obj_padding_px), upsample_factor=np.float64(pd.upsample_factor),
                   probe_init=_c64(probe_model._probe.detach().numpy()), propagators=_c64(pt._propagators.numpy()),
                   sampling=np.asarray(pt.sampling, dtype=np.float64),
                   fov_mask=np.asarray(obj_model.mask[0].detach().numpy(), dtype=np.float32),
                   obj_sampling=np.asarray(obj_model.sampling, dtype=np.float64),
                   probe_overlap=np.asarray(pt._get_probe_overlap(), dtype=np.float64))
        out["obj_perturbed"] = obj_model._obj.detach().numpy().copy()
        obj2 = obj_model.obj
        out["obj_constrained"] = obj2.detach().numpy().copy()
        soft = obj_model.apply_soft_constraints(obj2, mask=obj_model.mask)
        out["soft_loss"] = np.float64(soft.item())
        bi = np.arange(batch)
        obj_model._obj.grad = None
        probe_model._probe.grad = None
        pt.dset._set_targets("l2_amplitude")
        pt.compute_propagator_arrays()
        patch_indices, _pos, frac, descan = pt.dset.forward(bi, pt.obj_padding_px)
        sp = probe_model.forward(frac)
        op = obj_model.forward(patch_indices)
        prop, ov = pt.forward_operator(op, sp, descan)
        inten = pt.detector_model.forward(ov)
        loss, tg = pt.error_estimate(inten, bi)
        total = loss + pt._soft_constraints()
        pt.backward(total, True, op, prop, ov, patch_indices, tg)
        out.update(batch_indices=bi, batch_loss=np.float64(loss.item()), batch_total_loss=np.float64(total.item()),
                   batch_intensities=_f32(inten.detach().numpy()), grad_obj=obj_model._obj.grad.numpy().copy(),
                   grad_probe=_c64(probe_model._probe.grad.numpy()))
        obj_model._obj.grad = None
        probe_model._probe.grad = None
        pt.rng = seed + 3
        pt.reconstruct(num_iters=iters, batch_size=batch,
                       optimizer_params={"object": {"type": "adam"}, "probe": {"type": "adam"}},
                       constraints=constraints, device="cpu")
        out.update(recon_obj=obj_model._obj.detach().numpy().copy(),
                   recon_probe=_c64(probe_model._probe.detach().numpy()),
                   recon_losses=np.asarray(pt._iter_losses, dtype=np.float64), recon_rng_seed=np.int64(seed + 3))
        path = os.path.join(HERE, f"objcons_{name}64.npz")
        np.savez_compressed(path, **out)
        print(f"wrote {path}: soft={out['soft_loss']:.4g} loss={out['batch_loss']:.4g} "
              f"total={out['batch_total_loss']:.4g} losses={out['recon_losses']}")


def probeconstraints_cases(seed=131):
    """Optional probe constraints (probe_models.py:430-482): the centre-of-mass shift
    (``center_probe``) after Gram-Schmidt and the TV soft loss (``tv_weight``), on a raw probe
    moved off centre.  Each case records the constrained probe, the probe's soft loss, one
    batch's loss (consistency + soft) and autograd gradients, and 2 Adam iterations."""
    import torch
    from quantem.core.datastructures.dataset4dstem import Dataset4dstem
    from quantem.diffractive_imaging.complex_probe import real_space_probe
    from quantem.diffractive_imaging.dataset_models import PtychographyDatasetRaster
    from quantem.diffractive_imaging.detector_models import DetectorPixelated
    from quantem.diffractive_imaging.object_models import ObjectPixelated
    from quantem.diffractive_imaging.probe_models import ProbePixelated
    from quantem.diffractive_imaging.ptychography import Ptychography

    H, S, nscan, step_px, pad, dz, counts, batch, iters = 64, 2, 5, 6, 32, 20.0, 1e5, 10, 2
    px, energy = 0.2, 300e3
    rs = 1.0 / (H * px)
    # (name, probe modes, mode weights, probe constraints, roll of the raw probe in px)
    cases = [
        ("centertv", 2, [0.8, 0.2], {"orthogonalize_probe": True, "center_probe": True, "tv_weight": 0.05}, (3, -2)),
        ("center1", 1, [1.0], {"orthogonalize_probe": False, "center_probe": True, "tv_weight": 0.0}, (-4, 5)),
        ("tv3", 3, [0.7, 0.2, 0.1], {"orthogonalize_probe": True, "center_probe": False, "tv_weight": 0.1}, (0, 0)),
    ]
    for k, (name, P, weights, pcons, roll) in enumerate(cases):
        rng = np.random.default_rng(seed + k)
        probe1 = real_space_probe(gpts=(H, H), sampling=(px, px), energy=energy, semiangle_cutoff=20.0,
                                  aberration_coefs={"C10": -200.0}).numpy().astype(np.complex128)
        probes = np.stack([probe1 * np.sqrt(w) * np.exp(2j * np.pi * j * np.arange(H)[None, :] / H)
                           for j, w in enumerate(weights)])
        obj_hw = int((nscan - 1) * step_px + 2 * pad)
        obj_hw += (-obj_hw) % 8
        phase = np.stack([O.gaussian_atom_phase((obj_hw, obj_hw), obj_hw * obj_hw // 400, 1.5, 0.1, rng)
                          for _ in range(S)])
        grid = np.stack(np.meshgrid(np.arange(nscan), np.arange(nscan), indexing="ij"), -1).reshape(-1, 2)
        pos = grid * step_px + pad + rng.uniform(-0.5, 0.5, size=(nscan * nscan, 2))
        props_true = O.propagators((H, H), (px, px), energy, [dz] * (S - 1))
        data = simulate_data(np.exp(1j * phase), probes, pos, props_true, counts, rng)
        d4 = Dataset4dstem.from_array(data.reshape(nscan, nscan, H, H), sampling=(step_px * px, step_px * px, rs, rs),
                                      units=("A", "A", "A^-1", "A^-1"))
        pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
        pd.preprocess(com_fit_function="constant", force_com_rotation=0, force_com_transpose=False,
                      plot_rotation=False, plot_com=False, probe_energy=energy)
        obj_model = ObjectPixelated.from_uniform(num_slices=S, slice_thicknesses=dz, obj_type="complex")
        probe_model = ProbePixelated.from_params(
            probe_params={"energy": energy, "defocus": 200.0, "semiangle_cutoff": 20.0},
            num_probes=P, rng=seed + 1, initial_probe_weights=weights)
        pt = Ptychography.from_models(dset=pd, obj_model=obj_model, probe_model=probe_model,
                                      detector_model=DetectorPixelated(), device="cpu", verbose=0, rng=seed + 2)
        pt.preprocess(obj_padding_px=(pad, pad))
        constraints = {"probe": dict(pcons)}
        pt.constraints = constraints
        with torch.no_grad():
            shp = tuple(obj_model._obj.shape)
            amp = 1.0 - 0.3 * rng.random(shp)
            ph = 0.4 * rng.standard_normal(shp)
            obj_model._obj.data = torch.tensor(amp * np.exp(1j * ph), dtype=torch.complex64)
            raw = probe_model._probe.detach().numpy()
            raw = np.roll(raw, roll, axis=(-2, -1)) * np.exp(0.2j * rng.standard_normal(raw.shape))
            probe_model._probe.data = torch.tensor(raw, dtype=torch.complex64)
        out = dict(H=H, S=S, P=P, nscan=nscan, step_px=step_px, pad=pad, dz=dz, px=px, energy=energy, batch=batch,
                   iters=iters, seed=seed + k, counts=counts, weights=np.asarray(weights, dtype=np.float64),
                   probe_constraints=np.asarray(repr(pcons)), data=data,
                   targets=_f32(pd.targets.numpy()), mean_intensity=np.float64(pd.mean_diffraction_intensity),
                   positions=_f32(pd.scan_positions_px.detach().numpy()), obj_shape=np.asarray(pt.obj_shape_full),
                   obj_padding_px=np.asarray(pt.obj_padding_px), upsample_factor=np.float64(pd.upsample_factor),
                   probe_init=_c64(probe_model._probe.detach().numpy()), propagators=_c64(pt._propagators.numpy()),
                   obj_perturbed=obj_model._obj.detach().numpy().copy())
        probe2 = probe_model.probe
        out["probe_constrained"] = _c64(probe2.detach().numpy())
        out["probe_soft_loss"] = np.float64(probe_model.apply_soft_constraints(probe2).item())
        bi = np.arange(batch)
        obj_model._obj.grad = None
        probe_model._probe.grad = None
        pt.dset._set_targets("l2_amplitude")
        pt.compute_propagator_arrays()
        patch_indices, _pos, frac, descan = pt.dset.forward(bi, pt.obj_padding_px)
        sp = probe_model.forward(frac)
        op = obj_model.forward(patch_indices)
        prop, ov = pt.forward_operator(op, sp, descan)
        inten = pt.detector_model.forward(ov)
        loss, tg = pt.error_estimate(inten, bi)
        total = loss + pt._soft_constraints()
        pt.backward(total, True, op, prop, ov, patch_indices, tg)
        out.update(batch_indices=bi, batch_loss=np.float64(loss.item()), batch_total_loss=np.float64(total.item()),
                   batch_intensities=_f32(inten.detach().numpy()), grad_obj=obj_model._obj.grad.numpy().copy(),
                   grad_probe=_c64(probe_model._probe.grad.numpy()))
        obj_model._obj.grad = None
        probe_model._probe.grad = None
        pt.rng = seed + 3
        pt.reconstruct(num_iters=iters, batch_size=batch,
                       optimizer_params={"object": {"type": "adam"}, "probe": {"type": "adam"}},
                       constraints=constraints, device="cpu")
        out.update(recon_obj=obj_model._obj.detach().numpy().copy(),
                   recon_probe=_c64(probe_model._probe.detach().numpy()),
                   recon_losses=np.asarray(pt._iter_losses, dtype=np.float64), recon_rng_seed=np.int64(seed + 3))
        path = os.path.join(HERE, f"probecons_{name}64.npz")
        np.savez_compressed(path, **out)
        print(f"wrote {path}: soft={out['probe_soft_loss']:.4g} loss={out['batch_loss']:.4g} "
              f"total={out['batch_total_loss']:.4g} losses={out['recon_losses']}")


def bilinear_case():
    """preprocess(bilinear=True) (dataset_models.py:946-1025, 1372-1480 with shift_array's
    bilinear branch, ptycho_utils.py:273-284) on the mixed64 patterns, with a plane CoM fit
    (a different shift for every pattern): centred targets, mean intensity and the CoM fit."""
    from quantem.core.datastructures.dataset4dstem import Dataset4dstem
    from quantem.diffractive_imaging.dataset_models import PtychographyDatasetRaster

    z = np.load(os.path.join(HERE, "mixed64.npz"))
    H, nscan = int(z["H"]), int(z["nscan"])
    px, step = float(z["px"]), float(z["step_px"])
    rs = 1.0 / (H * px)
    out = dict(H=H, nscan=nscan, px=px, step_px=step, energy=z["energy"], data=z["data"])
    for fit in ("plane", "constant"):
        d4 = Dataset4dstem.from_array(z["data"].reshape(nscan, nscan, H, H), sampling=(step * px, step * px, rs, rs),
                                      units=("A", "A", "A^-1", "A^-1"))
        pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
        pd.preprocess(com_fit_function=fit, force_com_rotation=0, force_com_transpose=False, bilinear=True,
                      plot_rotation=False, plot_com=False, probe_energy=float(z["energy"]))
        out[f"targets_{fit}"] = _f32(pd.targets.numpy())
        out[f"mean_intensity_{fit}"] = np.float64(pd.mean_diffraction_intensity)
        out[f"com_fit_{fit}"] = np.asarray(pd.com_fit, dtype=np.float64)
    path = os.path.join(HERE, "bilinear64.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}")


def whitenoise_case():
    """The reference gradient test's fixture (test_ptychography.py:19-212), restated."""
    import torch
    from quantem.core.datastructures.dataset4dstem import Dataset4dstem
    from quantem.diffractive_imaging.dataset_models import PtychographyDatasetRaster
    from quantem.diffractive_imaging.detector_models import DetectorPixelated
    from quantem.diffractive_imaging.object_models import ObjectPixelated
    from quantem.diffractive_imaging.probe_models import ProbePixelated
    from quantem.diffractive_imaging.ptychography import Ptychography

    from tests.golden.whitenoise import whitenoise_inputs

    inp = whitenoise_inputs()
    N = inp["N"]
    d4 = Dataset4dstem.from_array(inp["data4d"], sampling=inp["sampling4d"],
                                  units=("A", "A", "A^-1", "A^-1"))
    pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
    pd.preprocess(com_fit_function="constant", plot_rotation=False, plot_com=False,
                  probe_energy=inp["energy"], force_com_rotation=0, force_com_transpose=False)
    out = {}
    for nprobe in (1, 2):
        for autograd in (True, False):
            obj_model = ObjectPixelated.from_uniform(num_slices=1, obj_type="complex",
                                                     slice_thicknesses=1)
            # a (P, N, N) stack: the reference's from_array concatenates a 2-D
            # array along rows when num_probes > 1 (probe_models.py:603-606)
            probe_model = ProbePixelated.from_array(
                num_probes=nprobe, probe_params=inp["probe_params"],
                probe_array=np.stack([inp["probe"]] * nprobe).astype(np.complex64))
            pt = Ptychography.from_models(dset=pd, obj_model=obj_model, probe_model=probe_model,
                                          detector_model=DetectorPixelated(), rng=42, verbose=0)
            pt.preprocess(obj_padding_px=(0, 0))
            pt.reconstruct(num_iters=1, reset=True, autograd=autograd,
                           constraints={"probe": {"orthogonalize_probe": False}},
                           optimizer_params={"object": {"type": "sgd", "lr": 0.5},
                                             "probe": {"type": "sgd", "lr": 0.5}},
                           batch_size=N * N, device="cpu")
            tag = f"p{nprobe}_{'ad' if autograd else 'an'}"
            out[f"probe_used_{tag}"] = _c64(probe_model._initial_probe.detach().numpy())
            out[f"grad_obj_{tag}"] = _c64(obj_model._obj.grad.numpy())
            out[f"grad_probe_{tag}"] = _c64(probe_model._probe.grad.numpy())
            out[f"loss_{tag}"] = np.asarray(pt._iter_losses, dtype=np.float64)
    out["targets_sum"] = np.float64(pd.targets.numpy().astype(np.float64).sum())
    out["mean_intensity"] = np.float64(pd.mean_diffraction_intensity)
    path = os.path.join(HERE, "whitenoise64.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}")
    del torch


def main(src):
    import torch

    torch.manual_seed(0)
    import_reference(src)
    if os.environ.get("GOLDEN_ONLY") == "whitenoise":
        whitenoise_case()
        return
    if os.environ.get("GOLDEN_ONLY") == "c2small":
        c2small_case()
        return
    if os.environ.get("GOLDEN_ONLY") == "objtypes":
        objtype_cases()
        return
    if os.environ.get("GOLDEN_ONLY") == "positions":
        positions_case()
        return
    if os.environ.get("GOLDEN_ONLY") == "descantilt":
        descan_tilt_case()
        return
    if os.environ.get("GOLDEN_ONLY") == "objconstraints":
        objconstraints_cases()
        return
    if os.environ.get("GOLDEN_ONLY") == "bilinear":
        bilinear_case()
        return
    if os.environ.get("GOLDEN_ONLY") == "probeconstraints":
        probeconstraints_cases()
        return
    run_case("single64", H=64, S=1, P=1, nscan=6, step_px=4, pad=32, dz=20.0, counts=1e5,
             jitter=False, batch=12, iters=3, seed=11)
    run_case("mixed64", H=64, S=3, P=3, nscan=5, step_px=6, pad=32, dz=20.0, counts=1e5,
             jitter=True, batch=10, iters=2, weights=[0.7, 0.2, 0.1], seed=21)
    run_case("mixed128", H=128, S=4, P=4, nscan=3, step_px=6, pad=64, dz=20.0, counts=1e5,
             jitter=True, batch=9, iters=2, weights=[0.7, 0.15, 0.1, 0.05], seed=31,
             keep_data=False)
    whitenoise_case()
    c2small_case()
    objtype_cases()
    positions_case()
    descan_tilt_case()
    objconstraints_cases()


def objtype_cases():
    """The pure-phase and potential object types (object_models.py:87, 123-136,
    289-339, 252-256) at the mixed64 geometry, default constraints (positivity on)."""
    run_case("purephase64", H=64, S=2, P=2, nscan=5, step_px=6, pad=32, dz=20.0, counts=1e5,
             jitter=True, batch=10, iters=2, weights=[0.8, 0.2], seed=51, obj_type="pure_phase")
    run_case("potential64", H=64, S=2, P=2, nscan=5, step_px=6, pad=32, dz=20.0, counts=1e5,
             jitter=True, batch=10, iters=2, weights=[0.8, 0.2], seed=61, obj_type="potential")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {os.path.relpath(__file__)} <reference source dir (the one holding quantem/)>")
    main(sys.argv[1])
