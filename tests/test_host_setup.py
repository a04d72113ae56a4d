"""Host-side set-up of the drop-in API against the reference's own set-up
products recorded in the golden fixtures (CPU only, no CUDA needed)."""
import numpy as np
import pytest
import torch

from tests.conftest import load_golden, rel


def build_from_golden(z, device="cpu"):
    from quantem_b200.diffractive_imaging import (Dataset4dstem, DetectorPixelated, ObjectPixelated,
                                                  ProbePixelated, Ptychography, PtychographyDatasetRaster)

    H, nscan = int(z["H"]), int(z["nscan"])
    px, step = float(z["px"]), float(z["step_px"])
    rs = 1.0 / (H * px)
    d4 = Dataset4dstem.from_array(z["data"].reshape(nscan, nscan, H, H), sampling=(step * px, step * px, rs, rs),
                                  units=("A", "A", "A^-1", "A^-1"))
    pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
    pd.preprocess(com_fit_function="constant", force_com_rotation=0, force_com_transpose=False,
                  plot_rotation=False, plot_com=False, probe_energy=float(z["energy"]), device=device)
    S, P, seed = int(z["S"]), int(z["P"]), int(z["seed"])
    w = z["weights"] if z["weights"].size else None
    obj = ObjectPixelated.from_uniform(num_slices=S, slice_thicknesses=float(z["dz"]), obj_type="complex")
    probe = ProbePixelated.from_params(probe_params={"energy": float(z["energy"]), "defocus": 200.0,
                                                     "semiangle_cutoff": 20.0},
                                       num_probes=P, rng=seed + 1, initial_probe_weights=w)
    pt = Ptychography.from_models(dset=pd, obj_model=obj, probe_model=probe, detector_model=DetectorPixelated(),
                                  device=device, verbose=0, rng=seed + 2)
    pad = int(z["pad"])
    pt.preprocess(obj_padding_px=(pad, pad))
    return pt


@pytest.mark.parametrize("case", ["single64", "mixed64", "c2small"])
def test_setup_matches_reference(case):
    z = load_golden(case)
    pt = build_from_golden(z)
    d = pt.dset
    assert abs(d.mean_diffraction_intensity - float(z["mean_intensity"])) / float(z["mean_intensity"]) < 1e-6
    assert rel(d.targets.numpy(), z["targets"]) < 1e-6
    np.testing.assert_allclose(d.initial_scan_positions_px.numpy(), z["initial_positions"], rtol=0, atol=1e-4)
    assert tuple(pt.obj_shape_full) == tuple(z["obj_shape"])
    np.testing.assert_array_equal(pt.obj_padding_px, z["obj_padding_px"])
    assert abs(d.upsample_factor - float(z["upsample_factor"])) < 1e-12
    assert rel(pt.probe_model._probe.detach().numpy(), z["probe_init"]) < 1e-5
    if int(z["S"]) > 1:
        assert rel(pt.propagators.numpy(), z["propagators"]) < 1e-6


def test_batcher_matches_reference_order():
    """Same numpy generator call sequence as the reference SimpleBatcher."""
    from quantem_b200.diffractive_imaging.ptycho_utils import SimpleBatcher

    b = SimpleBatcher(37, 10, rng=5)
    got = [x.tolist() for x in b]
    rng = np.random.default_rng(5)
    order = rng.permutation(np.arange(37))
    assert got == [order[i:i + 10].tolist() for i in range(0, 37, 10)]
    v = SimpleBatcher(20, 4, rng=1, val_ratio=0.25)
    assert len(v.val_indices) == 5 and len(v.train_indices) == 15


def test_gram_schmidt_matches_oracle():
    from oracle import ptycho_oracle as O
    from quantem_b200.diffractive_imaging.ptycho_utils import orthogonalize_probes

    rng = np.random.default_rng(0)
    p = rng.standard_normal((3, 16, 16)) + 1j * rng.standard_normal((3, 16, 16))
    p[1] *= 2.0
    ref, _, _ = O.gram_schmidt(p)
    got = orthogonalize_probes(torch.as_tensor(p)).numpy()
    assert rel(got, ref) < 1e-12


def test_unsupported_options_raise():
    from quantem_b200.diffractive_imaging import ObjectPixelated

    with pytest.raises(ValueError, match="Object type"):
        ObjectPixelated.from_uniform(num_slices=1, obj_type="absorption")
    o = ObjectPixelated.from_uniform(num_slices=1)
    o.add_constraint("tv_weight_xy", 0.1)  # every optional constraint is built for pixelated objects
    o.add_constraint("q_lowpass", 0.5)
    with pytest.raises(KeyError):
        o.add_constraint("no_such_constraint", 1)


@pytest.mark.parametrize("case", ["complex", "potential"])
def test_fov_mask_matches_reference(case):
    """The probe-overlap FOV mask Ptychography.preprocess builds (ptychography_base.py:
    191-216), on the host set-up path, against the reference's own (fixtures objcons_*)."""
    z = load_golden(f"objcons_{case}64")
    pt = build_from_golden(z)
    pt.probe_model._probe = torch.as_tensor(z["probe_init"]).requires_grad_(True)
    pt._set_obj_fov_mask()
    np.testing.assert_allclose(pt._get_probe_overlap(), z["probe_overlap"], rtol=1e-5, atol=1e-3)
    assert np.abs(pt.obj_model.mask.numpy() - z["fov_mask"]).max() < 1e-5


def test_reference_api_surface_on_the_host():
    """Members of the reference's Ptychography that need no GPU: units, snapshots, object
    type, probe intensities, optimiser bookkeeping, clone."""
    z = load_golden("mixed64")
    pt = build_from_golden(z)
    assert pt.reciprocal_units == ["A^-1", "A^-1"] and pt.angular_units == ["mrad", "mrad"]
    from quantem_b200.diffractive_imaging.complex_probe import electron_wavelength_angstrom

    np.testing.assert_allclose(pt.angular_sampling,
                               np.asarray(pt.dset.detector_sampling) * electron_wavelength_angstrom(float(z["energy"])) * 1e3)
    assert pt.iter_recon_types.size == 0 and pt.autograd
    pt.store_snapshots = True
    pt.store_snapshot_every = 2
    assert pt.store_snapshots and pt.store_snapshot_every == 2
    with pytest.raises(ValueError, match="No snapshots"):
        pt.get_snapshot_by_iter(0)
    o = pt.obj_model._obj.detach().numpy()  # snapshot objects are host arrays
    pt._snapshots = [dict(iteration=0, obj=o, probe=pt.probe), dict(iteration=4, obj=o, probe=pt.probe)]
    assert pt.get_snapshot_by_iter(3, closest=True)["iteration"] == 4
    assert pt.get_snapshot_by_iter(0, cropped=True)["obj"].shape == pt._crop_rotate_obj_fov(o).shape
    w = pt.get_probe_intensities()
    assert w.shape == (int(z["P"]),) and abs(w.sum() - 1) < 1e-6
    assert pt.obj_type == "complex"
    pt.set_obj_type("pure_phase")
    assert pt.obj_type == "pure_phase"
    pt.set_obj_type("complex")
    assert pt.schedulers == {}
    m = pt.obj_fov_mask
    assert m.shape == (1, *tuple(pt.obj_shape_full[-2:]))
    pt.obj_fov_mask = 0.5 * m[0]
    np.testing.assert_array_equal(pt.obj_fov_mask, 0.5 * m)
    c = pt.clone()
    assert c is not pt and c.obj_model is not pt.obj_model
    assert torch.equal(c.obj_model._obj.detach(), pt.obj_model._obj.detach())


@pytest.mark.parametrize("case", ["centertv", "center1", "tv3"])
def test_probe_constraints_on_the_host_match_reference(case):
    """The probe's optional constraints on host tensors (set-up code): the centred /
    orthogonalised probe and its TV loss against the reference's own (fixtures probecons_*64)."""
    from quantem_b200.diffractive_imaging import ProbePixelated
    from tests.test_oracle_golden import PROBECONS_CASES

    z = load_golden(f"probecons_{case}64")
    pm = ProbePixelated.from_params(probe_params={"energy": float(z["energy"]), "defocus": 200.0,
                                                  "semiangle_cutoff": 20.0}, num_probes=int(z["P"]))
    pm.constraints = PROBECONS_CASES[case]
    pm._probe = torch.as_tensor(z["probe_init"])
    p = pm.probe
    assert rel(p.numpy(), z["probe_constrained"]) < 2e-5
    soft = float(pm.apply_soft_constraints(p))
    assert abs(soft - float(z["probe_soft_loss"])) <= 1e-5 * max(float(z["probe_soft_loss"]), 1e-3)


@pytest.mark.parametrize("fit", ["plane", "constant"])
def test_bilinear_centring_matches_reference(fit):
    """preprocess(bilinear=True) on the host against the reference's own (fixture
    bilinear64): the CoM fit, the centred targets and the mean intensity."""
    from quantem_b200.diffractive_imaging import Dataset4dstem, PtychographyDatasetRaster

    z = load_golden("bilinear64")
    H, nscan = int(z["H"]), int(z["nscan"])
    px, step = float(z["px"]), float(z["step_px"])
    rs = 1.0 / (H * px)
    d4 = Dataset4dstem.from_array(z["data"].reshape(nscan, nscan, H, H), sampling=(step * px, step * px, rs, rs),
                                  units=("A", "A", "A^-1", "A^-1"))
    pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
    pd.preprocess(com_fit_function=fit, force_com_rotation=0, force_com_transpose=False, bilinear=True,
                  plot_rotation=False, plot_com=False, probe_energy=float(z["energy"]), device="cpu")
    np.testing.assert_allclose(pd.com_fit, z[f"com_fit_{fit}"], rtol=0, atol=1e-5)  # float32 CoM sums
    assert rel(pd.targets.numpy(), z[f"targets_{fit}"]) < 1e-6
    assert abs(pd.mean_diffraction_intensity - float(z[f"mean_intensity_{fit}"])) <= 1e-6 * pd.mean_diffraction_intensity


def test_model_api_members_on_the_host():
    """Members of the reference's dataset, probe and object models that need no GPU."""
    from quantem_b200.diffractive_imaging import PtychographyDatasetRaster

    z = load_golden("mixed64")
    pt = build_from_golden(z)
    d = pt.dset
    H, nscan = int(z["H"]), int(z["nscan"])
    assert tuple(d.shape) == (nscan, nscan, H, H) and tuple(d.dset.shape) == tuple(d.shape)
    assert d.reciprocal_units == ["A^-1", "A^-1"] and d.diffraction_padding.tolist() == [0, 0]
    assert tuple(d.intensities.shape) == (nscan * nscan, H, H)
    assert tuple(d.centered_intensities.shape) == (nscan * nscan, H, H)
    assert rel(d.centered_intensities.numpy(), d.centered_amplitudes.numpy() ** 2) < 1e-6
    assert not d.patch_indices_need_update()
    sh = torch.arange(12, dtype=torch.float32).reshape(6, 2) ** 2
    ref = 0.3 * (sh[:, 0].diff().abs().mean() + sh[:, 1].diff().abs().mean()) / 2
    assert torch.allclose(d.get_descan_tv_loss(sh, 0.3), ref)
    with pytest.raises(ValueError):
        d.intensities = np.zeros((2, H, H))
    d2 = PtychographyDatasetRaster.from_array(z["data"].reshape(nscan, nscan, H, H), sampling=(1, 1, 0.1, 0.1),
                                              units=("A", "A", "A^-1", "A^-1"), verbose=0)
    assert d2.num_gpts == nscan * nscan and d2.dset.name == "4D-STEM dataset"
    pm = pt.probe_model
    assert pm.name == "ProbePixelated" and tuple(pm.shape) == (int(z["P"]), H, H)
    assert torch.equal(pm.apply_hard_constraints(pm._probe.detach()), pm.probe.detach())
    om = pt.obj_model
    assert om.name == "ObjPixelized" and om.shape_2d == tuple(pt.obj_shape_full[-2:])


def test_host_probe_constraint_gradients_match_oracle():
    """The host (set-up) forms of the probe's centre-of-mass shift and TV loss: torch autograd
    through them against the FP64 oracle's reverse chain."""
    from oracle import ptycho_oracle as O
    from quantem_b200.diffractive_imaging.ptycho_utils import center_probe, probe_tv_loss

    rng = np.random.default_rng(12)
    n = 32
    y, x = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    p = np.stack([np.exp(-(((y - 4.2) % n) ** 2 + ((x - n + 6.1) % n) ** 2) / 25.0) * np.exp(0.3j * k * x)
                  for k in range(2)]) + 0.02 * rng.standard_normal((2, n, n))
    g = rng.standard_normal((2, n, n)) + 1j * rng.standard_normal((2, n, n))
    t = torch.as_tensor(p, dtype=torch.complex128).requires_grad_(True)
    out = center_probe(t)
    ref, cache = O.center_probe(p)
    # the host form forms -2 pi i k in complex64 first, as the reference's ramp does; the oracle
    # keeps it in float64
    assert rel(out.detach().numpy(), ref) < 1e-6
    (out.conj() * torch.as_tensor(g)).real.sum().backward()
    assert rel(t.grad.numpy(), O.center_probe_vjp(cache, g)) < 1e-6
    t.grad = None
    probe_tv_loss(t, 0.2).backward()
    assert rel(t.grad.numpy(), O.probe_tv_loss(p, 0.2)[1]) < 1e-12
