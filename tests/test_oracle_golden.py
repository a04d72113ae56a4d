"""Pins the FP64 CPU oracle to outputs of the reference itself (golden fixtures
made by tests/golden/make_golden.py from the reference package)."""
import numpy as np
import pytest

from oracle import ptycho_oracle as O
from tests.conftest import load_golden, rel


def obj_type_of(z):
    return str(z["obj_type"]) if "obj_type" in z else "complex"


def fp64(x):
    return x.astype(np.complex128) if np.iscomplexobj(x) else x.astype(np.float64)


@pytest.mark.parametrize("case", ["single64", "mixed64", "mixed128", "purephase64", "potential64"])
def test_oracle_matches_reference_batch(case):
    z = load_golden(case)
    S = int(z["S"])
    props = z["propagators"].astype(np.complex128) if S > 1 else np.zeros((0,) + z["targets"].shape[1:])
    bi = z["batch_indices"]
    pos = z["positions"].astype(np.float64)[bi]
    mask = np.ones(z["targets"].shape[1:])
    loss, g_obj, g_probe, st = O.full_gradients(
        fp64(z["obj_perturbed"]), z["probe_init"].astype(np.complex128), pos, props,
        z["targets"].astype(np.float64)[bi], mask, z["positions"].shape[0], float(z["mean_intensity"]),
        float(z["upsample_factor"]), orthogonalize=bool(z["orthogonalize"]), obj_type=obj_type_of(z))
    assert rel(O.detector_intensities(st), z["batch_intensities"]) < 2e-6
    assert abs(loss - float(z["batch_loss"])) / float(z["batch_loss"]) < 2e-6
    assert rel(g_obj, z["grad_obj"]) < 5e-6
    assert rel(g_probe, z["grad_probe"]) < 5e-6


def test_oracle_propagators_match_reference():
    z = load_golden("mixed64")
    p = O.propagators(z["targets"].shape[1:], z["sampling"], float(z["energy"]), [float(z["dz"])] * (int(z["S"]) - 1))
    assert rel(p, z["propagators"]) < 1e-6


def _cos(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.real(np.vdot(a, b)) / np.linalg.norm(a) / np.linalg.norm(b))


@pytest.mark.parametrize("nprobe", [1, 2])
def test_oracle_matches_reference_gradient_test_case(nprobe):
    """The reference's own gradient-test fixture (white-noise object, 1 px raster,
    4096 positions), autograd gradients after one full-batch step.

    At the uniform starting object all 4096 positions predict the same pattern
    and the per-position gradient terms largely cancel in the sums, so float32
    evaluations (the reference's, or the oracle run in complex64) differ from the
    float64 result by ~1e-2 in the object gradient and by ~0.3 in the probe
    gradient (measured: oracle complex64 vs complex128 object gradient 7.9e-3).
    The loss is well conditioned and keeps the 1e-5 bar; the gradients are
    checked at the level float32 arithmetic can reach here."""
    from tests.golden.whitenoise import whitenoise_inputs

    inp = whitenoise_inputs()
    z = load_golden("whitenoise64")
    tag = f"p{nprobe}_ad"
    N = inp["N"]
    # targets = centred amplitudes after the reference's constant-CoM preprocessing
    from quantem_b200.diffractive_imaging import Dataset4dstem, PtychographyDatasetRaster

    d4 = Dataset4dstem.from_array(inp["data4d"], sampling=inp["sampling4d"], units=("A", "A", "A^-1", "A^-1"))
    pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
    pd.preprocess(com_fit_function="constant", force_com_rotation=0, force_com_transpose=False,
                  probe_energy=inp["energy"])
    assert abs(pd.mean_diffraction_intensity - float(z["mean_intensity"])) / float(z["mean_intensity"]) < 1e-6
    probe = z[f"probe_used_{tag}"].astype(np.complex128)
    obj = np.ones((1, N, N), np.complex128)
    pos = pd.scan_positions_px.numpy().astype(np.float64)
    loss, g_obj, g_probe, _ = O.full_gradients(obj, probe, pos, np.zeros((0, N, N)),
                                               pd.targets.numpy().astype(np.float64), np.ones((N, N)),
                                               pd.num_gpts, pd.mean_diffraction_intensity, pd.upsample_factor,
                                               orthogonalize=False)
    assert abs(loss - z[f"loss_{tag}"][0]) / z[f"loss_{tag}"][0] < 1e-5
    assert rel(g_obj, z[f"grad_obj_{tag}"]) < 2e-2
    assert _cos(g_obj, z[f"grad_obj_{tag}"]) > 0.9999
    assert _cos(g_probe, z[f"grad_probe_{tag}"]) > 0.9


@pytest.mark.parametrize("case", ["single64", "mixed64", "mixed128"])
def test_oracle_analytic_update_matches_reference(case):
    z = load_golden(case)
    S, H = int(z["S"]), int(z["H"])
    props = z["propagators"].astype(np.complex128) if S > 1 else np.zeros((0, H, H))
    bi = z["batch_indices"]
    g_obj, g_probe, _ = O.analytic_gradients(z["obj_perturbed"].astype(np.complex128),
                                             z["probe_init"].astype(np.complex128),
                                             z["positions"].astype(np.float64)[bi], props,
                                             z["targets"].astype(np.float64)[bi],
                                             orthogonalize=bool(z["orthogonalize"]))
    assert rel(g_obj, z["grad_obj_an"]) < 5e-6
    assert rel(g_probe, z["grad_probe_an"]) < 5e-6


@pytest.mark.parametrize("loss_type", O.LOSS_TYPES)
def test_oracle_loss_types_match_reference(loss_type):
    """All five consistency losses and their dL/dI against the reference's own
    error_estimate (ptychography_base.py:908-932), fixture tests/golden/loss_types.npz."""
    z = load_golden("loss_types")
    inten, mask = z["intensity"], z["mask"]
    loss, dldi_cc = O.loss_and_seed(np.fft.ifftshift(inten, axes=(-2, -1)), z[f"{loss_type}_targets"], mask,
                                    int(z["num_gpts"]), float(z["mean_intensity"]), loss_type)
    assert abs(loss - float(z[f"{loss_type}_loss"])) <= 1e-12 * abs(float(z[f"{loss_type}_loss"]))
    assert rel(np.fft.fftshift(dldi_cc, axes=(-2, -1)), z[f"{loss_type}_dldi"]) < 1e-12


def test_oracle_matches_reference_c2small():
    """The headline geometry (8 slices, 4 modes with weights 0.7/0.15/0.1/0.05 at 128^2,
    512^2 object, two windows wrapping both edges): the reference's batch intensities,
    loss and autograd gradients (object gradient on the sampled pixels)."""
    from tests.golden.c2small import load_c2small, sampled

    z = load_c2small()
    bi = z["batch_indices"]
    H = int(z["H"])
    loss, g_obj, g_probe, st = O.full_gradients(
        z["obj_perturbed"].astype(np.complex128), z["probe_init"].astype(np.complex128),
        z["positions"].astype(np.float64)[bi], z["propagators"].astype(np.complex128),
        z["targets"].astype(np.float64)[bi], np.ones((H, H)), z["positions"].shape[0], float(z["mean_intensity"]),
        float(z["upsample_factor"]), orthogonalize=True)
    assert rel(O.detector_intensities(st), z["batch_intensities"]) < 2e-6
    assert abs(loss - float(z["batch_loss"])) / float(z["batch_loss"]) < 2e-6
    assert rel(sampled(g_obj, z["grad_idx"]), z["grad_obj_sampled"]) < 5e-6
    assert rel(g_probe, z["grad_probe"]) < 5e-6


@pytest.mark.parametrize("case", ["purephase64", "potential64"])
def test_oracle_reconstruct_matches_reference_object_types(case):
    """Two Adam iterations of the reference's reconstruct for pure-phase and potential
    objects: loss trajectory and final parameters against the FP64 oracle."""
    z = load_golden(case)
    H = int(z["H"])
    obj, probe, losses = O.reconstruct(fp64(z["obj_perturbed"]), z["probe_init"].astype(np.complex128),
                                       z["positions"].astype(np.float64), z["propagators"].astype(np.complex128),
                                       z["targets"].astype(np.float64), np.ones((H, H)), float(z["mean_intensity"]),
                                       float(z["upsample_factor"]), int(z["iters"]), int(z["batch"]),
                                       np.random.default_rng(int(z["recon_rng_seed"])), obj_type=obj_type_of(z))
    np.testing.assert_allclose(losses, z["recon_losses"], rtol=2e-6)
    assert rel(obj, z["recon_obj"]) < 1e-5
    assert rel(probe, z["recon_probe"]) < 1e-5


def test_oracle_position_gradients_and_learned_positions_match_reference():
    """Learned scan positions (fixture positions64, made by the reference with a dataset
    optimiser and learn_descan=False): the batch's autograd position gradient, and 3 Adam
    iterations moving object, probe and positions."""
    z = load_golden("positions64")
    H = int(z["H"])
    bi = z["batch_indices"]
    props = z["propagators"].astype(np.complex128)
    loss, _, _, st = O.full_gradients(
        z["obj_perturbed"].astype(np.complex128), z["probe_init"].astype(np.complex128),
        z["positions"].astype(np.float64)[bi], props, z["targets"].astype(np.float64)[bi], np.ones((H, H)),
        z["positions"].shape[0], float(z["mean_intensity"]), float(z["upsample_factor"]), orthogonalize=True)
    assert abs(loss - float(z["batch_loss"])) / float(z["batch_loss"]) < 2e-6
    g = O.position_gradients(st.probe_o, st, st.g_probe_plane)
    ref = z["grad_positions"][bi]
    assert np.abs(z["grad_positions"][len(bi):]).max() == 0.0  # positions outside the batch get none
    assert rel(g, ref) < 1e-5  # the reference's float32 ramp and FFTs
    obj, probe, losses, pos = O.reconstruct(
        z["obj_perturbed"].astype(np.complex128), z["probe_init"].astype(np.complex128),
        z["positions"].astype(np.float64), props, z["targets"].astype(np.float64), np.ones((H, H)),
        float(z["mean_intensity"]), float(z["upsample_factor"]), int(z["iters"]), int(z["batch"]),
        np.random.default_rng(int(z["recon_rng_seed"])), lr_positions=1e-2)
    np.testing.assert_allclose(losses, z["recon_losses"], rtol=1e-5)
    moved_ref = z["recon_positions"] - z["positions"]
    assert np.abs(moved_ref).max() > 0.02
    assert rel(pos - z["positions"], moved_ref) < 1e-3  # Adam's sign-like steps on float32 gradients
    assert rel(obj, z["recon_obj"]) < 1e-4


def test_oracle_descan_and_tilt_gradients_and_learning_match_reference():
    """Learned descan shifts and probe tilt (fixture descantilt64, made by the reference with
    a dataset optimiser over the descan shifts and learn_probe_tilt=True): the batch's
    autograd descan and tilt gradients against the uncentred targets, and 3 Adam
    iterations moving object, probe, tilt and descan."""
    z = load_golden("descantilt64")
    H, S = int(z["H"]), int(z["S"])
    bi = z["batch_indices"]
    geom = ((H, H), tuple(z["sampling"]), float(z["energy"]), [float(z["dz"])] * (S - 1))
    props = O.propagators(*geom, tilt_mrad=tuple(z["tilt"]))
    assert rel(props, z["propagators"]) < 1e-6  # the reference's complex64 propagators at the start tilt
    loss, g_obj, g_probe, st = O.full_gradients(
        z["obj_perturbed"].astype(np.complex128), z["probe_init"].astype(np.complex128),
        z["positions"].astype(np.float64)[bi], props, z["targets"].astype(np.float64)[bi], np.ones((H, H)),
        z["positions"].shape[0], float(z["mean_intensity"]), float(z["upsample_factor"]), orthogonalize=True,
        descan=z["descan"].astype(np.float64)[bi])
    assert abs(loss - float(z["batch_loss"])) / float(z["batch_loss"]) < 2e-6
    assert rel(np.fft.fftshift(st.intensity, axes=(-2, -1)), z["batch_intensities"]) < 2e-6
    assert rel(g_obj, z["grad_obj"]) < 5e-6
    assert rel(g_probe, z["grad_probe"]) < 5e-6
    gd = O.descan_gradients(st)
    assert np.abs(z["grad_descan"][len(bi):]).max() == 0.0
    assert rel(gd, z["grad_descan"][bi]) < 1e-5
    gt = O.tilt_gradients(st, tuple(z["tilt"]), geom[3], geom[1], geom[0])
    assert rel(gt, z["grad_tilt"]) < 1e-5
    obj, probe, losses, learned = O.reconstruct(
        z["obj_perturbed"].astype(np.complex128), z["probe_init"].astype(np.complex128),
        z["positions"].astype(np.float64), props, z["targets"].astype(np.float64), np.ones((H, H)),
        float(z["mean_intensity"]), float(z["upsample_factor"]), int(z["iters"]), int(z["batch"]),
        np.random.default_rng(int(z["recon_rng_seed"])), descan=z["descan"], lr_descan=1e-2,
        tilt=z["tilt"], prop_geometry=geom)
    np.testing.assert_allclose(losses, z["recon_losses"], rtol=1e-5)
    moved = z["recon_descan"] - z["descan"]
    assert np.abs(moved).max() > 0.02
    assert rel(learned["descan"] - z["descan"], moved) < 1e-3
    assert rel(learned["tilt"] - z["tilt"], z["recon_tilt"] - z["tilt"]) < 1e-3
    assert rel(obj, z["recon_obj"]) < 1e-4
    assert np.array_equal(z["recon_positions"], z["positions"])  # scan positions not learned


OBJCONS_CASES = {
    "complex": ("complex", {"gaussian_sigma": 1.0, "tv_weight_xy": 0.05, "tv_weight_z": 0.02,
                            "surface_zero_weight": 0.01}),
    "complexfov": ("complex", {"apply_fov_mask": True, "gaussian_sigma": 1.0}),
    "potential": ("potential", {"fix_potential_baseline": True, "apply_fov_mask": True, "identical_slices": True,
                                "tv_weight_xy": 0.05}),
    "pure_phase": ("pure_phase", {"gaussian_sigma": 0.7, "identical_slices": True, "tv_weight_xy": 0.04}),
    "butter_complex": ("complex", {"q_lowpass": 1.5, "q_highpass": 0.05, "butterworth_order": 3}),
    "butter_potential": ("potential", {"q_lowpass": 1.2, "gaussian_sigma": 0.8}),
}


@pytest.mark.parametrize("case", sorted(OBJCONS_CASES))
def test_oracle_object_constraints_match_reference(case):
    """Optional object constraints (fixtures objcons_*64, made by the reference): the
    probe-overlap FOV mask, the hard-constrained object, the soft-constraint loss, one
    batch's total loss and raw-object / probe gradients, and 2 Adam iterations."""
    obj_type, cons = OBJCONS_CASES[case]
    z = load_golden(f"objcons_{case}64")
    H = int(z["H"])
    probe_o = O.gram_schmidt(z["probe_init"].astype(np.complex128))[0]
    ov = O.probe_overlap(np.abs(probe_o[0]) ** 2, z["positions"].astype(np.float64), z["obj_shape"][-2:])
    assert rel(ov, z["probe_overlap"]) < 1e-5
    mask = O.fov_mask(ov, z["obj_padding_px"])
    assert np.abs(mask - z["fov_mask"]).max() < 1e-5
    raw = z["obj_perturbed"].astype(np.complex128 if obj_type != "potential" else np.float64)
    smp = tuple(z["obj_sampling"])
    ext = O._ext_args(cons, mask, raw.shape[-2:], smp)
    obj2 = O.constrain_object_ext(raw, obj_type, **ext)
    assert rel(obj2, z["obj_constrained"]) < 1e-5
    soft, _ = O.soft_constraint_loss(obj2, obj_type, cons.get("tv_weight_z", 0), cons.get("tv_weight_xy", 0),
                                     cons.get("surface_zero_weight", 0))
    assert abs(soft - float(z["soft_loss"])) <= 1e-5 * max(abs(float(z["soft_loss"])), 1e-3)
    bi = z["batch_indices"]
    props = z["propagators"].astype(np.complex128)
    args = (props, z["targets"].astype(np.float64)[bi], np.ones((H, H)), z["positions"].shape[0],
            float(z["mean_intensity"]), float(z["upsample_factor"]))
    loss, g_obj, g_probe, _ = O.full_gradients(raw, z["probe_init"].astype(np.complex128),
                                               z["positions"].astype(np.float64)[bi], *args, obj_type=obj_type,
                                               obj_constraints=cons, obj_mask=mask, obj_sampling=smp)
    assert abs(loss - float(z["batch_total_loss"])) / float(z["batch_total_loss"]) < 2e-6
    assert rel(g_obj, z["grad_obj"]) < 5e-5
    assert rel(g_probe, z["grad_probe"]) < 5e-6
    obj, probe, losses = O.reconstruct(
        raw, z["probe_init"].astype(np.complex128), z["positions"].astype(np.float64), props,
        z["targets"].astype(np.float64), np.ones((H, H)), float(z["mean_intensity"]), float(z["upsample_factor"]),
        int(z["iters"]), int(z["batch"]), np.random.default_rng(int(z["recon_rng_seed"])), obj_type=obj_type,
        obj_constraints=cons, obj_mask=mask, obj_sampling=smp)
    np.testing.assert_allclose(losses, z["recon_losses"], rtol=2e-5)
    assert rel(obj, z["recon_obj"]) < 2e-4


PROBECONS_CASES = {
    "centertv": {"orthogonalize_probe": True, "center_probe": True, "tv_weight": 0.05},
    "center1": {"orthogonalize_probe": False, "center_probe": True, "tv_weight": 0.0},
    "tv3": {"orthogonalize_probe": True, "center_probe": False, "tv_weight": 0.1},
}


@pytest.mark.parametrize("case", sorted(PROBECONS_CASES))
def test_oracle_probe_constraints_match_reference(case):
    """Optional probe constraints (fixtures probecons_*64, made by the reference): the
    centre-of-mass shifted / orthogonalised probe, the probe TV loss, one batch's total loss
    and gradients, and 2 Adam iterations."""
    cons = PROBECONS_CASES[case]
    z = load_golden(f"probecons_{case}64")
    H = int(z["H"])
    raw_p = z["probe_init"].astype(np.complex128)
    probe_c, _ = O.constrain_probe(raw_p, cons)
    assert rel(probe_c, z["probe_constrained"]) < 1e-5
    soft, _ = O.probe_tv_loss(probe_c, cons["tv_weight"])
    assert abs(soft - float(z["probe_soft_loss"])) <= 1e-5 * max(abs(float(z["probe_soft_loss"])), 1e-3)
    raw = z["obj_perturbed"].astype(np.complex128)
    bi = z["batch_indices"]
    props = z["propagators"].astype(np.complex128)
    args = (props, z["targets"].astype(np.float64)[bi], np.ones((H, H)), z["positions"].shape[0],
            float(z["mean_intensity"]), float(z["upsample_factor"]))
    loss, g_obj, g_probe, _ = O.full_gradients(raw, raw_p, z["positions"].astype(np.float64)[bi], *args,
                                               probe_constraints=cons)
    assert abs(loss - float(z["batch_total_loss"])) / float(z["batch_total_loss"]) < 2e-6
    assert rel(g_obj, z["grad_obj"]) < 5e-5
    assert rel(g_probe, z["grad_probe"]) < 5e-5
    obj, probe, losses = O.reconstruct(
        raw, raw_p, z["positions"].astype(np.float64), props, z["targets"].astype(np.float64), np.ones((H, H)),
        float(z["mean_intensity"]), float(z["upsample_factor"]), int(z["iters"]), int(z["batch"]),
        np.random.default_rng(int(z["recon_rng_seed"])), probe_constraints=cons)
    np.testing.assert_allclose(losses, z["recon_losses"], rtol=2e-5)
    assert rel(obj, z["recon_obj"]) < 2e-4
    assert rel(probe, z["recon_probe"]) < 2e-4


@pytest.mark.parametrize("case,obj_type", [("purephase64", "pure_phase"), ("potential64", "potential")])
def test_oracle_analytic_update_of_other_object_types_matches_reference(case, obj_type):
    """The analytic update directions of pure-phase and potential objects (object_models.py:
    705-712: a potential takes Re(-i conj(o) conj(psi) g)) against the reference's own."""
    z = load_golden(case)
    bi = z["batch_indices"]
    raw = z["obj_perturbed"].astype(np.float64 if obj_type == "potential" else np.complex128)
    g_obj, g_probe, _ = O.analytic_gradients(raw, z["probe_init"].astype(np.complex128),
                                             z["positions"].astype(np.float64)[bi],
                                             z["propagators"].astype(np.complex128),
                                             z["targets"].astype(np.float64)[bi],
                                             orthogonalize=bool(z["orthogonalize"]), obj_type=obj_type)
    assert np.isrealobj(g_obj) == (obj_type == "potential")
    assert rel(g_obj, z["grad_obj_an"]) < 5e-6
    assert rel(g_probe, z["grad_probe_an"]) < 5e-6
