"""FP64 central finite differences of the oracle's batch loss against its adjoint.

The loss is a function of the raw object (through the hard constraint, with its
mean-phase term) and of the raw probe modes (through Gram-Schmidt and the intensity
sort).  For random complex directions d the directional derivative
dL/dt (x + t d) at t = 0 equals Re<g, d> for a gradient g in torch's convention
(dL/dRe + i dL/dIm).  In FP64 a central difference with t ~ 1e-6 of the parameter
scale agrees with it to ~1e-8 relative (truncation ~t^2, rounding ~1e-16 / t).

The check is made at the fixtures' start object with its amplitude scaled by 0.999:
the hard constraint clamps |o| to 1, and the start objects (amplitude 1 - 0.3 U[0,1))
hold a few pixels within 1e-6 of that kink, where a difference quotient straddles two
branches (measured: up to 1.5e-3 relative at t = 1e-6 on the unscaled c2small start)."""
import numpy as np
import pytest

from oracle import ptycho_oracle as O
from tests.conftest import load_golden


def _loss(z, obj_raw, probe_raw):
    bi = z["batch_indices"]
    H = int(z["H"])
    S = int(z["S"])
    props = z["propagators"].astype(np.complex128) if S > 1 else np.zeros((0, H, H))
    obj_c = O.constrain_object(obj_raw)
    probe_o = O.gram_schmidt(probe_raw)[0] if int(z["orthogonalize"]) else probe_raw
    st = O.forward(obj_c, probe_o, z["positions"].astype(np.float64)[bi], props)
    loss, _ = O.loss_and_seed(st.intensity, z["targets"].astype(np.float64)[bi], np.ones((H, H)),
                              z["positions"].shape[0], float(z["mean_intensity"]))
    return loss


def _grads(z, obj_raw, probe_raw):
    bi = z["batch_indices"]
    H = int(z["H"])
    S = int(z["S"])
    props = z["propagators"].astype(np.complex128) if S > 1 else np.zeros((0, H, H))
    loss, g_obj, g_probe, _ = O.full_gradients(
        obj_raw, probe_raw, z["positions"].astype(np.float64)[bi], props, z["targets"].astype(np.float64)[bi],
        np.ones((H, H)), z["positions"].shape[0], float(z["mean_intensity"]), 1.0,
        orthogonalize=bool(int(z["orthogonalize"])))
    return loss, g_obj * 2.0, g_probe  # undo the upsample_factor^2 / 2 rescale (factor 1 here)


def fd_directional(z, obj_raw, probe_raw, d_obj, d_probe, t):
    """Central difference of the loss along (d_obj, d_probe)."""
    lp = _loss(z, obj_raw + t * d_obj, probe_raw + t * d_probe)
    lm = _loss(z, obj_raw - t * d_obj, probe_raw - t * d_probe)
    return (lp - lm) / (2 * t)


def random_directions(rng, obj_raw, probe_raw, which):
    """Unit-scale complex directions (scaled to the parameters' RMS) for the object, the
    probe, or both."""
    def rnd(x):
        d = rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape)
        return d * (np.sqrt(np.mean(np.abs(x) ** 2)) / np.sqrt(np.mean(np.abs(d) ** 2)))

    d_obj = rnd(obj_raw) if which in ("obj", "both") else np.zeros_like(obj_raw)
    d_probe = rnd(probe_raw) if which in ("probe", "both") else np.zeros_like(probe_raw)
    return d_obj, d_probe


def _inner(g, d):
    return float(np.sum(g.real * d.real + g.imag * d.imag))


@pytest.mark.parametrize("case", ["single64", "mixed64", "c2small"])
@pytest.mark.parametrize("which", ["obj", "probe", "both"])
def test_oracle_adjoint_matches_fp64_finite_differences(case, which):
    if case == "c2small":
        from tests.golden.c2small import load_c2small

        z = load_c2small()
    else:
        z = load_golden(case)
    obj_raw = z["obj_perturbed"].astype(np.complex128) * 0.999  # away from the |o| = 1 clamp
    probe_raw = z["probe_init"].astype(np.complex128)
    _, g_obj, g_probe = _grads(z, obj_raw, probe_raw)
    loss = _loss(z, obj_raw, probe_raw)
    t = 1e-6
    rng = np.random.default_rng(hash((case, which)) % 2**32)
    for _ in range(2):
        d_obj, d_probe = random_directions(rng, obj_raw, probe_raw, which)
        adj = _inner(g_obj, d_obj) + _inner(g_probe, d_probe)
        fd = fd_directional(z, obj_raw, probe_raw, d_obj, d_probe, t)
        # 1e-7 relative plus the difference quotient's own rounding floor, eps |L| / t
        # (random directions in ~10^5 dimensions cancel much of <g, d>)
        assert abs(fd - adj) <= 1e-7 * abs(adj) + 4 * np.finfo(np.float64).eps * abs(loss) / t, (fd, adj)


@pytest.mark.parametrize("case", ["single64", "mixed64", "c2small"])
def test_oracle_position_gradients_match_fp64_finite_differences(case):
    """dL/d(scan positions): only the fractional shift of the probe depends on a position
    (the rounded part picks the patch), so a central difference of 1e-6 px, far from the
    rounding boundaries of the fixture positions, checks O.position_gradients."""
    if case == "c2small":
        from tests.golden.c2small import load_c2small

        z = load_c2small()
    else:
        z = load_golden(case)
    H, S = int(z["H"]), int(z["S"])
    props = z["propagators"].astype(np.complex128) if S > 1 else np.zeros((0, H, H))
    bi = z["batch_indices"]
    obj_c = O.constrain_object(z["obj_perturbed"].astype(np.complex128))
    probe_o = O.gram_schmidt(z["probe_init"].astype(np.complex128))[0] if int(z["orthogonalize"]) else \
        z["probe_init"].astype(np.complex128)
    pos = z["positions"].astype(np.float64)[bi]
    tg = z["targets"].astype(np.float64)[bi]
    args = (props, tg, np.ones((H, H)), z["positions"].shape[0], float(z["mean_intensity"]))
    loss, _, _, st = O.batch_loss_and_grads(obj_c, probe_o, pos, *args)
    gpos = O.position_gradients(probe_o, st, st.g_probe_plane)
    frac = pos - np.round(pos)
    assert np.abs(np.abs(frac) - 0.5).min() > 1e-3  # no position sits on a rounding boundary
    rng = np.random.default_rng(5)
    d = rng.standard_normal(pos.shape)
    t = 1e-6

    def lossat(p):
        return O.batch_loss_and_grads(obj_c, probe_o, p, *args)[0]

    fd = (lossat(pos + t * d) - lossat(pos - t * d)) / (2 * t)
    adj = float(np.sum(gpos * d))
    assert abs(fd - adj) <= 1e-6 * abs(adj) + 4 * np.finfo(np.float64).eps * abs(loss) / t, (fd, adj)


@pytest.mark.parametrize("case", ["single64", "mixed64", "c2small"])
def test_oracle_descan_gradients_match_fp64_finite_differences(case):
    """dL/d(descan shift): the descan ramp multiplies the exit wave, so every batch
    entry's two shifts enter smoothly; central differences of 1e-6 px along a random
    direction check O.descan_gradients at random shifts of up to 0.8 px."""
    if case == "c2small":
        from tests.golden.c2small import load_c2small

        z = load_c2small()
    else:
        z = load_golden(case)
    H, S = int(z["H"]), int(z["S"])
    props = z["propagators"].astype(np.complex128) if S > 1 else np.zeros((0, H, H))
    bi = z["batch_indices"]
    obj_c = O.constrain_object(z["obj_perturbed"].astype(np.complex128))
    probe_o = O.gram_schmidt(z["probe_init"].astype(np.complex128))[0] if int(z["orthogonalize"]) else \
        z["probe_init"].astype(np.complex128)
    pos = z["positions"].astype(np.float64)[bi]
    tg = z["targets"].astype(np.float64)[bi]
    args = (props, tg, np.ones((H, H)), z["positions"].shape[0], float(z["mean_intensity"]))
    rng = np.random.default_rng(9)
    dsc = rng.uniform(-0.8, 0.8, size=pos.shape)
    loss, _, _, st = O.batch_loss_and_grads(obj_c, probe_o, pos, *args, descan=dsc)
    g = O.descan_gradients(st)
    d = rng.standard_normal(pos.shape)
    t = 1e-6

    def lossat(x):
        return O.batch_loss_and_grads(obj_c, probe_o, pos, *args, descan=x)[0]

    fd = (lossat(dsc + t * d) - lossat(dsc - t * d)) / (2 * t)
    adj = float(np.sum(g * d))
    assert abs(fd - adj) <= 1e-6 * abs(adj) + 4 * np.finfo(np.float64).eps * abs(loss) / t, (fd, adj)


@pytest.mark.parametrize("case", ["mixed64", "c2small"])
def test_oracle_tilt_gradients_match_fp64_finite_differences(case):
    """dL/d(probe tilt) through the propagators (probe_models.py:376-427) at a tilt of
    (1.5, -2.0) mrad: central differences of 1e-4 mrad of the loss with the propagators
    recomputed at each tilt; also the reference's zero-gradient rule at a zero tilt."""
    if case == "c2small":
        from tests.golden.c2small import load_c2small

        z = load_c2small()
    else:
        z = load_golden(case)
    H, S = int(z["H"]), int(z["S"])
    px = float(z["px"]) if "px" in z else 0.2
    energy = float(z["energy"]) if "energy" in z else 300e3
    dz = [float(z["dz"])] * (S - 1)
    bi = z["batch_indices"]
    obj_c = O.constrain_object(z["obj_perturbed"].astype(np.complex128))
    probe_o = O.gram_schmidt(z["probe_init"].astype(np.complex128))[0] if int(z["orthogonalize"]) else \
        z["probe_init"].astype(np.complex128)
    pos = z["positions"].astype(np.float64)[bi]
    tg = z["targets"].astype(np.float64)[bi]
    rest = (tg, np.ones((H, H)), z["positions"].shape[0], float(z["mean_intensity"]))

    def lossat(tilt):
        props = O.propagators((H, H), (px, px), energy, dz, tilt_mrad=tilt)
        return O.batch_loss_and_grads(obj_c, probe_o, pos, props, *rest)

    tilt = (1.5, -2.0)
    loss, _, _, st = lossat(tilt)
    g = O.tilt_gradients(st, tilt, dz, (px, px), (H, H))
    t = 1e-4
    for a in range(2):
        e = np.zeros(2)
        e[a] = t
        fd = (lossat(tuple(np.add(tilt, e)))[0] - lossat(tuple(np.subtract(tilt, e)))[0]) / (2 * t)
        assert abs(fd - g[a]) <= 1e-6 * abs(g[a]) + 4 * np.finfo(np.float64).eps * abs(loss) / t, (a, fd, g[a])
    _, _, _, st0 = lossat((0.0, 0.0))
    assert np.all(O.tilt_gradients(st0, (0.0, 0.0), dz, (px, px), (H, H)) == 0.0)


@pytest.mark.parametrize("obj_type", ["complex", "pure_phase", "potential"])
def test_oracle_constraint_chain_vjp_matches_fp64_finite_differences(obj_type):
    """The optional hard constraints (FOV mask, Gaussian blur, Butterworth filter; not
    identical slices, whose gradient is straight-through by design, nor the potential's
    fixed baseline, whose offset is detached by design, both as in the reference) and the
    soft-constraint loss: their VJPs against central differences."""
    import scipy.ndimage as ndi

    rng = np.random.default_rng(17)
    S, H, W = 3, 24, 20
    m = np.zeros((H, W))
    m[4:20, 3:17] = 1.0
    m = ndi.gaussian_filter(m, 1.5)
    if obj_type == "potential":
        x = 0.05 + 0.1 * rng.standard_normal((S, H, W))
        x = x + 0.5  # away from the positivity clamp's kink
        cons = {"apply_fov_mask": True, "gaussian_sigma": 0.9, "q_lowpass": 1.4}
    else:
        x = (0.5 + 0.4 * rng.random((S, H, W))) * np.exp(0.7j * rng.standard_normal((S, H, W)))
        cons = {"apply_fov_mask": True, "gaussian_sigma": 0.9, "q_lowpass": 1.4, "q_highpass": 0.1}
    ext = O._ext_args(cons, m, (H, W), (0.2, 0.2))
    cplx = np.iscomplexobj(x)
    G = rng.standard_normal(x.shape) + (1j * rng.standard_normal(x.shape) if cplx else 0)

    def L(v):
        y = O.constrain_object_ext(v, obj_type, **ext)
        return float(np.sum((np.conj(y) * G).real))

    g = O.constrain_object_ext_vjp(x, G, obj_type, **ext)
    d = rng.standard_normal(x.shape) + (1j * rng.standard_normal(x.shape) if cplx else 0)
    t = 1e-6
    fd = (L(x + t * d) - L(x - t * d)) / (2 * t)
    adj = float(np.sum((np.conj(g) * d).real))
    assert abs(fd - adj) <= 1e-6 * abs(adj) + 1e-8, (fd, adj)
    # soft constraints, at an object without zero-magnitude pixels (the phase of a zero pixel
    # has no derivative; both the kernels and the oracle give it a zero gradient there)
    y = x if obj_type == "potential" else x * np.exp(0.3j)
    loss, gs = O.soft_constraint_loss(y, obj_type, 0.03, 0.05, 0.02)
    dy = rng.standard_normal(y.shape) + (1j * rng.standard_normal(y.shape) if np.iscomplexobj(y) else 0)
    ls = lambda v: O.soft_constraint_loss(v, obj_type, 0.03, 0.05, 0.02)[0]  # noqa: E731
    fd = (ls(y + t * dy) - ls(y - t * dy)) / (2 * t)
    adj = float(np.sum((np.conj(gs) * dy).real))
    assert abs(fd - adj) <= 1e-5 * abs(adj) + 1e-8, (fd, adj)


@pytest.mark.parametrize("P", [1, 3])
def test_oracle_probe_constraints_match_fp64_finite_differences(P):
    """The probe's centre-of-mass shift (through the centre of mass itself) and its TV soft
    loss, after Gram-Schmidt, through a random linear functional of the constrained probe:
    Re<g, d> of the reverse chain against central differences along random directions."""
    rng = np.random.default_rng(61 + P)
    n = 32
    y, x = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    base = np.exp(-(((y - 5.3) % n) ** 2 + ((x - n + 4.1) % n) ** 2) / 30.0)  # off-centre blob
    probe = np.stack([base * np.exp(1j * 0.3 * k * x) + 0.05 * (rng.standard_normal((n, n))
                                                                 + 1j * rng.standard_normal((n, n)))
                      for k in range(P)])
    w = rng.standard_normal((P, n, n)) + 1j * rng.standard_normal((P, n, n))
    cons = {"orthogonalize_probe": True, "center_probe": True, "tv_weight": 0.07}

    def loss(p):
        c, _ = O.constrain_probe(p, cons)
        tv, _ = O.probe_tv_loss(c, cons["tv_weight"])
        return float(np.sum((np.conj(w) * c).real)) + tv

    c, cache = O.constrain_probe(probe, cons)
    _, g_tv = O.probe_tv_loss(c, cons["tv_weight"])
    g = O.constrain_probe_vjp(cache, w + g_tv)
    for _ in range(3):
        d = rng.standard_normal(probe.shape) + 1j * rng.standard_normal(probe.shape)
        t = 1e-6 * np.abs(probe).max() / np.abs(d).max()
        fd = (loss(probe + t * d) - loss(probe - t * d)) / (2 * t)
        an = float(np.sum((np.conj(g) * d).real))
        assert abs(fd - an) <= 1e-6 * abs(an) + 1e-9
