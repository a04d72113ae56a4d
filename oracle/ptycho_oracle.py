"""CPU oracle for the multislice mixed-probe ptychography iteration.

TEST INFRASTRUCTURE ONLY.  This module restates, in numpy/scipy, the algorithm
of quantem.diffractive_imaging's gradient-descent iteration so that the CUDA
path can be checked against it.  Only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg may import it; the product package never
does, and the product fails loudly when its CUDA library is missing.

Precision: every function is dtype-generic.  Parity checks run it in
complex128/float64 (with the reference's float32 constants restated in float64,
see ``propagators`` and ``translation_ramp``); the CPU baseline runs it in
complex64/float32 like the reference's default configuration.

Pinning: the reference ships no golden vectors for this path (its two gradient
tests compare autograd against analytic gradients by SSIM only).  This oracle is
pinned against fixtures produced by running the reference itself
(``tests/golden/make_golden.py``; see ``tests/test_oracle_golden.py``).

Conventions (all from the reference):
* complex gradients follow torch: grad = dL/dRe + i dL/dIm;
* FFT norms: propagation uses the unnormalised forward / 1/N inverse pair
  (ptychography_base.py:988), the detector the orthonormal FFT
  (detector_models.py:28);
* object patches are corner-centred windows with modulo wrap
  (dataset_models.py:514-535); positions are rounded half-to-even
  (dataset_models.py:1490, torch.round).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np
import scipy.fft as sfft

_WORKERS = int(os.environ.get("QUANTEM_ORACLE_WORKERS", "1"))


def set_workers(n: int) -> None:
    """Number of threads scipy.fft may use (CPU-baseline timing uses all)."""
    global _WORKERS
    _WORKERS = max(1, int(n))


def fft2(x, norm="backward"):
    return sfft.fft2(x, axes=(-2, -1), norm=norm, workers=_WORKERS)


def ifft2(x, norm="backward"):
    return sfft.ifft2(x, axes=(-2, -1), norm=norm, workers=_WORKERS)


def real_dtype(cdtype):
    return np.float64 if np.dtype(cdtype) == np.complex128 else np.float32


# ----------------------------------------------------------------------------
# constants and setup restatements
# ----------------------------------------------------------------------------

def electron_wavelength_angstrom(energy_ev: float) -> float:
    """Relativistic electron wavelength [A]; core/utils/utils.py:97-104."""
    m = 9.109383e-31
    e = 1.602177e-19
    c = 299792458.0
    h = 6.62607e-34
    return (
        h / math.sqrt(2 * m * e * energy_ev) / math.sqrt(1 + e * energy_ev / 2 / m / c**2) * 1e10
    )


def fftfreq_index(n: int) -> np.ndarray:
    """Integer fftfreq(n, d=1/n) used for corner-centred patches."""
    return np.fft.fftfreq(n, d=1.0 / n).astype(np.int64)


def propagators(roi_shape, sampling, energy, slice_thicknesses, tilt_mrad=(0.0, 0.0),
                cdtype=np.complex128):
    """Fresnel propagators (S-1, H, W); probe_models.py:376-427.

    The reference evaluates k^2 in complex64 (probe_models.py:407,413); this
    restatement evaluates the same formula in the precision of ``cdtype``.
    """
    dz = np.atleast_1d(np.asarray(slice_thicknesses, dtype=np.float64))
    if dz.size == 0:
        return np.zeros((0, *roi_shape), dtype=cdtype)
    kr = np.fft.fftfreq(int(roi_shape[0]), float(sampling[0]))
    kc = np.fft.fftfreq(int(roi_shape[1]), float(sampling[1]))
    k2 = kr[:, None] ** 2 + kc[None, :] ** 2
    lam = electron_wavelength_angstrom(energy)
    props = np.exp(-1j * np.pi * lam * dz[:, None, None] * k2[None])
    tr, tc = tilt_mrad
    if tr != 0:
        props = props * np.exp(-2j * np.pi * dz[:, None, None] * np.tan(tr / 1e3) * kr[None, :, None])
    if tc != 0:
        props = props * np.exp(-2j * np.pi * dz[:, None, None] * np.tan(tc / 1e3) * kc[None, None, :])
    return props.astype(cdtype)


def translation_ramp(frac: np.ndarray, shape, cdtype=np.complex128) -> np.ndarray:
    """Sub-pixel Fourier translation ramp (B, H, W); ptycho_utils.py:156-176."""
    nr, nc = shape
    kr = np.fft.fftfreq(nr, d=1.0)
    kc = np.fft.fftfreq(nc, d=1.0)
    r = frac[:, 0][:, None, None]
    c = frac[:, 1][:, None, None]
    ramp = np.exp(-2j * np.pi * kr[None, :, None] * r) * np.exp(-2j * np.pi * kc[None, None, :] * c)
    return ramp.astype(cdtype)


def round_half_even(x: np.ndarray) -> np.ndarray:
    return np.round(x)  # numpy rounds half to even, like torch.round


def split_positions(positions_px: np.ndarray):
    """(r0, c0) integer patch origins and fractional offsets; dataset_models.py:1487-1490."""
    rounded = round_half_even(positions_px)
    frac = positions_px - rounded
    return rounded.astype(np.int64), frac


def patch_rows_cols(origins: np.ndarray, roi_shape, obj_shape):
    """Wrapped row / column index grids of every patch; dataset_models.py:514-535."""
    fr = fftfreq_index(int(roi_shape[0]))
    fc = fftfreq_index(int(roi_shape[1]))
    rows = (origins[:, 0][:, None] + fr[None, :]) % int(obj_shape[0])
    cols = (origins[:, 1][:, None] + fc[None, :]) % int(obj_shape[1])
    return rows, cols  # (B, H), (B, W)


def gather_patches(obj: np.ndarray, rows: np.ndarray, cols: np.ndarray) -> np.ndarray:
    """(S, B, H, W) patches; object_models.py:252-265."""
    return obj[:, rows[:, :, None], cols[:, None, :]]


def scatter_patches(grad_patches: np.ndarray, rows, cols, obj_shape_3d) -> np.ndarray:
    """Adjoint of ``gather_patches`` (index_add); ptycho_utils.py:215-236."""
    out = np.zeros(obj_shape_3d, dtype=grad_patches.dtype)
    S = obj_shape_3d[0]
    for s in range(S):
        np.add.at(out[s], (rows[:, :, None], cols[:, None, :]), grad_patches[s])
    return out


# ----------------------------------------------------------------------------
# hard constraints
# ----------------------------------------------------------------------------

def constrain_object(obj: np.ndarray) -> np.ndarray:
    """Complex-object hard constraint; object_models.py:289-300.

    o' = clamp(|o|, 0, 1) * exp(i (angle(o) - mean(angle(o)))), mean over the
    whole (S, Ho, Wo) array.
    """
    amp = np.clip(np.abs(obj), 0.0, 1.0)
    ph = np.angle(obj)
    ph = ph - ph.mean()
    return (amp * np.exp(1j * ph)).astype(obj.dtype)


def constrain_object_vjp(obj: np.ndarray, grad_out: np.ndarray) -> np.ndarray:
    """Vector-Jacobian product of ``constrain_object`` (torch gradient convention).

    clamp passes the gradient where 0 <= |o| <= 1 (inclusive), abs contributes
    sgn(o) * g_a, angle contributes i o / |o|^2 * g_phi (zero at o == 0), and the
    mean removal subtracts the mean of g_phi over the whole object.
    """
    mag = np.abs(obj)
    amp = np.clip(mag, 0.0, 1.0)
    ph = np.angle(obj)
    th = ph - ph.mean()
    e = np.exp(1j * th)
    ge = grad_out * np.conj(e)
    g_amp = ge.real
    g_th = amp * ge.imag
    g_ph = g_th - g_th.mean()
    g_mag = np.where((mag >= 0.0) & (mag <= 1.0), g_amp, 0.0)
    safe = np.where(mag == 0, 1.0, mag)
    sgn = np.where(mag == 0, 0.0, obj / safe)
    dang = np.where(mag == 0, 0.0, 1j * obj / safe**2)
    return (g_mag * sgn + g_ph * dang).astype(obj.dtype)


def object_transmission(obj: np.ndarray, obj_type: str = "complex", positivity: bool = True,
                        fix_baseline: bool = False, baseline_factor: float = 1.0) -> np.ndarray:
    """Transmission multiplied into the wave, for every object type:
    apply_hard_constraints (object_models.py:289-339, no FOV mask) followed by the
    exp(i V) of _get_obj_patches for real potentials (object_models.py:252-256).

    complex: ``constrain_object``; pure_phase: exp(i (angle(o) - mean angle));
    potential: V' = V - offset (offset = factor * min V when the baseline is fixed),
    clamped at 0 with positivity, transmission exp(i V')."""
    if obj_type == "complex":
        return constrain_object(obj)
    if obj_type == "pure_phase":
        ph = np.angle(obj)
        return np.exp(1j * (ph - ph.mean())).astype(obj.dtype)
    if obj_type == "potential":
        v = obj - (obj.min() * baseline_factor if fix_baseline else 0.0)
        if positivity:
            v = np.maximum(v, 0.0)
        cdt = np.complex128 if obj.dtype == np.float64 else np.complex64
        return np.exp(1j * v).astype(cdt)
    raise ValueError(obj_type)


def object_transmission_vjp(obj: np.ndarray, grad_t: np.ndarray, obj_type: str = "complex",
                            positivity: bool = True, fix_baseline: bool = False,
                            baseline_factor: float = 1.0) -> np.ndarray:
    """VJP of ``object_transmission`` w.r.t. the raw object (torch convention).

    pure_phase: the amplitude does not enter, g = g_phi * i o / |o|^2 with g_phi the
    mean-removed Im(G conj(e)); potential: dL/dV = Re(conj(G) i t) where the clamp
    passes (V - offset >= 0, inclusive like torch.clamp) -- the offset is detached."""
    if obj_type == "complex":
        return constrain_object_vjp(obj, grad_t)
    if obj_type == "pure_phase":
        mag = np.abs(obj)
        th = np.angle(obj) - np.angle(obj).mean()
        g_th = (grad_t * np.exp(-1j * th)).imag
        g_ph = g_th - g_th.mean()
        safe = np.where(mag == 0, 1.0, mag)
        dang = np.where(mag == 0, 0.0, 1j * obj / safe**2)
        return (g_ph * dang).astype(obj.dtype)
    if obj_type == "potential":
        v = obj - (obj.min() * baseline_factor if fix_baseline else 0.0)
        passes = (v >= 0.0) if positivity else np.ones(v.shape, bool)
        t = np.exp(1j * (np.maximum(v, 0.0) if positivity else v))
        return np.where(passes, (np.conj(grad_t) * 1j * t).real, 0.0).astype(obj.dtype)
    raise ValueError(obj_type)


# ----------------------------------------------------------------------------
# optional object constraints (object_models.py:273-480) and the FOV mask
# (ptychography_base.py:191-216)
# ----------------------------------------------------------------------------

def probe_overlap(probe0_intensity: np.ndarray, positions_px: np.ndarray, obj_shape_2d) -> np.ndarray:
    """sum over positions of |probe mode 0|^2 placed at each position's patch window
    (ptychography_base.py:201-216, ptycho_utils.py:215-236; unshifted probe, rounded
    positions, wrapped windows)."""
    H, W = probe0_intensity.shape
    origins, _ = split_positions(np.asarray(positions_px, dtype=np.float64))
    rows, cols = patch_rows_cols(origins, (H, W), obj_shape_2d)
    out = np.zeros(tuple(int(x) for x in obj_shape_2d), dtype=np.float64)
    for b in range(origins.shape[0]):
        np.add.at(out, (rows[b][:, None], cols[b][None, :]), probe0_intensity)
    return out


def fov_mask(overlap: np.ndarray, obj_padding_px, gaussian_sigma: float = 2.0) -> np.ndarray:
    """ptychography_base.py:191-199: overlap > 0.3 max, binary closing (5 iterations),
    binary dilation (min(32, min(padding) // 4) iterations), Gaussian filter."""
    import scipy.ndimage as ndi

    ov = overlap > overlap.max() * 0.3
    ov = ndi.binary_closing(ov, iterations=5)
    ov = ndi.binary_dilation(ov, iterations=min(32, int(np.min(obj_padding_px)) // 4))
    return ndi.gaussian_filter(ov.astype(np.float32), sigma=gaussian_sigma)


def gaussian_taps(sigma: float) -> np.ndarray:
    """The normalised float32 Gaussian of object_models.py:445-451."""
    k = int(2 * math.ceil(3 * sigma) + 1)
    if k % 2 == 0:
        k += 1
    ax = np.arange(-k // 2 + 1.0, k // 2 + 1.0, dtype=np.float32)
    g = np.exp(-0.5 * (ax / np.float32(sigma)) ** 2).astype(np.float32)
    return (g / g.sum()).astype(np.float32)


def blur(x: np.ndarray, taps: np.ndarray) -> np.ndarray:
    """object_models.py:437-479: zero-padded 'same' correlation with the taps along the
    rows, then along the columns, of every slice (real and imaginary parts separately).
    Self-adjoint (symmetric taps, symmetric zero padding): the VJP is the same blur."""
    import scipy.ndimage as ndi

    t = np.asarray(taps, dtype=np.float64)

    def one(a):
        a = ndi.correlate1d(a, t, axis=-2, mode="constant", cval=0.0)
        return ndi.correlate1d(a, t, axis=-1, mode="constant", cval=0.0)

    if np.iscomplexobj(x):
        return one(x.real) + 1j * one(x.imag)
    return one(x)


def butterworth_env(shape, sampling, q_lowpass=None, q_highpass=None, order: int = 4) -> np.ndarray:
    """The float32 Butterworth envelope of object_models.py:495-507 on the (H, W) frequency
    grid of the object (fftfreq with the object sampling, |q| radial)."""
    qx = np.fft.fftfreq(int(shape[0]), float(sampling[0])).astype(np.float32)
    qy = np.fft.fftfreq(int(shape[1]), float(sampling[1])).astype(np.float32)
    qya, qxa = np.meshgrid(qy, qx, indexing="xy")
    qra = np.sqrt(qxa**2 + qya**2).astype(np.float32)
    env = np.ones_like(qra)
    if q_highpass:
        env = env * (1 - 1 / (1 + (qra / np.float32(q_highpass)) ** (2 * order)))
    if q_lowpass:
        env = env * (1 / (1 + (qra / np.float32(q_lowpass)) ** (2 * order)))
    return env.astype(np.float32)


def butterworth(x: np.ndarray, env: np.ndarray) -> np.ndarray:
    """object_models.py:509-520: per slice, mean removed, ifft2(fft2(x) env), mean added
    back; the real part for a real (potential) input."""
    mu = x.mean(axis=(-2, -1), keepdims=True)
    y = np.fft.ifft2(np.fft.fft2(x - mu) * env) + mu
    return y.real if not np.iscomplexobj(x) else y


def butterworth_vjp(g: np.ndarray, env: np.ndarray, real: bool) -> np.ndarray:
    """VJP of ``butterworth``: the filter P = ifft2 env fft2 is self-adjoint (a real,
    radially symmetric envelope), so g_x = P g - mean(P g) + mean(g) per slice (real part
    for a real input)."""
    pg = np.fft.ifft2(np.fft.fft2(g) * env)
    out = pg - pg.mean(axis=(-2, -1), keepdims=True) + g.mean(axis=(-2, -1), keepdims=True)
    return out.real if real else out


def constrain_object_ext(obj: np.ndarray, obj_type: str, mask=None, positivity: bool = True,
                         fix_baseline: bool = False, baseline_factor: float = 1.0, taps=None,
                         identical: bool = False, butter_env=None) -> np.ndarray:
    """ObjectConstraints.apply_hard_constraints (object_models.py:289-339) with the FOV mask
    (apply_fov_mask, the mask (H, W) applied to every slice), the Gaussian blur and identical
    slices: complex / pure phase -> amp mask exp(i (angle - mean angle) mask) times the mask
    again (the reference multiplies the amplitude by the mask twice); potential -> V - offset
    (offset = factor * mean of V over the background pixels, mask < 0.5 max mask, or factor *
    min V without a background), clamped at 0, times the mask.  Returns the complex object or
    the real potential before exp(i V)."""
    m = None if mask is None else np.asarray(mask, dtype=np.float64)[None]
    if obj_type in ("complex", "pure_phase"):
        amp = np.clip(np.abs(obj), 0.0, 1.0) if obj_type == "complex" else np.ones(obj.shape)
        ph = np.angle(obj) - np.angle(obj).mean()
        out = amp * np.exp(1j * ph) if m is None else amp * m * np.exp(1j * ph * m) * m
    elif obj_type == "potential":
        off = 0.0
        if fix_baseline:
            if m is not None:
                bg = np.broadcast_to(m < 0.5 * m.max(), obj.shape)
                off = obj[bg].mean() if bg.any() else obj.min()
            else:
                off = obj.min()
            off = off * baseline_factor
        out = obj - off
        if positivity:
            out = np.maximum(out, 0.0)
        if m is not None:
            out = out * m
    else:
        raise ValueError(obj_type)
    if taps is not None:
        out = blur(out, taps)
    if butter_env is not None:
        out = butterworth(out, butter_env)
    if identical and out.shape[0] > 1:
        out = np.broadcast_to(out.mean(axis=0, keepdims=True), out.shape).copy()
    return out


def constrain_object_ext_vjp(obj: np.ndarray, grad_out: np.ndarray, obj_type: str, mask=None,
                             positivity: bool = True, fix_baseline: bool = False, baseline_factor: float = 1.0,
                             taps=None, identical: bool = False, butter_env=None) -> np.ndarray:
    """VJP of ``constrain_object_ext`` w.r.t. the raw object (torch convention).  Identical
    slices pass the gradient straight through (the reference averages in place under
    no_grad), the blur is self-adjoint, the potential's offset is detached."""
    g = np.asarray(grad_out)
    if butter_env is not None:
        g = butterworth_vjp(g, butter_env, real=obj_type == "potential")
    if taps is not None:
        g = blur(g, taps)
    m = None if mask is None else np.asarray(mask, dtype=np.float64)[None]
    if obj_type in ("complex", "pure_phase"):
        mag = np.abs(obj)
        amp = np.clip(mag, 0.0, 1.0) if obj_type == "complex" else np.ones(obj.shape)
        th = np.angle(obj) - np.angle(obj).mean()
        mm = np.ones(obj.shape) if m is None else np.broadcast_to(m, obj.shape)
        A = amp * (mm if m is None else mm * mm)
        e = np.exp(1j * th * mm)
        g_amp = (mm * mm if m is not None else 1.0) * (np.conj(e) * g).real
        g_th = mm * A * (np.conj(e) * g).imag
        g_ph = g_th - g_th.mean()
        passes = (mag >= 0.0) & (mag <= 1.0) if obj_type == "complex" else np.zeros(obj.shape, bool)
        g_mag = np.where(passes, g_amp, 0.0)
        safe = np.where(mag == 0, 1.0, mag)
        r = np.where(mag == 0, 0.0, g_mag * obj / safe + g_ph * 1j * obj / safe**2)
        return r
    if obj_type == "potential":
        off = 0.0
        if fix_baseline:
            if m is not None:
                bg = np.broadcast_to(m < 0.5 * m.max(), obj.shape)
                off = obj[bg].mean() if bg.any() else obj.min()
            else:
                off = obj.min()
            off = off * baseline_factor
        v = obj - off
        passes = (v >= 0.0) if positivity else np.ones(v.shape, bool)
        gg = np.real(g) * (1.0 if m is None else m)
        return np.where(passes, gg, 0.0)
    raise ValueError(obj_type)


def phase_exp_vjp(v: np.ndarray, grad_t: np.ndarray) -> np.ndarray:
    """dL/dV of t = exp(i V) (object_models.py:252-256): Re(conj(G) i t)."""
    return (np.conj(grad_t) * 1j * np.exp(1j * v)).real


def soft_constraint_loss(obj2: np.ndarray, obj_type: str, tv_weight_z: float = 0.0, tv_weight_xy: float = 0.0,
                         surface_zero_weight: float = 0.0):
    """Soft constraints of the hard-constrained object (object_models.py:341-435): TV of
    the phase (and, for complex objects, the amplitude) or of the potential, along z with
    tv_weight_z and along rows / columns with tv_weight_xy, each term w * mean |diff|,
    divided by the number of weighted dimensions; surface-zero terms on the first and last
    slices (3 slices or more).  Returns (loss, gradient w.r.t. obj2 in torch convention)."""
    S = obj2.shape[0]
    w = (tv_weight_z, tv_weight_xy) if S > 1 else (0.0, tv_weight_xy)
    loss = 0.0
    cplx = np.iscomplexobj(obj2)
    g_ph = np.zeros(obj2.shape)
    g_amp = np.zeros(obj2.shape)
    g_real = np.zeros(obj2.shape)

    def tv(a, g):
        nonlocal loss
        ws = [w[0] if (d == 0) else w[1] for d in range(3)]
        nd = sum(1 for x in ws if x > 0)
        if nd == 0:
            return
        for d in range(3):
            if ws[d] <= 0:
                continue
            df = np.diff(a, axis=d)
            loss += ws[d] * np.mean(np.abs(df)) / nd
            sg = np.sign(df) * ws[d] / (df.size * nd)
            pad_hi = [(0, 0)] * 3
            pad_lo = [(0, 0)] * 3
            pad_hi[d] = (1, 0)
            pad_lo[d] = (0, 1)
            g += np.pad(sg, pad_hi) - np.pad(sg, pad_lo)

    if any(w):
        if cplx:
            tv(np.angle(obj2), g_ph)
            if obj_type == "complex":
                tv(np.abs(obj2), g_amp)
        else:
            tv(obj2, g_real)
    if surface_zero_weight and S >= 3:
        sw = surface_zero_weight
        for k in (0, S - 1):
            if cplx:
                ang = np.angle(obj2[k])
                ph = np.abs(ang)
                u = ph - ph.mean()
                n = u.size
                if obj_type == "complex":
                    loss += sw * np.mean(1.0 - np.abs(obj2[k]))
                    g_amp[k] += -sw / n
                loss += sw * np.mean(np.abs(u))
                su = np.sign(u)
                g_ph[k] += sw * (su - su.mean()) / n * np.sign(ang)
            else:
                loss += sw * np.mean(np.abs(obj2[k]))
                g_real[k] += sw * np.sign(obj2[k]) / obj2[k].size
    if cplx:
        a = np.abs(obj2)
        safe = np.where(a == 0, 1.0, a)
        grad = np.where(a == 0, 0.0, g_amp * obj2 / safe + 1j * g_ph * obj2 / safe**2)
        return float(loss), grad
    return float(loss), g_real


def gram_schmidt(probe: np.ndarray):
    """Mixed-state probe orthogonalisation + intensity sort; probe_models.py:484-525.

    Modified Gram-Schmidt with the running vector (as the reference loop), each
    mode rescaled to its original norm, then sorted by descending intensity.
    Returns (probes_sorted, order, cache-for-vjp).
    """
    P = probe.shape[0]
    flat = probe.reshape(P, -1)
    n0 = np.sqrt(np.sum(flat.real**2 + flat.imag**2, axis=1))
    qs, steps = [], []
    for i in range(P):
        u = flat[i].copy()
        hist = []
        for j in range(len(qs)):
            c = np.sum(np.conj(qs[j]) * u)
            hist.append((u.copy(), c))
            u = u - c * qs[j]
        nrm = np.sqrt(np.sum(u.real**2 + u.imag**2))
        nrm_c = max(nrm, 1e-12)
        qs.append(u / nrm_c)
        steps.append((hist, u, nrm, nrm_c))
    q = np.stack(qs)
    out = q * n0[:, None]
    inten = np.sum(np.abs(out) ** 2, axis=1)
    order = np.argsort(-inten, kind="stable")
    cache = dict(flat=flat, n0=n0, q=q, steps=steps, order=order)
    return out[order].reshape(probe.shape), order, cache


def gram_schmidt_vjp(cache, grad_sorted: np.ndarray) -> np.ndarray:
    """Reverse mode of ``gram_schmidt`` (torch gradient convention)."""
    flat, n0, q, steps, order = (cache[k] for k in ("flat", "n0", "q", "steps", "order"))
    P, n = flat.shape
    g_out = np.zeros_like(flat)
    g_out[order] = grad_sorted.reshape(P, n)
    g_q = g_out * n0[:, None]
    g_n0 = np.sum((np.conj(q) * g_out).real, axis=1)
    g_flat = np.zeros_like(flat)
    for i in range(P):
        g_flat[i] += flat[i] / max(n0[i], 1e-300) * g_n0[i]
    for i in reversed(range(P)):
        hist, u, nrm, nrm_c = steps[i]
        gq = g_q[i]
        g_u = gq / nrm_c
        if nrm >= 1e-12:
            g_nrm = -np.sum((np.conj(u) * gq).real) / nrm_c**2
            g_u = g_u + u / nrm * g_nrm
        for j in reversed(range(len(hist))):
            u_prev, c = hist[j]
            # u = u_prev - c q_j
            g_c = -np.sum(np.conj(q[j]) * g_u)
            g_q[j] += -np.conj(c) * g_u
            # c = sum(conj(q_j) * u_prev)
            g_uprev = g_u + q[j] * g_c
            g_q[j] += np.conj(g_c) * u_prev
            g_u = g_uprev
        g_flat[i] += g_u
    return g_flat.reshape(grad_sorted.shape)


def center_probe(probe: np.ndarray):
    """Probe centre-of-mass constraint; probe_models.py:467-482.

    Per mode: the centre of mass of |psi|^2 on the fftshifted grid, minus n // 2, and the
    mode Fourier-shifted by minus that offset (fourier_shift_expand with expand_dim=False,
    ptycho_utils.py:128-139; the ramp's frequencies are float32 fftfreq values,
    ptycho_utils.py:166-170).  An unshifted row y sits at (y + n // 2) mod n after the
    fftshift.  Returns (centred probe, cache for ``center_probe_vjp``)."""
    P, nr, nc = probe.shape
    inten = probe.real**2 + probe.imag**2
    wr = ((np.arange(nr) + nr // 2) % nr).astype(np.float64)
    wc = ((np.arange(nc) + nc // 2) % nc).astype(np.float64)
    tot = inten.sum(axis=(-2, -1))
    com = np.stack([(inten * wr[None, :, None]).sum(axis=(-2, -1)) / tot - nr // 2,
                    (inten * wc[None, None, :]).sum(axis=(-2, -1)) / tot - nc // 2], axis=-1)
    kr = np.fft.fftfreq(nr).astype(np.float32).astype(np.float64)
    kc = np.fft.fftfreq(nc).astype(np.float32).astype(np.float64)
    # shift by -com: exp(-2 pi i (kr (-com_r) + kc (-com_c)))
    ramp = np.exp(2j * np.pi * (kr[None, :, None] * com[:, 0, None, None] + kc[None, None, :] * com[:, 1, None, None]))
    spec = fft2(probe) * ramp
    cache = dict(probe=probe, spec=spec, ramp=ramp, com=com, tot=tot, wr=wr, wc=wc, kr=kr, kc=kc)
    return ifft2(spec), cache


def center_probe_vjp(cache, g: np.ndarray) -> np.ndarray:
    """Reverse mode of ``center_probe`` (torch gradient convention): the adjoint of the
    fixed shift, ifft2(fft2(g) conj(ramp)), plus the path through the centre of mass,
    dL/dcom = Re (1/n^2) sum_k conj(fft2(g)) spec 2 pi i k and dcom/d|psi|^2 = (w - n // 2
    - com) / sum |psi|^2, with d|psi|^2 -> 2 psi."""
    probe, spec, ramp, com, tot, wr, wc, kr, kc = (cache[k] for k in
                                                   ("probe", "spec", "ramp", "com", "tot", "wr", "wc", "kr", "kc"))
    P, nr, nc = probe.shape
    G = fft2(g)
    g_lin = ifft2(G * np.conj(ramp))
    cross = np.conj(G) * spec * (2j * np.pi) / (nr * nc)
    d_com_r = (cross * kr[None, :, None]).sum(axis=(-2, -1)).real
    d_com_c = (cross * kc[None, None, :]).sum(axis=(-2, -1)).real
    d_inten = (d_com_r[:, None, None] * (wr[None, :, None] - nr // 2 - com[:, 0, None, None])
               + d_com_c[:, None, None] * (wc[None, None, :] - nc // 2 - com[:, 1, None, None])) / tot[:, None, None]
    return g_lin + 2.0 * probe * d_inten


def probe_tv_loss(probe: np.ndarray, weight: float):
    """Probe total-variation soft constraint; probe_models.py:460-466: weight times the sum
    over the last two axes of mean |diff(probe)|.  Returns (loss, gradient); the gradient of
    |d| is d / |d| and 0 where d = 0 (torch's convention)."""
    if not weight:
        return 0.0, np.zeros_like(probe)
    loss, g = 0.0, np.zeros_like(probe)
    for axis in (-1, -2):
        d = np.diff(probe, axis=axis)
        a = np.abs(d)
        loss += a.mean()
        s = np.where(a > 0, d / np.where(a > 0, a, 1.0), 0.0) / d.size
        hi = [slice(None)] * probe.ndim
        lo = [slice(None)] * probe.ndim
        hi[axis], lo[axis] = slice(1, None), slice(None, -1)
        g[tuple(hi)] += s
        g[tuple(lo)] -= s
    return float(weight * loss), weight * g


def constrain_probe(probe_raw: np.ndarray, probe_constraints: dict | None = None):
    """The probe's hard constraints in the reference's order (probe_models.py:452-458):
    Gram-Schmidt + sort when ``orthogonalize_probe`` (default on), then the centre-of-mass
    shift when ``center_probe``.  Returns (probe, cache for ``constrain_probe_vjp``)."""
    c = {"orthogonalize_probe": True} if probe_constraints is None else probe_constraints
    p, gs_cache, ctr_cache = probe_raw, None, None
    if c.get("orthogonalize_probe", True):
        p, _, gs_cache = gram_schmidt(p)
    if c.get("center_probe", False):
        p, ctr_cache = center_probe(p)
    return p, (gs_cache, ctr_cache)


def constrain_probe_vjp(cache, g: np.ndarray) -> np.ndarray:
    gs_cache, ctr_cache = cache
    if ctr_cache is not None:
        g = center_probe_vjp(ctr_cache, g)
    if gs_cache is not None:
        g = gram_schmidt_vjp(gs_cache, g)
    return g


# ----------------------------------------------------------------------------
# forward model and loss
# ----------------------------------------------------------------------------

@dataclass
class ForwardState:
    rows: np.ndarray
    cols: np.ndarray
    ramp: np.ndarray
    patches: np.ndarray          # (S, B, H, W)
    waves: list = field(default_factory=list)  # incoming wave at each slice, (P, B, H, W)
    far: np.ndarray = None       # orthonormal far field (P, B, H, W)
    intensity: np.ndarray = None  # corner-centred sum over modes (B, H, W)
    g_probe_plane: np.ndarray = None  # set by adjoint: dL/d(shifted probe) (P, B, H, W)
    probe_o: np.ndarray = None        # set by full_gradients: the orthogonalised probe used
    descan_ramp: np.ndarray = None    # (B, H, W) descan ramp of the exit wave, or None
    exit: np.ndarray = None           # exit wave (P, B, H, W) after the descan ramp
    g_exit: np.ndarray = None         # set by adjoint: dL/d(exit) (P, B, H, W)
    prop_sums: np.ndarray = None      # set by adjoint: (S-1, 2) sum_k fftfreq_idx(k) Im(conj(G_Z) Z)


def forward(obj_c: np.ndarray, probe_o: np.ndarray, positions_px: np.ndarray,
            props: np.ndarray, descan: np.ndarray | None = None) -> ForwardState:
    """Batch forward model.

    probe shift: ptycho_utils.py:128-139 (fft2 -> ramp -> ifft2), probe_models.py:718-720;
    multislice: ptychography_base.py:934-947, 970-989;
    descan (optional, (B, 2) px): the exit wave times the translation ramp of the
    descan shift evaluated on the real-space grid (ptychography_base.py:903-905,
    ptycho_utils.py:156-176), which moves the far field by -descan pixels;
    detector: detector_models.py:22-30 (orthonormal FFT, |.|^2 summed over modes).
    The returned intensity is corner-centred (before the detector fftshift).
    """
    S = obj_c.shape[0]
    H, W = probe_o.shape[-2:]
    origins, frac = split_positions(positions_px)
    rows, cols = patch_rows_cols(origins, (H, W), obj_c.shape[-2:])
    ramp = translation_ramp(frac, (H, W), probe_o.dtype)
    patches = gather_patches(obj_c, rows, cols)
    psi = ifft2(fft2(probe_o)[:, None] * ramp[None])  # (P, B, H, W)
    st = ForwardState(rows=rows, cols=cols, ramp=ramp, patches=patches)
    for s in range(S):
        st.waves.append(psi)
        chi = patches[s][None] * psi
        if s < S - 1:
            psi = ifft2(fft2(chi) * props[s][None, None])
        else:
            psi = chi
    if descan is not None:
        st.descan_ramp = translation_ramp(np.asarray(descan, dtype=np.float64), (H, W), probe_o.dtype)
        psi = psi * st.descan_ramp[None]
    st.exit = psi
    st.far = fft2(psi, norm="ortho")
    st.intensity = np.sum(st.far.real**2 + st.far.imag**2, axis=0)
    return st


def detector_intensities(state: ForwardState) -> np.ndarray:
    """fftshifted predicted intensities (B, H, W) as DetectorPixelated.forward returns."""
    return np.fft.fftshift(state.intensity, axes=(-2, -1))


LOSS_TYPES = ("l2_amplitude", "l1_amplitude", "l2_intensity", "l1_intensity", "poisson")


def loss_and_seed(intensity_cc: np.ndarray, targets: np.ndarray, mask: np.ndarray,
                  num_gpts: int, mean_intensity: float, loss_type: str = "l2_amplitude"):
    """Consistency loss and dL/dI (corner-centred); ptychography_base.py:908-932.

    ``targets``/``mask`` are in detector (centred) layout, so they are
    ifftshifted onto the corner-centred intensity grid first.
    """
    B = intensity_cc.shape[0]
    t = np.fft.ifftshift(targets, axes=(-2, -1))
    m = np.fft.ifftshift(mask, axes=(-2, -1))
    scale = 1.0 / (B / num_gpts) / mean_intensity
    if "amplitude" in loss_type:
        pred = np.sqrt(intensity_cc + 1e-9)
        dpred_dI = 0.5 / pred
    else:
        pred = intensity_cc
        dpred_dI = np.ones_like(pred)
    diff = pred * m - t * m
    if loss_type.startswith("l2"):
        loss = np.sum(diff**2) * scale
        dL_dpred = 2 * diff * m * scale
    elif loss_type.startswith("l1"):
        loss = np.sum(np.abs(diff)) * scale
        dL_dpred = np.sign(diff) * m * scale
    elif loss_type == "poisson":
        loss = np.sum(pred - t * np.log(pred + 1e-6)) / mean_intensity
        dL_dpred = (1 - t / (pred + 1e-6)) / mean_intensity
    else:
        raise ValueError(loss_type)
    return float(loss), dL_dpred * dpred_dI


def adjoint(obj_c, probe_o, props, st: ForwardState, dL_dI: np.ndarray):
    """Gradients of the batch loss w.r.t. the constrained object and the
    orthogonalised probe (torch convention), by reversing ``forward``."""
    S = obj_c.shape[0]
    H, W = probe_o.shape[-2:]
    g_far = 2.0 * st.far * dL_dI[None]
    g = ifft2(g_far, norm="ortho")  # adjoint of the orthonormal FFT
    st.g_exit = g
    if st.descan_ramp is not None:
        g = g * np.conj(st.descan_ramp)[None]
    g_patch = np.zeros_like(st.patches)
    fr = fftfreq_index(H).astype(np.float64)[:, None]
    fc = fftfreq_index(W).astype(np.float64)[None, :]
    st.prop_sums = np.zeros((max(S - 1, 0), 2))
    for s in reversed(range(S)):
        psi = st.waves[s]
        g_patch[s] = np.sum(np.conj(psi) * g, axis=0)
        g = np.conj(st.patches[s])[None] * g
        if s > 0:
            # propagator sensitivity: Z = fft2(chi_{s-1}) K_{s-1} enters w_s = ifft2(Z), so
            # dL/dZ = fft2(g) / (H W) (torch convention) and sum_k k Im(conj(dL/dZ) Z) carries
            # every per-axis phase ramp of K (the tilt terms of probe_models.py:418-425)
            gz = fft2(g) / (H * W)
            z = fft2(st.patches[s - 1][None] * st.waves[s - 1]) * props[s - 1][None, None]
            im = np.imag(np.conj(gz) * z)
            st.prop_sums[s - 1] = (np.sum(fr * im), np.sum(fc * im))
            g = ifft2(fft2(g) * np.conj(props[s - 1])[None, None])
    # probe shift adjoint: ifft2(sum_b conj(ramp_b) * fft2(g_b))
    acc = np.sum(fft2(g) * np.conj(st.ramp)[None], axis=1)
    g_probe = ifft2(acc)
    g_obj = scatter_patches(g_patch, st.rows, st.cols, obj_c.shape)
    st.g_probe_plane = g  # (P, B, H, W): gradient w.r.t. the shifted probe, for position gradients
    return g_obj, g_probe


def position_gradients(probe_o, st: ForwardState, g_probe_plane: np.ndarray) -> np.ndarray:
    """dL/d(scan position) (B, 2) of the batch: the positions enter only through the
    fractional shift of the probe (dataset_models.py:1487-1490, ptycho_utils.py:128-176;
    the rounded part only picks the patch).  With Y = fft2(probe) * ramp(frac) and
    psi0 = ifft2(Y), G_Y = fft2(g) / (H W) for the probe-plane gradient g, and
    dL/dfrac_r = sum over modes and frequencies of Re(conj(G_Y) (-2 pi i k_r) Y)."""
    H, W = probe_o.shape[-2:]
    kr = np.fft.fftfreq(H, d=1.0)[None, None, :, None]
    kc = np.fft.fftfreq(W, d=1.0)[None, None, None, :]
    Y = fft2(probe_o)[:, None] * st.ramp[None]            # (P, B, H, W)
    t = np.conj(fft2(g_probe_plane) / (H * W)) * Y
    gr = np.sum(np.real(-2j * np.pi * kr * t), axis=(0, 2, 3))
    gc = np.sum(np.real(-2j * np.pi * kc * t), axis=(0, 2, 3))
    return np.stack([gr, gc], axis=-1)


def descan_gradients(st: ForwardState) -> np.ndarray:
    """dL/d(descan shift) (B, 2): the exit wave is E = Y ramp(d) with
    ramp = exp(-2 pi i (fftfreq_r d_r + fftfreq_c d_c)) on the real-space grid, so
    dL/dd_r = sum over modes and pixels of 2 pi fftfreq_r Im(conj(dL/dE) E)."""
    H, W = st.exit.shape[-2:]
    kr = np.fft.fftfreq(H, d=1.0)[None, None, :, None]
    kc = np.fft.fftfreq(W, d=1.0)[None, None, None, :]
    im = np.imag(np.conj(st.g_exit) * st.exit)
    return np.stack([np.sum(2 * np.pi * kr * im, axis=(0, 2, 3)), np.sum(2 * np.pi * kc * im, axis=(0, 2, 3))], -1)


def tilt_gradients(st: ForwardState, tilt_mrad, slice_thicknesses, sampling, roi_shape) -> np.ndarray:
    """dL/d(probe tilt) (2,) [1/mrad] of a batch.  K_s carries exp(-2 pi i dz_s tan(theta/1e3) k)
    per axis (probe_models.py:418-425), so dL/dtheta = sum_s 2 pi dz_s sec^2(theta/1e3)/1e3
    sum_k k Im(conj(dL/dZ_s) Z_s).  The reference multiplies the ramp in only when
    theta != 0 (probe_models.py:418, 421), so a zero tilt has a zero gradient."""
    dz = np.broadcast_to(np.atleast_1d(np.asarray(slice_thicknesses, dtype=np.float64)), (st.prop_sums.shape[0],))
    out = np.zeros(2)
    for a in range(2):
        th = float(tilt_mrad[a])
        if th == 0.0 or st.prop_sums.shape[0] == 0:
            continue
        k_unit = 1.0 / (int(roi_shape[a]) * float(sampling[a]))  # fftfreq(n, d) = index / (n d)
        sec2 = 1.0 / math.cos(th / 1e3) ** 2
        out[a] = float(np.sum(2 * np.pi * dz * st.prop_sums[:, a])) * k_unit * sec2 / 1e3
    return out


def batch_loss_and_grads(obj_c, probe_o, positions_px, props, targets, mask, num_gpts,
                         mean_intensity, loss_type="l2_amplitude", descan=None):
    st = forward(obj_c, probe_o, positions_px, props, descan)
    loss, dI = loss_and_seed(st.intensity, targets, mask, num_gpts, mean_intensity, loss_type)
    g_obj, g_probe = adjoint(obj_c, probe_o, props, st, dI)
    return loss, g_obj, g_probe, st


def _ext_args(obj_constraints: dict, obj_mask, obj_shape_2d=None, sampling=None):
    c = obj_constraints
    env = None
    if c.get("q_lowpass") or c.get("q_highpass"):
        env = butterworth_env(obj_shape_2d, sampling, c.get("q_lowpass"), c.get("q_highpass"),
                              int(c.get("butterworth_order", 4)))
    return dict(mask=obj_mask if c.get("apply_fov_mask") else None, positivity=c.get("positivity", True),
                fix_baseline=c.get("fix_potential_baseline", False),
                baseline_factor=c.get("fix_potential_baseline_factor", 1.0),
                taps=gaussian_taps(c["gaussian_sigma"]) if c.get("gaussian_sigma") is not None else None,
                identical=c.get("identical_slices", False), butter_env=env)


def full_gradients(obj_raw, probe_raw, positions_px, props, targets, mask, num_gpts,
                   mean_intensity, upsample_factor, orthogonalize=True,
                   loss_type="l2_amplitude", obj_type="complex", descan=None, obj_constraints=None,
                   obj_mask=None, obj_sampling=None, probe_constraints=None):
    """Loss and gradients w.r.t. the raw parameters, as Ptychography.backward
    leaves them (autograd branch, ptychography.py:326-332): the object gradient
    is scaled by upsample_factor**2 / 2.  ``obj_type``: complex, pure_phase or
    potential (default constraints: positivity on, baseline not fixed).  ``descan``:
    (B, 2) descan shifts of the batch or None; ``descan_gradients(st)`` and
    ``tilt_gradients(st, ...)`` read the returned state.  ``obj_constraints`` (a dict of the
    reference's object constraints) with ``obj_mask`` (the FOV mask) selects the full hard
    constraint (``constrain_object_ext``) and adds the soft-constraint loss, as the
    reference's batch loss does (ptychography.py:229-231).  ``probe_constraints`` (a dict of
    the reference's probe constraints; replaces ``orthogonalize``) adds the centre-of-mass
    shift and the probe TV soft loss on the hard-constrained probe (ptychography.py:134)."""
    if obj_constraints is not None:
        ext = _ext_args(obj_constraints, obj_mask, obj_raw.shape[-2:], obj_sampling)
        obj2 = constrain_object_ext(obj_raw, obj_type, **ext)
        obj_c = np.exp(1j * obj2) if obj_type == "potential" else obj2
    else:
        obj_c = object_transmission(obj_raw, obj_type)
    pc = {"orthogonalize_probe": bool(orthogonalize)} if probe_constraints is None else probe_constraints
    probe_o, pcache = constrain_probe(probe_raw, pc)
    loss, g_obj_c, g_probe_o, st = batch_loss_and_grads(
        obj_c, probe_o, positions_px, props, targets, mask, num_gpts, mean_intensity, loss_type, descan)
    st.probe_o = probe_o
    if pc.get("tv_weight", 0):
        tv, g_tv = probe_tv_loss(probe_o, pc["tv_weight"])
        loss = loss + tv
        g_probe_o = g_probe_o + g_tv
    if obj_constraints is not None:
        c = obj_constraints
        g2 = phase_exp_vjp(obj2, g_obj_c) if obj_type == "potential" else g_obj_c
        if c.get("tv_weight_z", 0) or c.get("tv_weight_xy", 0) or c.get("surface_zero_weight", 0):
            soft, g_soft = soft_constraint_loss(obj2, obj_type, c.get("tv_weight_z", 0), c.get("tv_weight_xy", 0),
                                                c.get("surface_zero_weight", 0))
            loss = loss + soft
            g2 = g2 + g_soft
        g_obj = constrain_object_ext_vjp(obj_raw, g2, obj_type, **ext) * (upsample_factor**2 / 2)
    else:
        g_obj = object_transmission_vjp(obj_raw, g_obj_c, obj_type) * (upsample_factor**2 / 2)
    g_probe = constrain_probe_vjp(pcache, g_probe_o)
    return loss, g_obj, g_probe, st


# ----------------------------------------------------------------------------
# optimiser
# ----------------------------------------------------------------------------

@dataclass
class AdamState:
    step: int = 0
    exp_avg: np.ndarray = None
    exp_avg_sq: np.ndarray = None


def adam_step(param: np.ndarray, grad: np.ndarray, st: AdamState, lr, betas=(0.9, 0.999),
              eps=1e-8, weight_decay=0.0, decoupled=False):
    """torch.optim.Adam / AdamW update on the real view of a complex parameter
    (optimizer_mixin.py:117-123 selects the torch optimiser)."""
    rd = real_dtype(param.dtype) if np.iscomplexobj(param) else param.dtype
    p = param.view(rd) if np.iscomplexobj(param) else param
    g = grad.astype(param.dtype).view(rd) if np.iscomplexobj(param) else grad
    if st.exp_avg is None:
        st.exp_avg = np.zeros_like(p)
        st.exp_avg_sq = np.zeros_like(p)
    st.step += 1
    b1, b2 = betas
    if weight_decay != 0:
        if decoupled:
            p *= 1 - lr * weight_decay
        else:
            g = g + weight_decay * p
    st.exp_avg += (g - st.exp_avg) * (1 - b1)
    st.exp_avg_sq *= b2
    st.exp_avg_sq += (1 - b2) * g * g
    bc1 = 1 - b1**st.step
    bc2 = 1 - b2**st.step
    denom = np.sqrt(st.exp_avg_sq) / math.sqrt(bc2) + eps
    p -= (lr / bc1) * st.exp_avg / denom
    return param


def sgd_step(param, grad, lr):
    param -= lr * grad.astype(param.dtype)
    return param


# ----------------------------------------------------------------------------
# batching
# ----------------------------------------------------------------------------

def batch_order(rng: np.random.Generator, num: int, batch_size: int):
    """One epoch of SimpleBatcher without validation split; ptycho_utils.py:91-96."""
    order = rng.permutation(np.arange(num))
    return [order[i:i + batch_size] for i in range(0, num, batch_size)]


# ----------------------------------------------------------------------------
# synthetic data helpers
# ----------------------------------------------------------------------------

def gaussian_atom_phase(shape, n_atoms, sigma_px, peak_rad, rng):
    """Sum of isotropic Gaussian atoms at uniform positions (periodic)."""
    H, W = shape
    out = np.zeros((H, W), dtype=np.float64)
    rr = np.arange(H)[:, None]
    cc = np.arange(W)[None, :]
    pos = rng.uniform(0, 1, size=(n_atoms, 2)) * np.array([H, W])
    for r0, c0 in pos:
        dr = (rr - r0 + H / 2) % H - H / 2
        dc = (cc - c0 + W / 2) % W - W / 2
        out += np.exp(-(dr**2 + dc**2) / (2 * sigma_px**2))
    return peak_rad * out


# ----------------------------------------------------------------------------
# iteration driver
# ----------------------------------------------------------------------------

def reconstruct(obj_raw, probe_raw, positions_px, props, targets, mask, mean_intensity, upsample_factor,
                num_iters, batch_size, rng, lr_obj=5e-3, lr_probe=1e-3, orthogonalize=True,
                loss_type="l2_amplitude", obj_type="complex", lr_positions=None, descan=None, lr_descan=None,
                tilt=None, prop_geometry=None, obj_constraints=None, obj_mask=None, obj_sampling=None,
                probe_constraints=None):
    """Adam iterations of Ptychography.reconstruct (ptychography.py:208-245) on
    the given state; batches from a numpy generator like SimpleBatcher.  With
    ``lr_positions`` the scan positions are a parameter too (a dataset optimiser,
    dataset_models.py:98-110): Adam over the whole (N, 2) array, the gradient zero
    outside the batch.  ``descan`` ((N, 2) start) applies descan shifts, learned with
    Adam at ``lr_descan`` (the same dataset optimiser).  ``tilt`` ((2,) mrad start, with
    ``prop_geometry`` = (roi_shape, sampling, energy, slice_thicknesses)) learns the probe
    tilt in the probe's Adam (lr_probe; probe_models.py:295-304), the propagators
    recomputed from it for every batch.  Returns (obj, probe, per-iteration mean batch
    losses), plus the positions with ``lr_positions``, plus a dict with "descan" / "tilt"
    when either is given."""
    obj = obj_raw.copy()
    probe = probe_raw.copy()
    pos = positions_px.astype(np.float64).copy()
    dsc = None if descan is None else np.asarray(descan, dtype=np.float64).copy()
    th = None if tilt is None else np.asarray(tilt, dtype=np.float64).copy()
    so, sp, spos, sdsc, sth = AdamState(), AdamState(), AdamState(), AdamState(), AdamState()
    npos = positions_px.shape[0]
    losses = []
    for _ in range(num_iters):
        tot, nb = 0.0, 0
        for bi in batch_order(rng, npos, batch_size):
            if th is not None:
                roi, samp, energy, dz = prop_geometry
                props = propagators(roi, samp, energy, dz, tilt_mrad=tuple(th))
            loss, g_obj, g_probe, st = full_gradients(obj, probe, pos[bi], props, targets[bi], mask, npos,
                                                      mean_intensity, upsample_factor, orthogonalize, loss_type,
                                                      obj_type, descan=None if dsc is None else dsc[bi],
                                                      obj_constraints=obj_constraints, obj_mask=obj_mask,
                                                      obj_sampling=obj_sampling, probe_constraints=probe_constraints)
            if lr_positions is not None:
                g_pos = np.zeros_like(pos)
                g_pos[bi] = position_gradients(st.probe_o, st, st.g_probe_plane)
            if dsc is not None and lr_descan is not None:
                g_dsc = np.zeros_like(dsc)
                g_dsc[bi] = descan_gradients(st)
            if th is not None:
                g_th = tilt_gradients(st, th, prop_geometry[3], prop_geometry[1], prop_geometry[0])
            adam_step(obj, g_obj, so, lr_obj)
            adam_step(probe, g_probe, sp, lr_probe)
            if th is not None:
                adam_step(th, g_th, sth, lr_probe)
            if lr_positions is not None:
                adam_step(pos, g_pos, spos, lr_positions)
            if dsc is not None and lr_descan is not None:
                adam_step(dsc, g_dsc, sdsc, lr_descan)
            tot += loss
            nb += 1
        losses.append(tot / nb)
    res = (obj, probe, np.array(losses))
    if lr_positions is not None:
        res = res + (pos,)
    if dsc is not None or th is not None:
        res = res + ({"descan": dsc, "tilt": th},)
    return res


# ----------------------------------------------------------------------------
# analytic (autograd=False) update directions
# ----------------------------------------------------------------------------

def fourier_projection_seed(far: np.ndarray, targets: np.ndarray) -> np.ndarray:
    """Fourier-space seed m(Psi) - Psi of the analytic update (ptychography.py:350-372).

    ``far`` is the orthonormal far field (P, B, H, W), ``targets`` the measured
    amplitudes in detector (centred) layout.  One mode: measured amplitude with
    the estimated phase; several modes: Psi * measured / estimated amplitude with
    the estimate sqrt(sum_p |Psi_p + 1e-9|^2) (ptychography_base.py:949-961) and
    zero estimates mapped to infinity.  Returns (mod - Psi) in Fourier space.
    """
    meas = np.fft.fftshift(targets, axes=(-2, -1))[None]
    P = far.shape[0]
    if P == 1:
        mod = meas * np.exp(1j * np.angle(far))
    else:
        amps = np.sqrt(np.sum(np.abs(far + 1e-9) ** 2, axis=0))
        amps = np.where(amps == 0, np.inf, amps)
        mod = (meas / amps) * far
    return mod - far


def analytic_gradients(obj_raw, probe_raw, positions_px, props, targets, orthogonalize=False, obj_type="complex",
                       obj_c=None, probe_o=None):
    """Object and probe update directions of the analytic path, as
    ``Ptychography.backward(autograd=False)`` leaves them in ``.grad``
    (ptychography.py:339-348, object_models.py:686-725, probe_models.py:774-783).
    ``obj_type``: complex and pure-phase objects take sum_patches(conj(psi) g); a potential
    takes the real sum_patches(Re(-i conj(o) conj(psi) g)) with o its transmission patches.
    ``obj_c`` / ``probe_o`` (optional) replace the default hard-constrained transmission and
    probe, for the optional constraints, which act through the forward model only.
    """
    if obj_c is None:
        obj_c = constrain_object(obj_raw) if obj_type == "complex" else object_transmission(obj_raw, obj_type)
    if probe_o is None:
        probe_o = gram_schmidt(probe_raw)[0] if orthogonalize else probe_raw
    S = obj_c.shape[0]
    P, H, W = probe_o.shape
    st = forward(obj_c, probe_o, positions_px, props)
    grad = ifft2(fourier_projection_seed(st.far, targets), norm="ortho")
    pot = obj_type == "potential"
    g_obj = np.zeros(obj_c.shape, dtype=obj_c.real.dtype if pot else obj_c.dtype)
    for s in reversed(range(S)):
        psi = st.waves[s]
        norm = 0.0
        upd = np.zeros(obj_c.shape[1:], dtype=g_obj.dtype)
        for a in range(P):
            inten = scatter_patches((np.abs(psi[a]) ** 2)[None], st.rows, st.cols, (1,) + obj_c.shape[1:])[0]
            norm += inten.max()
            term = np.conj(psi[a]) * grad[a]
            if pot:
                term = np.real(-1j * np.conj(st.patches[s]) * term)
            upd += scatter_patches(term[None], st.rows, st.cols, (1,) + obj_c.shape[1:])[0]
        g_obj[s] = upd / norm
        grad = np.conj(st.patches[s])[None] * grad
        if s > 0:
            grad = ifft2(fft2(grad) * np.conj(props[s - 1])[None, None])
    obj_norm = np.max(np.sum(np.abs(st.patches) ** 2, axis=(-2, -1)))
    ortho_norm = 2 * np.sqrt(H * W) if P == 1 else 1 / (2 * np.sqrt(H * W))
    g_probe = np.sum(grad, axis=1) / obj_norm / ortho_norm
    return -g_obj, -g_probe, st
