"""Inputs of the reference's own gradient test, restated.

Recipe of tests/diffractive_imaging/test_ptychography.py:19-146 in the
reference: a 64x64 white-noise phase object (numpy seed 42, zero-mean uniform
noise), an analytic soft-aperture probe (Q_PROBE = 0.25 A^-1, C10 = 50 A,
300 kV), a 1 px raster over the whole object with periodic wrap, and
intensities = fftshift(|fft2(patch * probe)|^2 * 100).
"""
from __future__ import annotations

import numpy as np

from oracle.ptycho_oracle import electron_wavelength_angstrom

N = 64
Q_MAX = 0.5
Q_PROBE = Q_MAX / 2
ENERGY = 300e3
C10 = 50.0


def whitenoise_inputs():
    rng = np.random.default_rng(42)
    arr = rng.random((N, N))
    arr -= arr.mean()
    obj = np.exp(1.0j * arr.astype(np.float32))
    sampling = 1 / Q_MAX / 2
    rsamp = 2 * Q_MAX / N
    q = np.fft.fftfreq(N, sampling)
    qq = np.sqrt(q[:, None] ** 2 + q[None, :] ** 2)
    aperture = np.sqrt(np.clip((Q_PROBE - qq) / rsamp + 0.5, 0, 1))
    chi = qq**2 * electron_wavelength_angstrom(ENERGY) * np.pi * C10
    pf = aperture * np.exp(-1j * chi)
    pf /= np.sqrt(np.sum(np.abs(pf) ** 2))
    probe = np.fft.ifft2(pf) * N
    x = np.arange(0.0, N, 1.0)
    xx, yy = np.meshgrid(x, x, indexing="ij")
    positions = np.stack((xx.ravel(), yy.ravel()), axis=-1)
    ind = np.fft.fftfreq(N, d=1 / N).astype(int)
    x0 = np.round(positions[:, 0]).astype(int)
    y0 = np.round(positions[:, 1]).astype(int)
    row = (x0[:, None, None] + ind[None, :, None]) % N
    col = (y0[:, None, None] + ind[None, None, :]) % N
    exit_waves = obj[row, col] * probe
    inten = np.abs(np.fft.fft2(exit_waves)) ** 2
    data4d = np.fft.fftshift(inten * 100, axes=(-2, -1)).reshape((N, N, N, N))
    return dict(
        N=N, obj=obj, probe=probe, positions=positions, data4d=data4d,
        sampling4d=(1, 1, rsamp, rsamp), energy=ENERGY,
        probe_params={"energy": ENERGY, "C10": C10,
                      "semiangle_cutoff": electron_wavelength_angstrom(ENERGY) * 1e3},
    )
