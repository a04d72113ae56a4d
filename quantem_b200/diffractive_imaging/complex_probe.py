"""Probe synthesis (set-up of the ptychography path), restated in torch.

Follows quantem.diffractive_imaging.complex_probe of the reference:
soft/hard aperture (complex_probe.py:33-125), polar aberration surface chi
(164-215), Fourier-space probe (434-472) and real-space probe (475-507).
Frequencies are evaluated in float32 like the reference (404-405).
"""
from __future__ import annotations

import math
from typing import Mapping

import torch

POLAR_ALIASES = {
    "defocus": "C10", "astigmatism": "C12", "astigmatism_angle": "phi12", "coma": "C21",
    "coma_angle": "phi21", "Cs": "C30", "C5": "C50",
}
POLAR_SYMBOLS = (
    "C10", "C12", "phi12", "C21", "phi21", "C23", "phi23", "C30", "C32", "phi32", "C34", "phi34",
    "C41", "phi41", "C43", "phi43", "C45", "phi45", "C50", "C52", "phi52", "C54", "phi54", "C56", "phi56",
)


def electron_wavelength_angstrom(energy_ev: float) -> float:
    """Relativistic electron wavelength in Angstrom (core/utils/utils.py:97-104)."""
    m = 9.109383e-31
    e = 1.602177e-19
    c = 299792458
    h = 6.62607e-34
    return h / math.sqrt(2 * m * e * energy_ev) / math.sqrt(1 + e * energy_ev / 2 / m / c**2) * 1e10


def spatial_frequencies(gpts, sampling, device="cpu"):
    kx = torch.fft.fftfreq(int(gpts[0]), float(sampling[0]), device=device, dtype=torch.float32)
    ky = torch.fft.fftfreq(int(gpts[1]), float(sampling[1]), device=device, dtype=torch.float32)
    return kx[:, None].broadcast_to(*gpts), ky[None, :].broadcast_to(*gpts)


def polar_coordinates(kx, ky):
    return torch.sqrt(kx.square() + ky.square()), torch.arctan2(ky, kx)


def hard_aperture(alpha, semiangle_cutoff):
    return (alpha <= semiangle_cutoff * 1e-3).to(torch.float32)


def soft_aperture(alpha, phi, semiangle_cutoff, angular_sampling):
    semiangle_rad = semiangle_cutoff * 1e-3
    denom = torch.sqrt((torch.cos(phi) * angular_sampling[0] * 1e-3).square()
                       + (torch.sin(phi) * angular_sampling[1] * 1e-3).square())
    return torch.clip((semiangle_rad - alpha) / denom + 0.5, 0, 1).to(torch.float32)


def aberration_surface(alpha, phi, wavelength, coefs: Mapping[str, float]):
    a2 = alpha.square()
    chi = torch.zeros_like(alpha)

    def g(name):
        return coefs.get(name, 0.0)

    if any(k in coefs for k in ("C10", "C12", "phi12")):
        chi = chi + 0.5 * a2 * (g("C10") + g("C12") * torch.cos(2 * (phi - g("phi12"))))
    if any(k in coefs for k in ("C21", "phi21", "C23", "phi23")):
        chi = chi + (1 / 3) * a2 * alpha * (g("C21") * torch.cos(phi - g("phi21"))
                                            + g("C23") * torch.cos(3 * (phi - g("phi23"))))
    if any(k in coefs for k in ("C30", "C32", "phi32", "C34", "phi34")):
        chi = chi + 0.25 * a2.square() * (g("C30") + g("C32") * torch.cos(2 * (phi - g("phi32")))
                                          + g("C34") * torch.cos(4 * (phi - g("phi34"))))
    if any(k in coefs for k in ("C41", "phi41", "C43", "phi43", "C45", "phi45")):
        chi = chi + 0.2 * a2.square() * alpha * (g("C41") * torch.cos(phi - g("phi41"))
                                                 + g("C43") * torch.cos(3 * (phi - g("phi43")))
                                                 + g("C45") * torch.cos(5 * (phi - g("phi45"))))
    if any(k in coefs for k in ("C50", "C52", "phi52", "C54", "phi54", "C56", "phi56")):
        chi = chi + (1 / 6) * a2 * a2 * a2 * (g("C50") + g("C52") * torch.cos(2 * (phi - g("phi52")))
                                              + g("C54") * torch.cos(4 * (phi - g("phi54")))
                                              + g("C56") * torch.cos(6 * (phi - g("phi56"))))
    return 2 * math.pi / wavelength * chi


def fourier_space_probe(gpts, sampling, energy, semiangle_cutoff, soft_edges=True,
                        vacuum_probe_intensity=None, aberration_coefs=None, normalized=True, device="cpu"):
    wavelength = electron_wavelength_angstrom(energy)
    k, phi = polar_coordinates(*spatial_frequencies(gpts, sampling, device))
    alpha = k * wavelength
    angular_sampling = (alpha[1, 0] * 1e3, alpha[0, 1] * 1e3)
    if vacuum_probe_intensity is not None:
        ap = torch.sqrt(vacuum_probe_intensity.to(device)).to(torch.float32)
    elif soft_edges:
        ap = soft_aperture(alpha, phi, semiangle_cutoff, angular_sampling)
    else:
        ap = hard_aperture(alpha, semiangle_cutoff)
    fp = ap * torch.exp(-1j * aberration_surface(alpha, phi, wavelength, aberration_coefs or {}))
    if normalized:
        fp = fp / fp.abs().square().sum().sqrt()
    return fp


def real_space_probe(gpts, sampling, energy, semiangle_cutoff, soft_edges=True, vacuum_probe_intensity=None,
                     aberration_coefs=None, normalized=True, device="cpu"):
    fp = fourier_space_probe(gpts, sampling, energy, semiangle_cutoff, soft_edges, vacuum_probe_intensity,
                             aberration_coefs, True, device)
    probe = torch.fft.ifft2(fp)
    if normalized:
        probe = probe / probe.abs().square().sum().sqrt()
    return probe
