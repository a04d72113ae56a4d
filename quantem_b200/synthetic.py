"""Seeded synthetic multislice mixed-probe datasets, simulated on the GPU with
this package's own forward kernels.

Geometry follows the benchmark configurations of the ptychography path:
300 kV, 0.2 A real-space pixels, 20 mrad aperture, 200 A defocus, Gaussian-atom
phase objects, raster scans with optional +-0.5 px jitter and Poisson noise.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import ops
from .diffractive_imaging.complex_probe import electron_wavelength_angstrom, real_space_probe
from .diffractive_imaging.ptycho_utils import orthogonalize_probes


@dataclass
class SyntheticConfig:
    n: int = 128                  # probe window
    slices: int = 8
    modes: int = 4
    mode_weights: tuple = (0.7, 0.15, 0.1, 0.05)
    scan: tuple = (64, 64)
    step_px: float = 6.0
    jitter_px: float = 0.5
    pad_px: int = 67
    slice_thickness: float = 20.0
    peak_phase: float = 0.1
    atom_density: float = 0.003   # atoms / px^2 / slice
    sigma_px: float = 1.5
    counts: float = 1e5
    energy: float = 300e3
    pixel: float = 0.2
    semiangle: float = 20.0
    defocus: float = 200.0
    seed: int = 0


def gaussian_atom_phase(shape, n_atoms, sigma, peak, gen: torch.Generator, device):
    """Sum of periodic isotropic Gaussians at uniform positions (one slice)."""
    H, W = shape
    pos = torch.rand((n_atoms, 2), generator=gen, device=device, dtype=torch.float64) * torch.tensor(
        [H, W], device=device, dtype=torch.float64)
    rad = int(np.ceil(5 * sigma))
    off = torch.arange(-rad, rad + 1, device=device)
    base = torch.floor(pos).long()
    rr = base[:, 0, None, None] + off[None, :, None]
    cc = base[:, 1, None, None] + off[None, None, :]
    val = torch.exp(-((rr - pos[:, 0, None, None]) ** 2 + (cc - pos[:, 1, None, None]) ** 2) / (2 * sigma**2))
    out = torch.zeros(H * W, device=device, dtype=torch.float64)
    idx = (rr % H) * W + (cc % W)
    out.index_put_((idx.reshape(-1),), val.reshape(-1), accumulate=True)
    return peak * out.reshape(H, W)


def fresnel_propagators(n, sampling, energy, dz, slices, device):
    """(S-1, n, n) propagators; probe_models.py:376-427 evaluated like the reference."""
    if slices <= 1:
        return torch.zeros((0, n, n), dtype=torch.complex64, device=device)
    kr = torch.fft.fftfreq(n, sampling, device=device)
    kc = torch.fft.fftfreq(n, sampling, device=device)
    k2 = (kr[:, None] ** 2 + kc[None] ** 2).to(torch.complex64)
    lam = electron_wavelength_angstrom(energy)
    dzt = torch.full((slices - 1,), float(dz), device=device, dtype=k2.dtype)
    return torch.exp((-1.0j * torch.pi * lam * dzt[:, None, None]) * k2)


def make_probe_modes(cfg: SyntheticConfig, device):
    base = real_space_probe((cfg.n, cfg.n), (cfg.pixel, cfg.pixel), cfg.energy, cfg.semiangle,
                            aberration_coefs={"C10": -cfg.defocus}, device=device).to(torch.complex64)
    modes = [base]
    k = torch.fft.fftfreq(cfg.n, device=device)
    g = torch.Generator(device="cpu").manual_seed(cfg.seed + 11)
    for _ in range(1, cfg.modes):
        sr, sc = (torch.rand(2, generator=g) - 0.5).tolist()
        ramp = torch.exp(-2j * torch.pi * (sr * k[:, None] * 4 + sc * k[None, :] * 4))
        modes.append(base * ramp.to(torch.complex64))
    probes = torch.stack(modes)
    w = torch.tensor(cfg.mode_weights[:cfg.modes], dtype=torch.float32, device=device)
    w = w / w.sum()
    norms = probes.abs().square().sum(dim=(-2, -1))
    return probes * torch.sqrt(w / norms)[:, None, None]


def make_dataset(cfg: SyntheticConfig, device="cuda"):
    """Returns a dict with the true object/probe, positions [px], object shape,
    Poisson intensities (npos, n, n) in detector layout and their amplitudes."""
    dev = torch.device(device)
    gen = torch.Generator(device=dev).manual_seed(cfg.seed)
    nr, nc = cfg.scan
    ext = (np.array(cfg.scan) - 1) * cfg.step_px
    Ho = int(ext[0] + 2 * cfg.pad_px)
    Wo = int(ext[1] + 2 * cfg.pad_px)
    Ho += (-Ho) % 8
    Wo += (-Wo) % 8
    n_atoms = max(4, int(cfg.atom_density * Ho * Wo))
    phase = torch.stack([gaussian_atom_phase((Ho, Wo), n_atoms, cfg.sigma_px, cfg.peak_phase, gen, dev)
                         for _ in range(cfg.slices)])
    obj = torch.exp(1j * phase).to(torch.complex64)
    rr, cc = torch.meshgrid(torch.arange(nr, device=dev), torch.arange(nc, device=dev), indexing="ij")
    pos = torch.stack([rr.reshape(-1), cc.reshape(-1)], -1).double() * cfg.step_px + cfg.pad_px
    if cfg.jitter_px:
        pos = pos + (torch.rand(pos.shape, generator=gen, device=dev, dtype=torch.float64) * 2 - 1) * cfg.jitter_px
    pos = pos.float().contiguous()
    # simulate with the orthogonalised, intensity-sorted modes: the reconstruction
    # applies the same Gram-Schmidt (probe_models.py:484-525) to its probe, which
    # leaves these modes unchanged, so data and model describe one mixed state
    probes = orthogonalize_probes(make_probe_modes(cfg, dev))
    props = ops.separable_propagators(cfg.n, (cfg.pixel, cfg.pixel), cfg.energy,
                                      [cfg.slice_thickness] * (cfg.slices - 1), device=dev)
    npos = pos.shape[0]
    dummy_t = torch.zeros((npos, cfg.n, cfg.n), device=dev, dtype=torch.float32)
    mask = torch.ones((cfg.n, cfg.n), device=dev, dtype=torch.float32)
    inten = torch.empty((npos, cfg.n, cfg.n), device=dev, dtype=torch.float32)
    chunk = 1024
    for s in range(0, npos, chunk):
        idx = torch.arange(s, min(s + chunk, npos), device=dev, dtype=torch.int64)
        out = ops.batch_forward(obj, probes, props, pos, idx, dummy_t, mask, npos, 1.0)
        inten[s:s + idx.numel()] = out["intensity"]
    scale = cfg.counts / inten.sum(dim=(-2, -1)).mean()
    counts = torch.poisson(inten.double() * scale, generator=gen).float()
    return dict(obj=obj, probes=probes, positions=pos, obj_shape=(cfg.slices, Ho, Wo), intensities=counts,
                amplitudes=torch.sqrt(counts), propagators=props, mean_intensity=float(counts.sum() / npos))
