"""Pixelated detector (quantem detector_models.DetectorPixelated).

forward: orthonormal 2-D FFT of every exit wave, |.|^2 summed over probe modes,
fftshift to the detector's centred layout (detector_models.py:22-30).  On the
training path this runs fused inside the batch kernel; this method serves
callers that hold explicit exit waves.
"""
from __future__ import annotations

import torch


class DetectorPixelated:
    def forward(self, exit_waves: torch.Tensor) -> torch.Tensor:
        from .. import ops

        n = exit_waves.shape[-1]
        far = ops.fft2(exit_waves.detach().to(torch.complex64).contiguous(), scale=1.0 / n)
        inten = torch.sum(far.real.square() + far.imag.square(), dim=0)
        return torch.fft.fftshift(inten, dim=(-2, -1))


DetectorModelType = DetectorPixelated
