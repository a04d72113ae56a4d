"""Golden values of the reference's consistency losses (all five loss types).

Run in a container where the reference source tree is mounted:

    python tests/golden/make_golden_loss.py <reference checkout>/src

Calls the reference's own ``PtychographyBase.error_estimate``
(ptychography_base.py:908-932) on seeded predicted intensities, targets and a
detector mask (detector layout), with torch autograd for dL/dI, and stores the
inputs, losses and gradients in ``loss_types.npz``.
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from baseline.reference_import import import_reference  # noqa: E402

LOSS_TYPES = ("l2_amplitude", "l1_amplitude", "l2_intensity", "l1_intensity", "poisson")


def main(src):
    import torch

    import_reference(src)
    from quantem.diffractive_imaging.ptychography_base import PtychographyBase

    rng = np.random.default_rng(17)
    B, n, num_gpts, mean_i = 3, 16, 40, 7.5
    inten = (rng.random((B, n, n)) * 9 + 0.05).astype(np.float64)
    mask = (rng.random((n, n)) > 0.2).astype(np.float64)
    out = dict(intensity=inten, mask=mask, num_gpts=np.int64(num_gpts), mean_intensity=np.float64(mean_i))
    for lt in LOSS_TYPES:
        t = np.sqrt(rng.random((B, n, n)) * 9) if "amplitude" in lt else rng.random((B, n, n)) * 9
        dset = types.SimpleNamespace(targets=torch.tensor(t), detector_mask=torch.tensor(mask), num_gpts=num_gpts,
                                     mean_diffraction_intensity=mean_i)
        me = types.SimpleNamespace(dset=dset)
        pred = torch.tensor(inten, requires_grad=True)
        loss, _ = PtychographyBase.error_estimate(me, pred, np.arange(B), loss_type=lt)
        loss.backward()
        out[f"{lt}_targets"] = t
        out[f"{lt}_loss"] = np.float64(loss.item())
        out[f"{lt}_dldi"] = pred.grad.numpy()
    np.savez_compressed(os.path.join(HERE, "loss_types.npz"), **out)
    print("wrote loss_types.npz")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {os.path.relpath(__file__)} <reference source dir (the one holding quantem/)>")
    main(sys.argv[1])
