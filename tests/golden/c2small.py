"""The c2small fixture (headline geometry at a 3 x 3 scan, made by
``make_golden.py`` from the reference itself): the perturbed start object is not
stored but regenerated from its seed, and object-sized arrays are stored on
sampled pixels only."""
from __future__ import annotations

import numpy as np


def perturbed_object(shape, seed):
    """The perturbed start object: amplitude 1 - 0.3 U[0,1), phase 0.4 N(0,1), rounded
    to complex64 (the reference run received exactly this array)."""
    rng = np.random.default_rng(seed)
    amp = 1.0 - 0.3 * rng.random(shape)
    ph = 0.4 * rng.standard_normal(shape)
    return (amp * np.exp(1j * ph)).astype(np.complex64)


def load_c2small():
    """The fixture with ``obj_perturbed`` regenerated (and checked against its stored
    checksum)."""
    from tests.conftest import load_golden

    z = load_golden("c2small")
    obj = perturbed_object(tuple(int(v) for v in z["obj_shape"]), int(z["perturb_seed"]))
    got = float(np.abs(obj.astype(np.complex128)).sum())
    if abs(got - float(z["obj_perturbed_abs_sum"])) > 1e-9 * got:
        raise AssertionError("regenerated c2small start object differs from the recorded one")
    z["obj_perturbed"] = obj
    return z


def sampled(arr, idx):
    """Values of a (S, Ho, Wo) array at the flat per-slice indices ``idx``."""
    a = np.asarray(arr)
    return a.reshape(a.shape[0], -1)[:, idx]
