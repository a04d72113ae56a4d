"""Global configuration keys used by the ptychography path.

Mirrors the keys of quantem.core.config that the path reads (quantem.yaml:4-14,
core/config.py:153-179, 491-553): ``device``, ``dtype_real`` and
``dtype_complex``.  The CUDA path computes in float32/complex64 only.
"""
from __future__ import annotations

import torch

_CONFIG = {"device": "cpu", "dtype_real": "float32", "dtype_complex": "complex64", "has_torch": True}


def get(key: str, default=None):
    return _CONFIG.get(key, default)


def set(values: dict) -> None:  # noqa: A001 - same name as the reference API
    for k, v in values.items():
        if k in ("dtype_real", "dtype_complex") and v not in ("float32", "complex64"):
            raise ValueError(f"{k}={v!r}: the B200 path computes in float32/complex64 only")
        _CONFIG[k] = v


def validate_device(device) -> tuple[str, int | None]:
    """Normalise 'cpu' | 'gpu' | 'cuda' | 'cuda:X' | int | torch.device."""
    if device is None:
        device = _CONFIG["device"]
    if isinstance(device, torch.device):
        device = str(device)
    if isinstance(device, int):
        return f"cuda:{device}", device
    d = str(device).lower()
    if d == "cpu":
        return "cpu", None
    if d in ("gpu", "cuda"):
        return "cuda:0", 0
    if d.startswith("cuda:"):
        idx = int(d.split(":")[1])
        return f"cuda:{idx}", idx
    raise ValueError(f"Unknown device {device!r}")
