"""4D-STEM input container (the part of quantem.core.datastructures the path uses).

Dataset4dstem.from_array(array, name, origin, sampling, units) mirrors
core/datastructures/dataset4dstem.py:117-157; only the array and its
calibration are kept.
"""
from __future__ import annotations

import numpy as np


class Dataset4dstem:
    _token = object()

    def __init__(self, array, name, origin, sampling, units, signal_units="arb. units", _token=None):
        if _token is not self._token:
            raise RuntimeError("Use Dataset4dstem.from_array() to instantiate this class.")
        self.array = array
        self.name = name
        self.origin = np.asarray(origin, dtype=float)
        self.sampling = np.asarray(sampling, dtype=float)
        self.units = list(units)
        self.signal_units = signal_units
        self.file_path = None

    @classmethod
    def from_array(cls, array, name=None, origin=None, sampling=None, units=None, signal_units="arb. units"):
        arr = np.asarray(array)
        if arr.ndim != 4:
            raise ValueError(f"Dataset4dstem needs a 4-D array, got shape {arr.shape}")
        return cls(arr, name if name is not None else "4D-STEM dataset",
                   origin if origin is not None else np.zeros(4),
                   sampling if sampling is not None else np.ones(4),
                   units if units is not None else ["pixels"] * 4, signal_units, _token=cls._token)

    @property
    def shape(self):
        return self.array.shape
