"""Drop-in B200 implementation of quantem.diffractive_imaging's gradient ptychography path."""
from ..core.datasets import Dataset4dstem
from .dataset_models import PtychographyDatasetRaster
from .detector_models import DetectorPixelated
from .object_models import ObjectDIP, ObjectPixelated
from .probe_models import ProbePixelated
from .ptychography import Ptychography
from .ptychography_lite import PtychoLite, PtychoLiteDIP
from .ptycho_utils import SimpleBatcher

__all__ = ["Dataset4dstem", "PtychographyDatasetRaster", "DetectorPixelated", "ObjectPixelated", "ObjectDIP", "ProbePixelated",
           "Ptychography", "PtychoLite", "PtychoLiteDIP", "SimpleBatcher"]
