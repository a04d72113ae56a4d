"""B200-native multislice mixed-probe ptychography (drop-in for quantem.diffractive_imaging)."""
__version__ = "0.1.0"
