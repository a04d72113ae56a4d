"""Minimal core utilities the ptychography path needs (config, datasets, optimiser mixin, RNG)."""
