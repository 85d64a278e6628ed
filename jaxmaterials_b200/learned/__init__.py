"""Learned warm start: a spectral-convolution network trained on solver output."""
