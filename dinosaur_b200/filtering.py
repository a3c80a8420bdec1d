"""Spectral filters (dinosaur/filtering.py:27-100).

The per-l scalings are FP64 on the host, as in the reference.  Inside the
fused SIL3 step they are applied by the final stage kernel; the standalone
filter functions here scale every leaf whose shape broadcasts with the
scaling (filtering.py:27-35).
"""

from __future__ import annotations

import numpy as np
import torch

from dinosaur_b200 import pytree


def exponential_scaling(grid, attenuation=16, order=18, cutoff=0.0):
  """exp(-a ((k - c)/(1 - c))^(2p)) for k > c, k = l / l_max (filtering.py:38-89)."""
  _, total_wavenumber = grid.modal_axes
  k = total_wavenumber / total_wavenumber.max()
  a, c, p = attenuation, cutoff, order
  return np.exp((k > c) * (-a * (((k - c) / (1 - c)) ** (2 * p))))


def diffusion_scaling(grid, scale, order=1):
  """exp(-scale (-lambda_l)^order) (filtering.py:92-100)."""
  eigenvalues = grid.laplacian_eigenvalues
  return np.exp(-scale * (-eigenvalues) ** order)


def apply_scaling(scaling, tree):
  scaling = np.asarray(scaling)

  def rescale(x):
    if not isinstance(x, (torch.Tensor, np.ndarray)) or x.ndim == 0:
      return x
    if tuple(x.shape) != tuple(np.broadcast_shapes(tuple(x.shape),
                                                   scaling.shape)):
      return x
    if isinstance(x, torch.Tensor):
      return x * torch.as_tensor(scaling, device=x.device, dtype=x.dtype)
    return x * scaling

  return pytree.tree_map(rescale, tree)


def exponential_filter(grid, attenuation=16, order=18, cutoff=0.0):
  scaling = exponential_scaling(grid, attenuation, order, cutoff)
  return lambda tree: apply_scaling(scaling, tree)


def horizontal_diffusion_filter(grid, scale, order=1):
  scaling = diffusion_scaling(grid, scale, order)
  return lambda tree: apply_scaling(scaling, tree)
