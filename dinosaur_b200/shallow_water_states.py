"""Steady zonal-flow states of the shallow-water equations
(dinosaur/shallow_water_states.py:50-119), built with the GPU transforms."""

from __future__ import annotations

import numpy as np
import torch

from dinosaur_b200 import shallow_water
from dinosaur_b200 import spherical_harmonic as sh


def one_layer(u, grid: sh.Grid) -> shallow_water.State:
  """Steady state of one layer: d(phi + u^2/2)/dlat + (zeta + f) u = 0 with
  v = 0 (shallow_water_states.py:50-85); u(lat) is nodal, shape [lat]."""
  sec_lat = torch.as_tensor(1 / grid.cos_lat, device='cuda', dtype=torch.float32)
  lon, _ = grid.nodal_axes
  u = sh.as_device_tensor(np.ones_like(lon)[..., np.newaxis] * np.asarray(u))
  sec_lat_u = u * sec_lat
  vorticity = -grid.sec_lat_d_dlat_cos2(grid.to_modal(sec_lat_u))
  f = torch.as_tensor(shallow_water.get_coriolis(grid), device='cuda',
                      dtype=torch.float32)
  total_vorticity = grid.to_nodal(vorticity) + f
  potential_plus_energy = -grid.inverse_laplacian(
      grid.sec_lat_d_dlat_cos2(grid.to_modal(sec_lat_u * total_vorticity)))
  potential = potential_plus_energy - grid.to_modal(u ** 2 / 2)
  potential = potential.clone()
  potential[0, 0] = 0
  return shallow_water.State(vorticity, torch.zeros_like(vorticity), potential)


def multi_layer(u, density, coords) -> shallow_water.State:
  """Steady state of n layers (shallow_water_states.py:88-119): the one-layer
  potentials, then (D + I) phi = phi_one_layer across layers."""
  states = [one_layer(ui, coords.horizontal) for ui in np.asarray(u)]
  vort = torch.stack([s.vorticity for s in states])
  div = torch.stack([s.divergence for s in states])
  pot = torch.stack([s.potential for s in states])
  n = coords.vertical.layers
  if n > 1:
    ratios = shallow_water.get_density_ratios(density) + np.eye(n)
    flat = pot.reshape(n, -1).double().cpu().numpy()
    pot = torch.as_tensor(np.linalg.solve(ratios, flat).reshape(pot.shape),
                          device='cuda', dtype=torch.float32)
  return shallow_water.State(vort, div, pot)
