"""Held-Suarez forcing on sigma levels (dinosaur/held_suarez.py:47-167).

Constants are given in SI units (the reference takes pint quantities) and are
nondimensionalised with the default scale.  On the hot path the forcing runs
fused with the primitive equations: ``time_integration.compose_equations(
[pe, hs])`` returns a primitive-equation object whose explicit-terms kernel
adds Rayleigh drag and Newtonian cooling from the same diagnostic state (the
reference recomputes that state, held_suarez.py:126-128).  Evaluated on its
own, ``explicit_terms`` computes the forcing with the CUDA transforms and
spectral operators of the grid and elementwise nodal arithmetic on the GPU.
"""

from __future__ import annotations

import functools

import numpy as np
import torch

from dinosaur_b200 import spherical_harmonic as sh
from dinosaur_b200 import time_integration
from dinosaur_b200 import units


class HeldSuarezForcingSigma(time_integration.ExplicitODE):

  def __init__(self, coords, physics_specs, reference_temperature,
               p0: float = 1e5, sigma_b: float = 0.7,
               kf: float = 1 / units.SECONDS_PER_DAY,
               ka: float = 1 / (40 * units.SECONDS_PER_DAY),
               ks: float = 1 / (4 * units.SECONDS_PER_DAY),
               minT: float = 200.0, maxT: float = 315.0, dTy: float = 60.0,
               dThz: float = 10.0):
    self.coords = coords
    self.physics_specs = physics_specs
    self.reference_temperature = np.asarray(reference_temperature)
    self.p0 = units.nondim_pressure(p0)
    self.sigma_b = sigma_b
    # Rates in 1/s -> nondimensional rates.
    self.kf = kf * units.TIME_SCALE
    self.ka = ka * units.TIME_SCALE
    self.ks = ks * units.TIME_SCALE
    self.minT, self.maxT, self.dTy, self.dThz = minT, maxT, dTy, dThz
    self.sigma = coords.vertical.centers

  @functools.cached_property
  def lat(self):
    """Latitude of every nodal point, (lon, lat) (built on first use: the
    Gauss nodes come from the grid's GPU plan)."""
    _, sin_lat = self.coords.horizontal.nodal_mesh
    return np.arcsin(sin_lat)

  def _cutoff(self):
    # Boundary-layer profile: 0 above sigma_b, rising linearly to 1 at the
    # surface.
    return np.maximum(0, (self.sigma - self.sigma_b) / (1 - self.sigma_b))

  def kv(self):
    """Rayleigh-drag rate per level, (K, 1, 1) (held_suarez.py:99-103)."""
    return (self.kf * self._cutoff())[:, None, None]

  def kt(self):
    """Newtonian-cooling rate, (K, lon, lat) (held_suarez.py:105-109)."""
    return self.ka + (self.ks - self.ka) * (
        self._cutoff()[:, None, None] * np.cos(self.lat) ** 4)

  def equilibrium_temperature(self, nodal_surface_pressure):
    """Radiative-equilibrium temperature (held_suarez.py:111-120).

    T_eq = max(minT, (p / p0)^kappa (maxT - dTy sin^2(lat)
    - dThz ln(p / p0) cos^2(lat))) with p = sigma p_s on every level; a torch
    surface pressure gives a torch result on its device, an array a NumPy one.
    """
    kappa = self.physics_specs.kappa
    if isinstance(nodal_surface_pressure, torch.Tensor):
      ps = nodal_surface_pressure
      dev = lambda a: torch.as_tensor(np.asarray(a), device=ps.device, dtype=ps.dtype)
      sigma, lat = dev(self.sigma)[:, None, None], dev(self.lat)
      ratio = sigma * ps / self.p0
      t = ratio ** kappa * (self.maxT - self.dTy * torch.sin(lat) ** 2
                            - self.dThz * torch.log(ratio) * torch.cos(lat) ** 2)
      return torch.clamp(t, min=self.minT)
    ratio = self.sigma[:, None, None] * np.asarray(nodal_surface_pressure) / self.p0
    t = ratio ** kappa * (self.maxT - self.dTy * np.sin(self.lat) ** 2
                          - self.dThz * np.log(ratio) * np.cos(self.lat) ** 2)
    return np.maximum(self.minT, t)

  def explicit_terms(self, state):
    """Rayleigh drag and Newtonian cooling tendencies (held_suarez.py:122-167).

    The winds times cos(lat) come from the modal vorticity and divergence
    (unclipped, as in the reference's diagnostic state), the drag acts on
    them divided by cos^2(lat), and the vorticity and divergence tendencies
    are the clipped curl and divergence of its modal transform; the
    temperature relaxes towards T_eq(sigma p_s).  The surface-pressure (and
    any tracer) tendency is zero.  Members may be stacked on a leading axis.
    """
    grid = self.coords.horizontal
    vort = sh.as_device_tensor(state.vorticity)
    div = sh.as_device_tensor(state.divergence)
    dev = lambda a: torch.as_tensor(np.asarray(a), device=vort.device,
                                    dtype=torch.float32)
    cos2 = dev(grid.cos_lat ** 2)
    kv = dev(self.kv())
    cos_lat_u = sh.get_cos_lat_vector(vort, div, grid, clip=False)
    velocity = tuple(grid.to_modal(-kv * grid.to_nodal(c) / cos2) for c in cos_lat_u)
    temperature = (dev(self.reference_temperature)[:, None, None]
                   + grid.to_nodal(sh.as_device_tensor(state.temperature_variation)))
    ps = torch.exp(grid.to_nodal(sh.as_device_tensor(state.log_surface_pressure)))
    teq = self.equilibrium_temperature(ps)
    t_tend = -dev(self.kt()) * (temperature - teq)
    from dinosaur_b200 import primitive_equations  # pylint: disable=g-import-not-at-top
    return primitive_equations.State(
        vorticity=grid.curl_cos_lat(velocity),
        divergence=grid.div_cos_lat(velocity),
        temperature_variation=grid.to_modal(t_tend),
        log_surface_pressure=torch.zeros_like(
            sh.as_device_tensor(state.log_surface_pressure)),
        tracers={k: torch.zeros_like(sh.as_device_tensor(v))
                 for k, v in state.tracers.items()})
